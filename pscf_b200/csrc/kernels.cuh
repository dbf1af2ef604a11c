// kernels.cuh -- MDE propagator, contour-integral and reduction kernels.
//
// The propagator step is the reference's step_exp (src/step_mod.f90:146-176):
//   q1 = eo1 . F^-1[ek1 . F[eo1 . q]] / N                     (full step)
//   qh = eo1 . F^-1[ek2 . F[eo2 . q]] / N                     (first half step)
//   q2 = eo2 . F^-1[ek2 . F[qh]] / N                           (second half step)
//   q_out = (4 q2 - q1) / 3                                    (Richardson)
// with eo1 = exp(-w ds/2), eo2 = exp(-w ds/4), ek1 = exp(-ds b^2 k^2/6),
// ek2 = exp(-ds b^2 k^2/12) (make_propg, src/step_mod.f90:109-129).
#pragma once
#include "fft_dev.cuh"

namespace pscfg {

#define PSCFG_MAXB 8

// One contour sweep of one chain of one instance, in one direction.
template <typename T>
struct SweepField {
    T *slab;                // slices [ns+1][nr], slice s at slab + s*nr
    int ns;                 // number of steps (= last slice index)
    int dir;                // +1: s -> s+1 from s=0; -1: s -> s-1 from s=ns
    int nblk;
    int bgn[PSCFG_MAXB + 1];  // 0-based slice index of each block start
    const T *eo1[PSCFG_MAXB];
    const T *eo2[PSCFG_MAXB];
    const T *ek1[PSCFG_MAXB];
    const T *ek2[PSCFG_MAXB];
    // scratch for the multi-pass 3-D step (unused for dim <= 2)
    cx<T> *S1, *S2;
    T *q1;
    // optional separable k-space factors per block (plane kernels of
    // kernels3p.cuh, orthogonal cells): exp(-ds b^2 k^2/6) and /12 as
    // products of 1-D factors over the spectrum's x, y and z positions;
    // nullptr: the ek1/ek2 tables are read instead
    const T *ekf[PSCFG_MAXB];
    // optional single-step overrides (adjoint): read `in` instead of the
    // source slice, write `out` instead of the destination slice, and store
    // the step intermediates P1 x (into q1), h = E1 C2 E2 x and P2 x
    const T *in;
    T *out;
    T *h_out;
    T *q2_out;
};

template <typename T>
__device__ __forceinline__ const T *src_slice(const SweepField<T> &f, int src, long nr)
{
    return f.in ? f.in : f.slab + (long)src * nr;
}
template <typename T>
__device__ __forceinline__ T *dst_slice(const SweepField<T> &f, int dst, long nr)
{
    return f.out ? f.out : f.slab + (long)dst * nr;
}

// Block index and source/destination slices of step t (0-based).
template <typename T>
__device__ __forceinline__ bool step_slices(const SweepField<T> &f, int t, int &blk, int &src, int &dst)
{
    if (t >= f.ns) return false;
    if (f.dir > 0) {
        src = t;
        dst = t + 1;
        blk = 0;
        while (blk < f.nblk - 1 && src >= f.bgn[blk + 1]) blk++;
    } else {
        src = f.ns - t;
        dst = src - 1;
        blk = f.nblk - 1;
        while (blk > 0 && src <= f.bgn[blk]) blk--;
    }
    return true;
}

// ---------------------------------------------------------------------
// Propagator tables (make_propg, src/step_mod.f90:109-129)
// ---------------------------------------------------------------------
template <typename T>
struct TableJob {
    const double *omega;  // nr, monomer field of the block
    const double *ksq;    // nk
    T *eo1, *eo2, *ek1, *ek2;
    double ds, b;
};

template <typename T>
__global__ void k_make_tables(const TableJob<T> *jobs, long nr, long nk)
{
    const TableJob<T> J = jobs[blockIdx.y];
    const double lap = J.ds * (J.b * J.b) / 6.0;
    const double pot = J.ds / 2.0;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += stride) {
        double w = J.omega[i];
        J.eo1[i] = (T)exp(-pot * w);
        J.eo2[i] = (T)exp(-(pot / 2.0) * w);
    }
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nk; i += stride) {
        double k = J.ksq[i];
        J.ek1[i] = (T)exp(-lap * k);
        J.ek2[i] = (T)exp(-(lap / 2.0) * k);
    }
}

// Fill slice 0 (forward) or slice ns (backward) with 1 (src/scf_mod.fp.f90:330, 345).
template <typename T>
__global__ void k_init_ends(const SweepField<T> *fields, long nr)
{
    const SweepField<T> &f = fields[blockIdx.y];
    T *s = f.slab + (f.dir > 0 ? 0 : (long)f.ns * nr);
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += (long)gridDim.x * blockDim.x) s[i] = (T)1;
}

template <typename T>
__device__ __forceinline__ void mul_spec(cx<T> *S, const T *ek, const PlaneGeom &g, int plane_off)
{
    for (int i = threadIdx.x; i < g.n1h * g.n2; i += blockDim.x) {
        int y = i / g.n1h, x = i - y * g.n1h;
        T e = ek[plane_off + i];
        cx<T> v = S[y * g.LS + x];
        S[y * g.LS + x] = mk<T>(e * v.x, e * v.y);
    }
}

// ---------------------------------------------------------------------
// dim <= 2: one CTA owns a whole grid and runs steps [t0, t1) of its
// sweep in shared memory.  grid.x = field.
// smem: q[nr], q1[nr] (T) + A, B [n2*LS] (cx<T>)
// ---------------------------------------------------------------------
template <typename T>
__global__ void k_sweep_plane(const SweepField<T> *fields, PlaneGeom g, int t0, int t1)
{
    const SweepField<T> &f = fields[blockIdx.x];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nr = g.n1 * g.n2;
    cx<T> *A = (cx<T> *)smem_raw;
    cx<T> *B = A + g.n2 * g.LS;
    T *q = (T *)(B + g.n2 * g.LS);
    T *q1 = q + nr;
    const T rn = (T)nr;

    int blk, src, dst;
    if (!step_slices(f, t0, blk, src, dst)) return;
    {
        const T *qs = src_slice(f, src, nr);
        for (int i = threadIdx.x; i < nr; i += blockDim.x) q[i] = qs[i];
    }
    __syncthreads();

    for (int t = t0; t < t1; t++) {
        if (!step_slices(f, t, blk, src, dst)) break;
        const T *eo1 = f.eo1[blk], *eo2 = f.eo2[blk], *ek1 = f.ek1[blk], *ek2 = f.ek2[blk];
        // full step
        pack_rows<T>(A, g, [&](int r) { return eo1[r] * q[r]; });
        cx<T> *F = plane_forward<T>(A, B, g);
        mul_spec<T>(F, ek1, g, 0);
        cx<T> *Z = plane_inverse<T>(F, F == A ? B : A, g);
        for (int i = threadIdx.x; i < nr; i += blockDim.x) {
            const T v = eo1[i] * unpack_real<T>(Z, g, i) / rn;
            q1[i] = v;
            if (f.q1) f.q1[i] = v;
        }
        __syncthreads();
        // two half steps
        pack_rows<T>(A, g, [&](int r) { return eo2[r] * q[r]; });
        F = plane_forward<T>(A, B, g);
        mul_spec<T>(F, ek2, g, 0);
        Z = plane_inverse<T>(F, F == A ? B : A, g);
        cx<T> *O = (Z == A) ? B : A;
        if (f.h_out)
            for (int i = threadIdx.x; i < nr; i += blockDim.x) f.h_out[i] = eo1[i] * unpack_real<T>(Z, g, i) / rn;
        pack_rows<T>(O, g, [&](int r) { return eo1[r] * unpack_real<T>(Z, g, r) / rn; });
        F = plane_forward<T>(O, Z, g);
        mul_spec<T>(F, ek2, g, 0);
        Z = plane_inverse<T>(F, F == A ? B : A, g);
        T *out = dst_slice(f, dst, nr);
        for (int i = threadIdx.x; i < nr; i += blockDim.x) {
            T q2 = eo2[i] * unpack_real<T>(Z, g, i) / rn;
            T v = ((T)4 * q2 - q1[i]) / (T)3;
            q[i] = v;
            out[i] = v;
            if (f.q2_out) f.q2_out[i] = q2;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------
// dim 3: multi-pass step.  Spectral scratch layout [z][y][kx] (compact,
// row length n1h).  grid = (n3, nfields) for xy kernels.
// smem for xy kernels: A, B [n2*LS] cx<T>
// ---------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void store_plane(cx<T> *dstg, const cx<T> *S, const PlaneGeom &g)
{
    for (int i = threadIdx.x; i < g.n1h * g.n2; i += blockDim.x) {
        int y = i / g.n1h, x = i - y * g.n1h;
        dstg[i] = S[y * g.LS + x];
    }
}
template <typename T>
__device__ __forceinline__ void load_plane(cx<T> *S, const cx<T> *srcg, const PlaneGeom &g)
{
    for (int i = threadIdx.x; i < g.n1h * g.n2; i += blockDim.x) {
        int y = i / g.n1h, x = i - y * g.n1h;
        S[y * g.LS + x] = srcg[i];
    }
}

// K1: S1 = Fxy[eo1 q], S2 = Fxy[eo2 q]
template <typename T>
__global__ void k3_fwd_pair(const SweepField<T> *fields, PlaneGeom g, int t)
{
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *A = (cx<T> *)smem_raw;
    cx<T> *B = A + g.n2 * g.LS;
    const int z = blockIdx.x;
    const long np = (long)g.n1 * g.n2, nkp = (long)g.n1h * g.n2;
    const long nr = np * g.n3;
    const T *q = src_slice(f, src, nr) + z * np;
    const T *eo1 = f.eo1[blk] + z * np, *eo2 = f.eo2[blk] + z * np;
    pack_rows<T>(A, g, [&](int r) { return eo1[r] * q[r]; });
    cx<T> *F = plane_forward<T>(A, B, g);
    store_plane<T>(f.S1 + z * nkp, F, g);
    __syncthreads();
    pack_rows<T>(A, g, [&](int r) { return eo2[r] * q[r]; });
    F = plane_forward<T>(A, B, g);
    store_plane<T>(f.S2 + z * nkp, F, g);
}

// K2/K4: along z for a tile of TC columns: S <- F_z^-1[ek . F_z[S]]
// which = 1: S1 with ek1; 2: S2 with ek2; 3: both (grid.z selects)
template <typename T, int TC>
__global__ void k3_zconv(const SweepField<T> *fields, PlaneGeom g, int t, int which)
{
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    int sel = which == 3 ? (int)blockIdx.z + 1 : which;
    cx<T> *S = (sel == 1) ? f.S1 : f.S2;
    const T *ek = (sel == 1) ? f.ek1[blk] : f.ek2[blk];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *A = (cx<T> *)smem_raw;
    cx<T> *B = A + g.n3 * TC;
    const long P = (long)g.n1h * g.n2;   // plane size (columns)
    const long c0 = (long)blockIdx.x * TC;
    const int nc = (int)min((long)TC, P - c0);
    for (int i = threadIdx.x; i < g.n3 * TC; i += blockDim.x) {
        int z = i / TC, c = i - z * TC;
        A[i] = (c < nc) ? S[z * P + c0 + c] : mk<T>((T)0, (T)0);
    }
    cx<T> *F = fft_lines<-1, T>(A, B, g.zp, TC, TC, 1, true);
    for (int i = threadIdx.x; i < g.n3 * TC; i += blockDim.x) {
        int z = i / TC, c = i - z * TC;
        if (c < nc) {
            T e = ek[z * P + c0 + c];
            F[i] = mk<T>(e * F[i].x, e * F[i].y);
        }
    }
    cx<T> *Z = fft_lines<1, T>(F, F == A ? B : A, g.zp, TC, TC, 1, true);
    for (int i = threadIdx.x; i < g.n3 * TC; i += blockDim.x) {
        int z = i / TC, c = i - z * TC;
        if (c < nc) S[z * P + c0 + c] = Z[i];
    }
}

// K3: q1 = eo1 Fxy^-1[S1]/N ; S2 <- Fxy[eo1 Fxy^-1[S2]/N]
template <typename T>
__global__ void k3_inv_mid(const SweepField<T> *fields, PlaneGeom g, int t)
{
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *A = (cx<T> *)smem_raw;
    cx<T> *B = A + g.n2 * g.LS;
    const int z = blockIdx.x;
    const long np = (long)g.n1 * g.n2, nkp = (long)g.n1h * g.n2;
    const T rn = (T)(np * g.n3);
    const T *eo1 = f.eo1[blk] + z * np;
    T *q1 = f.q1 + z * np;
    load_plane<T>(A, f.S1 + z * nkp, g);
    cx<T> *Z = plane_inverse<T>(A, B, g);
    for (int i = threadIdx.x; i < (int)np; i += blockDim.x) q1[i] = eo1[i] * unpack_real<T>(Z, g, i) / rn;
    __syncthreads();
    load_plane<T>(A, f.S2 + z * nkp, g);
    Z = plane_inverse<T>(A, B, g);
    cx<T> *O = (Z == A) ? B : A;
    if (f.h_out)
        for (int i = threadIdx.x; i < (int)np; i += blockDim.x) f.h_out[z * np + i] = eo1[i] * unpack_real<T>(Z, g, i) / rn;
    pack_rows<T>(O, g, [&](int r) { return eo1[r] * unpack_real<T>(Z, g, r) / rn; });
    cx<T> *F = plane_forward<T>(O, Z, g);
    store_plane<T>(f.S2 + z * nkp, F, g);
}

// K5: q_out = (4 eo2 Fxy^-1[S2]/N - q1)/3
template <typename T>
__global__ void k3_inv_final(const SweepField<T> *fields, PlaneGeom g, int t)
{
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *A = (cx<T> *)smem_raw;
    cx<T> *B = A + g.n2 * g.LS;
    const int z = blockIdx.x;
    const long np = (long)g.n1 * g.n2, nkp = (long)g.n1h * g.n2;
    const long nr = np * g.n3;
    const T rn = (T)nr;
    const T *eo2 = f.eo2[blk] + z * np;
    const T *q1 = f.q1 + z * np;
    T *out = dst_slice(f, dst, nr) + z * np;
    load_plane<T>(A, f.S2 + z * nkp, g);
    cx<T> *Z = plane_inverse<T>(A, B, g);
    for (int i = threadIdx.x; i < (int)np; i += blockDim.x) {
        T q2 = eo2[i] * unpack_real<T>(Z, g, i) / rn;
        out[i] = ((T)4 * q2 - q1[i]) / (T)3;
        if (f.q2_out) f.q2_out[z * np + i] = q2;
    }
}

// ---------------------------------------------------------------------
// Contour integrals (src/scf_mod.fp.f90:358-426)
// ---------------------------------------------------------------------

// Deterministic block-wide sum in double (fixed tree order).
__device__ __forceinline__ double block_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        for (int i = 0; i < nw; i++) s += red[i];
    }
    return s;  // valid in thread 0
}

// Partial sums of an array (per job, per CTA) -> part[job*gridDim.x + cta].
template <typename T>
__global__ void k_partial_sum(const T *const *ptrs, long n, double *part)
{
    __shared__ double red[32];
    const T *p = ptrs[blockIdx.y];
    double s = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) s += (double)p[i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) part[(long)blockIdx.y * gridDim.x + blockIdx.x] = s;
}

// Fixed-order final reduction of npart partials per job: out[j] = sum/div.
static __global__ void k_final_sum(const double *part, int npart, double div, double *out, int njobs)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    double s = 0.0;
    for (int i = 0; i < npart; i++) s += part[(long)j * npart + i];
    out[j] = s / div;
}

// Same, writing job j's result to *outs[j].
static __global__ void k_final_sum_ptr(const double *part, int npart, double div, double *const *outs, int njobs)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    double s = 0.0;
    for (int i = 0; i < npart; i++) s += part[(long)j * npart + i];
    *outs[j] = s / div;
}

// Simpson contour integral for one (instance, chain): rho of each block,
// accumulated into the monomer density with weight phi/(L Q).
struct SimpsonJob {
    const void *qf, *qr;        // slabs
    double *rho;                // instance density base [M][nr]
    const double *Q;            // device scalar
    double phi, length;
    int nblk;
    int bgn[PSCFG_MAXB + 1];
    int mon[PSCFG_MAXB];
    double bds[PSCFG_MAXB];
    int accumulate;             // 1: add to the existing rho (solvent terms already there)
    int n_monomer;
    int grand;                  // 1: phi = Q exp(mu) from the device Q (grand ensemble)
    double mu;
};

// Simpson contributions of the slices [s0, s1) of one chain, held in
// segment buffers (slice s at qf + (s - s0) nr), added to rho:
// rho_a += scale sum_s w[s][a] qf_s qr_s with w the per-slice Simpson
// weights (ds/3 x 1, 4, 2 of each block containing the slice) and
// scale = phi / (L Q).  Jobs grouped per instance (grid.y), as k_simpson.
struct SimpsonSegJob {
    const void *qf, *qr;
    const double *w;        // [ns + 1][PSCFG_MAXM]
    const double *Q;
    double phi_over_L;
    int s0, s1;
    int n_monomer;
    double *rho;
};

template <typename T>
__global__ void k_simpson_seg(const SimpsonSegJob *jobs, const int *job_start, long nr)
{
    const int inst = blockIdx.y;
    const int j0 = job_start[inst], j1 = job_start[inst + 1];
    if (j1 <= j0) return;
    const int M = jobs[j0].n_monomer;
    double *rho = jobs[j0].rho;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += (long)gridDim.x * blockDim.x) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int a = 0; a < M; a++) acc[a] = rho[(long)a * nr + r];
        for (int jb = j0; jb < j1; jb++) {
            const SimpsonSegJob &J = jobs[jb];
            const T *qf = (const T *)J.qf, *qr = (const T *)J.qr;
            const double scale = J.phi_over_L / *J.Q;
            for (int s = J.s0; s < J.s1; s++) {
                const double p = (double)qf[(long)(s - J.s0) * nr + r] * (double)qr[(long)(s - J.s0) * nr + r] * scale;
                for (int a = 0; a < M; a++) acc[a] += J.w[s * PSCFG_MAXM + a] * p;
            }
        }
        for (int a = 0; a < M; a++) rho[(long)a * nr + r] = acc[a];
    }
}

// Jobs of one instance must run in order (they accumulate into one rho);
// jobs are grouped per instance in grid.y = instance, looping over its chains.
template <typename T>
__global__ void k_simpson(const SimpsonJob *jobs, const int *job_start, long nr)
{
    const int inst = blockIdx.y;
    const int j0 = job_start[inst], j1 = job_start[inst + 1];
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += (long)gridDim.x * blockDim.x) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        if (j1 > j0 && jobs[j0].accumulate)
            for (int a = 0; a < jobs[j0].n_monomer; a++) acc[a] = jobs[j0].rho[(long)a * nr + r];
        for (int jb = j0; jb < j1; jb++) {
            const SimpsonJob &J = jobs[jb];
            const T *qf = (const T *)J.qf, *qr = (const T *)J.qr;
            const double Q = *J.Q;
            const double phi = J.grand ? Q * exp(J.mu) : J.phi;
            for (int b = 0; b < J.nblk; b++) {
                const int ib = J.bgn[b], ie = J.bgn[b + 1];
                double s = (double)qf[(long)ib * nr + r] * (double)qr[(long)ib * nr + r];
                s = s + (double)qf[(long)ie * nr + r] * (double)qr[(long)ie * nr + r];
                for (int j = ib + 1; j <= ie - 1; j += 2)
                    s = s + (double)qf[(long)j * nr + r] * (double)qr[(long)j * nr + r] * 4.0;
                for (int j = ib + 2; j <= ie - 2; j += 2)
                    s = s + (double)qf[(long)j * nr + r] * (double)qr[(long)j * nr + r] * 2.0;
                s = s * J.bds[b] / 3.0;
                s = s / J.length / Q;
                acc[J.mon[b]] = acc[J.mon[b]] + phi * s;
            }
        }
        if (j1 > j0) {
            const SimpsonJob &J0 = jobs[j0];
            for (int a = 0; a < J0.n_monomer; a++) J0.rho[(long)a * nr + r] = acc[a];
        }
    }
}

}  // namespace pscfg
