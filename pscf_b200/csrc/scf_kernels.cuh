// scf_kernels.cuh -- stress, solvent, free-energy and Anderson-mixing kernels.
#pragma once
#include "kernels.cuh"

namespace pscfg {

// Batched copies of double arrays, job j = blockIdx.y: the per-instance
// scalars (Q, stress) gathered into one staging block before a single
// device-to-host copy, and the per-instance field copies of an Anderson
// step, as one launch instead of one copy per instance.
struct CopyJob {
    const double *src;
    double *dst;
    long n;
};

static __global__ void k_copy_list(const CopyJob *jobs)
{
    const CopyJob j = jobs[blockIdx.y];
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < j.n; i += (long)gridDim.x * blockDim.x)
        j.dst[i] = j.src[i];
}

// ---------------------------------------------------------------------
// Stress (scf_stress, src/scf_mod.fp.f90:451-550).  Per contour slice i:
//   inc_b(i) = sum_k w(k) dGsq_b(k) Re(qf^_i(k) conj(qr^_i(k)))
// (unnormalised FFTs).  The slice sums are reduced on the device in a
// fixed order; the Simpson weights, b^2 ds / (N^2 3 6) and the mixing
// over chains are applied by k_stress_final.
// ---------------------------------------------------------------------
template <typename T>
struct StressJob {
    const T *qf, *qr;          // slabs of one (instance, chain)
    const double *wdgsq;       // [PSCFG_MAXCP][nk] of the instance
    int ncp;
    int nslices;               // ns + 1
    double *inc;               // [nslices][PSCFG_MAXCP] output (slice sums)
};

// dim <= 2: one CTA per (job, slice); 4 plane buffers in shared memory.
template <typename T>
static __global__ void k2_stress_slices(const StressJob<T> *jobs, PlaneGeom g)
{
    const StressJob<T> &J = jobs[blockIdx.y];
    const int s = blockIdx.x;
    if (s >= J.nslices) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int pb = g.n2 * g.LS;
    cx<T> *A = (cx<T> *)smem_raw, *B = A + pb, *C = B + pb, *D = C + pb;
    __shared__ double red[32];
    const long nr = (long)g.n1 * g.n2;
    const T *qf = J.qf + (long)s * nr, *qr = J.qr + (long)s * nr;
    pack_rows<T>(A, g, [&](int r) { return qf[r]; });
    pack_rows<T>(C, g, [&](int r) { return qr[r]; });
    cx<T> *F = plane_forward<T>(A, B, g);
    cx<T> *R = plane_forward<T>(C, D, g);
    const long nk = (long)g.n1h * g.n2;
    for (int b = 0; b < J.ncp; b++) {
        double acc = 0.0;
        for (int i = threadIdx.x; i < (int)nk; i += blockDim.x) {
            int y = i / g.n1h, x = i - y * g.n1h;
            cx<T> f = F[y * g.LS + x], r = R[y * g.LS + x];
            acc += J.wdgsq[(long)b * nk + i] * ((double)f.x * (double)r.x + (double)f.y * (double)r.y);
        }
        double tot = block_sum(acc, red);
        if (threadIdx.x == 0) J.inc[(long)s * PSCFG_MAXCP + b] = tot;
        __syncthreads();
    }
}

// dim 3, pass 1: xy-forward of slices [s0, s0+cs) of qf and qr into
// spec[(slice-s0)*2 + fr][z][y][kx].  grid = (n3, cs, 2).
template <typename T>
static __global__ void k3_stress_xy(const StressJob<T> *job, PlaneGeom g, int s0, cx<T> *spec)
{
    const StressJob<T> &J = *job;
    const int s = s0 + blockIdx.y;
    if (s >= J.nslices) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *A = (cx<T> *)smem_raw;
    cx<T> *B = A + g.n2 * g.LS;
    const int z = blockIdx.x;
    const long np = (long)g.n1 * g.n2, nkp = (long)g.n1h * g.n2;
    const long nr = np * g.n3, nk = nkp * g.n3;
    const T *q = (blockIdx.z == 0 ? J.qf : J.qr) + (long)s * nr + z * np;
    pack_rows<T>(A, g, [&](int r) { return q[r]; });
    cx<T> *F = plane_forward<T>(A, B, g);
    store_plane<T>(spec + ((long)blockIdx.y * 2 + blockIdx.z) * nk + z * nkp, F, g);
}

// dim 3, pass 2: z-forward of both spectra on a tile of TC columns and the
// weighted dot products.  grid = (ntiles, cs).  Writes
// part[((slice-s0)*ntiles + tile)*PSCFG_MAXCP + b].
template <typename T, int TC>
static __global__ void k3_stress_z(const StressJob<T> *job, PlaneGeom g, int s0, const cx<T> *spec, double *part)
{
    const StressJob<T> &J = *job;
    const int s = s0 + blockIdx.y;
    if (s >= J.nslices) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *A = (cx<T> *)smem_raw, *B = A + g.n3 * TC, *C = B + g.n3 * TC, *D = C + g.n3 * TC;
    __shared__ double red[32];
    const long P = (long)g.n1h * g.n2, nk = P * g.n3;
    const long c0 = (long)blockIdx.x * TC;
    const int nc = (int)min((long)TC, P - c0);
    const cx<T> *sf = spec + ((long)blockIdx.y * 2) * nk, *sr = sf + nk;
    for (int i = threadIdx.x; i < g.n3 * TC; i += blockDim.x) {
        int z = i / TC, c = i - z * TC;
        A[i] = (c < nc) ? sf[z * P + c0 + c] : mk<T>((T)0, (T)0);
        C[i] = (c < nc) ? sr[z * P + c0 + c] : mk<T>((T)0, (T)0);
    }
    cx<T> *F = fft_lines<-1, T>(A, B, g.zp, TC, TC, 1, true);
    cx<T> *R = fft_lines<-1, T>(C, D, g.zp, TC, TC, 1, true);
    for (int b = 0; b < J.ncp; b++) {
        double acc = 0.0;
        for (int i = threadIdx.x; i < g.n3 * TC; i += blockDim.x) {
            int z = i / TC, c = i - z * TC;
            if (c < nc) {
                cx<T> f = F[i], r = R[i];
                acc += J.wdgsq[(long)b * nk + z * P + c0 + c] * ((double)f.x * (double)r.x + (double)f.y * (double)r.y);
            }
        }
        double tot = block_sum(acc, red);
        if (threadIdx.x == 0) part[((long)blockIdx.y * gridDim.x + blockIdx.x) * PSCFG_MAXCP + b] = tot;
        __syncthreads();
    }
}

// dim 3, pass 3: fixed-order sum of tile partials -> inc.  grid = cs.
template <typename T>
static __global__ void k3_stress_sum(const StressJob<T> *job, int s0, int ntiles, const double *part)
{
    const StressJob<T> &J = *job;
    const int s = s0 + blockIdx.x;
    if (s >= J.nslices || threadIdx.x >= J.ncp) return;
    const int b = threadIdx.x;
    double acc = 0.0;
    for (int t = 0; t < ntiles; t++) acc += part[((long)blockIdx.x * ntiles + t) * PSCFG_MAXCP + b];
    J.inc[(long)s * PSCFG_MAXCP + b] = acc;
}

// Assemble the stress of each instance from the slice sums, in the order of
// src/scf_mod.fp.f90:484-546.  One thread per instance.
struct StressFinal {
    int nchain;
    int ncp;
    int ensemble;
    const double *inc[PSCFG_MAXC];
    const double *Q;                   // [PSCFG_MAXC]
    int nblk[PSCFG_MAXC];
    int bgn[PSCFG_MAXC][PSCFG_MAXB + 1];
    double bds[PSCFG_MAXC][PSCFG_MAXB];
    double b[PSCFG_MAXC][PSCFG_MAXB];  // kuhn length of each block's monomer
    double phi[PSCFG_MAXC], mu[PSCFG_MAXC], length[PSCFG_MAXC];
    double rnodes;
    double *out;                        // [PSCFG_MAXCP]
};

static __global__ void k_stress_final(const StressFinal *jobs, int n)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const StressFinal &F = jobs[j];
    const double normal = F.rnodes * F.rnodes * 3.0 * 6.0;
    double stress[PSCFG_MAXCP];
    for (int b = 0; b < F.ncp; b++) stress[b] = 0.0;
    for (int c = 0; c < F.nchain; c++) {
        double dQ[PSCFG_MAXCP];
        for (int b = 0; b < F.ncp; b++) dQ[b] = 0.0;
        for (int blk = 0; blk < F.nblk[c]; blk++) {
            const double bb = F.b[c][blk];
            const double ds0 = F.bds[c][blk];
            const int ib = F.bgn[c][blk], ie = F.bgn[c][blk + 1];
            for (int s = ib; s <= ie; s++) {
                // 1-based slice index i = s+1: interior i even -> 4 ds, odd -> 2 ds
                double ds = ds0;
                if (s != ib && s != ie) ds = (((s + 1) % 2) == 0) ? 4.0 * ds0 : 2.0 * ds0;
                for (int b = 0; b < F.ncp; b++) {
                    double inc = F.inc[c][(long)s * PSCFG_MAXCP + b];
                    inc = inc * (bb * bb) * ds / normal;
                    dQ[b] = dQ[b] - inc;
                }
            }
        }
        const double Q = F.Q[c];
        for (int b = 0; b < F.ncp; b++) {
            if (F.ensemble == 0) stress[b] = stress[b] - (dQ[b] / Q) * F.phi[c] / F.length[c];
            else stress[b] = stress[b] - (dQ[b] / Q) * exp(F.mu[c]) * Q / F.length[c];
        }
    }
    for (int b = 0; b < F.ncp; b++) F.out[b] = stress[b];
}

// ---------------------------------------------------------------------
// Solvents (solvent_density, src/scf_mod.fp.f90:251-295)
// ---------------------------------------------------------------------
struct SolventJob {
    const double *omega;   // monomer field
    double *rho;           // monomer density field (accumulated)
    double size;
    const double *Q;       // device scalar (mean of exp(-v w))
    double phi, mu;
    int grand;
};

static __global__ void k_solvent_boltz_partial(const SolventJob *jobs, long nr, double *part)
{
    __shared__ double red[32];
    const SolventJob &J = jobs[blockIdx.y];
    double s = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += (long)gridDim.x * blockDim.x)
        s += exp((-J.size) * J.omega[i]);
    s = block_sum(s, red);
    if (threadIdx.x == 0) part[(long)blockIdx.y * gridDim.x + blockIdx.x] = s;
}

static __global__ void k_solvent_rho(const SolventJob *jobs, int njobs, long nr)
{
    for (int j = 0; j < njobs; j++) {
        const SolventJob &J = jobs[j];
        const double Q = *J.Q;
        const double phi = J.grand ? Q * exp(J.mu) : J.phi;
        for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += (long)gridDim.x * blockDim.x)
            J.rho[i] = J.rho[i] + phi * exp((-J.size) * J.omega[i]) / Q;
    }
}

static __global__ void k_axpy(double *y, const double *x, long n)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) y[i] += x[i];
}

static __global__ void k_zero(double *p, long n)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) p[i] = 0.0;
}

// ---------------------------------------------------------------------
// Free energy field term (src/scf_mod.fp.f90:861-869) as a grid average:
//   sum_r [ sum_{a<b} rho_a chi_ab rho_b - sum_a omega_a rho_a ]
// grid = (nctas, ninst); partials reduced by k_final_sum.
// ---------------------------------------------------------------------
struct FieldJob {
    const double *omega, *rho;
    double chi[PSCFG_MAXM][PSCFG_MAXM];
    int M;
};

static __global__ void k_fe_partial(const FieldJob *jobs, long nr, double *part)
{
    __shared__ double red[32];
    const FieldJob &J = jobs[blockIdx.y];
    double acc = 0.0;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += (long)gridDim.x * blockDim.x) {
        double t = 0.0;
        for (int a = 0; a < J.M; a++) {
            double ra = J.rho[(long)a * nr + r];
            for (int b = a + 1; b < J.M; b++) t += ra * J.chi[a][b] * J.rho[(long)b * nr + r];
            t -= J.omega[(long)a * nr + r] * ra;
        }
        acc += t;
    }
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) part[(long)blockIdx.y * gridDim.x + blockIdx.x] = acc;
}

// ---------------------------------------------------------------------
// Anderson mixing (src/iterate_mod.fp.f90:1171-1416) on grid fields.
// ---------------------------------------------------------------------
struct AmJob {
    const double *omega, *rho;
    double *dev;                        // current deviation slot [M][nr]
    double chi[PSCFG_MAXM][PSCFG_MAXM];
    int M;
};

// dev_a = sum_b chi_ba rho_b + (sum_b omega_b [+ chi12 rho3 + chi23 rho1 + chi13 rho2])/M - omega_a;
// partial sums of dev_a for the mean (uniform component removal).
static __global__ void k_am_dev(const AmJob *jobs, long nr, double *part)
{
    __shared__ double red[32];
    const AmJob &J = jobs[blockIdx.y];
    double sums[PSCFG_MAXM] = {0.0, 0.0, 0.0, 0.0};
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += (long)gridDim.x * blockDim.x) {
        double rho[PSCFG_MAXM], om[PSCFG_MAXM];
        double sw = 0.0;
        for (int a = 0; a < J.M; a++) {
            rho[a] = J.rho[(long)a * nr + r];
            om[a] = J.omega[(long)a * nr + r];
            sw += om[a];
        }
        if (J.M == 3) sw += J.chi[0][1] * rho[2] + J.chi[1][2] * rho[0] + J.chi[0][2] * rho[1];
        for (int a = 0; a < J.M; a++) {
            double d = 0.0;
            for (int b = 0; b < J.M; b++) d += J.chi[b][a] * rho[b];
            d += sw / J.M - om[a];
            J.dev[(long)a * nr + r] = d;
            sums[a] += d;
        }
    }
    for (int a = 0; a < J.M; a++) {
        double t = block_sum(sums[a], red);
        if (threadIdx.x == 0) part[((long)blockIdx.y * PSCFG_MAXM + a) * gridDim.x + blockIdx.x] = t;
        __syncthreads();
    }
}

// Subtract the mean of each dev_a and return partial max |dev|.
struct AmFix {
    double *dev;
    const double *mean;    // [PSCFG_MAXM] device
    int M;
};

static __global__ void k_am_fix(const AmFix *jobs, long nr, double *part)
{
    __shared__ double red[32];
    const AmFix &J = jobs[blockIdx.y];
    double mx = 0.0;
    for (int a = 0; a < J.M; a++) {
        const double m = J.mean[a];
        double *d = J.dev + (long)a * nr;
        for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += (long)gridDim.x * blockDim.x) {
            double v = d[r] - m;
            d[r] = v;
            mx = fmax(mx, fabs(v));
        }
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int i = 0; i < (int)((blockDim.x + 31) >> 5); i++) m = fmax(m, red[i]);
        part[(long)blockIdx.y * gridDim.x + blockIdx.x] = m;
    }
}

static __global__ void k_final_max(const double *part, int npart, double *out, int njobs)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    double m = 0.0;
    for (int i = 0; i < npart; i++) m = fmax(m, part[(long)j * npart + i]);
    out[j] = m;
}

// Status word of each instance's Anderson iteration, computed on the device
// from the iteration's reductions and read back with its other scalars:
// 0 finite; 1 non-finite (<dev, dev> or max |dev| is NaN or Inf: a NaN or
// Inf in omega, rho or the propagators; max |dev| alone would miss a NaN,
// fmax drops NaN operands); 2 diverged (max |dev| above `large`).
static __global__ void k_am_status(const double *emax, const double *g, int gstride, double large, double *status,
                                   int njobs)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= njobs) return;
    const double e = emax[k], g0 = g[(long)k * gstride];
    status[k] = (!isfinite(e) || !isfinite(g0)) ? 1.0 : (e > large ? 2.0 : 0.0);
}

// Dot products of the current deviation with the stored ones:
// g[h] = <dev_cur, dev_h> (sum over monomers and grid), h < nh.
#define PSCFG_MAXH 32
struct AmDot {
    const double *cur;
    const double *hist[PSCFG_MAXH + 1];
    int nh;
    long len;                           // M * nr
};

static __global__ void k_am_dots(const AmDot *jobs, double *part)
{
    __shared__ double red[32];
    const AmDot &J = jobs[blockIdx.y];
    double acc[PSCFG_MAXH + 1];
#pragma unroll
    for (int h = 0; h <= PSCFG_MAXH; h++) acc[h] = 0.0;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < J.len; r += (long)gridDim.x * blockDim.x) {
        const double c = J.cur[r];
#pragma unroll
        for (int h = 0; h <= PSCFG_MAXH; h++)
            if (h < J.nh) acc[h] += c * J.hist[h][r];
    }
    for (int h = 0; h < J.nh; h++) {
        double t = block_sum(acc[h], red);
        if (threadIdx.x == 0) part[((long)blockIdx.y * (PSCFG_MAXH + 1) + h) * gridDim.x + blockIdx.x] = t;
        __syncthreads();
    }
}

// Mixing: omega <- omega + sum_n C_n (om_n - om_cur) + lam (d_cur + sum_n C_n (d_n - d_cur))
struct AmMix {
    double *omega;
    const double *om_cur, *d_cur;
    const double *om[PSCFG_MAXH];
    const double *d[PSCFG_MAXH];
    double C[PSCFG_MAXH];
    int n;
    double lam;
    long len;
};

static __global__ void k_am_mix(const AmMix *jobs)
{
    const AmMix &J = jobs[blockIdx.y];
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < J.len; r += (long)gridDim.x * blockDim.x) {
        double ww = J.omega[r], dd = J.d_cur[r];
        const double oc = J.om_cur[r], dc = dd;
        for (int k = 0; k < J.n; k++) {
            ww += J.C[k] * (J.om[k][r] - oc);
            dd += J.C[k] * (J.d[k][r] - dc);
        }
        J.omega[r] = ww + J.lam * dd;
    }
}

}  // namespace pscfg

namespace pscfg {

// ---------------------------------------------------------------------
// k^2 and stress weights on the device (make_ksq + G_to_bz,
// src/grid_mod.f90:141-160, 225-283; make_dGsq src/basis_mod.f90:1993-2014).
// One thread per half-grid point; the 3^dim images are tried in the
// reference order (+1, 0, -1 per used dimension) with the 1e-8 tie rule.
// ---------------------------------------------------------------------
struct GeomJob {
    double G[3][3];
    double dGG[PSCFG_MAXCP][3][3];
    int ncp;
    double *ksq;     // [nk]
    double *wdgsq;   // [PSCFG_MAXCP][nk]
    const double *kweight;   // [nk] star weights or nullptr (all 1)
    double *wdg0;            // [PSCFG_MAXCP][nk] w(kx) G^T dGG_b G without star weights, or nullptr
    const int *gate;         // nullptr, or a device flag: the job runs only when it is nonzero
};

__device__ __forceinline__ double gnorm_dev(int dim, const int Gt[3], const double G[3][3])
{
    double v0 = 0, v1 = 0, v2 = 0;
    for (int i = 0; i < dim; i++) {
        v0 += Gt[i] * G[i][0];
        v1 += Gt[i] * G[i][1];
        v2 += Gt[i] * G[i][2];
    }
    double s = v0 * v0;
    if (dim > 1) s += v1 * v1;
    if (dim > 2) s += v2 * v2;
    return s;
}

static __global__ void k_make_geom(const GeomJob *jobs, int dim, int n1, int n2, int n3)
{
    const GeomJob &J = jobs[blockIdx.y];
    if (J.gate && *J.gate == 0) return;
    const int n1h = n1 / 2 + 1;
    const long nk = (long)n1h * n2 * n3;
    const int n[3] = {n1, n2, n3};
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < nk; idx += (long)gridDim.x * blockDim.x) {
        const int i1 = (int)(idx % n1h);
        const int i2 = (int)((idx / n1h) % n2);
        const int i3 = (int)(idx / ((long)n1h * n2));
        const int Gin[3] = {i1, i2, i3};
        int Gmin[3] = {0, 0, 0}, Gt[3] = {0, 0, 0};
        double gmin = 1.0e10;
        const int h0 = 1, h1 = dim > 1 ? 1 : 0, h2 = dim > 2 ? 1 : 0;
        for (int a = h0; a >= -h0; a--) {
            Gt[0] = Gin[0] + a * n[0];
            for (int b = h1; b >= -h1; b--) {
                Gt[1] = dim > 1 ? Gin[1] + b * n[1] : 0;
                for (int c = h2; c >= -h2; c--) {
                    Gt[2] = dim > 2 ? Gin[2] + c * n[2] : 0;
                    double g = gnorm_dev(dim, Gt, J.G);
                    if (g < gmin - 1.0e-8) {
                        Gmin[0] = Gt[0];
                        Gmin[1] = Gt[1];
                        Gmin[2] = Gt[2];
                        gmin = g;
                    }
                }
            }
        }
        J.ksq[idx] = gnorm_dev(dim, Gmin, J.G);
        const double w0 = (i1 == 0 || (n1 % 2 == 0 && i1 == n1 / 2)) ? 1.0 : 2.0;
        const double w = J.kweight ? w0 * J.kweight[idx] : w0;
        for (int b = 0; b < PSCFG_MAXCP; b++) {
            double v = 0;
            if (b < J.ncp)
                for (int j = 0; j < dim; j++)
                    for (int l = 0; l < dim; l++) v += (double)Gmin[j] * (double)Gmin[l] * J.dGG[b][j][l];
            J.wdgsq[(long)b * nk + idx] = w * v;
            if (J.wdg0) J.wdg0[(long)b * nk + idx] = w0 * v;
        }
    }
}

// ---------------------------------------------------------------------
// Space-group projection: dst[a](i) = mean over ops of src[a](M i + t mod n).
// ops: [nops][12] = 9 entries of M (row major) + 3 of t.
// ---------------------------------------------------------------------
struct SymJob {
    double *f;              // [M][nr], projected in place
    const int *perm;        // grid points grouped by orbit
    const int *start;       // orbit o = perm[start[o] .. start[o+1])
    int norb;
    int M;
    const int *gate;        // nullptr, or a device flag: project only when it is nonzero
};

// Space-group projection f <- (1/|G|) sum_g f(g r) as the orbit mean: a
// point's images under the group cover its orbit |G|/|orbit| times each.
// One thread per orbit reads and rewrites all of its points.
static __global__ void k_symmetrize(const SymJob *jobs, long nr)
{
    const SymJob &J = jobs[blockIdx.y];
    if (J.gate && *J.gate == 0) return;
    for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < J.norb; o += gridDim.x * blockDim.x) {
        const int b = J.start[o], e = J.start[o + 1];
        const double inv = 1.0 / (double)(e - b);
        for (int a = 0; a < J.M; a++) {
            double *f = J.f + (long)a * nr;
            double acc = 0.0;
            for (int k = b; k < e; k++) acc += f[J.perm[k]];
            acc *= inv;
            for (int k = b; k < e; k++) f[J.perm[k]] = acc;
        }
    }
}

}  // namespace pscfg

namespace pscfg {

// ---------------------------------------------------------------------
// Forward r2c of FP64 grid fields into compact half spectra [nk]
// (layout [z][y][kx]).  Used by the star-weighted free energy.
// ---------------------------------------------------------------------
static __global__ void k2_fft_fields(const double *const *src, cx<double> *const *dst, PlaneGeom g)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<double> *A = (cx<double> *)smem_raw;
    cx<double> *B = A + g.n2 * g.LS;
    const double *f = src[blockIdx.x];
    pack_rows<double>(A, g, [&](int r) { return f[r]; });
    cx<double> *F = plane_forward<double>(A, B, g);
    store_plane<double>(dst[blockIdx.x], F, g);
}

static __global__ void k3_fft_fields_xy(const double *const *src, cx<double> *const *dst, PlaneGeom g)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<double> *A = (cx<double> *)smem_raw;
    cx<double> *B = A + g.n2 * g.LS;
    const int z = blockIdx.x;
    const long np = (long)g.n1 * g.n2, nkp = (long)g.n1h * g.n2;
    const double *f = src[blockIdx.y] + z * np;
    pack_rows<double>(A, g, [&](int r) { return f[r]; });
    cx<double> *F = plane_forward<double>(A, B, g);
    store_plane<double>(dst[blockIdx.y] + z * nkp, F, g);
}

template <int TC>
static __global__ void k3_fft_fields_z(cx<double> *const *dst, PlaneGeom g)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<double> *A = (cx<double> *)smem_raw;
    cx<double> *B = A + g.n3 * TC;
    cx<double> *S = dst[blockIdx.y];
    const long P = (long)g.n1h * g.n2;
    const long c0 = (long)blockIdx.x * TC;
    const int nc = (int)min((long)TC, P - c0);
    for (int i = threadIdx.x; i < g.n3 * TC; i += blockDim.x) {
        int z = i / TC, c = i - z * TC;
        A[i] = (c < nc) ? S[z * P + c0 + c] : mk<double>(0.0, 0.0);
    }
    cx<double> *F = fft_lines<-1, double>(A, B, g.zp, TC, TC, 1, true);
    for (int i = threadIdx.x; i < g.n3 * TC; i += blockDim.x) {
        int z = i / TC, c = i - z * TC;
        if (c < nc) S[z * P + c0 + c] = F[i];
    }
}

// Star-weighted field term of the free energy (src/scf_mod.fp.f90:861-869
// with the star weights of the reference basis): per instance
//   sum_k w(kx) r(k) [ sum_{a<b} chi_ab Re(R_a R_b*) - sum_a Re(W_a R_a*) ]
struct FeSpecJob {
    const cx<double> *R[PSCFG_MAXM], *W[PSCFG_MAXM];
    const double *kweight;
    double chi[PSCFG_MAXM][PSCFG_MAXM];
    int M;
};

static __global__ void k_fe_spectral(const FeSpecJob *jobs, long nk, int n1, double *part)
{
    __shared__ double red[32];
    const FeSpecJob &J = jobs[blockIdx.y];
    const int n1h = n1 / 2 + 1;
    double acc = 0.0;
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += (long)gridDim.x * blockDim.x) {
        const int i1 = (int)(k % n1h);
        const double w = (i1 == 0 || ((n1 & 1) == 0 && i1 == n1 / 2)) ? 1.0 : 2.0;
        double t = 0.0;
        for (int a = 0; a < J.M; a++) {
            const cx<double> ra = J.R[a][k];
            for (int b = a + 1; b < J.M; b++) {
                const cx<double> rb = J.R[b][k];
                t += J.chi[a][b] * (ra.x * rb.x + ra.y * rb.y);
            }
            const cx<double> wa = J.W[a][k];
            t -= wa.x * ra.x + wa.y * ra.y;
        }
        acc += w * (J.kweight ? J.kweight[k] : 1.0) * t;
    }
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) part[(long)blockIdx.y * gridDim.x + blockIdx.x] = acc;
}

}  // namespace pscfg
