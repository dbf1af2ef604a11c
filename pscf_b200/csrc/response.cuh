// response.cuh -- complex (Bloch) propagation for the linear response of a
// periodic state (src/response_mod.f90:389-468, 864-1186;
// src/response_step_mod.f90:114-219).
//
// A perturbation exp(ik.r) dw(r) of one monomer's field makes the
// propagators exp(ik.r) dq(r,s) with dq complex and periodic.  Its step
// fftc_step(x) = E IFFT[K FFT[E x]] (E = exp(-w ds_l/2), K =
// exp(-|G+k|^2 ds_l b^2/6) on the full grid) has no G -> -G symmetry, so
// the transforms are complex-to-complex over the whole grid.  One transform
// is a sequence of line passes, one per grid axis: every pass loads TL
// lines of one job into shared memory, transforms them (Stockham, the same
// codelets as the real path) and writes them back in place.  The first pass
// builds its input on the fly, the pass of the last axis applies K between
// the forward and the inverse transform, and the final pass applies E.
#pragma once
#include "fft_dev.cuh"

namespace pscfg {

// input x = ca A + cb B + cw W (qa + qb)/2, then times E (first pass)
struct CJob {
    const cx<double> *A, *B, *W;
    const double *qa, *qb;
    double ca, cb, cw;
    const double *E;     // [nr] or null
    const double *K;     // [nr] full grid or null
    cx<double> *out;     // [nr] work buffer and result
};

struct CPass {
    int axis;            // 0: x, 1: y, 2: z
    int L;               // line length n[axis]
    int nl;              // number of lines nr / L
    int TL;              // lines per CTA
    int first, fwd, kmul, inv, last;
    LinePlan plan;
};

__device__ __forceinline__ long cline_base(int axis, long l, int n1, int n2)
{
    if (axis == 0) return l * n1;
    if (axis == 1) return (l % n1) + (l / n1) * (long)n1 * n2;
    return l;
}

__device__ __forceinline__ long cline_stride(int axis, int n1, int n2)
{
    return axis == 0 ? 1 : (axis == 1 ? n1 : (long)n1 * n2);
}

// grid = (ceil(nl / TL), njobs); dynamic smem 2 * TL * L complex
static __global__ void __launch_bounds__(128) k_cline(const CJob *jobs, CPass P, int n1, int n2, double inv_n)
{
    const CJob &J = jobs[blockIdx.y];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<double> *a = (cx<double> *)smem_raw;
    cx<double> *b = a + (long)P.TL * P.L;
    const long l0 = (long)blockIdx.x * P.TL;
    const int nl = (int)min((long)P.TL, (long)P.nl - l0);
    const long es = cline_stride(P.axis, n1, n2);
    // shared layout: x lines line-major (contiguous rows), y/z lines
    // element-major (consecutive threads take consecutive lines = x)
    const bool lm = P.axis == 0;
    const int ses = lm ? 1 : P.TL, sls = lm ? P.L : 1;
    const int tot = nl * P.L;
    for (int i = threadIdx.x; i < tot; i += blockDim.x) {
        const int li = lm ? i / P.L : i % nl, e = lm ? i % P.L : i / nl;
        const long r = cline_base(P.axis, l0 + li, n1, n2) + e * es;
        cx<double> v;
        if (P.first) {
            v = mk<double>(0.0, 0.0);
            if (J.A) v = v + scale(J.A[r], J.ca);
            if (J.B) v = v + scale(J.B[r], J.cb);
            if (J.W) {
                const double qs = ((J.qa ? J.qa[r] : 0.0) + (J.qb ? J.qb[r] : 0.0)) / 2.0;
                v = v + scale(J.W[r], J.cw * qs);
            }
            if (J.E) v = scale(v, J.E[r]);
        } else {
            v = J.out[r];
        }
        a[li * sls + e * ses] = v;
    }
    cx<double> *res = a;
    if (P.fwd) res = fft_lines<-1, double>(a, b, P.plan, nl, ses, sls, !lm);
    if (P.kmul) {
        for (int i = threadIdx.x; i < tot; i += blockDim.x) {
            const int li = lm ? i / P.L : i % nl, e = lm ? i % P.L : i / nl;
            const long r = cline_base(P.axis, l0 + li, n1, n2) + e * es;
            const double f = (J.K ? J.K[r] : 1.0) * inv_n;
            cx<double> &z = res[li * sls + e * ses];
            z = scale(z, f);
        }
    }
    if (P.inv) res = fft_lines<1, double>(res, res == a ? b : a, P.plan, nl, ses, sls, !lm);
    __syncthreads();
    for (int i = threadIdx.x; i < tot; i += blockDim.x) {
        const int li = lm ? i / P.L : i % nl, e = lm ? i % P.L : i / nl;
        const long r = cline_base(P.axis, l0 + li, n1, n2) + e * es;
        cx<double> v = res[li * sls + e * ses];
        if (P.last && J.E) v = scale(v, J.E[r]);
        J.out[r] = v;
    }
}

// One segment of a perturbed propagator (ps_propagate at orders 0 and 1,
// then (4 d1 - d0)/3), and its Simpson term of the density response:
//   d0 = A1 - ds A2,  d1 = B - (ds/2) A5   (A2, A5 null: no source)
//   dq <- (4 d1 - d0)/3;   acc_m += coef_m * other * dq.
struct CCombine {
    cx<double> *dq;
    const cx<double> *A1, *A2, *A5, *B;
    double ds;
    const double *other;          // the unperturbed propagator of the other direction at the new node
    cx<double> *acc;              // [M][nr]
    double coef[PSCFG_MAXM];
    int M;
};

static __global__ void k_resp_combine(const CCombine *jobs, long nr)
{
    const CCombine &J = jobs[blockIdx.y];
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += (long)gridDim.x * blockDim.x) {
        cx<double> d0 = J.A1[r], d1 = J.B[r];
        if (J.A2) d0 = d0 - scale(J.A2[r], J.ds);
        if (J.A5) d1 = d1 - scale(J.A5[r], J.ds / 2.0);
        const cx<double> q = mk<double>((4.0 * d1.x - d0.x) / 3.0, (4.0 * d1.y - d0.y) / 3.0);
        J.dq[r] = q;
        const double o = J.other[r];
        for (int m = 0; m < J.M; m++)
            if (J.coef[m] != 0.0) {
                cx<double> &a = J.acc[(long)m * nr + r];
                a = a + scale(q, J.coef[m] * o);
            }
    }
}

// dst[i] (+)= sum of the listed complex arrays (fixed order)
struct CSum {
    cx<double> *dst;
    const cx<double> *src[2 * PSCFG_MAXC];
    int n;
};

static __global__ void k_csum(const CSum *jobs, long len)
{
    const CSum &J = jobs[blockIdx.y];
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long)gridDim.x * blockDim.x) {
        cx<double> v = mk<double>(0.0, 0.0);
        for (int k = 0; k < J.n; k++) v = v + J.src[k][i];
        J.dst[i] = v;
    }
}

// out[k] = Re(spec[idx[k]] / coef[k]) (kgrid_to_basis with no_parity)
struct CRead {
    const cx<double> *spec;
    double *out;
};

static __global__ void k_resp_readout(const CRead *jobs, const int *idx, const double *coef, int nread)
{
    const CRead &J = jobs[blockIdx.y];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nread; k += gridDim.x * blockDim.x) {
        const cx<double> z = J.spec[idx[k]];
        const double cr = coef[2 * k], ci = coef[2 * k + 1];
        const double den = cr * cr + ci * ci;
        J.out[k] = (z.x * cr + z.y * ci) / den;
    }
}

// midpoint of the half-step chain: h / exp(-w ds/4) (the step kernels
// store h = exp(-w ds/2) C2 exp(-w ds/4) q)
struct CDiv {
    double *x;
    const double *d;
};

static __global__ void k_resp_div(const CDiv *jobs, long nr)
{
    const CDiv &J = jobs[blockIdx.y];
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += (long)gridDim.x * blockDim.x)
        J.x[r] = J.x[r] / J.d[r];
}

// exp tables of the perturbed step: E = exp(-w ds_l/2), K = exp(-ksq ds_l b^2/6)
struct CTab {
    const double *w;      // omega of the block's monomer
    const double *ksq;    // |G+k|^2 full grid
    double *E, *K;
    double ds, b2;
};

static __global__ void k_resp_tables(const CTab *jobs, long nr)
{
    const CTab &J = jobs[blockIdx.y];
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += (long)gridDim.x * blockDim.x) {
        J.E[r] = exp(-J.w[r] * J.ds / 2.0);
        J.K[r] = exp(-J.ksq[r] * J.ds * J.b2 / 6.0);
    }
}

}  // namespace pscfg
