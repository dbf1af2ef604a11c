// adjoint.cuh -- reverse-mode derivative of density() with respect to omega.
//
// For a scalar L(rho, lnQ) with upstream gradients G_m(r) = dL/drho_m(r)
// and gQ_c = dL/dlnQ_c, the derivative dL/domega_m(r) of the discrete
// reference algorithm (step_exp src/step_mod.f90:146-176, Simpson
// src/scf_mod.fp.f90:364-426, bigQ :359) is obtained by two adjoint sweeps
// per chain that reuse the forward step kernels: the step operator
// P = (4 P2 - P1)/3 with P1 = E1 C1 E1, P2 = E2 C2 E1 C2 E2 (E diagonal
// Boltzmann factors, C real even k-space filters) is symmetric, so
//   lambda_j = P lambda_{j+1} + direct_j        (adjoint of the qf chain)
//   lambda_s = P lambda_{s-1} + direct_s        (adjoint of the qr chain)
// and the omega derivative of one step lambda . P(omega) q is pointwise:
//   D1 = -(ds/2) [lambda P1 q + q P1 lambda]
//   D2 = -(ds/4) [lambda P2 q + q P2 lambda] - (ds/2) h_lambda h_q / eo1
//   D  = (4 D2 - D1) / 3,        h_x = E1 C2 E2 x.
#pragma once
#include "kernels.cuh"

namespace pscfg {

struct AdjPoint {
    // step intermediates of the adjoint state (lam) and of the stored slice (q)
    const void *lam, *p1l, *hl, *p2l;
    const void *q, *p1q, *hq, *p2q;
    const void *eo1;            // block table exp(-w ds/2)
    double ds;
    double *grad;               // dL/domega of the block's monomer (accumulated)
    void *lam_new;              // output: P lam + direct
    // direct term sum_m coef[m] G_m(r) * other(r) at the new slice
    const double *G;            // [M][nr] upstream dL/drho
    const void *other;          // the other chain's slice at the new index
    double coef[PSCFG_MAXM];
    int M;
};

template <typename T>
__global__ void k_adj_point(const AdjPoint *jobs, long nr)
{
    const AdjPoint &J = jobs[blockIdx.y];
    const T *lam = (const T *)J.lam, *p1l = (const T *)J.p1l, *hl = (const T *)J.hl, *p2l = (const T *)J.p2l;
    const T *q = (const T *)J.q, *p1q = (const T *)J.p1q, *hq = (const T *)J.hq, *p2q = (const T *)J.p2q;
    const T *eo1 = (const T *)J.eo1, *other = (const T *)J.other;
    T *ln = (T *)J.lam_new;
    const double ds = J.ds;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += (long)gridDim.x * blockDim.x) {
        const double l = lam[r], x = q[r];
        const double d1 = -(ds / 2.0) * (l * (double)p1q[r] + x * (double)p1l[r]);
        const double d2 = -(ds / 4.0) * (l * (double)p2q[r] + x * (double)p2l[r]) -
                          (ds / 2.0) * (double)hl[r] * (double)hq[r] / (double)eo1[r];
        J.grad[r] += (4.0 * d2 - d1) / 3.0;
        double dir = 0.0;
        for (int m = 0; m < J.M; m++) dir += J.coef[m] * J.G[(long)m * nr + r];
        ln[r] = (T)((4.0 * (double)p2l[r] - (double)p1l[r]) / 3.0 + dir * (double)other[r]);
    }
}

// lambda at the first adjoint slice: direct term plus the constant from the
// Q dependence (added to the qf-chain adjoint only).
struct AdjInit {
    void *lam;
    const double *G;
    const void *other;
    double coef[PSCFG_MAXM];
    double cst;
    int M;
};

template <typename T>
__global__ void k_adj_init(const AdjInit *jobs, long nr)
{
    const AdjInit &J = jobs[blockIdx.y];
    T *lam = (T *)J.lam;
    const T *other = (const T *)J.other;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += (long)gridDim.x * blockDim.x) {
        double dir = 0.0;
        for (int m = 0; m < J.M; m++) dir += J.coef[m] * J.G[(long)m * nr + r];
        lam[r] = (T)(dir * (double)other[r] + J.cst);
    }
}

// Overlap S_c = sum_r sum_m G_m(r) rho^(c)_m(r) of one chain's density
// contribution with the upstream gradient: sum over slices of
// coef_j . G(r) qf_j qr_j.  Partials per (job, CTA).
struct AdjOverlap {
    const void *qf, *qr;
    const double *G;
    const double *coef;         // [nslices][PSCFG_MAXM] device
    int nslices;
    int M;
};

template <typename T>
__global__ void k_adj_overlap(const AdjOverlap *jobs, long nr, double *part)
{
    __shared__ double red[32];
    const AdjOverlap &J = jobs[blockIdx.y];
    const T *qf = (const T *)J.qf, *qr = (const T *)J.qr;
    double acc = 0.0;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += (long)gridDim.x * blockDim.x) {
        double g[PSCFG_MAXM];
        for (int m = 0; m < J.M; m++) g[m] = J.G[(long)m * nr + r];
        for (int j = 0; j < J.nslices; j++) {
            double c = 0.0;
            for (int m = 0; m < J.M; m++) c += J.coef[j * PSCFG_MAXM + m] * g[m];
            acc += c * (double)qf[(long)j * nr + r] * (double)qr[(long)j * nr + r];
        }
    }
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) part[(long)blockIdx.y * gridDim.x + blockIdx.x] = acc;
}

// Real-field pairs whose weighted spectral products give the cell
// derivative of one adjoint step <lambda, P(cell) q>: with the symmetric
// k-space filters C1 = C(ds), C2 = C(ds/2) and E1 = exp(-w ds/2),
// E2 = exp(-w ds/4), h_x = E1 C2 E2 x,
//   d<lambda, P1 q> = <E1 lambda, dC1 (E1 q)>,  C1 E1 q = P1 q / E1
//   d<lambda, P2 q> = <E2 lambda, dC2 h_q> + <h_lambda, dC2 E2 q>,
//                     C2 h_q = P2 q / E2,  C2 E2 q = h_q / E1
// so the pairs (a, b) = (E1 lam, P1q/E1), (E2 lam, P2q/E2), (h_lam, h_q/E1)
// carry the k-space filter in b.
struct AdjCellPair {
    const double *lam, *hl, *p1q, *hq, *p2q;
    const double *eo1, *eo2;
    double *a, *b;        // [3][nr] each
};

static __global__ void k_adj_cellpairs(const AdjCellPair *jobs, long nr)
{
    const AdjCellPair &J = jobs[blockIdx.y];
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += (long)gridDim.x * blockDim.x) {
        const double e1 = J.eo1[r], e2 = J.eo2[r], l = J.lam[r];
        J.a[r] = e1 * l;
        J.b[r] = J.p1q[r] / e1;
        J.a[nr + r] = e2 * l;
        J.b[nr + r] = J.p2q[r] / e2;
        J.a[2 * nr + r] = J.hl[r];
        J.b[2 * nr + r] = J.hq[r] / e1;
    }
}

// g[b] += sum over jobs and pairs of coef[pair] * inc[pair][b], fixed order
struct AdjCellAcc {
    const double *inc;    // [3][PSCFG_MAXCP]
    double coef[3];
    double *g;            // [PSCFG_MAXCP]
    int ncp;
};

static __global__ void k_adj_cellacc(const AdjCellAcc *jobs, int n)
{
    const int b = threadIdx.x;
    for (int k = 0; k < n; k++) {
        const AdjCellAcc &J = jobs[k];
        if (b < J.ncp)
            for (int p = 0; p < 3; p++) J.g[b] += J.coef[p] * J.inc[p * PSCFG_MAXCP + b];
    }
}

}  // namespace pscfg
