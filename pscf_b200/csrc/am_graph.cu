// am_graph.cu -- the device control kernels of the graph-driven Anderson
// iteration (am_graph.cuh).  This file is compiled with -fmad=false: the
// Gram updates, the coefficient solve, the mixing of the cell parameters and
// the unit cell then round exactly as the host-driven iteration does, so the
// two give the same iterates.
#include <cuda_runtime.h>

#include "am_graph.cuh"

namespace pscfg {

__device__ __forceinline__ int amg_slot(int head, int back, int S) { return ((head - back) % S + S) % S; }

// Start of an iteration: count it, and point the deviation, mean and Gram
// jobs of act position k at the instance's current ring slot.
static __global__ void k_amg_prep(AmgInst *st, const int *act, int na, int S, AmJob *aj, AmFix *fx, AmDot *dots)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= na) return;
    AmgInst &A = st[act[k]];
    if (!A.done) A.itr++;
    double *dev = A.dev_hist + (long)A.head * A.fl;
    aj[k].dev = dev;
    fx[k].dev = dev;
    AmDot &D = dots[k];
    D.cur = dev;
    D.len = A.fl;
    const int nst = min(A.nstore + 1, S);
    D.nh = nst;
    for (int h = 0; h < nst; h++) D.hist[h] = A.dev_hist + (long)amg_slot(A.head, h, S) * A.fl;
}

// After the density and the free-energy field terms: mu (or phi) from Q,
// then f_Helmholtz and the pressure (src/scf_mod.fp.f90:834-886).
// terms[tidx[k]] is the field term of act position k.
static __global__ void k_amg_finish(AmgInst *st, const int *act, int na, const double *terms, const int *tidx)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= na) return;
    AmgInst &A = st[act[k]];
    for (int c = 0; c < A.n_chain; c++) A.Qv[c] = A.Q[c];
    for (int s = 0; s < A.n_solvent; s++) A.Qsv[s] = A.Qs[s];
    for (int c = 0; c < A.n_chain; c++) {
        if (A.ensemble == 0) A.mu[c] = log(A.phi[c] / A.Q[c]);
        else A.phi[c] = A.Q[c] * exp(A.mu[c]);
    }
    for (int s = 0; s < A.n_solvent; s++) {
        if (A.ensemble == 0) A.mus[s] = log(A.phis[s] / A.Qs[s]);
        else A.phis[s] = A.Qs[s] * exp(A.mus[s]);
    }
    double fe = 0.0;
    for (int c = 0; c < A.n_chain; c++)
        if (A.phi[c] > 1.0e-8) fe = fe + A.phi[c] * (A.mu[c] - 1.0) / A.length[c];
    for (int s = 0; s < A.n_solvent; s++)
        if (A.phis[s] > 1.0e-8) fe = fe + A.phis[s] * (A.mus[s] - 1.0) / A.solvent_size[s];
    fe += terms[tidx[k]];
    double pr = -fe;
    for (int c = 0; c < A.n_chain; c++)
        if (A.phi[c] > 1.0e-8) pr = pr + A.mu[c] * A.phi[c] / A.length[c];
    for (int s = 0; s < A.n_solvent; s++)
        if (A.phis[s] > 1.0e-8) pr = pr + A.mus[s] * A.phis[s] / A.solvent_size[s];
    A.f_new = fe;
    A.p_new = pr;
}

// The Anderson step of act position k, one warp per instance (block k):
// Gram row and cell deviation of the new entry, error and exit status,
// lambda, the coefficient solve, the mixing job, the new cell and its
// geometry job, the history copy.  emax[k]: max |dev|; gres[k][h]:
// <dev_cur, dev_h>; word[k]: the status word of k_am_status.  Each matrix
// entry goes through the same operations in the same order as in the host
// loop's solve_dense (Gaussian elimination with partial pivoting, the first
// of equal pivots); lanes own rows.
static __global__ void __launch_bounds__(32) k_amg_update(AmgParam P, AmgInst *st, const int *act, int na,
                                                          const double *emax, const double *gres,
                                                          const double *word, AmMix *mix, CopyJob *hist_copy,
                                                          GeomJob *geo)
{
    __shared__ double U[PSCFG_MAXH * PSCFG_MAXH], V[PSCFG_MAXH];
    __shared__ int sl[PSCFG_MAXH];
    __shared__ int s_n, s_go;
    __shared__ double s_lam;
    const int k = blockIdx.x, lane = threadIdx.x;
    if (k >= na) return;
    AmgInst &A = st[act[k]];
    const int S = P.H + 1;
    const int ncp = P.domain ? A.ncp : 0;
    if (lane == 0) {
        mix[k].len = 0;
        hist_copy[k].n = 0;
    }
    const bool was_done = A.done != 0;
    __syncwarp();
    if (was_done) {
        if (lane == 0) A.mixed = 0;
        return;
    }
    // Gram row of the new entry (lane h)
    const int nst = min(A.nstore + 1, S);
    const double *g = gres + (long)k * (PSCFG_MAXH + 1);
    if (lane < nst) {
        const int slot = amg_slot(A.head, lane, S);
        A.gram[A.head * S + slot] = g[lane] / P.nr;
        A.gram[slot * S + A.head] = g[lane] / P.nr;
    }
    __syncwarp();
    if (lane == 0) {
        A.mixed = 0;
        A.f = A.f_new;
        A.p = A.p_new;
        for (int b = 0; b < PSCFG_MAXCP; b++) A.stress[b] = P.domain ? A.stress_dev[b] : 0.0;
        for (int b = 0; b < ncp; b++) A.devcp[A.head][b] = -A.stress[b];
        const double e1 = emax[k];
        double e2 = 0.0;
        for (int b = 0; b < ncp; b++) e2 = (e2 < fabs(A.stress[b])) ? fabs(A.stress[b]) : e2;
        A.error = (e1 < e2) ? e2 : e1;
        A.nstore = nst;
        s_go = 0;
        if (word[k] == 1.0 || !isfinite(A.error)) {
            A.error = nan("");
            A.status = PSCFG_AM_NONFINITE;
            A.done = 1;
        } else if (A.error < P.error_max) {
            A.status = PSCFG_AM_CONVERGED;
            A.done = 1;
        } else if (!(A.error <= 100.0 * P.large)) {
            A.status = PSCFG_AM_DIVERGED;
            A.done = 1;
        } else if (A.itr > P.max_itr) {
            A.status = PSCFG_AM_MAXITER;
            A.done = 1;
        } else {
            if (P.restart > 0 && A.itr - A.k0 > 1 && A.error > P.restart * A.best_run) {
                A.k0 = A.itr - 1;
                A.nstore = 1;
                A.best_run = A.error;
            }
            A.best_run = (A.error < A.best_run) ? A.error : A.best_run;
            const int kk = A.itr - A.k0;
            int itr_prev;
            double lam;
            if (kk < P.H + 1) {
                itr_prev = kk - 1;
                lam = am_lambda_ramp(kk);
            } else {
                itr_prev = P.H;
                lam = 1.0;
            }
            itr_prev = min(itr_prev, A.nstore - 1);
            if (P.mix_max > 0) lam = (P.mix_max < lam) ? P.mix_max : lam;
            s_n = itr_prev;
            s_lam = lam;
            s_go = 1;
        }
    }
    __syncwarp();
    if (!s_go) return;
    const int n = s_n, cur = A.head;
    if (lane < n) sl[lane] = amg_slot(cur, 1 + lane, S);
    __syncwarp();
    // U_mn, V_m (src/iterate_mod.fp.f90:1349-1381), lane m
    if (lane < n) {
        const int mm = lane;
        auto G = [&](int a, int b) { return A.gram[a * S + b]; };
        for (int nn = mm; nn < n; nn++) {
            double u = G(cur, cur) - G(cur, sl[nn]) - G(sl[mm], cur) + G(sl[mm], sl[nn]);
            for (int b = 0; b < ncp; b++)
                u += (A.devcp[cur][b] - A.devcp[sl[mm]][b]) * (A.devcp[cur][b] - A.devcp[sl[nn]][b]);
            U[mm * n + nn] = u;
            U[nn * n + mm] = u;
        }
        double v = G(cur, cur) - G(sl[mm], cur);
        for (int b = 0; b < ncp; b++) v += (A.devcp[cur][b] - A.devcp[sl[mm]][b]) * A.devcp[cur][b];
        V[mm] = v;
    }
    __syncwarp();
    // elimination with partial pivoting
    bool singular = false;
    for (int c = 0; c < n && !singular; c++) {
        double a = (lane >= c && lane < n) ? fabs(U[lane * n + c]) : -1.0;
        int p = lane;
        for (int o = 16; o > 0; o >>= 1) {
            const double a2 = __shfl_down_sync(0xffffffffu, a, o);
            const int p2 = __shfl_down_sync(0xffffffffu, p, o);
            if (a2 > a || (a2 == a && p2 < p)) {
                a = a2;
                p = p2;
            }
        }
        p = __shfl_sync(0xffffffffu, p, 0);
        if (U[p * n + c] == 0.0) {
            singular = true;
            break;
        }
        if (p != c) {
            if (lane < n) {
                const double t = U[c * n + lane];
                U[c * n + lane] = U[p * n + lane];
                U[p * n + lane] = t;
            }
            if (lane == 0) {
                const double t = V[c];
                V[c] = V[p];
                V[p] = t;
            }
        }
        __syncwarp();
        if (lane > c && lane < n) {
            const int r = lane;
            const double f = U[r * n + c] / U[c * n + c];
            for (int q = c; q < n; q++) U[r * n + q] -= f * U[c * n + q];
            V[r] -= f * V[c];
        }
        __syncwarp();
    }
    if (lane != 0) return;
    AmMix &m = mix[k];
    if (n > 0) {
        if (singular) {
            A.error = INFINITY;
            A.status = PSCFG_AM_SINGULAR;
            A.done = 1;
            return;
        }
        for (int r = n - 1; r >= 0; r--) {
            double s = V[r];
            for (int q = r + 1; q < n; q++) s -= U[r * n + q] * V[q];
            V[r] = s / U[r * n + r];
        }
    }
    const double lam = s_lam;
    m.omega = A.omega;
    m.om_cur = A.om_hist + (long)cur * A.fl;
    m.d_cur = A.dev_hist + (long)cur * A.fl;
    m.lam = lam;
    m.n = n;
    double cp_new[PSCFG_MAXCP];
    for (int nn = 0; nn < n; nn++) {
        m.C[nn] = V[nn];
        m.om[nn] = A.om_hist + (long)sl[nn] * A.fl;
        m.d[nn] = A.dev_hist + (long)sl[nn] * A.fl;
    }
    for (int b = 0; b < ncp; b++) {
        if (n == 0) {
            cp_new[b] = A.cell[b] + lam * A.devcp[cur][b];
        } else {
            double ww = A.cell[b], dd = A.devcp[cur][b];
            for (int nn = 0; nn < n; nn++) {
                ww += V[nn] * (A.cph[sl[nn]][b] - A.cph[cur][b]);
                dd += V[nn] * (A.devcp[sl[nn]][b] - A.devcp[cur][b]);
            }
            cp_new[b] = ww + lam * dd;
        }
    }
    m.len = A.fl;
    for (int b = 0; b < ncp; b++) A.cell[b] = cp_new[b];
    A.head = (A.head + 1) % S;
    for (int b = 0; b < A.ncp; b++) A.cph[A.head][b] = A.cell[b];
    A.mixed = 1;
    // omega after the projection is recorded in the new ring slot
    hist_copy[k].src = A.omega;
    hist_copy[k].dst = A.om_hist + (long)A.head * A.fl;
    hist_copy[k].n = A.fl;
    if (P.domain) {
        Cell c;
        make_unit_cell(A.dim, A.crystal, A.cell, c);
        GeomJob &J = geo[k];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) J.G[i][j] = c.G[i][j];
        for (int b = 0; b < PSCFG_MAXCP; b++)
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) J.dGG[b][i][j] = c.dGG[b][i][j];
        J.ncp = c.ncp;
    }
}

void amg_launch_prep(cudaStream_t st, AmgInst *A, const int *act, int na, int S, AmJob *aj, AmFix *fx, AmDot *dots)
{
    k_amg_prep<<<(unsigned)((na + 127) / 128), 128, 0, st>>>(A, act, na, S, aj, fx, dots);
}

void amg_launch_finish(cudaStream_t st, AmgInst *A, const int *act, int na, const double *terms, const int *tidx)
{
    k_amg_finish<<<(unsigned)((na + 127) / 128), 128, 0, st>>>(A, act, na, terms, tidx);
}

void amg_launch_update(cudaStream_t st, const AmgParam &P, AmgInst *A, const int *act, int na, const double *emax,
                       const double *gres, const double *word, AmMix *mix, CopyJob *hist_copy, GeomJob *geo)
{
    k_amg_update<<<(unsigned)na, 32, 0, st>>>(P, A, act, na, emax, gres, word, mix, hist_copy, geo);
}

}  // namespace pscfg
