// am_graph.cuh -- Anderson mixing with its per-iteration control on the
// device, so that whole iterations (density, stress, free energy, the
// Anderson sums, the coefficient solve, the mixing, the projection and the
// cell update) replay from one captured CUDA graph with no host round trip.
//
// The control flow is the host iteration's (src/iterate_mod.fp.f90:1042-1490:
// deviation and error, the lambda = 1 - 0.9^k ramp of :1147-1153, U_mn / V_m
// of :1349-1381 solved by Gaussian elimination with partial pivoting, the
// mixing of omega and of the cell parameters), restated per instance in one
// device thread.  An instance that has finished keeps its state: the kernels
// of its density still run until the graph is rebuilt without it, but its
// omega, cell and results no longer change.  The kernels are in am_graph.cu.
#pragma once
#include "host_geom.h"
#include "scf_kernels.cuh"

namespace pscfg {

// Run parameters (pscfg_am_param) for the device control kernels.
struct AmgParam {
    int H;              // history length n_hist
    int max_itr;
    int domain;         // relax the unit cell
    double error_max;
    double mix_max;     // cap on lambda (0: none)
    double restart;     // restart factor (0: never)
    double large;       // divergence bound / 100 (the host loop's 100)
    double nr;          // grid points (Gram normalisation)
};

// State of one instance in a graph-driven run (device memory).
struct AmgInst {
    // constants
    int n_chain, n_solvent, ensemble;
    int ncp;            // cell parameters of the crystal system
    int dim, crystal;
    double length[PSCFG_MAXC], solvent_size[PSCFG_MAXS];
    double *omega, *om_hist, *dev_hist;
    long fl;            // M * nr
    const double *Q, *Qs, *stress_dev;
    // chemistry (mu_phi_chain / mu_phi_solvent, src/scf_mod.fp.f90:768-820):
    // canonical: phi given, mu = ln(phi / Q); grand: mu given, phi = Q exp(mu)
    double phi[PSCFG_MAXC], mu[PSCFG_MAXC], phis[PSCFG_MAXS], mus[PSCFG_MAXS];
    double Qv[PSCFG_MAXC], Qsv[PSCFG_MAXS];   // the last Q, Q_solvent
    // Anderson state (everything up to devcp is read back at each host check)
    int itr, status, done, mixed, k0, nstore, head, pad;
    double error, best_run, f, p, f_new, p_new;
    double stress[PSCFG_MAXCP], cell[PSCFG_MAXCP];
    double devcp[PSCFG_MAXH + 1][PSCFG_MAXCP], cph[PSCFG_MAXH + 1][PSCFG_MAXCP];
    double gram[(PSCFG_MAXH + 1) * (PSCFG_MAXH + 1)];   // ring-indexed <d_i, d_j> / nr
};

// Launches of the control kernels (am_graph.cu, compiled without
// multiply-add contraction so that they round as the host iteration does).
void amg_launch_prep(cudaStream_t st, AmgInst *A, const int *act, int na, int S, AmJob *aj, AmFix *fx, AmDot *dots);
void amg_launch_finish(cudaStream_t st, AmgInst *A, const int *act, int na, const double *terms, const int *tidx);
void amg_launch_update(cudaStream_t st, const AmgParam &P, AmgInst *A, const int *act, int na, const double *emax,
                       const double *gres, const double *word, AmMix *mix, CopyJob *hist_copy, GeomJob *geo);

}  // namespace pscfg
