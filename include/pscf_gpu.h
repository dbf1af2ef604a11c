/*
 * pscf_gpu.h -- C ABI of the B200 SCFT propagator engine (libpscfgpu.so).
 *
 * Drop-in boundary for the hot path of the Fortran PSCF solver.  Each entry
 * point names the reference routine it replaces.  The reference keeps its
 * state in module globals and exits with `stop` on errors; here the state
 * lives in an opaque engine handle and every call returns a status code
 * (0 = OK, see PSCFG_E*), with a message from pscfg_last_error().
 *
 * Conventions (kept from the reference so a Fortran host can pass its
 * arrays through ISO_C_BINDING without copies):
 *   - grid fields are x-fastest (Fortran column-major (0:n1-1,0:n2-1,0:n3-1)),
 *     unused dimensions have extent 1 (src/grid_mod.f90:84-93);
 *   - a multi-monomer field is [n_monomer][nr] with nr = n1*n2*n3, i.e. the
 *     Fortran omega_grid(0:,0:,0:,1:N_monomer) (src/grid_mod.f90:43-46);
 *   - monomer indices are 0-based (1-based in Fortran input);
 *   - all values are double precision on the host side.
 *
 * An engine holds a batch of n_inst independent SCFT instances that share
 * one grid shape (dim, n1, n2, n3) and precision; each instance has its own
 * chemistry and unit cell.  Batch calls act on every instance.  Host-side
 * arrays are laid out instance-major ([n_inst][...]).  Calls on one engine
 * are not thread safe; an engine owns one CUDA stream.
 */
#ifndef PSCF_GPU_H
#define PSCF_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define PSCFG_MAXM 4      /* monomer types   */
#define PSCFG_MAXC 4      /* chain species   */
#define PSCFG_MAXB 8      /* blocks per chain */
#define PSCFG_MAXS 4      /* solvent species */
#define PSCFG_MAXCP 6     /* cell parameters */

/* status codes */
#define PSCFG_OK 0
#define PSCFG_EINVAL 1     /* invalid argument */
#define PSCFG_ECUDA 2      /* CUDA runtime error */
#define PSCFG_ENOMEM 3     /* device allocation failed */
#define PSCFG_ESTATE 4     /* call order violated (e.g. stress before density) */
#define PSCFG_ENOTCONV 5   /* iteration did not converge (results still written) */

/* precision of the propagator */
#define PSCFG_FP64 0
#define PSCFG_FP32 1       /* FP32 propagation + FFT, FP64 contour sums */
#define PSCFG_MIXED 2      /* Anderson runs start in FP32 and switch each instance
                              to FP64 once its error is below the switch error or
                              stops improving; other calls run in FP64 */

/* OR-ed into pscfg_create's precision: propagator checkpointing.  Each
 * chain keeps every K-th slice of qf and qr (K = ceil(sqrt(Ns)) of the
 * batch's longest chain) and two K + 1 slice working segments instead of
 * all Ns + 1 slices; density, stress and the adjoint recompute each segment
 * from its checkpoint with the same step kernels: a density takes 3 Ns
 * steps per chain instead of 2 Ns; the stress and the adjoint recompute
 * both propagators, 2 Ns steps more each.  The reference
 * stores every slice (chain_grid_type%qf/qr, src/chain_mod.f90:159-165);
 * results agree with the stored-slice engine to roundoff.  Not available
 * with pscfg_response. */
#define PSCFG_CHECKPOINT 0x100

/* crystal systems (src/unit_cell_mod.f90:309-664) */
#define PSCFG_LAMELLAR 0
#define PSCFG_SQUARE 10
#define PSCFG_RECTANGULAR 11
#define PSCFG_HEXAGONAL2D 12
#define PSCFG_OBLIQUE 13
#define PSCFG_CUBIC 20
#define PSCFG_TETRAGONAL 21
#define PSCFG_ORTHORHOMBIC 22
#define PSCFG_HEXAGONAL3D 23
#define PSCFG_MONOCLINIC 24

/* One SCFT instance: the module globals read by the reference hot path
 * (src/chemistry_mod.f90:41-46 chemistry, src/grid_mod.f90:43-46 grid,
 * src/unit_cell_mod.f90 cell, chain_step from DISCRETIZATION). */
typedef struct pscfg_system {
    int dim;                                /* 1, 2 or 3 */
    int n[3];                               /* grid; unused entries = 1 */
    int n_monomer;
    int n_chain;
    int n_solvent;
    int ensemble;                           /* 0 canonical, 1 grand */
    int n_block[PSCFG_MAXC];
    int block_monomer[PSCFG_MAXC][PSCFG_MAXB];
    double block_length[PSCFG_MAXC][PSCFG_MAXB];
    double kuhn[PSCFG_MAXM];
    double chi[PSCFG_MAXM][PSCFG_MAXM];
    double phi_chain[PSCFG_MAXC];
    double mu_chain[PSCFG_MAXC];
    int solvent_monomer[PSCFG_MAXS];
    double solvent_size[PSCFG_MAXS];
    double phi_solvent[PSCFG_MAXS];
    double mu_solvent[PSCFG_MAXS];
    double chain_step;                      /* ds */
    int crystal_system;                     /* PSCFG_LAMELLAR ... */
    double cell_param[PSCFG_MAXCP];
} pscfg_system;

typedef struct pscfg_engine pscfg_engine;

/* Anderson-mixing parameters (src/iterate_mod.fp.f90:983-1021 startup,
 * iterate_AM input: max_itr, error_max, N_hist, domain). */
typedef struct pscfg_am_param {
    int max_itr;
    int n_hist;
    int domain;              /* 1: relax the unit cell (stress -> 0) */
    double error_max;
    double switch_error;     /* PSCFG_MIXED: FP32 -> FP64 below this error (0: 1e-3), on
                                stagnation within 1000x of it, when the error rises to 10x the
                                best FP32 error, or after 500 FP32 iterations */
    /* Stabilisers for starts far from a solution (no counterpart in the
     * reference, whose iterate_AM always ramps lambda = 1 - 0.9^k to 1 and
     * keeps its history): 0 selects the reference behaviour. */
    double mix_max;          /* cap on lambda (0: 1) */
    double restart;          /* restart the history and the lambda ramp when the error exceeds
                                restart x its best value since the last restart (0: never) */
    /* 0: the host drives each iteration (one synchronisation per iteration,
     * the coefficient solve on the host).  n > 0: every iteration -- density,
     * stress, free energy, Anderson sums, coefficient solve, mixing,
     * projection, cell update -- replays from one captured CUDA graph with
     * its control on the device, and the host reads the instances' status
     * words every n iterations (the graph is rebuilt without the finished
     * instances once a quarter of them have finished).  FP64 engines without
     * PSCFG_CHECKPOINT. */
    int graph_check;
} pscfg_am_param;

/* Per-instance exit status of an Anderson run (pscfg_am_result.status).
 * The reference stops the whole program on these conditions
 * (src/iterate_mod.fp.f90:412-420); here each instance retires on its own
 * and the others go on. */
#define PSCFG_AM_CONVERGED 0   /* error below error_max */
#define PSCFG_AM_RUNNING 1     /* not finished yet (pscfg_am_results during a run) */
#define PSCFG_AM_NONFINITE 2   /* NaN or Inf in the deviation (detected on the device) */
#define PSCFG_AM_DIVERGED 3    /* error above 1e4 */
#define PSCFG_AM_MAXITER 4     /* max_itr iterations without converging */
#define PSCFG_AM_SINGULAR 5    /* singular Anderson coefficient system */

/* Per-instance result of pscfg_iterate_am. */
typedef struct pscfg_am_result {
    int itr;
    int itr_fp32;            /* PSCFG_MIXED: iterations run with FP32 propagation */
    int converged;           /* 1 converged, 0 not (max_itr or diverged) */
    int status;              /* PSCFG_AM_* */
    double error;            /* max(|dev|, |stress|) at exit */
    double f_helmholtz;      /* free energy per monomer / kT */
    double pressure;
    double stress[PSCFG_MAXCP];
    double cell_param[PSCFG_MAXCP];
    double q[PSCFG_MAXC];
    double mu_chain[PSCFG_MAXC];
} pscfg_am_result;

/* Create an engine for n_inst instances of one grid shape.
 * Replaces density_startup + make_chain_grid + init_step
 * (src/scf_mod.fp.f90:82-117, src/chain_mod.f90:97-175,
 * src/step_mod.f90:60-92), the unit cell setup make_unit_cell + make_ksq
 * (src/unit_cell_mod.f90:309-664, src/grid_mod.f90:141-160).
 * `precision` is PSCFG_FP64 or PSCFG_FP32. */
int pscfg_create(const pscfg_system *systems, int n_inst, int precision, pscfg_engine **out);
void pscfg_destroy(pscfg_engine *e);

/* Message of the last failed call on this engine (or of the last failed
 * pscfg_create when e is NULL). */
const char *pscfg_last_error(const pscfg_engine *e);

/* New unit cell for instance `inst`: G_basis, dGG and the k^2 table are
 * rebuilt (make_unit_cell + make_ksq, src/iterate_mod.fp.f90:1453-1459). */
int pscfg_set_cell_param(pscfg_engine *e, int inst, const double *cell_param);

/* k^2 table of instance `inst` on the r2c half grid (0:n1/2,0:n2-1,0:n3-1),
 * x fastest (ksq_grid, src/grid_mod.f90:141-160).  nk doubles. */
int pscfg_get_ksq(pscfg_engine *e, int inst, double *ksq);

/* density() on grid fields for every instance
 * (src/scf_mod.fp.f90:144-229 between basis_to_kgrid/ifft and
 * fft/kgrid_to_basis).  omega, rho: host [n_inst][n_monomer][nr];
 * q: host [n_inst][PSCFG_MAXC] chain partition functions (bigQ);
 * q_solvent: host [n_inst][PSCFG_MAXS] or NULL. */
int pscfg_density(pscfg_engine *e, const double *omega, double *rho, double *q, double *q_solvent);

/* Same with device-resident omega/rho (cudaMalloc'd, same layout). */
int pscfg_density_device(pscfg_engine *e, const double *omega_dev, double *rho_dev, double *q, double *q_solvent);

/* scf_stress (src/scf_mod.fp.f90:451-550) after a density call:
 * stress: host [n_inst][PSCFG_MAXCP] = d f_Helmholtz / d cell_param. */
int pscfg_stress(pscfg_engine *e, double *stress);

/* free_energy (src/scf_mod.fp.f90:834-886) and mu_phi_chain
 * (src/scf_mod.fp.f90:768-785) for the fields of the last density call.
 * out: host [n_inst][2] = {f_Helmholtz, pressure};
 * mu_chain: host [n_inst][PSCFG_MAXC] or NULL. */
int pscfg_free_energy(pscfg_engine *e, double *out, double *mu_chain);

/* Anderson-mixing solve of every instance (iterate_AM,
 * src/iterate_mod.fp.f90:1042-1490) with density, stress, deviations,
 * Gram matrix and mixing on the device.  omega: host
 * [n_inst][n_monomer][nr], in: initial guess, out: solution.  rho: host
 * output or NULL.  results: host [n_inst]. */
int pscfg_iterate_am(pscfg_engine *e, double *omega, const pscfg_am_param *prm, double *rho,
                     pscfg_am_result *results);

/* Reverse-mode derivative of the last density call (no counterpart
 * routine in the reference; it differentiates the reference's discrete
 * algorithm: step_exp src/step_mod.f90:146-176, Simpson sums
 * src/scf_mod.fp.f90:364-426, bigQ :359).  Given upstream gradients
 * grad_rho [n_inst][n_monomer][nr] = dL/drho and, optionally,
 * grad_lnq [n_inst][PSCFG_MAXC] = dL/dlnQ, writes
 * grad_omega [n_inst][n_monomer][nr] = dL/domega (per grid point).  Two
 * adjoint sweeps per chain run through the same step kernels.  FP64
 * propagators only.  Host arrays; the _device form takes device arrays
 * (grad_lnq stays on the host). */
int pscfg_density_adjoint(pscfg_engine *e, const double *grad_rho, const double *grad_lnq, double *grad_omega);
int pscfg_density_adjoint_device(pscfg_engine *e, const double *grad_rho_dev, const double *grad_lnq,
                                 double *grad_omega_dev);

/* pscfg_density_adjoint plus the derivative with respect to the cell
 * parameters: grad_cell [n_inst][PSCFG_MAXCP] (host) = dL/d cell_param.
 * Exact derivative of the discrete algorithm (the k-space filters
 * exp(-ds b^2 k^2/6), exp(-ds b^2 k^2/12) of step_exp depend on the cell
 * through k^2 = G^T GG G, src/unit_cell_mod.f90:723-757); for
 * L = -(phi/N) lnQ it is the continuum stress of scf_stress
 * (src/scf_mod.fp.f90:451-550) up to the contour discretisation.  No
 * counterpart routine in the reference. */
int pscfg_density_adjoint_cell(pscfg_engine *e, const double *grad_rho, const double *grad_lnq, double *grad_omega,
                               double *grad_cell);

/* Ideal-gas linear response of instance `inst` to Bloch perturbations
 * (replaces drho_domega_id's loop over perturbations, calc_q0 / calc_delq /
 * calc_delrho, src/response_mod.f90:389-468, 697-1186, with the steps of
 * src/response_step_mod.f90:114-219 at the order the reference uses, 1).
 * Perturbation p adds exp(i k.r) W_p(r) to the field of monomer
 * pert_monomer[p]; W_p is given on the grid (pert_field: host
 * [n_pert][nr][2], re/im interleaved; the reference builds it from one
 * basis function, calc_perturb_field :1275-1291).  kvec: k in units of
 * the reciprocal basis vectors (3 entries, those beyond dim ignored);
 * ktrans_sq is added to every |G+k|^2 (calc_ksqgrid_new :1203-1238).
 * For every perturbation and monomer m the periodic part of the density
 * response is transformed (fftc(+1), /N) and read at n_read waves:
 * out[p][m][j] = Re(FFT(drho_m)[read_index[j]] / read_coef[j])
 * (kgrid_to_basis with no_parity, src/grid_basis_mod.f90:146-200);
 * read_coef: [n_read][2].  Uses the propagators of the preceding
 * pscfg_density call (FP64).  Host arrays. */
int pscfg_response(pscfg_engine *e, int inst, const double *kvec, double ktrans_sq, int n_pert,
                   const int *pert_monomer, const double *pert_field, int n_read, const int *read_index,
                   const double *read_coef, double *out);

/* Stepwise form of pscfg_iterate_am for callers that interleave their own
 * work or time single iterations: pscfg_am_begin loads omega (host, or
 * NULL to keep the engine's fields) and runs the initial density;
 * pscfg_am_iterate runs up to `iters` iterations of every unfinished
 * instance and returns how many are still iterating; pscfg_am_results
 * writes the per-instance results and, when non-NULL, omega/rho (host). */
int pscfg_am_begin(pscfg_engine *e, const double *omega, const pscfg_am_param *prm);
int pscfg_am_iterate(pscfg_engine *e, int iters, int *remaining);
int pscfg_am_results(pscfg_engine *e, double *omega, double *rho, pscfg_am_result *results);

/* Impose a space group on instance `inst`: omega is projected onto the
 * group-invariant fields (the span of the reference's symmetry-adapted
 * star basis, src/basis_mod.f90 / src/grid_basis_mod.f90:47-200) at the
 * start of an Anderson run and after every mixing step.  ops: [nops][12]
 * ints, 9 entries of the integer grid-index matrix M (row major) then 3 of
 * the translation t in grid units: i -> M i + t (mod n).  nops = 0 removes
 * the constraint. */
int pscfg_set_symmetry(pscfg_engine *e, int inst, int nops, const int *ops);

/* The CUDA stream (cudaStream_t) every kernel of this engine runs on. */
void *pscfg_stream(const pscfg_engine *e);

/* Phase timing with CUDA events on the engine stream (the reference's
 * cpu_time stopwatches scf_time/basis_time, src/pscf.fp.f90:492-494, per
 * phase).  pscfg_set_profiling(e, 1) resets and enables the accumulators;
 * pscfg_get_profile writes out[6] = {sweep ms, contour-integral ms,
 * stress ms, mixing ms, MDE steps in the timed sweeps, sweep launches}. */
int pscfg_set_profiling(pscfg_engine *e, int on);
int pscfg_get_profile(const pscfg_engine *e, double *out);

/* nsteps applications of step_exp (src/step_mod.f90:146-176) to q for
 * instance `inst`, with the tables of make_propg(ds, b, ksq, omega_m)
 * (src/step_mod.f90:109-129).  omega_m, q_in, q_out: host [nr]. */
int pscfg_propagate(pscfg_engine *e, int inst, const double *omega_m, double b, double ds,
                    const double *q_in, double *q_out, int nsteps);

/* Limits of pscfg_propagate_noalloc. */
#define PSCFG_NOALLOC_MAX_NR 65536     /* grid points (n1*n2*n3) */
#define PSCFG_NOALLOC_MAX_LINE 1024    /* points along any one axis */

/* step_exp applied nsteps times (src/step_mod.f90:146-176), like
 * pscfg_propagate, for callers that cannot let a library allocate device
 * memory: hosts whose whole device budget is handed to their own memory
 * pool (a Fortran host running many solver instances side by side, or a
 * framework whose caching allocator owns the device) and therefore need
 * every call to stay inside memory they already account for.  This entry
 * point has no counterpart in the reference.
 *
 * It takes no engine handle and calls no cudaMalloc/cudaFree: its scratch
 * (propagator tables, spectra, working slices, twiddles, step descriptors)
 * is one file-scope device array of about 5.6 MB, which every GPU that
 * loads the library holds until the process exits.  Grids must have at
 * most PSCFG_NOALLOC_MAX_NR points and PSCFG_NOALLOC_MAX_LINE points per
 * axis, extents with no prime factor above 7, and fit the shared memory of
 * the kernels (227 KB): for dim <= 2, 32 n2 (n1/2+1) + 16 n1 n2 bytes
 * (64 x 64 fits, 128 x 128 does not); for dim = 3, 32 n2 (n1/2+1) and
 * 512 n3 bytes each.  Other grids are rejected with PSCFG_EINVAL, before
 * any GPU work is queued, and a message from pscfg_last_error(NULL).  The
 * first call on a device does a one-time set-up with that device current:
 * it looks up the array's device address (cudaGetSymbolAddress) and copies
 * the codelet constants to the device (cudaMemcpyToSymbol).  After that a
 * call queues kernel launches only (no host-device copies).  All calls
 * on a device share the array: calls whose GPU work overlaps (other host
 * threads, or streams with no ordering between them) race on it.  Each
 * call writes every scratch entry it reads, so nothing carries over from
 * the previous call.
 *
 * All arrays are device pointers, FP64, x-fastest: ksq_dev [nk] (the k^2
 * table, e.g. from pscfg_get_ksq), omega_dev [nr] (the block's monomer
 * field), q_in_dev / q_out_dev [nr] (may alias).  Work is queued on
 * `stream` (a cudaStream_t, NULL for the default stream); the call returns
 * without synchronising. */
int pscfg_propagate_noalloc(int dim, const int *n, const double *ksq_dev, const double *omega_dev, double b,
                            double ds, const double *q_in_dev, double *q_out_dev, int nsteps, void *stream);

/* Star basis of instance `inst` for pscfg_density_basis (the reference's
 * basis_mod / grid_basis_mod tables, src/basis_mod.f90,
 * src/grid_basis_mod.f90:47-200): n_wave waves of the r2c half grid, wave j
 * at flat index wave_k[j] = kx + (n1/2+1)(ky + n2 kz) (0 <= kx <= n1/2), in
 * real basis function wave_star[j] (0-based), with complex coefficient
 * (coeff[2j], coeff[2j+1]) of f_s(r) = sum_G c_s(G) exp(i G.r) over all
 * waves G; the waves outside the half grid are the Hermitian partners,
 * c_s(-G) = conj c_s(G).  A half-grid wave belongs to one function, or to
 * two: the cosine- and sine-like functions (phi +- conj phi) / sqrt(+-2) of
 * a pair of stars related by inversion in a group without inversion (the
 * reference's star_invert = +1 / -1); waves of cancelled stars are left
 * out.  The tables (sorted by function) stay on the device. */
int pscfg_set_basis(pscfg_engine *e, int inst, int n_star, int n_wave, const int *wave_k, const int *wave_star,
                    const double *coeff);

/* density() with omega and rho as star coefficients, as the reference's
 * density(N, omega, rho, qout, q_solvent) takes them
 * (src/scf_mod.fp.f90:144-229): basis_to_kgrid and the inverse FFT of omega,
 * the propagators and contour integrals, the forward FFT and kgrid_to_basis
 * of rho, all on the device (one gather/scatter kernel each).  Coefficients
 * a_s = <f, f_s> (grid averages).  omega_basis / rho_basis: host
 * [n_inst][n_monomer][n_star_i], instances one after another (each with its
 * own n_star); rho_basis may be NULL; q, q_solvent as in pscfg_density.
 * Every instance needs pscfg_set_basis first (PSCFG_ESTATE otherwise). */
int pscfg_density_basis(pscfg_engine *e, const double *omega_basis, double *rho_basis, double *q, double *q_solvent);

/* Stored propagators of chain `chain` of instance `inst` after a density
 * call (chain_grid_type%qf/qr, src/chain_mod.f90:39-50): host
 * [n_slices][nr] each (either may be NULL); returns the slice count in
 * *n_slices when non-NULL. */
int pscfg_get_propagators(pscfg_engine *e, int inst, int chain, double *qf, double *qr, int *n_slices);

/* Number of MDE steps (step_exp calls) in one density() of the whole
 * batch: sum over instances and chains of 2 * Ns. */
long pscfg_steps_per_density(const pscfg_engine *e);

/* Kernel launches issued by this engine since creation (all streams). */
long pscfg_launch_count(const pscfg_engine *e);

/* Planes per CTA that the 3-D register sweep of this engine's grid uses for
 * a sweep of n_fields fields in FP64 (fp32 != 0: FP32), as measured by the
 * engine (one timed trial sweep per candidate before the first real sweep
 * of each class of field counts -- up to the same power of two -- the
 * fastest kept for the process); -1 when the thread-block-cluster sweep
 * (32^3, FP64) was the fastest; 0 while undecided or for grids without the
 * register sweep (16^3, 32^3). */
int pscfg_sweep_planes(const pscfg_engine *e, int n_fields, int fp32);

#ifdef __cplusplus
}
#endif
#endif /* PSCF_GPU_H */
