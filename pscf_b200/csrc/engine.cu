// engine.cu -- batched SCFT propagator engine behind the C ABI of
// include/pscf_gpu.h.
//
// One engine = a batch of independent SCFT instances sharing one grid shape
// and precision.  All instances of the batch advance together: every kernel
// launch covers every active (instance, chain, direction) field, so a batch
// of small grids fills the 148 SMs that one instance alone cannot.
//
// Device memory per instance (one bump-allocated arena per engine):
//   omega, rho           [M][nr] double   (x fastest, like omega_grid)
//   ksq                  [nk]    double   (r2c half grid, like ksq_grid)
//   wdgsq                [MAXCP][nk] double  stress weights
//   qf, qr per chain     [ns+1][nr] T     (chain_grid_type%qf/qr)
//   eo1, eo2 per block   [nr] T ; ek1, ek2 per block [nk] T  (make_propg)
//   3-D step scratch per field: S1, S2 [nk] cx<T>, q1 [nr] T
//   Anderson history     (n_hist+1) x 2 x [M][nr] double
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/pscf_gpu.h"
#include "host_geom.h"
#include "launch_util.h"
#include "scf_kernels.cuh"
#include "kernels3c.cuh"
#include "adjoint.cuh"
#include "kernels3x.cuh"
#include "response.cuh"
#include "kernels3l.cuh"
#include "kernels3p.cuh"
#include "basis.cuh"
#include "am_graph.cuh"

namespace pscfg {

static thread_local std::string g_create_error;

// Error text of calls made without an engine handle, for pscfg_last_error(NULL).
void set_global_error(const std::string &msg) { g_create_error = msg; }

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t _e = (call);                                                                 \
        if (_e != cudaSuccess) {                                                                 \
            throw Err(PSCFG_ECUDA, std::string(#call) + ": " + cudaGetErrorString(_e));          \
        }                                                                                        \
    } while (0)

struct Err {
    int code;
    std::string msg;
    Err(int c, std::string m) : code(c), msg(std::move(m)) {}
};

static const int Z_TILE = 16;

// Device buffers owned by one call.
struct CallScratch {
    std::vector<void *> p;
    void *get(size_t bytes)
    {
        void *d = nullptr;
        cudaError_t e = cudaMalloc(&d, std::max(bytes, (size_t)16));
        if (e != cudaSuccess) throw Err(PSCFG_ENOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
        p.push_back(d);
        return d;
    }
    ~CallScratch()
    {
        for (void *d : p) cudaFree(d);
    }
};

struct Inst {
    pscfg_system sys;
    Cell cell;
    int ns[PSCFG_MAXC];
    int bgn[PSCFG_MAXC][PSCFG_MAXB + 1];
    double bds[PSCFG_MAXC][PSCFG_MAXB];
    double length[PSCFG_MAXC];
    double *omega = nullptr, *rho = nullptr, *ksq = nullptr, *wdgsq = nullptr;
    void *qf[PSCFG_MAXC] = {}, *qr[PSCFG_MAXC] = {};
    void *eo1[PSCFG_MAXC][PSCFG_MAXB] = {}, *eo2[PSCFG_MAXC][PSCFG_MAXB] = {};
    void *ek1[PSCFG_MAXC][PSCFG_MAXB] = {}, *ek2[PSCFG_MAXC][PSCFG_MAXB] = {};
    void *S1[2 * PSCFG_MAXC] = {}, *S2[2 * PSCFG_MAXC] = {}, *q1[2 * PSCFG_MAXC] = {};
    double *Qdev = nullptr;       // [MAXC] chain partition functions
    double *Qsolv = nullptr;      // [MAXS]
    double *inc[PSCFG_MAXC] = {}; // stress slice sums [ns+1][MAXCP]
    double *stress_dev = nullptr; // [MAXCP]
    double Q[PSCFG_MAXC] = {}, Qs[PSCFG_MAXS] = {};
    bool have_density = false;
    int dens_prec = PSCFG_FP64;   // precision of the stored propagators
    int prec_now = PSCFG_FP64;    // propagation precision of the next density call
    // Anderson
    double *om_hist = nullptr, *dev_hist = nullptr;
    // adjoint scratch per (chain, direction): lambda ping-pong, step
    // intermediates of lambda and of the stored slice, spectra, gradient
    void *adj_real[PSCFG_MAXC][2] = {};   // 10 fields of nr T
    void *adj_spec[PSCFG_MAXC][2] = {};   // 4 spectra of nk cx<T>
    double *adj_grad[PSCFG_MAXC][2] = {}; // [M][nr]
    double *adj_coef[PSCFG_MAXC] = {};    // [ns+1][MAXM] device
    // space group imposed on omega (0 ops: none)
    int nops = 0;
    int *d_orb_perm = nullptr;   // real-space orbits of the group on the grid
    int *d_orb_start = nullptr;
    int norb = 0;
    // star basis for basis-coefficient fields (pscfg_set_basis): CSR tables
    // sorted by star in one device buffer
    int n_star = 0, n_wave = 0;
    void *basis_buf = nullptr;
    const int *b_start = nullptr, *b_k = nullptr, *b_star = nullptr;
    const cx<double> *b_c = nullptr;
    // checkpointing (PSCFG_CHECKPOINT): qf/qr hold the checkpoint slices
    // min(j K, ns), j = 0..nseg; segA/segB are K + 1 slice working segments
    int nseg[PSCFG_MAXC] = {};
    void *segA[PSCFG_MAXC] = {}, *segB[PSCFG_MAXC] = {};
    double *simp_w[PSCFG_MAXC] = {};   // [ns + 1][MAXM] per-slice Simpson weights
    double *kweight = nullptr;    // [nk] star weights (nullptr: exact Parseval weights)
    double *wdg0 = nullptr;       // [MAXCP][nk] stress weights without star weights (set with kweight)
};

struct Engine {
    int prec = PSCFG_FP64;
    int dim = 1;
    int n[3] = {1, 1, 1};
    long nr = 1, nk = 1;
    int M = 0;
    std::vector<Inst> inst;
    cudaStream_t st = nullptr;
    // second branch of the plane-kernel sweeps: the fields of a small batch
    // split in two independent kernel chains (fork/join events on st)
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool no_branch = false;          // PSCFG_NO_BRANCH=1: one chain
    bool ckpt = false;               // PSCFG_CHECKPOINT
    int ckK = 0;                     // checkpoint interval (slices)
    std::string err;
    long launches = 0;
    int n_hist_alloc = 0;
    bool no_fixed_kernels = false;   // force the run-time sized kernels (tests)
    bool cluster_step = false;       // one-launch cluster step for 32^3 (PSCFG_CLUSTER_STEP=1)
    bool smem_zconv = false;         // shared-memory z pass instead of register columns (PSCFG_SMEM_ZCONV=1)
    bool smem_fft = false;           // shared-memory x-y column passes (PSCFG_SMEM_FFT=1)
    bool no_graphs = false;          // launch the 3-D sweeps directly (PSCFG_NO_GRAPHS=1)
    bool line_step = false;          // line-pass 3-D step even where the plane kernels fit (PSCFG_LINE_STEP=1)
    int plane_p = 1;                 // shared-memory plane kernels (kernels3p.cuh) for 64x128x224 and 64^3; 0: off (PSCFG_PLANE_P)
    int planes = 0;                  // planes per CTA of the register sweep, 0 = by launch size (PSCFG_PLANES)
    // CUDA graphs of 3-D sweeps, keyed by descriptor address, field and step count
    struct SweepGraph {
        const void *dfl;
        int nf, ns, tsize, t0, variant;
        cudaGraphExec_t exec;
        long launches;
    };
    std::vector<SweepGraph> graphs;
    // events timing the trial sweeps of the planes-per-CTA choice
    cudaEvent_t tune_e0 = nullptr, tune_e1 = nullptr;
    // optional CUDA-event timing of the phases (ms, accumulated)
    bool profiling = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double t_sweep = 0, t_contour = 0, t_stress = 0, t_mix = 0;
    long n_steps_timed = 0;     // MDE steps in the timed sweeps
    long sweep_launches = 0;

    // FFT plan / twiddle tables
    PlaneGeom g64, g32;
    std::vector<void *> allocs;

    // descriptor scratch (device), grown on demand
    void *d_desc = nullptr;
    size_t d_desc_bytes = 0;
    size_t geom_off = (size_t)8 << 20;   // descriptor offset reserved for geometry jobs
    double *d_part = nullptr;
    size_t d_part_len = 0;
    double *d_small = nullptr;   // scalars [n_inst][64]
    double *dstage = nullptr;    // device twin of hpin: per-instance scalars gathered for one copy
    // pinned host staging of per-instance scalars read back each Anderson
    // iteration (one synchronisation per iteration): [n_inst][16] Q and
    // Q_solvent, [n_inst][8] stress, [n_inst] free-energy terms, from
    // n_inst*32 the Anderson sums
    double *hpin = nullptr;
    int hpin_inst = 0;
    double *hq(int i) { return hpin + (size_t)i * 16; }
    double *hst(int i) { return hpin + (size_t)hpin_inst * 16 + (size_t)i * 8; }
    double *hfe() { return hpin + (size_t)hpin_inst * 24; }
    double *hsm() { return hpin + (size_t)hpin_inst * 32; }
    void *spec = nullptr;        // 3-D stress spectra scratch
    void *fe_spec = nullptr;     // spectra for the star-weighted free energy
    void *basis_scr = nullptr;   // pscfg_density_basis: spectra and coefficients
    size_t basis_scr_bytes = 0;
    size_t fe_spec_bytes = 0;
    size_t spec_bytes = 0;
    double *stress_part = nullptr;
    size_t stress_part_len = 0;

    // Graph-driven Anderson iterations: amg selects the device-side forms
    // of the iteration's host steps (no host copies or waits, table k-space
    // factors); while capturing, descriptors go to an arena that lives as
    // long as the captured graph (amg_exec), copied on st_up outside the
    // capture.
    bool amg = false;
    bool capturing = false;
    cudaStream_t st_up = nullptr;
    std::vector<void *> cap_blocks;
    char *cap_cur = nullptr;
    size_t cap_left = 0;
    cudaGraphExec_t amg_exec = nullptr;
    std::vector<const double *> amg_G;   // per instance: its cell's G on the device (GeomJob of the run)

    ~Engine()
    {
        if (tune_e0) cudaEventDestroy(tune_e0);
        if (tune_e1) cudaEventDestroy(tune_e1);
        if (amg_exec) cudaGraphExecDestroy(amg_exec);
        for (void *p : cap_blocks) cudaFree(p);
        if (st_up) cudaStreamDestroy(st_up);
        for (void *p : allocs) cudaFree(p);
        if (d_desc) cudaFree(d_desc);
        for (void *p : desc_retired) cudaFree(p);
        if (d_part) cudaFree(d_part);
        if (d_small) cudaFree(d_small);
        if (dstage) cudaFree(dstage);
        if (spec) cudaFree(spec);
        if (fe_spec) cudaFree(fe_spec);
        if (stress_part) cudaFree(stress_part);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (auto &g : graphs) cudaGraphExecDestroy(g.exec);
        for (auto &I : inst)
            if (I.basis_buf) cudaFree(I.basis_buf);
        if (basis_scr) cudaFree(basis_scr);
        if (hpin) cudaFreeHost(hpin);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (st2) cudaStreamDestroy(st2);
        if (st) cudaStreamDestroy(st);
    }

    void *dalloc(size_t bytes)
    {
        void *p = nullptr;
        if (bytes == 0) bytes = 16;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) throw Err(PSCFG_ENOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
        allocs.push_back(p);
        return p;
    }

    int cur = PSCFG_FP64;          // precision of the kernels being launched
    size_t tsize() const { return prec == PSCFG_FP32 ? sizeof(float) : sizeof(double); }
    const PlaneGeom &geom() const { return cur == PSCFG_FP32 ? g32 : g64; }

    // Growing the descriptor scratch retires the old buffer instead of
    // freeing it: descriptors uploaded earlier in the same host sequence may
    // still be waiting for their launches.  Retired buffers (a geometric
    // series, so at most about the final size) are freed with the engine.
    void *desc(size_t bytes)
    {
        if (bytes > d_desc_bytes) {
            if (d_desc) desc_retired.push_back(d_desc);
            d_desc = nullptr;
            size_t nb = std::max(bytes + bytes / 2, (size_t)16 << 20);
            CK(cudaMalloc(&d_desc, nb));
            d_desc_bytes = nb;
        }
        return d_desc;
    }
    std::vector<void *> desc_retired;
    void *cap_alloc(size_t bytes)
    {
        bytes = (bytes + 255) / 256 * 256;
        if (bytes > cap_left) {
            const size_t nb = std::max(bytes, (size_t)4 << 20);
            void *p = nullptr;
            CK(cudaMalloc(&p, nb));
            cap_blocks.push_back(p);
            cap_cur = (char *)p;
            cap_left = nb;
        }
        void *r = cap_cur;
        cap_cur += bytes;
        cap_left -= bytes;
        return r;
    }
    // the arena of a destroyed graph (the stream must be idle)
    void cap_free()
    {
        for (void *p : cap_blocks) cudaFree(p);
        cap_blocks.clear();
        cap_cur = nullptr;
        cap_left = 0;
    }
    // a scratch buffer would have to grow inside a capture
    void no_growth_in_capture() const
    {
        if (capturing) throw Err(PSCFG_ECUDA, "scratch buffer growth while capturing an Anderson iteration");
    }
    // upload host descriptors into a sub-range of the descriptor scratch
    // (while capturing: into the arena, each upload its own range)
    template <typename D>
    D *upload(const std::vector<D> &v, size_t offset_bytes)
    {
        if (capturing) {
            D *p = (D *)cap_alloc(v.size() * sizeof(D) + 16);
            if (!v.empty()) {
                CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(D), cudaMemcpyHostToDevice, st_up));
                CK(cudaStreamSynchronize(st_up));
            }
            return p;
        }
        char *base = (char *)desc(offset_bytes + v.size() * sizeof(D) + 256);
        D *p = (D *)(base + offset_bytes);
        if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(D), cudaMemcpyHostToDevice, st));
        return p;
    }
    double *part(size_t len)
    {
        if (len > d_part_len) {
            no_growth_in_capture();
            if (d_part) cudaFree(d_part);
            d_part = nullptr;
            CK(cudaMalloc(&d_part, len * sizeof(double)));
            d_part_len = len;
        }
        return d_part;
    }
    void launched(cudaError_t e = cudaGetLastError())
    {
        launches++;
        if (e != cudaSuccess) throw Err(PSCFG_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    }
};

// ---------------------------------------------------------------------
// FFT plans
// ---------------------------------------------------------------------
template <typename T>
static void *twiddle_table(Engine &E, int n)
{
    std::vector<cx<T>> h(std::max(n, 1));
    for (int m = 0; m < n; m++) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
        h[m].x = (T)cosl(a);
        h[m].y = (T)sinl(a);
    }
    void *d = E.dalloc(h.size() * sizeof(cx<T>));
    CK(cudaMemcpy(d, h.data(), h.size() * sizeof(cx<T>), cudaMemcpyHostToDevice));
    return d;
}

template <typename T>
static void make_line_plan(Engine &E, int n, LinePlan &p)
{
    p.n = n;
    if (!plan_radices(n, p.rad, p.nst))
        throw Err(PSCFG_EINVAL, "grid size " + std::to_string(n) + " has a prime factor other than 2, 3, 5, 7");
    p.tw = twiddle_table<T>(E, n);
}

template <typename T>
static void make_geom(Engine &E, PlaneGeom &g)
{
    g.n1 = E.n[0];
    g.n2 = E.n[1];
    g.n3 = E.n[2];
    g.n1h = g.n1 / 2 + 1;
    g.even = (g.n1 % 2 == 0) ? 1 : 0;
    g.LS = g.even ? g.n1h : g.n1;
    make_line_plan<T>(E, g.even ? g.n1 / 2 : g.n1, g.row);
    make_line_plan<T>(E, g.n2, g.col);
    make_line_plan<T>(E, g.n3, g.zp);
    g.rtw = twiddle_table<T>(E, g.n1);
}

// W_N^m tables of the plane kernels (kernels3p.cuh), FP64 and FP32.
template <int N>
static void upload_ptw(const void *sym_d, const void *sym_f)
{
    double d[2][N];
    float f[2][N];
    for (int m = 0; m < N; m++) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * m / (long double)N;
        d[0][m] = (double)cosl(a);
        d[1][m] = (double)sinl(a);
        f[0][m] = (float)cosl(a);
        f[1][m] = (float)sinl(a);
    }
    CK(cudaMemcpyToSymbol(sym_d, d, sizeof(d)));
    CK(cudaMemcpyToSymbol(sym_f, f, sizeof(f)));
}

static void upload_p_twiddles()
{
    upload_ptw<32>(c_ptw32, c_ptw32f);
    upload_ptw<64>(c_ptw64, c_ptw64f);
    upload_ptw<128>(c_ptw128, c_ptw128f);
    upload_ptw<224>(c_ptw224, c_ptw224f);
}

static void upload_dft_constants()
{
    // row 0: cos(2 pi m/R), row 1: sin(2 pi m/R); the codelet forms
    // W = (cos, S*sin) with S = -1 forward, +1 inverse.
    double t5[2][5], t7[2][7];
    for (int m = 0; m < 5; m++) {
        long double a = 2.0L * 3.14159265358979323846264338327950288L * m / 5.0L;
        t5[0][m] = (double)cosl(a);
        t5[1][m] = (double)sinl(a);
    }
    for (int m = 0; m < 7; m++) {
        long double a = 2.0L * 3.14159265358979323846264338327950288L * m / 7.0L;
        t7[0][m] = (double)cosl(a);
        t7[1][m] = (double)sinl(a);
    }
    CK(cudaMemcpyToSymbol(c_dft5, t5, sizeof(t5)));
    CK(cudaMemcpyToSymbol(c_dft7, t7, sizeof(t7)));
    double w64[2][64];
    for (int m = 0; m < 64; m++) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * m / 64.0L;
        w64[0][m] = (double)cosl(a);
        w64[1][m] = (double)sinl(a);
    }
    CK(cudaMemcpyToSymbol(c_w64, w64, sizeof(w64)));
    upload_p_twiddles();
}

// ---------------------------------------------------------------------
// Setup
// ---------------------------------------------------------------------
static void validate_system(const pscfg_system &s, int dim, const int n[3])
{
    if (s.dim != dim || s.n[0] != n[0] || s.n[1] != n[1] || s.n[2] != n[2])
        throw Err(PSCFG_EINVAL, "all instances of an engine must share one grid shape");
    if (s.n_monomer < 1 || s.n_monomer > PSCFG_MAXM) throw Err(PSCFG_EINVAL, "n_monomer out of range");
    if (s.n_chain < 0 || s.n_chain > PSCFG_MAXC) throw Err(PSCFG_EINVAL, "n_chain out of range");
    if (s.n_solvent < 0 || s.n_solvent > PSCFG_MAXS) throw Err(PSCFG_EINVAL, "n_solvent out of range");
    if (s.chain_step <= 0) throw Err(PSCFG_EINVAL, "chain_step must be positive");
    for (int c = 0; c < s.n_chain; c++) {
        if (s.n_block[c] < 1 || s.n_block[c] > PSCFG_MAXB) throw Err(PSCFG_EINVAL, "n_block out of range");
        for (int b = 0; b < s.n_block[c]; b++)
            if (s.block_monomer[c][b] < 0 || s.block_monomer[c][b] >= s.n_monomer)
                throw Err(PSCFG_EINVAL, "block_monomer out of range");
    }
    for (int i = 0; i < s.n_solvent; i++)
        if (s.solvent_monomer[i] < 0 || s.solvent_monomer[i] >= s.n_monomer)
            throw Err(PSCFG_EINVAL, "solvent_monomer out of range");
}

// New unit cell for a set of instances: G_basis/dGG on the host
// (make_unit_cell), k^2 and stress weights on the device (k_make_geom).
static void update_cells(Engine &E, const std::vector<int> &which)
{
    if (which.empty()) return;
    std::vector<GeomJob> jobs;
    for (int i : which) {
        Inst &I = E.inst[i];
        Cell c;
        if (!make_unit_cell(E.dim, I.sys.crystal_system, I.sys.cell_param, c))
            throw Err(PSCFG_EINVAL, "unknown crystal system for this dimension");
        I.cell = c;
        GeomJob j;
        std::memset(&j, 0, sizeof(j));
        std::memcpy(j.G, c.G, sizeof(j.G));
        std::memcpy(j.dGG, c.dGG, sizeof(j.dGG));
        j.ncp = c.ncp;
        j.ksq = I.ksq;
        j.wdgsq = I.wdgsq;
        j.kweight = I.kweight;
        if (I.kweight && !I.wdg0) I.wdg0 = (double *)E.dalloc(sizeof(double) * PSCFG_MAXCP * E.nk);
        j.wdg0 = I.kweight ? I.wdg0 : nullptr;
        jobs.push_back(j);
        I.have_density = false;
    }
    GeomJob *dj = E.upload(jobs, E.geom_off);
    dim3 grid((unsigned)std::min<long>((E.nk + 255) / 256, 512), (unsigned)jobs.size());
    k_make_geom<<<grid, 256, 0, E.st>>>(dj, E.dim, E.n[0], E.n[1], E.n[2]);
    E.launched();
}

static void upload_cell(Engine &E, Inst &I)
{
    update_cells(E, std::vector<int>{(int)(&I - &E.inst[0])});
    CK(cudaStreamSynchronize(E.st));
}

// Phase timer: events recorded on the engine stream around a phase.
struct PhaseTimer {
    Engine &E;
    double *acc;
    PhaseTimer(Engine &e, double *a) : E(e), acc(a)
    {
        if (E.profiling) CK(cudaEventRecord(E.ev0, E.st));
    }
    ~PhaseTimer() noexcept(false)
    {
        if (E.profiling) {
            CK(cudaEventRecord(E.ev1, E.st));
            CK(cudaEventSynchronize(E.ev1));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, E.ev0, E.ev1));
            *acc += ms;
        }
    }
};

static void create_engine(Engine &E, const pscfg_system *sys, int n_inst, int precision)
{
    if (n_inst < 1) throw Err(PSCFG_EINVAL, "n_inst must be >= 1");
    E.ckpt = (precision & PSCFG_CHECKPOINT) != 0;
    precision &= ~PSCFG_CHECKPOINT;
    if (E.ckpt && precision != PSCFG_FP64) {
        long nr = 1;
        for (int d = 0; d < sys[0].dim && d < 3; d++) nr *= sys[0].n[d];
        if (nr % 2) throw Err(PSCFG_EINVAL, "PSCFG_CHECKPOINT with FP32 propagation needs an even number of grid points");
    }
    if (precision != PSCFG_FP64 && precision != PSCFG_FP32 && precision != PSCFG_MIXED)
        throw Err(PSCFG_EINVAL, "unknown precision");
    E.prec = precision;
    E.dim = sys[0].dim;
    if (E.dim < 1 || E.dim > 3) throw Err(PSCFG_EINVAL, "dim must be 1, 2 or 3");
    for (int d = 0; d < 3; d++) E.n[d] = (d < E.dim) ? sys[0].n[d] : 1;
    for (int d = 0; d < 3; d++)
        if (E.n[d] < 1) throw Err(PSCFG_EINVAL, "grid extents must be >= 1");
    E.nr = (long)E.n[0] * E.n[1] * E.n[2];
    E.nk = (long)(E.n[0] / 2 + 1) * E.n[1] * E.n[2];
    E.M = sys[0].n_monomer;
    // PSCFG_GENERIC_KERNELS=1 forces the run-time sized step kernels (used by
    // the tests that cross-check the two implementations)
    {
        const char *v = std::getenv("PSCFG_GENERIC_KERNELS");
        E.no_fixed_kernels = v && v[0] && v[0] != '0';
        const char *c = std::getenv("PSCFG_CLUSTER_STEP");
        E.cluster_step = c && c[0] && c[0] != '0';
        const char *z = std::getenv("PSCFG_SMEM_ZCONV");
        E.smem_zconv = z && z[0] && z[0] != '0';
        const char *xy = std::getenv("PSCFG_SMEM_FFT");
        E.smem_fft = xy && xy[0] && xy[0] != '0';
        const char *ng = std::getenv("PSCFG_NO_GRAPHS");
        E.no_graphs = ng && ng[0] && ng[0] != '0';
        const char *ls = std::getenv("PSCFG_LINE_STEP");
        E.line_step = ls && ls[0] && ls[0] != '0';
        const char *pl = std::getenv("PSCFG_PLANES");
        E.planes = pl ? std::atoi(pl) : 0;
        const char *pp = std::getenv("PSCFG_PLANE_P");
        if (pp && pp[0]) E.plane_p = std::atoi(pp);
        const char *nb = std::getenv("PSCFG_NO_BRANCH");
        E.no_branch = nb && nb[0] && nb[0] != '0';
    }
    CK(cudaStreamCreateWithFlags(&E.st, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&E.st2, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&E.st_up, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&E.ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&E.ev_join, cudaEventDisableTiming));
    upload_dft_constants();
    make_geom<double>(E, E.g64);
    if (precision != PSCFG_FP64) make_geom<float>(E, E.g32);

    const size_t ts = E.tsize();
    if (E.ckpt) {
        // K = ceil(sqrt(Ns)) of the longest chain of the batch
        int ns_max = 1;
        for (int i = 0; i < n_inst; i++)
            for (int c = 0; c < sys[i].n_chain && c < PSCFG_MAXC; c++) {
                if (sys[i].n_block[c] < 1 || sys[i].n_block[c] > PSCFG_MAXB) continue;
                int bgn[PSCFG_MAXB + 1];
                double bds[PSCFG_MAXB];
                ns_max = std::max(ns_max, chain_grid(sys[i].n_block[c], sys[i].block_length[c], sys[i].chain_step, bgn, bds));
            }
        E.ckK = std::max(1, (int)std::ceil(std::sqrt((double)ns_max)));
    }
    E.inst.resize(n_inst);
    for (int i = 0; i < n_inst; i++) {
        pscfg_system s = sys[i];
        for (int d = s.dim; d < 3; d++) s.n[d] = 1;
        validate_system(s, E.dim, E.n);
        if (s.n_monomer != E.M) throw Err(PSCFG_EINVAL, "all instances must have the same n_monomer");
        Inst &I = E.inst[i];
        I.sys = s;
        I.prec_now = (precision == PSCFG_FP32) ? PSCFG_FP32 : PSCFG_FP64;
        I.omega = (double *)E.dalloc(sizeof(double) * E.M * E.nr);
        I.rho = (double *)E.dalloc(sizeof(double) * E.M * E.nr);
        I.ksq = (double *)E.dalloc(sizeof(double) * E.nk);
        I.wdgsq = (double *)E.dalloc(sizeof(double) * PSCFG_MAXCP * E.nk);
        I.Qdev = (double *)E.dalloc(sizeof(double) * PSCFG_MAXC);
        I.Qsolv = (double *)E.dalloc(sizeof(double) * PSCFG_MAXS);
        I.stress_dev = (double *)E.dalloc(sizeof(double) * PSCFG_MAXCP);
        for (int c = 0; c < s.n_chain; c++) {
            I.ns[c] = chain_grid(s.n_block[c], s.block_length[c], s.chain_step, I.bgn[c], I.bds[c]);
            I.length[c] = 0;
            for (int b = 0; b < s.n_block[c]; b++) I.length[c] += s.block_length[c][b];
            if (E.ckpt) {
                const int K = E.ckK;
                I.nseg[c] = (I.ns[c] + K - 1) / K;
                I.qf[c] = E.dalloc(ts * E.nr * (I.nseg[c] + 1));
                I.qr[c] = E.dalloc(ts * E.nr * (I.nseg[c] + 1));
                I.segA[c] = E.dalloc(ts * E.nr * (K + 1));
                I.segB[c] = E.dalloc(ts * E.nr * (K + 1));
                std::vector<double> w((size_t)(I.ns[c] + 1) * PSCFG_MAXM, 0.0);
                for (int b = 0; b < s.n_block[c]; b++) {
                    const int ib = I.bgn[c][b], ie = I.bgn[c][b + 1], m = s.block_monomer[c][b];
                    for (int j = ib; j <= ie; j++) {
                        const double wt = (j == ib || j == ie) ? 1.0 : (((j - ib) % 2 == 1) ? 4.0 : 2.0);
                        w[(size_t)j * PSCFG_MAXM + m] += I.bds[c][b] / 3.0 * wt;
                    }
                }
                I.simp_w[c] = (double *)E.dalloc(sizeof(double) * w.size());
                CK(cudaMemcpy(I.simp_w[c], w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice));
            } else {
                I.qf[c] = E.dalloc(ts * E.nr * (I.ns[c] + 1));
                I.qr[c] = E.dalloc(ts * E.nr * (I.ns[c] + 1));
            }
            I.inc[c] = (double *)E.dalloc(sizeof(double) * PSCFG_MAXCP * (I.ns[c] + 1));
            for (int b = 0; b < s.n_block[c]; b++) {
                I.eo1[c][b] = E.dalloc(ts * E.nr);
                I.eo2[c][b] = E.dalloc(ts * E.nr);
                I.ek1[c][b] = E.dalloc(ts * E.nk);
                I.ek2[c][b] = E.dalloc(ts * E.nk);
            }
            if (E.dim == 3) {
                for (int d = 0; d < 2; d++) {
                    I.S1[2 * c + d] = E.dalloc(2 * ts * E.nk);
                    I.S2[2 * c + d] = E.dalloc(2 * ts * E.nk);
                    I.q1[2 * c + d] = E.dalloc(ts * E.nr);
                }
            }
        }
    }
    {
        std::vector<int> all(n_inst);
        for (int i = 0; i < n_inst; i++) all[i] = i;
        update_cells(E, all);
        CK(cudaStreamSynchronize(E.st));
    }
    E.d_small = nullptr;
    CK(cudaMalloc(&E.d_small, sizeof(double) * 64 * n_inst));
    CK(cudaMallocHost(&E.hpin, sizeof(double) * 128 * n_inst));
    CK(cudaMalloc(&E.dstage, sizeof(double) * 128 * n_inst));
    E.hpin_inst = n_inst;
    E.part((size_t)64 * n_inst * (PSCFG_MAXH + 2 * PSCFG_MAXM + 8) + 1024);
}

// ---------------------------------------------------------------------
// Density
// ---------------------------------------------------------------------
static int red_ctas(long n) { return (int)std::min<long>(std::max<long>((n + 255) / 256, 1), 64); }
// CTAs per job of a batched reduction over n points with njobs jobs: 64 per
// job for a batch, up to 4 per SM when a few jobs (one large instance) would
// otherwise leave most SMs idle and the loads without parallelism
static int red_ctas(long n, int njobs)
{
    const long cap = std::max<long>(64, 592 / std::max(njobs, 1));
    return (int)std::min<long>(std::max<long>((n + 255) / 256, 1), cap);
}

// One 3-D MDE step of every field with compile-time-shaped kernels.
template <typename T, int N1, int N2, int N3, int PPC>
static void step3c(Engine &E, const SweepField<T> *dfl, int nf, int t)
{
    constexpr int TC = (N3 >= 64) ? 16 : 32;
    constexpr int P = N2 * (N1 / 2 + 1);
    const PlaneGeom &g = E.geom();
    const int ntile = (P + TC - 1) / TC;
    const size_t sm = sizeof(cx<T>) * PPC * P;
    CK(allow_dyn_smem((const void *)k3c_fwd_pair<T, N1, N2, N3, PPC>));
    CK(allow_dyn_smem((const void *)k3c_inv_mid<T, N1, N2, N3, PPC>));
    CK(allow_dyn_smem((const void *)k3c_inv_final<T, N1, N2, N3, PPC>));
    k3c_fwd_pair<T, N1, N2, N3, PPC><<<dim3(N3 / PPC, nf), 256, sm, E.st>>>(dfl, g, t);
    E.launched();
    // z pass: register columns for N3 <= 32 (a 64-point column does not fit
    // a thread's registers in FP64), shared-memory tiles otherwise
    constexpr bool REGZ = N3 <= 32;
    const bool regz = REGZ && !E.smem_zconv;
    const unsigned rtile = (unsigned)((P + 127) / 128);
    auto zpass = [&](int which, int nz) {
        if constexpr (REGZ) {
            if (regz) {
                k3r_zconv<T, N1, N2, N3><<<dim3(rtile, nf, nz), 128, 0, E.st>>>(dfl, t, which);
                return;
            }
        }
        k3c_zconv<T, N1, N2, N3, TC><<<dim3(ntile, nf, nz), 256, 0, E.st>>>(dfl, g, t, which);
    };
    zpass(3, 2);
    E.launched();
    k3c_inv_mid<T, N1, N2, N3, PPC><<<dim3(N3 / PPC, nf), 256, sm, E.st>>>(dfl, g, t);
    E.launched();
    zpass(2, 1);
    E.launched();
    k3c_inv_final<T, N1, N2, N3, PPC><<<dim3(N3 / PPC, nf), 256, sm, E.st>>>(dfl, g, t);
    E.launched();
}

// One 3-D MDE step with register-column x-y kernels (natural y order) and
// the split-column z pass: 128 threads and PPC planes per CTA.
template <typename T, int N1, int N2, int N3, int PPC>
static void step3r(Engine &E, const SweepField<T> *dfl, int nf, int t)
{
    constexpr int P = N2 * (N1 / 2 + 1);
    const size_t sm = sizeof(cx<T>) * PPC * P;
    CK(allow_dyn_smem((const void *)k3r_fwd_pair<T, N1, N2, N3, PPC>));
    CK(allow_dyn_smem((const void *)k3r_inv_mid<T, N1, N2, N3, PPC>));
    CK(allow_dyn_smem((const void *)k3r_inv_final<T, N1, N2, N3, PPC>));
    const dim3 gp(N3 / PPC, nf);
    const unsigned rtile = (unsigned)((P + 63) / 64);
    k3r_fwd_pair<T, N1, N2, N3, PPC><<<gp, 128, sm, E.st>>>(dfl, t);
    E.launched();
    k3s_zconv<T, N1, N2, N3, true><<<dim3(rtile, nf, 2), 128, 0, E.st>>>(dfl, t, 3);
    E.launched();
    k3r_inv_mid<T, N1, N2, N3, PPC><<<gp, 128, sm, E.st>>>(dfl, t);
    E.launched();
    k3s_zconv<T, N1, N2, N3, true><<<dim3(rtile, nf, 1), 128, 0, E.st>>>(dfl, t, 2);
    E.launched();
    k3r_inv_final<T, N1, N2, N3, PPC><<<gp, 128, sm, E.st>>>(dfl, t);
    E.launched();
}

// Planes per CTA of the register sweep for nf fields of an n3-plane grid: the
// largest power of two up to pmax whose x-y launches still have 512 CTAs or
// more (the register limit allows 4 CTAs on each of the 148 SMs, 592 slots).
// Few fields (one or a few instances) take fewer planes per CTA so that more
// SMs share the work: at 32^3, 20 Anderson iterations of one BCC instance
// sweep in 61 ms with one plane per CTA against 107 ms with four, while 64
// instances are fastest with four (465 ms against 473 with two).
// Planes per CTA of the register sweep (pmax, pmax/2, ..., 1), measured.
// The first sweep of each (grid, precision, field-count class) is
// preceded by one trial sweep per candidate, timed with CUDA events on the
// engine stream (a graph replay, after its capture); the fastest is kept
// for the process (all engines) and the real sweep runs with it.  A trial
// writes only the slices that the real sweep then writes again, so every
// result comes from the chosen count -- which matters: the largest count's
// column pass pairs the real columns kx = 0 and n/2 into one complex column
// and rounds differently from the others.  PSCFG_PLANES forces a choice;
// inside a captured Anderson iteration the decided choice, or until then
// the launch-size rule (the largest count whose launch still has >= 512
// CTAs), is used.
static std::mutex g_planes_mu;
static std::map<long, int> g_planes_best;

static int planes_rule(int nf, int n3, int pmax)
{
    int p = pmax;
    while (p > 1 && (long)nf * (n3 / p) < 512) p /= 2;
    return p;
}

// the choice is shared by field counts up to the same power of two, so that
// a batch whose running instances dwindle measures a handful of times
static long planes_key(int n3, int tsize, int nf)
{
    long b = 1;
    while (b < nf) b *= 2;
    return ((long)n3 * 16 + tsize) * 100000 + b;
}

// trial(p, e0, e1) enqueues one sweep with p planes per CTA, recording e0
// just before its first launch and e1 after its last.
template <typename Trial>
static int sweep_planes(Engine &E, int nf, int n3, int pmax, int tsize, Trial trial, bool cluster = false)
{
    if (E.planes > 0) {
        for (int p = pmax; p >= 1; p /= 2)
            if (E.planes == p) return p;
    }
    if (E.planes < 0 && cluster) return 0;   // PSCFG_PLANES=-1: the cluster sweep
    const long key = planes_key(n3, tsize, nf);
    {
        std::lock_guard<std::mutex> lk(g_planes_mu);
        auto it = g_planes_best.find(key);
        if (it != g_planes_best.end()) return it->second;
    }
    if (E.capturing) return planes_rule(nf, n3, pmax);
    if (!E.tune_e0) {
        CK(cudaEventCreate(&E.tune_e0));
        CK(cudaEventCreate(&E.tune_e1));
    }
    int best = pmax;
    float best_ms = 0;
    for (int p = pmax; p >= (cluster ? 0 : 1); p = (p > 1 ? p / 2 : p - 1)) {
        trial(p, E.tune_e0, E.tune_e1);
        CK(cudaEventSynchronize(E.tune_e1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, E.tune_e0, E.tune_e1));
        if (p == pmax || ms < best_ms) {
            best = p;
            best_ms = ms;
        }
    }
    std::lock_guard<std::mutex> lk(g_planes_mu);
    auto ins = g_planes_best.emplace(key, best);   // another engine may have decided meanwhile
    return ins.first->second;
}

// Runs emit() -- a fixed sequence of sweep launches whose jobs are read from
// the descriptors at dfl -- through a CUDA graph captured once per (dfl,
// field count, step count, precision) and replayed after each descriptor
// upload (PSCFG_NO_GRAPHS=1 launches directly).
template <typename Emit>
static void graph_sweep(Engine &E, const void *dfl, int nf, int ns_max, int tsize, int t0, Emit emit,
                        int variant = 0, cudaEvent_t before = nullptr)
{
    if (E.no_graphs || E.capturing) {   // inside a captured Anderson iteration: its own nodes
        if (before) CK(cudaEventRecord(before, E.st));
        emit();
        return;
    }
    for (auto &g : E.graphs)
        if (g.dfl == dfl && g.nf == nf && g.ns == ns_max && g.tsize == tsize && g.t0 == t0 && g.variant == variant) {
            if (before) CK(cudaEventRecord(before, E.st));
            CK(cudaGraphLaunch(g.exec, E.st));
            E.launches += g.launches;
            return;
        }
    Engine::SweepGraph sg;
    sg.dfl = dfl;
    sg.nf = nf;
    sg.ns = ns_max;
    sg.tsize = tsize;
    sg.t0 = t0;
    sg.variant = variant;
    const long l0 = E.launches;
    CK(cudaStreamBeginCapture(E.st, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    try {
        emit();
    } catch (...) {
        cudaStreamEndCapture(E.st, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    CK(cudaStreamEndCapture(E.st, &graph));
    cudaError_t ie = cudaGraphInstantiate(&sg.exec, graph, 0);
    cudaGraphDestroy(graph);
    CK(ie);
    sg.launches = E.launches - l0;
    if (E.graphs.size() >= (E.ckpt ? 96u : 16u)) {
        cudaGraphExecDestroy(E.graphs.front().exec);
        E.graphs.erase(E.graphs.begin());
    }
    E.graphs.push_back(sg);
    if (before) CK(cudaGraphUpload(sg.exec, E.st));   // a timed first replay excludes the upload
    if (before) CK(cudaEventRecord(before, E.st));
    CK(cudaGraphLaunch(sg.exec, E.st));
}

// A whole 3-D sweep with the register-column kernels, the last kernel of
// every step fused with the first of the next.  Returns false where the
// grid has no such kernels (or another path was requested).
template <typename T>
static bool sweep3r(Engine &E, const SweepField<T> *dfl, int nf, int ns_max, int t0 = 0)
{
    if (E.no_fixed_kernels || E.smem_fft || E.cluster_step) return false;
    // The sweep is a fixed sequence of 1 + 4 ns_max launches whose jobs are
    // read from the descriptors at dfl, so it is captured once into a CUDA
    // graph per (dfl, nf, ns_max) and replayed after each descriptor upload.
    auto run = [&](auto n1c, auto ppcc, cudaEvent_t e0, cudaEvent_t e1) {
        constexpr int N = decltype(n1c)::value, PPC = decltype(ppcc)::value;
        constexpr int P = N * (N / 2 + 1);
        const size_t sm = sizeof(cx<T>) * PPC * P;
        CK(allow_dyn_smem((const void *)k3r_fwd_pair<T, N, N, N, PPC>));
        CK(allow_dyn_smem((const void *)k3r_inv_mid<T, N, N, N, PPC>));
        CK(allow_dyn_smem((const void *)k3r_final_fwd<T, N, N, N, PPC>));
        const dim3 gp(N / PPC, nf);
        const unsigned rtile = (unsigned)((P + 63) / 64);
        auto emit = [&]() {
            k3r_fwd_pair<T, N, N, N, PPC><<<gp, 128, sm, E.st>>>(dfl, t0);
            E.launched();
            for (int t = t0; t < ns_max; t++) {
                k3s_zconv<T, N, N, N, true><<<dim3(rtile, nf, 2), 128, 0, E.st>>>(dfl, t, 3);
                E.launched();
                k3r_inv_mid<T, N, N, N, PPC><<<gp, 128, sm, E.st>>>(dfl, t);
                E.launched();
                k3s_zconv<T, N, N, N, true><<<dim3(rtile, nf, 1), 128, 0, E.st>>>(dfl, t, 2);
                E.launched();
                k3r_final_fwd<T, N, N, N, PPC><<<gp, 128, sm, E.st>>>(dfl, t);
                E.launched();
            }
        };
        graph_sweep(E, dfl, nf, ns_max, (int)sizeof(T), t0, emit, PPC, e0);
        if (e1) CK(cudaEventRecord(e1, E.st));
    };
    const int a = E.n[0], b = E.n[1], c = E.n[2];
    if (a == 32 && b == 32 && c == 32) {
        using N = std::integral_constant<int, 32>;
        // candidate 0: the thread-block-cluster sweep (kernels3x.cuh), one
        // launch for the whole sweep, each field walked by one cluster
        auto cluster = [&](cudaEvent_t e0, cudaEvent_t e1) {
            const size_t sm = Cl32<T>::smem_bytes();
            CK(allow_dyn_smem((const void *)k3x_sweep32<T>));
            const PlaneGeom g = E.geom();
            auto emit = [&]() {
                k3x_sweep32<T><<<dim3(8 * nf), 512, sm, E.st>>>(dfl, g, t0, ns_max);
                E.launched();
            };
            graph_sweep(E, dfl, nf, ns_max, (int)sizeof(T), t0, emit, 100, e0);
            if (e1) CK(cudaEventRecord(e1, E.st));
        };
        auto go = [&](int p, cudaEvent_t e0, cudaEvent_t e1) {
            switch (p) {
            case 4: run(N(), std::integral_constant<int, 4>(), e0, e1); break;
            case 2: run(N(), std::integral_constant<int, 2>(), e0, e1); break;
            case 1: run(N(), std::integral_constant<int, 1>(), e0, e1); break;
            default: cluster(e0, e1); break;
            }
        };
        go(sweep_planes(E, nf, 32, 4, (int)sizeof(T), go, sizeof(T) == 8), nullptr, nullptr);
        return true;
    }
    if (a == 16 && b == 16 && c == 16) {
        using N = std::integral_constant<int, 16>;
        auto go = [&](int p, cudaEvent_t e0, cudaEvent_t e1) {
            switch (p) {
            case 8: run(N(), std::integral_constant<int, 8>(), e0, e1); break;
            case 4: run(N(), std::integral_constant<int, 4>(), e0, e1); break;
            case 2: run(N(), std::integral_constant<int, 2>(), e0, e1); break;
            default: run(N(), std::integral_constant<int, 1>(), e0, e1); break;
            }
        };
        go(sweep_planes(E, nf, 16, 8, (int)sizeof(T), go), nullptr, nullptr);
        return true;
    }
    return false;
}

// Whether the sweep of this engine runs the plane kernels (kernels3p.cuh).
static bool plane_kernels_apply(const Engine &E)
{
    if (E.dim != 3 || E.no_fixed_kernels || E.smem_fft || E.cluster_step || E.line_step || E.plane_p == 0) return false;
    const int a = E.n[0], b = E.n[1], c = E.n[2];
    return (a == 64 && b == 128 && c == 224) || (a == 64 && b == 64 && c == 64);
}

// Position p of a forward four-step transform of length N (Split<N> of
// fft_ct.cuh / kernels3p.cuh) -> frequency index.
__host__ __device__ static inline int host_iperm(int N, int p)
{
    int P = 1, Q = 1;
    switch (N) {
    case 32: P = 4; Q = 8; break;
    case 64: P = 8; Q = 8; break;
    case 128: P = 8; Q = 16; break;
    case 224: P = 16; Q = 14; break;
    default: P = N; Q = 1; break;
    }
    return p / Q + P * (p % Q);
}

// 1-D factors of exp(-lap k^2/6) and exp(-lap k^2/12) (lap = ds b^2) of an
// orthogonal cell over the plane kernels' spectrum positions: x (N1/2 + 1),
// y (N2) and z (N3), each index folded to its minimum image (G_to_bz,
// src/grid_mod.f90:225-283, along each axis).  Appends 2 (N1/2+1+N2+N3).
template <typename T>
static void append_ek_factors(const Engine &E, const Cell &cell, double lap, std::vector<T> &out)
{
    const int n1 = E.n[0], n2 = E.n[1], n3 = E.n[2], M = n1 / 2;
    auto g2 = [&](int axis, int k) {
        const int n = E.n[axis];
        const long double kf = (k > n / 2) ? k - n : k;
        const long double g = (long double)cell.G[axis][axis] * kf;
        return g * g;
    };
    for (int div : {6, 12}) {
        const long double c = (long double)lap / div;
        for (int xp = 0; xp <= M; xp++) out.push_back((T)expl(-c * g2(0, xp < M ? host_iperm(M, xp) : M)));
        for (int yp = 0; yp < n2; yp++) out.push_back((T)expl(-c * g2(1, host_iperm(n2, yp))));
        for (int zp = 0; zp < n3; zp++) out.push_back((T)expl(-c * g2(2, host_iperm(n3, zp))));
    }
}

// The same factors computed on the device from a cell held there (the
// graph-driven Anderson iteration updates the cell on the device): job j
// writes 2 (N1/2+1+N2+N3) values from G (row-major 3 x 3, diagonal) and
// lap.  grid = njobs, 256 threads.
struct EkfJob {
    const double *G;
    double lap;
    void *out;
};

template <typename T>
static __global__ void k_ek_factors(const EkfJob *jobs, int n1, int n2, int n3)
{
    const EkfJob &J = jobs[blockIdx.x];
    const int M = n1 / 2, L3 = M + 1 + n2 + n3;
    T *out = (T *)J.out;
    for (int i = threadIdx.x; i < 2 * L3; i += blockDim.x) {
        const double c = J.lap / (i < L3 ? 6.0 : 12.0);
        const int j = i % L3;
        int axis, n, k;
        if (j <= M) {
            axis = 0;
            n = n1;
            k = j < M ? host_iperm(M, j) : M;
        } else if (j < M + 1 + n2) {
            axis = 1;
            n = n2;
            k = host_iperm(n2, j - M - 1);
        } else {
            axis = 2;
            n = n3;
            k = host_iperm(n3, j - M - 1 - n2);
        }
        const double kf = (k > n / 2) ? (double)(k - n) : (double)k;
        const double g = J.G[axis * 3 + axis] * kf;
        out[i] = (T)exp(-c * g * g);
    }
}

// A whole 3-D sweep with the shared-memory plane kernels of kernels3p.cuh
// (64 x 128 x 224 and 64^3; PSCFG_PLANE_P=0 selects the other kernels:
// run-time shaped at 64 x 128 x 224, k3c at 64^3).  Returns false where not
// applicable.  64^3, 4 instances, FP64 sweep: 61.3k field-steps/s against
// 30.8k with the k3c kernels; 64 x 128 x 224, 1 instance: 8.0k against 2.5k.
template <typename T>
static bool sweep3p(Engine &E, const SweepField<T> *dfl, int nf, int ns_max, int t0 = 0)
{
    if (E.no_fixed_kernels || E.smem_fft || E.cluster_step || E.line_step || E.plane_p == 0) return false;
    auto run = [&](auto n1c, auto n2c, auto n3c, auto tcc) {
        constexpr int N1 = decltype(n1c)::value, N2 = decltype(n2c)::value, N3 = decltype(n3c)::value;
        constexpr int TC = decltype(tcc)::value;
        using PL = PlaneP<T, N1, N2>;
        const size_t smp = sizeof(cx<T>) * PL::PS, smz = sizeof(cx<T>) * N3 * TC;
        CK(allow_dyn_smem((const void *)k3p_fwd_pair<T, N1, N2, N3>));
        CK(allow_dyn_smem((const void *)k3p_mid<T, N1, N2, N3>));
        CK(allow_dyn_smem((const void *)k3p_final_fwd<T, N1, N2, N3>));
        CK(allow_dyn_smem((const void *)k3p_zconv<T, N1, N2, N3, TC>));
        const PlaneGeom g = E.geom();
        const unsigned ztiles = (unsigned)(PL::PS / TC);
        int dev = 0, nsm = 148;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const int pf = 2 * nsm;   // CTAs of k3p_zconv resident at once (2 per SM)
        // a small batch's fields run as two independent kernel chains (the
        // qf and qr sweeps of one instance, for instance), so that each
        // launch's last, partly empty wave overlaps the other chain's work
        const int h = (nf >= 2 && nf <= 8 && !E.no_branch) ? nf / 2 : 0;
        auto step = [&](const SweepField<T> *d, int n, cudaStream_t s, int t) {
            if (t < t0) {
                k3p_fwd_pair<T, N1, N2, N3><<<dim3(N3, n), 256, smp, s>>>(d, g, t0);
                E.launched();
                return;
            }
            k3p_zconv<T, N1, N2, N3, TC><<<dim3(ztiles, n, 2), 256, smz, s>>>(d, g, t, 3, pf);
            E.launched();
            k3p_mid<T, N1, N2, N3><<<dim3(N3, n, 2), 256, smp, s>>>(d, g, t);
            E.launched();
            k3p_zconv<T, N1, N2, N3, TC><<<dim3(ztiles, n, 1), 256, smz, s>>>(d, g, t, 2, pf);
            E.launched();
            k3p_final_fwd<T, N1, N2, N3><<<dim3(N3, n), 256, smp, s>>>(d, g, t);
            E.launched();
        };
        auto emit = [&]() {
            if (h == 0) {
                for (int t = t0 - 1; t < ns_max; t++) step(dfl, nf, E.st, t);
                return;
            }
            CK(cudaEventRecord(E.ev_fork, E.st));
            CK(cudaStreamWaitEvent(E.st2, E.ev_fork, 0));
            for (int t = t0 - 1; t < ns_max; t++) {
                step(dfl, h, E.st, t);
                step(dfl + h, nf - h, E.st2, t);
            }
            CK(cudaEventRecord(E.ev_join, E.st2));
            CK(cudaStreamWaitEvent(E.st, E.ev_join, 0));
        };
        graph_sweep(E, dfl, nf, ns_max, (int)sizeof(T), t0, emit);
    };
    const int a = E.n[0], b = E.n[1], c = E.n[2];
    if (a == 64 && b == 128 && c == 224) {
        run(std::integral_constant<int, 64>(), std::integral_constant<int, 128>(), std::integral_constant<int, 224>(),
            std::integral_constant<int, 16>());
        return true;
    }
    if (a == 64 && b == 64 && c == 64) {
        run(std::integral_constant<int, 64>(), std::integral_constant<int, 64>(), std::integral_constant<int, 64>(),
            std::integral_constant<int, 32>());
        return true;
    }
    return false;
}

// One 3-D MDE step as line passes (kernels3l.cuh), for grids with an even
// n1 whose x-y plane (or z tile) does not fit the shared memory of the
// whole-plane kernels (or with PSCFG_LINE_STEP=1).  Returns false if not
// applicable.  (Where both fit, the whole-plane kernels measured as fast or
// faster: C5-size 64 x 128 x 224 FP64 2.5k vs 2.7k steps/s, FP32 4.3k vs
// 2.8k.)
template <typename T>
static bool step3l(Engine &E, const SweepField<T> *dfl, int nf, int t)
{
    if (E.n[0] % 2 != 0) return false;
    const PlaneGeom &g = E.geom();
    const size_t smxy_plane = 2 * (size_t)g.n2 * g.LS * sizeof(cx<T>);
    const size_t smz_plane = 2 * (size_t)g.n3 * Z_TILE * sizeof(cx<T>);
    const bool plane_fits = smxy_plane <= 227 * 1024 && smz_plane <= 227 * 1024;
    if (plane_fits && !E.line_step) return false;
    const int M = g.n1 / 2, NH = M + 1;
    const long nrow = (long)g.n2 * g.n3;
    const int TLr = l3_rows_per_cta<T>(M);
    const unsigned gr = (unsigned)((nrow + TLr - 1) / TLr);
    const size_t smr = 2 * (size_t)TLr * NH * sizeof(cx<T>);
    auto lines_tl = [&](int L) { return std::max(1, std::min(32, (int)(65536 / (2 * L * (int)sizeof(cx<T>))))); };
    const int TLy = lines_tl(g.n2), TLz = lines_tl(g.n3);
    const unsigned gy = (unsigned)(((long)NH * g.n3 + TLy - 1) / TLy);
    const unsigned gz = (unsigned)(((long)NH * g.n2 + TLz - 1) / TLz);
    const size_t smy = 2 * (size_t)TLy * g.n2 * sizeof(cx<T>), smz = 2 * (size_t)TLz * g.n3 * sizeof(cx<T>);
    CK(allow_dyn_smem((const void *)k3l_rows<T, 0>));
    CK(allow_dyn_smem((const void *)k3l_rows<T, 1>));
    CK(allow_dyn_smem((const void *)k3l_rows<T, 2>));
    CK(allow_dyn_smem((const void *)k3l_lines<T>));
    auto yz = [&](int which, int nz) {
        k3l_lines<T><<<dim3(gy, nf, nz), L3_THREADS, smy, E.st>>>(dfl, g, t, 1, 0, which, TLy);
        E.launched();
        k3l_lines<T><<<dim3(gz, nf, nz), L3_THREADS, smz, E.st>>>(dfl, g, t, 2, 2, which, TLz);
        E.launched();
        k3l_lines<T><<<dim3(gy, nf, nz), L3_THREADS, smy, E.st>>>(dfl, g, t, 1, 1, which, TLy);
        E.launched();
    };
    k3l_rows<T, 0><<<dim3(gr, nf, 2), L3_THREADS, smr, E.st>>>(dfl, g, t, TLr);
    E.launched();
    yz(3, 2);
    k3l_rows<T, 1><<<dim3(gr, nf, 2), L3_THREADS, smr, E.st>>>(dfl, g, t, TLr);
    E.launched();
    yz(2, 1);
    k3l_rows<T, 2><<<dim3(gr, nf, 1), L3_THREADS, smr, E.st>>>(dfl, g, t, TLr);
    E.launched();
    return true;
}

// Returns true if the grid has a compile-time-shaped step (and runs it).
template <typename T>
static bool step3_fixed(Engine &E, const SweepField<T> *dfl, int nf, int t)
{
    if (E.no_fixed_kernels) return false;
    const int a = E.n[0], b = E.n[1], c = E.n[2];
    if (a == 32 && b == 32 && c == 32) {
        if (E.cluster_step) {
            const size_t sm = Cl32<T>::smem_bytes();
            CK(allow_dyn_smem((const void *)k3x_step32<T>));
            k3x_step32<T><<<dim3(8 * nf), 512, sm, E.st>>>(dfl, E.geom(), t);
            E.launched();
            return true;
        }
        if (E.smem_fft) step3c<T, 32, 32, 32, 8>(E, dfl, nf, t);
        else step3r<T, 32, 32, 32, 4>(E, dfl, nf, t);
        return true;
    }
    if (a == 16 && b == 16 && c == 16) {
        if (E.smem_fft) step3c<T, 16, 16, 16, 8>(E, dfl, nf, t);
        else step3r<T, 16, 16, 16, 8>(E, dfl, nf, t);
        return true;
    }
    if (a == 64 && b == 64 && c == 64) { step3c<T, 64, 64, 64, 1>(E, dfl, nf, t); return true; }
    return false;
}

template <typename T>
static void sweep_steps(Engine &E, const SweepField<T> *dfl, int nf, int t0, int t1);

template <typename T>
static void run_sweeps(Engine &E, const std::vector<int> &act)
{
    const PlaneGeom &g = E.geom();
    // tables
    std::vector<TableJob<T>> tj;
    for (int i : act) {
        Inst &I = E.inst[i];
        for (int c = 0; c < I.sys.n_chain; c++)
            for (int b = 0; b < I.sys.n_block[c]; b++) {
                TableJob<T> j;
                int m = I.sys.block_monomer[c][b];
                j.omega = I.omega + (long)m * E.nr;
                j.ksq = I.ksq;
                j.eo1 = (T *)I.eo1[c][b];
                j.eo2 = (T *)I.eo2[c][b];
                j.ek1 = (T *)I.ek1[c][b];
                j.ek2 = (T *)I.ek2[c][b];
                j.ds = I.bds[c][b];
                j.b = I.sys.kuhn[m];
                tj.push_back(j);
            }
    }
    std::vector<SweepField<T>> fl;
    int ns_max = 0;
    for (int i : act) {
        Inst &I = E.inst[i];
        for (int c = 0; c < I.sys.n_chain; c++)
            for (int d = 0; d < 2; d++) {
                SweepField<T> f;
                std::memset(&f, 0, sizeof(f));
                f.slab = (T *)(d == 0 ? I.qf[c] : I.qr[c]);
                f.ns = I.ns[c];
                f.dir = d == 0 ? 1 : -1;
                f.nblk = I.sys.n_block[c];
                for (int b = 0; b <= f.nblk; b++) f.bgn[b] = I.bgn[c][b];
                for (int b = 0; b < f.nblk; b++) {
                    f.eo1[b] = (const T *)I.eo1[c][b];
                    f.eo2[b] = (const T *)I.eo2[c][b];
                    f.ek1[b] = (const T *)I.ek1[c][b];
                    f.ek2[b] = (const T *)I.ek2[c][b];
                }
                f.S1 = (cx<T> *)I.S1[2 * c + d];
                f.S2 = (cx<T> *)I.S2[2 * c + d];
                f.q1 = (T *)I.q1[2 * c + d];
                fl.push_back(f);
                ns_max = std::max(ns_max, f.ns);
            }
    }
    if (fl.empty()) return;
    // separable k-space factors for the plane kernels when every cell of
    // the launch is orthogonal (written after the descriptors)
    // (graph-driven iterations: from the cell on the device, k_ek_factors)
    std::vector<T> ekf;
    std::vector<EkfJob> ekj;
    const int L3 = (int)(E.n[0] / 2 + 1) + E.n[1] + E.n[2];
    if (plane_kernels_apply(E)) {
        bool ortho = true;
        for (int i : act) {
            if (E.amg) {
                const int cs = E.inst[i].sys.crystal_system;
                if ((cs != PSCFG_CUBIC && cs != PSCFG_TETRAGONAL && cs != PSCFG_ORTHORHOMBIC) ||
                    i >= (int)E.amg_G.size() || !E.amg_G[i])
                    ortho = false;
            } else {
                for (int a = 0; a < 3; a++)
                    for (int b2 = 0; b2 < 3; b2++)
                        if (a != b2 && E.inst[i].cell.G[a][b2] != 0.0) ortho = false;
            }
        }
        if (ortho) {
            for (int i : act) {
                Inst &I = E.inst[i];
                for (int c = 0; c < I.sys.n_chain; c++)
                    for (int d = 0; d < 2; d++)
                        for (int b = 0; b < I.sys.n_block[c]; b++) {
                            const double kb = I.sys.kuhn[I.sys.block_monomer[c][b]];
                            if (E.amg) {
                                ekj.push_back(EkfJob{E.amg_G[i], I.bds[c][b] * kb * kb, nullptr});
                                ekf.resize(ekf.size() + 2 * (size_t)L3, (T)0);
                            } else {
                                append_ek_factors<T>(E, I.cell, I.bds[c][b] * kb * kb, ekf);
                            }
                        }
            }
        }
    }
    TableJob<T> *dtj = E.upload(tj, 0);
    size_t off = ((tj.size() * sizeof(TableJob<T>) + 255) / 256) * 256;
    if (!ekf.empty()) {
        const size_t off_tab = off + ((fl.size() * sizeof(SweepField<T>) + 255) / 256) * 256;
        const size_t off_ekj = off_tab + ((ekf.size() * sizeof(T) + 255) / 256) * 256;
        if (!E.capturing) {   // capacity first: no reallocation below
            E.desc(off_ekj + ekj.size() * sizeof(EkfJob) + 256);
            dtj = E.upload(tj, 0);
        }
        T *dtab = E.upload(ekf, off_tab);
        size_t k = 0;
        for (auto &f : fl)
            for (int b = 0; b < f.nblk; b++, k += 2 * (size_t)L3) f.ekf[b] = dtab + k;
        if (!ekj.empty()) {
            for (size_t j = 0; j < ekj.size(); j++) ekj[j].out = dtab + j * 2 * (size_t)L3;
            EkfJob *dj = E.upload(ekj, off_ekj);
            k_ek_factors<T><<<(unsigned)ekj.size(), 256, 0, E.st>>>(dj, E.n[0], E.n[1], E.n[2]);
            E.launched();
        }
    }
    SweepField<T> *dfl = E.upload(fl, off);
    {
        dim3 grid((unsigned)std::min<long>((E.nr + 255) / 256, 256), (unsigned)tj.size());
        k_make_tables<T><<<grid, 256, 0, E.st>>>(dtj, E.nr, E.nk);
        E.launched();
        dim3 g2((unsigned)std::min<long>((E.nr + 255) / 256, 256), (unsigned)fl.size());
        k_init_ends<T><<<g2, 256, 0, E.st>>>(dfl, E.nr);
        E.launched();
    }
    sweep_steps<T>(E, dfl, (int)fl.size(), 0, ns_max);
}

// Steps t in [t0, t1) of every field at dfl (t counts the steps of each
// field's own sweep, step_slices), on whichever kernels the grid has.
template <typename T>
static void sweep_steps(Engine &E, const SweepField<T> *dfl, int nf, int t0, int t1)
{
    const PlaneGeom &g = E.geom();
    const int ns_max = t1;
    if (E.dim == 2 && !E.no_fixed_kernels && E.n[0] == 64 && E.n[1] == 64) {
        // fixed-shape whole-sweep kernel: tables and q in shared memory
        const size_t sm = Sweep2P<T, 64, 64>::smem_bytes();
        CK(allow_dyn_smem((const void *)k2p_sweep<T, 64, 64>));
        k2p_sweep<T, 64, 64><<<nf, 256, sm, E.st>>>(dfl, t0, t1);
        E.launched();
        return;
    }
    if (E.dim <= 2) {
        size_t sm = 2 * (size_t)g.n2 * g.LS * sizeof(cx<T>) + 2 * (size_t)E.nr * sizeof(T);
        if (sm > 227 * 1024) throw Err(PSCFG_EINVAL, "grid too large for the single-CTA plane step");
        CK(allow_dyn_smem((const void *)k_sweep_plane<T>));
        // one CTA per field: a sweep of few fields is bound by the latency of
        // its FFT phases, which more warps hide (64 x 64 with this kernel,
        // one instance: 5.30 -> 4.28 ms per density with 512 threads instead
        // of 256; k2p_sweep above: 2.16 ms)
        int threads = (int)std::min<long>(512, std::max<long>(32, ((E.nr / 2 + 31) / 32) * 32));
        k_sweep_plane<T><<<nf, threads, sm, E.st>>>(dfl, g, t0, t1);
        E.launched();
    } else {
        size_t smxy = 2 * (size_t)g.n2 * g.LS * sizeof(cx<T>);
        size_t smz = 2 * (size_t)g.n3 * Z_TILE * sizeof(cx<T>);
        if ((smxy > 227 * 1024 || smz > 227 * 1024) && E.n[0] % 2 != 0)
            throw Err(PSCFG_EINVAL, "grid plane too large for the whole-plane kernels (odd n1)");
        CK(allow_dyn_smem((const void *)k3_fwd_pair<T>));
        CK(allow_dyn_smem((const void *)k3_inv_mid<T>));
        CK(allow_dyn_smem((const void *)k3_inv_final<T>));
        CK(allow_dyn_smem((const void *)k3_zconv<T, Z_TILE>));
        const long P = (long)g.n1h * g.n2;
        const int ntile = (int)((P + Z_TILE - 1) / Z_TILE);
        const int txy = 256, tz = 256;
        if (sweep3r<T>(E, dfl, nf, ns_max, t0)) return;
        if (sweep3p<T>(E, dfl, nf, ns_max, t0)) return;
        for (int t = t0; t < ns_max; t++) {
            if (step3_fixed<T>(E, dfl, nf, t)) continue;
            if (step3l<T>(E, dfl, nf, t)) continue;
            k3_fwd_pair<T><<<dim3(g.n3, nf), txy, smxy, E.st>>>(dfl, g, t);
            E.launched();
            k3_zconv<T, Z_TILE><<<dim3(ntile, nf, 2), tz, smz, E.st>>>(dfl, g, t, 3);
            E.launched();
            k3_inv_mid<T><<<dim3(g.n3, nf), txy, smxy, E.st>>>(dfl, g, t);
            E.launched();
            k3_zconv<T, Z_TILE><<<dim3(ntile, nf, 1), tz, smz, E.st>>>(dfl, g, t, 2);
            E.launched();
            k3_inv_final<T><<<dim3(g.n3, nf), txy, smxy, E.st>>>(dfl, g, t);
            E.launched();
        }
    }
}

// Q of every chain, solvents, Simpson density
template <typename T>
static void run_contour(Engine &E, const std::vector<int> &act)
{
    // Q = mean(qf[ns])  (src/scf_mod.fp.f90:358-360)
    std::vector<const T *> qp;
    std::vector<double *> qout;
    for (int i : act) {
        Inst &I = E.inst[i];
        for (int c = 0; c < I.sys.n_chain; c++) {
            qp.push_back((const T *)I.qf[c] + (long)(E.ckpt ? I.nseg[c] : I.ns[c]) * E.nr);
            qout.push_back(I.Qdev + c);
        }
    }
    const int nct = red_ctas(E.nr, (int)qp.size());
    size_t off = 0;
    if (!qp.empty()) {
        const T **dqp = (const T **)E.upload(qp, 0);
        off = ((qp.size() * sizeof(void *) + 255) / 256) * 256;
        double *part = E.part((size_t)nct * qp.size());
        k_partial_sum<T><<<dim3(nct, (unsigned)qp.size()), 256, 0, E.st>>>(dqp, E.nr, part);
        E.launched();
        double **dq = (double **)E.upload(qout, off);
        off += ((qout.size() * sizeof(void *) + 255) / 256) * 256;
        k_final_sum_ptr<<<(unsigned)((qp.size() + 127) / 128), 128, 0, E.st>>>(part, nct, (double)E.nr, dq, (int)qp.size());
        E.launched();
    }
    // solvents (src/scf_mod.fp.f90:193-200, 251-295): Q_s = <exp(-v w)>,
    // rho_alpha = phi_s exp(-v w)/Q_s added before the chain densities
    bool any_solvent = false, any_grand = false;
    std::vector<SolventJob> sj;
    std::vector<double *> qsout;
    for (int i : act) {
        Inst &I = E.inst[i];
        if (I.sys.ensemble == 1) any_grand = true;
        for (int s = 0; s < I.sys.n_solvent; s++) {
            SolventJob j;
            int m = I.sys.solvent_monomer[s];
            j.omega = I.omega + (long)m * E.nr;
            j.rho = I.rho + (long)m * E.nr;
            j.size = I.sys.solvent_size[s];
            j.Q = I.Qsolv + s;
            j.phi = I.sys.phi_solvent[s];
            j.mu = I.sys.mu_solvent[s];
            j.grand = I.sys.ensemble == 1;
            sj.push_back(j);
            qsout.push_back(I.Qsolv + s);
            any_solvent = true;
        }
    }
    std::vector<int> with_solvent;
    if (any_solvent) {
        for (int i : act) {
            Inst &I = E.inst[i];
            if (I.sys.n_solvent > 0) {
                k_zero<<<(unsigned)std::min<long>((E.M * E.nr + 255) / 256, 1024), 256, 0, E.st>>>(I.rho, (long)E.M * E.nr);
                E.launched();
                with_solvent.push_back(i);
            }
        }
        SolventJob *dsj0 = E.upload(sj, off);
        off += ((sj.size() * sizeof(SolventJob) + 255) / 256) * 256;
        double **dqs = (double **)E.upload(qsout, off);
        off += ((qsout.size() * sizeof(void *) + 255) / 256) * 256;
        double *part = E.part((size_t)nct * sj.size());
        k_solvent_boltz_partial<<<dim3(nct, (unsigned)sj.size()), 256, 0, E.st>>>(dsj0, E.nr, part);
        E.launched();
        k_final_sum_ptr<<<(unsigned)((sj.size() + 127) / 128), 128, 0, E.st>>>(part, nct, (double)E.nr, dqs, (int)sj.size());
        E.launched();
        k_solvent_rho<<<(unsigned)std::min<long>((E.nr + 255) / 256, 1024), 256, 0, E.st>>>(dsj0, (int)sj.size(), E.nr);
        E.launched();
    }
    // grand ensemble: phi = Q exp(mu) (mu_phi_chain/mu_phi_solvent,
    // src/scf_mod.fp.f90:202-209) is needed by the chain weights below
    // (graph-driven iterations: formed from the device Q by k_simpson)
    if (any_grand && !E.amg) {
        for (int i : act) {
            Inst &I = E.inst[i];
            if (I.sys.ensemble != 1) continue;
            CK(cudaMemcpyAsync(I.Q, I.Qdev, sizeof(double) * PSCFG_MAXC, cudaMemcpyDeviceToHost, E.st));
            CK(cudaMemcpyAsync(I.Qs, I.Qsolv, sizeof(double) * PSCFG_MAXS, cudaMemcpyDeviceToHost, E.st));
        }
        CK(cudaStreamSynchronize(E.st));
        for (int i : act) {
            Inst &I = E.inst[i];
            if (I.sys.ensemble != 1) continue;
            for (int c = 0; c < I.sys.n_chain; c++) I.sys.phi_chain[c] = I.Q[c] * std::exp(I.sys.mu_chain[c]);
            for (int s = 0; s < I.sys.n_solvent; s++) I.sys.phi_solvent[s] = I.Qs[s] * std::exp(I.sys.mu_solvent[s]);
        }
    }
    if (E.ckpt) {
        // the checkpointed density accumulates its Simpson sums segment by
        // segment (density_ckpt); start rho from the solvent part or zero
        for (int i : act) {
            Inst &I = E.inst[i];
            if (I.sys.n_solvent == 0) {
                k_zero<<<(unsigned)std::min<long>((E.M * E.nr + 255) / 256, 1024), 256, 0, E.st>>>(I.rho, (long)E.M * E.nr);
                E.launched();
            }
        }
        return;
    }
    // Simpson jobs grouped by instance
    std::vector<SimpsonJob> simp;
    std::vector<int> start;
    for (int i : act) {
        Inst &I = E.inst[i];
        start.push_back((int)simp.size());
        for (int c = 0; c < I.sys.n_chain; c++) {
            SimpsonJob j;
            std::memset(&j, 0, sizeof(j));
            j.qf = I.qf[c];
            j.qr = I.qr[c];
            j.rho = I.rho;
            j.Q = I.Qdev + c;
            j.phi = I.sys.phi_chain[c];
            j.length = I.length[c];
            j.nblk = I.sys.n_block[c];
            for (int b = 0; b <= j.nblk; b++) j.bgn[b] = I.bgn[c][b];
            for (int b = 0; b < j.nblk; b++) {
                j.mon[b] = I.sys.block_monomer[c][b];
                j.bds[b] = I.bds[c][b];
            }
            j.n_monomer = I.sys.n_monomer;
            j.accumulate = I.sys.n_solvent > 0 ? 1 : 0;
            j.grand = (E.amg && I.sys.ensemble == 1) ? 1 : 0;
            j.mu = I.sys.mu_chain[c];
            simp.push_back(j);
        }
        if (I.sys.n_chain == 0 && I.sys.n_solvent == 0)
            throw Err(PSCFG_EINVAL, "an instance needs at least one chain or solvent species");
    }
    start.push_back((int)simp.size());
    SimpsonJob *dsj = E.upload(simp, off);
    off += ((simp.size() * sizeof(SimpsonJob) + 255) / 256) * 256;
    int *dst = E.upload(start, off);
    dim3 grid((unsigned)std::min<long>((E.nr + 255) / 256, 1024), (unsigned)act.size());
    k_simpson<T><<<grid, 256, 0, E.st>>>(dsj, dst, E.nr);
    E.launched();
}


static void copy_list(Engine &E, const std::vector<CopyJob> &jobs, long maxn);
template <typename T>
static void slice_dots(Engine &E, const std::vector<StressJob<T>> &jobs);

// ---------------------------------------------------------------------
// Propagator checkpointing (PSCFG_CHECKPOINT)
// ---------------------------------------------------------------------
// A chain's slices are cut into segments [j K, min((j+1) K, ns)], j < nseg.
// qf/qr hold the checkpoint slices min(j K, ns), j = 0..nseg; a segment is
// recomputed from its checkpoint into segA (qf, upward) or segB (qr,
// downward) by the ordinary sweep kernels, through descriptors whose slab
// points K slices before the segment buffer (step_slices indexes the
// absolute slice).  A recomputed segment repeats the checkpointing pass's
// operations exactly, so it equals the slices that pass produced; against
// an uninterrupted sweep the slices agree to the last bits (a segment's
// first step starts from the checkpoint in global memory, where the fused
// sweep kernels carry it over from the previous step).
struct CkChain {
    int inst, c;
};

// the k-space tables of every block, and the separable factors of the plane
// kernels, for the chains of `act` (as run_sweeps builds them)
template <typename T>
static void ckpt_tables(Engine &E, const std::vector<int> &act, std::vector<const T *> &ekf_of)
{
    std::vector<TableJob<T>> tj;
    for (int i : act) {
        Inst &I = E.inst[i];
        for (int c = 0; c < I.sys.n_chain; c++)
            for (int b = 0; b < I.sys.n_block[c]; b++) {
                TableJob<T> j;
                int m = I.sys.block_monomer[c][b];
                j.omega = I.omega + (long)m * E.nr;
                j.ksq = I.ksq;
                j.eo1 = (T *)I.eo1[c][b];
                j.eo2 = (T *)I.eo2[c][b];
                j.ek1 = (T *)I.ek1[c][b];
                j.ek2 = (T *)I.ek2[c][b];
                j.ds = I.bds[c][b];
                j.b = I.sys.kuhn[m];
                tj.push_back(j);
            }
    }
    ekf_of.clear();
    std::vector<T> ekf;
    const int L3 = (int)(E.n[0] / 2 + 1) + E.n[1] + E.n[2];
    bool sep = plane_kernels_apply(E);
    for (int i : act)
        for (int a = 0; a < 3; a++)
            for (int b2 = 0; b2 < 3; b2++)
                if (a != b2 && E.inst[i].cell.G[a][b2] != 0.0) sep = false;
    const size_t off_tab = (size_t)6 << 20;
    if (sep) {
        for (int i : act) {
            Inst &I = E.inst[i];
            for (int c = 0; c < I.sys.n_chain; c++)
                for (int b = 0; b < I.sys.n_block[c]; b++) {
                    const double kb = I.sys.kuhn[I.sys.block_monomer[c][b]];
                    append_ek_factors<T>(E, I.cell, I.bds[c][b] * kb * kb, ekf);
                }
        }
        if (ekf.size() * sizeof(T) > ((size_t)2 << 20)) sep = false;   // keep below the geometry region
    }
    E.desc(((size_t)8 << 20) + 256);
    TableJob<T> *dtj = E.upload(tj, 0);
    dim3 grid((unsigned)std::min<long>((E.nr + 255) / 256, 256), (unsigned)tj.size());
    k_make_tables<T><<<grid, 256, 0, E.st>>>(dtj, E.nr, E.nk);
    E.launched();
    if (sep) {
        T *dtab = E.upload(ekf, off_tab);
        size_t k = 0;
        for (int i : act) {
            Inst &I = E.inst[i];
            for (int c = 0; c < I.sys.n_chain; c++) {
                ekf_of.push_back(dtab + k);
                k += (size_t)I.sys.n_block[c] * 2 * L3;
            }
        }
    }
}

// Recomputes (or, with store, computes and checkpoints) segment j of the
// chains `ch`: dir > 0 qf into segA from checkpoint j (store: its top into
// checkpoint j + 1); dir < 0 qr into segB from checkpoint j + 1 (store: its
// bottom into checkpoint j).  Chains whose nseg <= j are skipped.
template <typename T>
static void ckpt_segment(Engine &E, const std::vector<CkChain> &ch, const std::vector<const T *> &ekf_of, int j,
                         int dir, bool store)
{
    const int K = E.ckK;
    const long nr = E.nr;
    const int L3 = (int)(E.n[0] / 2 + 1) + E.n[1] + E.n[2];
    // qr segments of chains with different ns need different step ranges:
    // one launch group per ns
    std::vector<int> groups;
    for (size_t k = 0; k < ch.size(); k++) {
        const Inst &I = E.inst[ch[k].inst];
        if (j >= I.nseg[ch[k].c]) continue;
        const int key = dir > 0 ? 0 : I.ns[ch[k].c];
        if (std::find(groups.begin(), groups.end(), key) == groups.end()) groups.push_back(key);
    }
    for (int key : groups) {
        std::vector<SweepField<T>> fl;
        std::vector<CopyJob> pre, post;
        int t0 = 0, t1 = 0;
        for (size_t k = 0; k < ch.size(); k++) {
            Inst &I = E.inst[ch[k].inst];
            const int c = ch[k].c, ns = I.ns[c];
            if (j >= I.nseg[c] || (dir < 0 && ns != key)) continue;
            const int s0 = j * K, s1 = std::min((j + 1) * K, ns), len = s1 - s0;
            T *seg = (T *)(dir > 0 ? I.segA[c] : I.segB[c]);
            T *ck = (T *)(dir > 0 ? I.qf[c] : I.qr[c]);
            SweepField<T> f;
            std::memset(&f, 0, sizeof(f));
            f.slab = seg - (long)s0 * nr;   // slice s at seg + (s - s0) nr
            f.ns = ns;
            f.dir = dir;
            f.nblk = I.sys.n_block[c];
            for (int b = 0; b <= f.nblk; b++) f.bgn[b] = I.bgn[c][b];
            for (int b = 0; b < f.nblk; b++) {
                f.eo1[b] = (const T *)I.eo1[c][b];
                f.eo2[b] = (const T *)I.eo2[c][b];
                f.ek1[b] = (const T *)I.ek1[c][b];
                f.ek2[b] = (const T *)I.ek2[c][b];
                if (!ekf_of.empty()) f.ekf[b] = ekf_of[k] + (size_t)b * 2 * L3;
            }
            const int d = dir > 0 ? 0 : 1;
            f.S1 = (cx<T> *)I.S1[2 * c + d];
            f.S2 = (cx<T> *)I.S2[2 * c + d];
            f.q1 = (T *)I.q1[2 * c + d];
            fl.push_back(f);
            if (dir > 0) {
                pre.push_back(CopyJob{(const double *)(ck + (long)j * nr), (double *)seg, 0});
                if (store) post.push_back(CopyJob{(const double *)(seg + (long)len * nr), (double *)(ck + (long)(j + 1) * nr), 0});
                t0 = s0;
                t1 = std::max(t1, s1);
            } else {
                pre.push_back(CopyJob{(const double *)(ck + (long)(j + 1) * nr), (double *)(seg + (long)len * nr), 0});
                if (store) post.push_back(CopyJob{(const double *)seg, (double *)(ck + (long)j * nr), 0});
                t0 = ns - s1;
                t1 = ns - s0;
            }
        }
        if (fl.empty()) continue;
        // CopyJob counts doubles: a slice of nr T is nr * sizeof(T) / 8 doubles
        const long ncopy = nr * (long)sizeof(T) / (long)sizeof(double);
        for (auto &cj : pre) cj.n = ncopy;
        for (auto &cj : post) cj.n = ncopy;
        copy_list(E, pre, ncopy);
        SweepField<T> *dfl = E.upload(fl, 0);
        sweep_steps<T>(E, dfl, (int)fl.size(), t0, t1);
        if (store) copy_list(E, post, ncopy);
    }
}

// density() with checkpoints: qf segment by segment (checkpointing), Q and
// solvents, then from the last segment down: qf recomputed, qr propagated
// (checkpointing), and the segment's Simpson sums added to rho.
template <typename T>
static void density_ckpt(Engine &E, const std::vector<int> &act)
{
    std::vector<CkChain> ch;
    int nseg_max = 0;
    for (int i : act)
        for (int c = 0; c < E.inst[i].sys.n_chain; c++) {
            ch.push_back(CkChain{i, c});
            nseg_max = std::max(nseg_max, E.inst[i].nseg[c]);
        }
    {
        long l0 = E.launches;
        PhaseTimer pt(E, &E.t_sweep);
        std::vector<const T *> ekf_of;
        ckpt_tables<T>(E, act, ekf_of);
        // qf(0) = 1 and qr(ns) = 1: the first and the last checkpoints
        std::vector<SweepField<T>> ends;
        for (auto &k : ch) {
            Inst &I = E.inst[k.inst];
            SweepField<T> f;
            std::memset(&f, 0, sizeof(f));
            f.slab = (T *)I.qf[k.c];
            f.ns = I.nseg[k.c];
            f.dir = 1;
            ends.push_back(f);
            f.slab = (T *)I.qr[k.c];
            f.dir = -1;
            ends.push_back(f);
        }
        SweepField<T> *de = E.upload(ends, 0);
        dim3 g2((unsigned)std::min<long>((E.nr + 255) / 256, 256), (unsigned)ends.size());
        k_init_ends<T><<<g2, 256, 0, E.st>>>(de, E.nr);
        E.launched();
        for (int j = 0; j < nseg_max; j++) ckpt_segment<T>(E, ch, ekf_of, j, +1, true);
        if (E.profiling) {
            for (int i : act)
                for (int c = 0; c < E.inst[i].sys.n_chain; c++) E.n_steps_timed += 2L * E.inst[i].ns[c];
            E.sweep_launches += E.launches - l0;
        }
    }
    {
        PhaseTimer pc(E, &E.t_contour);
        run_contour<T>(E, act);   // Q from the last checkpoint, solvents, rho zeroed
    }
    {
        PhaseTimer pt(E, &E.t_sweep);
        std::vector<const T *> ekf_of;
        ckpt_tables<T>(E, act, ekf_of);
        const int K = E.ckK;
        for (int j = nseg_max - 1; j >= 0; j--) {
            ckpt_segment<T>(E, ch, ekf_of, j, +1, false);
            ckpt_segment<T>(E, ch, ekf_of, j, -1, true);
            std::vector<SimpsonSegJob> sj;
            std::vector<int> start;
            for (int i : act) {
                Inst &I = E.inst[i];
                start.push_back((int)sj.size());
                for (int c = 0; c < I.sys.n_chain; c++) {
                    if (j >= I.nseg[c]) continue;
                    SimpsonSegJob J;
                    J.qf = I.segA[c];
                    J.qr = I.segB[c];
                    J.w = I.simp_w[c];
                    J.Q = I.Qdev + c;
                    J.phi_over_L = I.sys.phi_chain[c] / I.length[c];
                    J.s0 = j * K;
                    J.s1 = (j == I.nseg[c] - 1) ? I.ns[c] + 1 : (j + 1) * K;   // each slice once
                    J.n_monomer = E.M;
                    J.rho = I.rho;
                    sj.push_back(J);
                }
            }
            start.push_back((int)sj.size());
            if (sj.empty()) continue;
            SimpsonSegJob *dsj = E.upload(sj, 0);
            const size_t o2 = ((sj.size() * sizeof(SimpsonSegJob) + 255) / 256) * 256;
            int *dst = E.upload(start, o2);
            dim3 grid((unsigned)std::min<long>((E.nr + 255) / 256, 1024), (unsigned)act.size());
            k_simpson_seg<T><<<grid, 256, 0, E.st>>>(dsj, dst, E.nr);
            E.launched();
        }
    }
}

// The stress slice sums with checkpoints: both propagators of every
// segment recomputed from their checkpoints, then slice_dots on the
// segment buffers into the slice sums of its slices.
template <typename T>
static void stress_slices_ckpt(Engine &E, const std::vector<int> &act)
{
    std::vector<CkChain> ch;
    int nseg_max = 0;
    for (int i : act)
        for (int c = 0; c < E.inst[i].sys.n_chain; c++) {
            ch.push_back(CkChain{i, c});
            nseg_max = std::max(nseg_max, E.inst[i].nseg[c]);
        }
    std::vector<const T *> ekf_of;
    ckpt_tables<T>(E, act, ekf_of);
    const int K = E.ckK;
    for (int j = 0; j < nseg_max; j++) {
        ckpt_segment<T>(E, ch, ekf_of, j, +1, false);
        ckpt_segment<T>(E, ch, ekf_of, j, -1, false);
        std::vector<StressJob<T>> jobs;
        for (auto &k : ch) {
            Inst &I = E.inst[k.inst];
            if (j >= I.nseg[k.c]) continue;
            const int s0 = j * K, s1 = std::min((j + 1) * K, I.ns[k.c]);
            StressJob<T> sjob;
            sjob.qf = (const T *)I.segA[k.c];
            sjob.qr = (const T *)I.segB[k.c];
            sjob.wdgsq = I.wdgsq;
            sjob.ncp = I.cell.ncp;
            sjob.nslices = s1 - s0 + 1;
            sjob.inc = I.inc[k.c] + (long)s0 * PSCFG_MAXCP;
            jobs.push_back(sjob);
        }
        if (!jobs.empty()) slice_dots<T>(E, jobs);
    }
}

template <typename T>
static void density_impl(Engine &E, const std::vector<int> &act)
{
    if (E.ckpt) {
        density_ckpt<T>(E, act);
        return;
    }
    {
        long l0 = E.launches;
        PhaseTimer pt(E, &E.t_sweep);
        run_sweeps<T>(E, act);
        if (E.profiling) {
            for (int i : act)
                for (int c = 0; c < E.inst[i].sys.n_chain; c++) E.n_steps_timed += 2L * E.inst[i].ns[c];
            E.sweep_launches += E.launches - l0;
        }
    }
    PhaseTimer pt(E, &E.t_contour);
    run_contour<T>(E, act);
}

static void split_prec(Engine &E, const std::vector<int> &act, std::vector<int> &a64, std::vector<int> &a32)
{
    for (int i : act) (E.inst[i].prec_now == PSCFG_FP32 ? a32 : a64).push_back(i);
}

static void density_finish(Engine &E, const std::vector<int> &act);

// One launch for a list of device copies (descriptors in their own
// region of the descriptor scratch).
static void copy_list(Engine &E, const std::vector<CopyJob> &jobs, long maxn)
{
    const unsigned gx = (unsigned)red_ctas(maxn, (int)std::min<size_t>(jobs.size(), 65535));
    for (size_t j0 = 0; j0 < jobs.size(); j0 += 65535) {
        const size_t cnt = std::min<size_t>(65535, jobs.size() - j0);
        std::vector<CopyJob> part(jobs.begin() + j0, jobs.begin() + j0 + cnt);
        CopyJob *dj = E.upload(part, E.geom_off + ((size_t)2 << 20));
        k_copy_list<<<dim3(gx, (unsigned)cnt), 256, 0, E.st>>>(dj);
        E.launched();
    }
}

static void density_all(Engine &E, const std::vector<int> &act, bool finish = true)
{
    std::vector<int> a64, a32;
    split_prec(E, act, a64, a32);
    if (!a64.empty()) {
        E.cur = PSCFG_FP64;
        density_impl<double>(E, a64);
    }
    if (!a32.empty()) {
        E.cur = PSCFG_FP32;
        density_impl<float>(E, a32);
    }
    // pull Q to the host (needed for mu and for the caller): gathered on the
    // device, one copy into the pinned staging buffer; finish = false leaves
    // the synchronisation and density_finish to the caller
    if (E.amg) {   // graph-driven iterations: Q stays on the device (k_amg_finish)
        for (int i : act) {
            E.inst[i].have_density = true;
            E.inst[i].dens_prec = E.inst[i].prec_now;
        }
        return;
    }
    std::vector<CopyJob> cj;
    for (int i : act) {
        Inst &I = E.inst[i];
        cj.push_back(CopyJob{I.Qdev, E.dstage + (size_t)i * 16, PSCFG_MAXC});
        cj.push_back(CopyJob{I.Qsolv, E.dstage + (size_t)i * 16 + 8, PSCFG_MAXS});
        I.have_density = true;
        I.dens_prec = I.prec_now;
    }
    copy_list(E, cj, 8);
    CK(cudaMemcpyAsync(E.hq(0), E.dstage, sizeof(double) * 16 * E.hpin_inst, cudaMemcpyDeviceToHost, E.st));
    if (finish) {
        CK(cudaStreamSynchronize(E.st));
        density_finish(E, act);
    }
}

// Q, Q_solvent from the staging buffer, then mu_phi_chain / mu_phi_solvent.
static void density_finish(Engine &E, const std::vector<int> &act)
{
    for (int i : act) {
        Inst &I = E.inst[i];
        std::memcpy(I.Q, E.hq(i), sizeof(double) * PSCFG_MAXC);
        std::memcpy(I.Qs, E.hq(i) + 8, sizeof(double) * PSCFG_MAXS);
        // mu_phi_chain / mu_phi_solvent (src/scf_mod.fp.f90:768-820)
        for (int c = 0; c < I.sys.n_chain; c++) {
            if (I.sys.ensemble == 0) I.sys.mu_chain[c] = std::log(I.sys.phi_chain[c] / I.Q[c]);
            else I.sys.phi_chain[c] = I.Q[c] * std::exp(I.sys.mu_chain[c]);
        }
        for (int s = 0; s < I.sys.n_solvent; s++) {
            if (I.sys.ensemble == 0) I.sys.mu_solvent[s] = std::log(I.sys.phi_solvent[s] / I.Qs[s]);
            else I.sys.phi_solvent[s] = I.Qs[s] * std::exp(I.sys.mu_solvent[s]);
        }
    }
}

// ---------------------------------------------------------------------
// Stress
// ---------------------------------------------------------------------
template <typename T, int N1, int N2, int N3, int PPC>
static void stress3c(Engine &E, const StressJob<T> *dj, int s0, int cnt)
{
    constexpr int TC = 16;
    constexpr int P = N2 * (N1 / 2 + 1);
    const int ntile = (P + TC - 1) / TC;
    const PlaneGeom &g = E.geom();
    const size_t sm = sizeof(cx<T>) * PPC * P;
    CK(allow_dyn_smem((const void *)k3c_stress_xy<T, N1, N2, N3, PPC>));
    k3c_stress_xy<T, N1, N2, N3, PPC><<<dim3(N3 / PPC, cnt, 2), 256, sm, E.st>>>(dj, g, s0, (cx<T> *)E.spec);
    E.launched();
    k3c_stress_z<T, N1, N2, N3, TC><<<dim3(ntile, cnt), 256, 0, E.st>>>(dj, g, s0, (const cx<T> *)E.spec, E.stress_part);
    E.launched();
    k3_stress_sum<T><<<cnt, 32, 0, E.st>>>(dj, s0, ntile, E.stress_part);
    E.launched();
}

// Stress slice sums with the register-column kernels (N3 <= 32).
template <typename T, int N1, int N2, int N3, int PPC>
static void stress3r(Engine &E, const StressJob<T> *dj, int s0, int cnt)
{
    constexpr int P = N2 * (N1 / 2 + 1);
    const int ntile = (P + 63) / 64;
    const size_t sm = sizeof(cx<T>) * PPC * P;
    CK(allow_dyn_smem((const void *)k3r_stress_xy<T, N1, N2, N3, PPC>));
    k3r_stress_xy<T, N1, N2, N3, PPC><<<dim3(N3 / PPC, cnt, 2), 128, sm, E.st>>>(dj, s0, (cx<T> *)E.spec);
    E.launched();
    k3s_stress_z<T, N1, N2, N3><<<dim3(ntile, cnt), 128, 0, E.st>>>(dj, s0, (const cx<T> *)E.spec, E.stress_part);
    E.launched();
    k3_stress_sum<T><<<cnt, 32, 0, E.st>>>(dj, s0, ntile, E.stress_part);
    E.launched();
}

// The stress slice pass with the plane kernels (kernels3p.cuh), for the
// shapes whose sweep uses them.
template <typename T, int N1, int N2, int N3, int TC>
static void stress3p(Engine &E, const StressJob<T> *dj, int s0, int cnt)
{
    using PL = PlaneP<T, N1, N2>;
    const size_t smp = sizeof(cx<T>) * PL::PS, smz = 2 * sizeof(cx<T>) * N3 * TC;
    CK(allow_dyn_smem((const void *)k3p_stress_xy<T, N1, N2, N3>));
    CK(allow_dyn_smem((const void *)k3p_stress_z<T, N1, N2, N3, TC>));
    const int ntile = PL::PS / TC;
    k3p_stress_xy<T, N1, N2, N3><<<dim3(N3, cnt, 2), 256, smp, E.st>>>(dj, s0, (cx<T> *)E.spec);
    E.launched();
    k3p_stress_z<T, N1, N2, N3, TC><<<dim3(ntile, cnt), 256, smz, E.st>>>(dj, s0, (const cx<T> *)E.spec, E.stress_part);
    E.launched();
    k3_stress_sum<T><<<cnt, 32, 0, E.st>>>(dj, s0, ntile, E.stress_part);
    E.launched();
}

template <typename T>
static bool stress3_fixed(Engine &E, const StressJob<T> *dj, int s0, int cnt)
{
    if (E.no_fixed_kernels) return false;
    const int a = E.n[0], b = E.n[1], c = E.n[2];
    const bool pk = !(E.smem_fft || E.cluster_step || E.line_step || E.plane_p == 0);
    if (pk && a == 64 && b == 128 && c == 224) { stress3p<T, 64, 128, 224, 8>(E, dj, s0, cnt); return true; }
    if (pk && a == 64 && b == 64 && c == 64) { stress3p<T, 64, 64, 64, 16>(E, dj, s0, cnt); return true; }
    if (a == 32 && b == 32 && c == 32) {
        if (E.smem_fft) stress3c<T, 32, 32, 32, 8>(E, dj, s0, cnt);
        else stress3r<T, 32, 32, 32, 4>(E, dj, s0, cnt);
        return true;
    }
    if (a == 16 && b == 16 && c == 16) {
        if (E.smem_fft) stress3c<T, 16, 16, 16, 8>(E, dj, s0, cnt);
        else stress3r<T, 16, 16, 16, 8>(E, dj, s0, cnt);
        return true;
    }
    if (a == 64 && b == 64 && c == 64) { stress3c<T, 64, 64, 64, 1>(E, dj, s0, cnt); return true; }
    return false;
}

// Per slice s of every job: inc[s][b] = sum_k wdgsq_b(k) Re(F[qf_s] conj F[qr_s])
// on the half spectrum (the stress slice sums; also the adjoint's cell pairs).
// All jobs of slice_dots in batched launches with the register-column
// kernels (16^3, 32^3).  Returns false where they do not apply.
template <typename T>
static bool slice_dots_r(Engine &E, const StressJob<T> *dj, int njobs, int maxs)
{
    if (E.no_fixed_kernels || E.smem_fft || E.dim != 3) return false;
    auto run = [&](auto n1c, auto ppcc) {
        constexpr int N = decltype(n1c)::value, PPC = decltype(ppcc)::value;
        constexpr int P = N * (N / 2 + 1);
        const int ntile = (P + 63) / 64;
        const size_t per_slice = 2 * (size_t)E.nk * sizeof(cx<T>);
        const int cs = (int)std::max<size_t>(1, std::min<size_t>((size_t)maxs, ((size_t)1 << 30) / (per_slice * njobs)));
        if (E.spec_bytes < per_slice * cs * njobs) {
            E.no_growth_in_capture();
            if (E.spec) cudaFree(E.spec);
            E.spec = nullptr;
            CK(cudaMalloc(&E.spec, per_slice * cs * njobs));
            E.spec_bytes = per_slice * cs * njobs;
        }
        const size_t plen = (size_t)cs * njobs * ntile * PSCFG_MAXCP;
        if (E.stress_part_len < plen) {
            E.no_growth_in_capture();
            if (E.stress_part) cudaFree(E.stress_part);
            E.stress_part = nullptr;
            CK(cudaMalloc(&E.stress_part, plen * sizeof(double)));
            E.stress_part_len = plen;
        }
        const size_t sm = sizeof(cx<T>) * PPC * P;
        CK(allow_dyn_smem((const void *)k3r_stress_xy_b<T, N, N, N, PPC>));
        for (int s0 = 0; s0 < maxs; s0 += cs) {
            const int cnt = std::min(cs, maxs - s0);
            k3r_stress_xy_b<T, N, N, N, PPC><<<dim3(N / PPC, cnt, 2 * njobs), 128, sm, E.st>>>(dj, s0, cs, (cx<T> *)E.spec);
            E.launched();
            k3s_stress_z_b<T, N, N, N><<<dim3(ntile, cnt, njobs), 128, 0, E.st>>>(dj, s0, cs, (const cx<T> *)E.spec,
                                                                                   E.stress_part);
            E.launched();
            k3_stress_sum_b<T><<<dim3(cnt, njobs), 32, 0, E.st>>>(dj, s0, cs, ntile, E.stress_part);
            E.launched();
        }
    };
    const int a = E.n[0], b = E.n[1], c = E.n[2];
    if (2 * njobs > 65535) return false;
    if (a == 32 && b == 32 && c == 32) {
        run(std::integral_constant<int, 32>(), std::integral_constant<int, 4>());
        return true;
    }
    if (a == 16 && b == 16 && c == 16) {
        run(std::integral_constant<int, 16>(), std::integral_constant<int, 8>());
        return true;
    }
    return false;
}

template <typename T>
static void slice_dots(Engine &E, const std::vector<StressJob<T>> &jobs)
{
    const PlaneGeom &g = E.geom();
    if (jobs.empty()) return;
    StressJob<T> *dj = E.upload(jobs, 0);
    {
        int maxs = 0;
        for (auto &j : jobs) maxs = std::max(maxs, j.nslices);
        if (slice_dots_r<T>(E, dj, (int)jobs.size(), maxs)) return;
    }
    size_t off = ((jobs.size() * sizeof(StressJob<T>) + 255) / 256) * 256;
    if (E.dim <= 2) {
        int maxs = 0;
        for (auto &j : jobs) maxs = std::max(maxs, j.nslices);
        size_t sm = 4 * (size_t)g.n2 * g.LS * sizeof(cx<T>);
        if (sm > 227 * 1024) throw Err(PSCFG_EINVAL, "grid too large for the plane stress kernel");
        CK(allow_dyn_smem((const void *)k2_stress_slices<T>));
        int threads = (int)std::min<long>(256, std::max<long>(32, ((E.nr / 2 + 31) / 32) * 32));
        k2_stress_slices<T><<<dim3(maxs, (unsigned)jobs.size()), threads, sm, E.st>>>(dj, g);
        E.launched();
    } else {
        const long P = (long)g.n1h * g.n2;
        const int ntile = (int)((P + Z_TILE - 1) / Z_TILE);
        size_t smxy = 2 * (size_t)g.n2 * g.LS * sizeof(cx<T>);
        size_t smz = 4 * (size_t)g.n3 * Z_TILE * sizeof(cx<T>);
        CK(allow_dyn_smem((const void *)k3_stress_xy<T>));
        CK(allow_dyn_smem((const void *)k3_stress_z<T, Z_TILE>));
        // chunk of slices so that the spectra scratch stays below ~1 GB
        const size_t per_slice = 2 * (size_t)E.nk * sizeof(cx<T>);
        int cs = (int)std::max<size_t>(1, std::min<size_t>(256, ((size_t)1 << 30) / per_slice));
        if (E.spec_bytes < per_slice * cs) {
            E.no_growth_in_capture();
            if (E.spec) cudaFree(E.spec);
            E.spec = nullptr;
            CK(cudaMalloc(&E.spec, per_slice * cs));
            E.spec_bytes = per_slice * cs;
        }
        // partial sums per (slice, column tile): the plane kernels' stress
        // pass (stress3p) tiles by 8 columns, the generic one by Z_TILE
        const long ntile_max = std::max<long>(ntile, (P + 7) / 8);
        size_t plen = (size_t)cs * ntile_max * PSCFG_MAXCP;
        if (E.stress_part_len < plen) {
            E.no_growth_in_capture();
            if (E.stress_part) cudaFree(E.stress_part);
            E.stress_part = nullptr;
            CK(cudaMalloc(&E.stress_part, plen * sizeof(double)));
            E.stress_part_len = plen;
        }
        for (size_t jb = 0; jb < jobs.size(); jb++) {
            for (int s0 = 0; s0 < jobs[jb].nslices; s0 += cs) {
                int cnt = std::min(cs, jobs[jb].nslices - s0);
                if (stress3_fixed<T>(E, dj + jb, s0, cnt)) continue;
                k3_stress_xy<T><<<dim3(g.n3, cnt, 2), 256, smxy, E.st>>>(dj + jb, g, s0, (cx<T> *)E.spec);
                E.launched();
                k3_stress_z<T, Z_TILE><<<dim3(ntile, cnt), 256, smz, E.st>>>(dj + jb, g, s0, (const cx<T> *)E.spec, E.stress_part);
                E.launched();
                k3_stress_sum<T><<<cnt, 32, 0, E.st>>>(dj + jb, s0, ntile, E.stress_part);
                E.launched();
            }
        }
    }
}

template <typename T>
static void stress_impl(Engine &E, const std::vector<int> &act)
{
    const PlaneGeom &g = E.geom();
    std::vector<StressJob<T>> jobs;
    if (E.ckpt) stress_slices_ckpt<T>(E, act);
    for (int i : act) {
        Inst &I = E.inst[i];
        for (int c = 0; c < I.sys.n_chain; c++) {
            StressJob<T> j;
            j.qf = (const T *)I.qf[c];
            j.qr = (const T *)I.qr[c];
            j.wdgsq = I.wdgsq;
            j.ncp = I.cell.ncp;
            j.nslices = I.ns[c] + 1;
            j.inc = I.inc[c];
            jobs.push_back(j);
        }
    }
    if (jobs.empty()) return;
    if (!E.ckpt) slice_dots<T>(E, jobs);
    const size_t off = ((jobs.size() * sizeof(StressJob<T>) + 255) / 256) * 256;
    std::vector<StressFinal> fin;
    for (int i : act) {
        Inst &I = E.inst[i];
        StressFinal f;
        std::memset(&f, 0, sizeof(f));
        f.nchain = I.sys.n_chain;
        f.ncp = I.cell.ncp;
        f.ensemble = I.sys.ensemble;
        f.Q = I.Qdev;
        f.rnodes = (double)E.nr;
        f.out = I.stress_dev;
        for (int c = 0; c < I.sys.n_chain; c++) {
            f.inc[c] = I.inc[c];
            f.nblk[c] = I.sys.n_block[c];
            for (int b = 0; b <= f.nblk[c]; b++) f.bgn[c][b] = I.bgn[c][b];
            for (int b = 0; b < f.nblk[c]; b++) {
                f.bds[c][b] = I.bds[c][b];
                f.b[c][b] = I.sys.kuhn[I.sys.block_monomer[c][b]];
            }
            f.phi[c] = I.sys.phi_chain[c];
            f.mu[c] = I.sys.mu_chain[c];
            f.length[c] = I.length[c];
        }
        fin.push_back(f);
    }
    StressFinal *df = E.upload(fin, off);
    k_stress_final<<<(unsigned)((fin.size() + 63) / 64), 64, 0, E.st>>>(df, (int)fin.size());
    E.launched();
}

static void stress_all(Engine &E, const std::vector<int> &act)
{
    for (int i : act)
        if (!E.inst[i].have_density) throw Err(PSCFG_ESTATE, "stress requires a preceding density call");
    PhaseTimer pt(E, &E.t_stress);
    std::vector<int> a64, a32;
    split_prec(E, act, a64, a32);
    if (!a64.empty()) {
        E.cur = PSCFG_FP64;
        stress_impl<double>(E, a64);
    }
    if (!a32.empty()) {
        E.cur = PSCFG_FP32;
        stress_impl<float>(E, a32);
    }
}

// ---------------------------------------------------------------------
// Free energy (src/scf_mod.fp.f90:834-886)
// ---------------------------------------------------------------------
// Field term sum_k w r [..] / nr^2 for instances with star weights, from
// the spectra of rho and omega (FP64 forward FFTs).
static void fe_spectral(Engine &E, const std::vector<int> &which, double *hout, bool dev_out = false)
{
    const PlaneGeom &g = E.g64;
    const int M = E.M;
    const size_t per = (size_t)2 * M * E.nk * sizeof(cx<double>);
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>(which.size(), ((size_t)512 << 20) / per));
    if (E.fe_spec_bytes < per * chunk) {
        E.no_growth_in_capture();
        if (E.fe_spec) cudaFree(E.fe_spec);
        E.fe_spec = nullptr;
        CK(cudaMalloc(&E.fe_spec, per * chunk));
        E.fe_spec_bytes = per * chunk;
    }
    const int nct = red_ctas(E.nk, (int)std::min<size_t>(chunk, which.size()));
    for (size_t c0 = 0; c0 < which.size(); c0 += chunk) {
        const int cn = (int)std::min<size_t>(chunk, which.size() - c0);
        std::vector<const double *> src;
        std::vector<cx<double> *> dst;
        std::vector<FeSpecJob> jobs;
        cx<double> *base = (cx<double> *)E.fe_spec;
        for (int k = 0; k < cn; k++) {
            Inst &I = E.inst[which[c0 + k]];
            FeSpecJob j;
            std::memset(&j, 0, sizeof(j));
            for (int a = 0; a < M; a++) {
                cx<double> *R = base + ((size_t)k * 2 * M + a) * E.nk;
                cx<double> *W = base + ((size_t)k * 2 * M + M + a) * E.nk;
                src.push_back(I.rho + (long)a * E.nr);
                dst.push_back(R);
                src.push_back(I.omega + (long)a * E.nr);
                dst.push_back(W);
                j.R[a] = R;
                j.W[a] = W;
            }
            j.kweight = I.kweight;
            j.M = M;
            for (int a = 0; a < M; a++)
                for (int b = 0; b < M; b++) j.chi[a][b] = I.sys.chi[a][b];
            jobs.push_back(j);
        }
        const double **dsrc = (const double **)E.upload(src, 0);
        size_t off = ((src.size() * sizeof(void *) + 255) / 256) * 256;
        cx<double> **ddst = (cx<double> **)E.upload(dst, off);
        off += ((dst.size() * sizeof(void *) + 255) / 256) * 256;
        FeSpecJob *dj = E.upload(jobs, off);
        const int nf = (int)src.size();
        size_t smxy = 2 * (size_t)g.n2 * g.LS * sizeof(cx<double>);
        if (E.dim <= 2) {
            CK(allow_dyn_smem((const void *)k2_fft_fields));
            int threads = (int)std::min<long>(256, std::max<long>(32, ((E.nr / 2 + 31) / 32) * 32));
            k2_fft_fields<<<nf, threads, smxy, E.st>>>(dsrc, ddst, g);
            E.launched();
        } else {
            const long P = (long)g.n1h * g.n2;
            const int ntile = (int)((P + Z_TILE - 1) / Z_TILE);
            size_t smz = 2 * (size_t)g.n3 * Z_TILE * sizeof(cx<double>);
            CK(allow_dyn_smem((const void *)k3_fft_fields_xy));
            CK(allow_dyn_smem((const void *)k3_fft_fields_z<Z_TILE>));
            k3_fft_fields_xy<<<dim3(g.n3, nf), 256, smxy, E.st>>>(dsrc, ddst, g);
            E.launched();
            k3_fft_fields_z<Z_TILE><<<dim3(ntile, nf), 256, smz, E.st>>>(ddst, g);
            E.launched();
        }
        double *part = E.part((size_t)nct * cn);
        k_fe_spectral<<<dim3(nct, cn), 256, 0, E.st>>>(dj, E.nk, E.n[0], part);
        E.launched();
        const double rn2 = (double)E.nr * (double)E.nr;
        k_final_sum<<<(unsigned)((cn + 127) / 128), 128, 0, E.st>>>(part, nct, rn2, E.d_small, cn);
        E.launched();
        CK(cudaMemcpyAsync(hout + c0, E.d_small, sizeof(double) * cn,
                           dev_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, E.st));
    }
}

// Instances without star weights first (real-space field terms), then
// those with star weights (spectral), in act order within each group.
static void fe_partition(Engine &E, const std::vector<int> &act, std::vector<size_t> &pos_plain,
                         std::vector<size_t> &pos_w)
{
    for (size_t k = 0; k < act.size(); k++) (E.inst[act[k]].kweight ? pos_w : pos_plain).push_back(k);
}

static void fe_finish(Engine &E, const std::vector<int> &act, std::vector<double> &f, std::vector<double> &p);

// Field terms of the free energy into the staging buffer; with finish, the
// synchronisation and the assembly (fe_finish) follow.  dterms (device):
// the terms go there instead, plain instances first, in act order, then
// the star-weighted ones (graph-driven iterations).
static void free_energy_all(Engine &E, const std::vector<int> &act, std::vector<double> &f, std::vector<double> &p,
                            bool finish = true, double *dterms = nullptr)
{
    std::vector<size_t> pos_plain, pos_w;
    fe_partition(E, act, pos_plain, pos_w);
    double *hfe = dterms ? dterms : E.hfe();
    const cudaMemcpyKind kind = dterms ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (!pos_plain.empty()) {
        std::vector<FieldJob> fj;
        for (size_t k : pos_plain) {
            Inst &I = E.inst[act[k]];
            FieldJob j;
            std::memset(&j, 0, sizeof(j));
            j.omega = I.omega;
            j.rho = I.rho;
            j.M = I.sys.n_monomer;
            for (int a = 0; a < j.M; a++)
                for (int b = 0; b < j.M; b++) j.chi[a][b] = I.sys.chi[a][b];
            fj.push_back(j);
        }
        FieldJob *dj = E.upload(fj, 0);
        const int nct = red_ctas(E.nr, (int)fj.size());
        double *part = E.part((size_t)nct * fj.size());
        k_fe_partial<<<dim3(nct, (unsigned)fj.size()), 256, 0, E.st>>>(dj, E.nr, part);
        E.launched();
        k_final_sum<<<(unsigned)((fj.size() + 127) / 128), 128, 0, E.st>>>(part, nct, (double)E.nr, E.d_small, (int)fj.size());
        E.launched();
        CK(cudaMemcpyAsync(hfe, E.d_small, sizeof(double) * fj.size(), kind, E.st));
    }
    if (!pos_w.empty()) {
        std::vector<int> weighted;
        for (size_t k : pos_w) weighted.push_back(act[k]);
        fe_spectral(E, weighted, hfe + pos_plain.size(), dterms != nullptr);
    }
    if (finish && !dterms) {
        CK(cudaStreamSynchronize(E.st));
        fe_finish(E, act, f, p);
    }
}

// f_Helmholtz and pressure (src/scf_mod.fp.f90:834-886) from the staged
// field terms and the host mu / phi.
static void fe_finish(Engine &E, const std::vector<int> &act, std::vector<double> &f, std::vector<double> &p)
{
    std::vector<size_t> pos_plain, pos_w;
    fe_partition(E, act, pos_plain, pos_w);
    std::vector<double> terms(act.size(), 0.0);
    const double *hfe = E.hfe();
    for (size_t k = 0; k < pos_plain.size(); k++) terms[pos_plain[k]] = hfe[k];
    for (size_t k = 0; k < pos_w.size(); k++) terms[pos_w[k]] = hfe[pos_plain.size() + k];
    f.assign(act.size(), 0.0);
    p.assign(act.size(), 0.0);
    for (size_t k = 0; k < act.size(); k++) {
        Inst &I = E.inst[act[k]];
        double fe = 0.0;
        for (int c = 0; c < I.sys.n_chain; c++)
            if (I.sys.phi_chain[c] > 1.0e-8) fe = fe + I.sys.phi_chain[c] * (I.sys.mu_chain[c] - 1.0) / I.length[c];
        for (int s = 0; s < I.sys.n_solvent; s++)
            if (I.sys.phi_solvent[s] > 1.0e-8)
                fe = fe + I.sys.phi_solvent[s] * (I.sys.mu_solvent[s] - 1.0) / I.sys.solvent_size[s];
        fe += terms[k];
        double pr = -fe;
        for (int c = 0; c < I.sys.n_chain; c++)
            if (I.sys.phi_chain[c] > 1.0e-8) pr = pr + I.sys.mu_chain[c] * I.sys.phi_chain[c] / I.length[c];
        for (int s = 0; s < I.sys.n_solvent; s++)
            if (I.sys.phi_solvent[s] > 1.0e-8) pr = pr + I.sys.mu_solvent[s] * I.sys.phi_solvent[s] / I.sys.solvent_size[s];
        f[k] = fe;
        p[k] = pr;
    }
}

// ---------------------------------------------------------------------
// Anderson mixing (src/iterate_mod.fp.f90:1042-1490)
// ---------------------------------------------------------------------
struct AmState {
    int itr = 0;
    int itr_fp32 = 0;          // iterations run with FP32 propagation
    double best = INFINITY;    // best FP32 error so far (stall detection)
    int since_best = 0;
    bool done = false;
    bool converged = false;
    double error = 0;
    int status = PSCFG_AM_RUNNING;
    int k0 = 0;                // iteration of the last history restart (lambda ramp origin)
    double best_run = INFINITY; // best error since the last restart
    int nstore = 0;            // number of valid history entries (<= H+1)
    int head = 0;              // ring slot of the most recent entry
    std::vector<double> gram;  // (H+1)x(H+1) ring-indexed <d_i, d_j>
    std::vector<std::vector<double>> devcp, cph;  // [H+1][ncp]
    double f = 0, p = 0;
    double stress[PSCFG_MAXCP] = {};
};

static bool solve_dense(int n, std::vector<double> &U, std::vector<double> &v)
{
    for (int c = 0; c < n; c++) {
        int p = c;
        for (int r = c + 1; r < n; r++)
            if (std::fabs(U[r * n + c]) > std::fabs(U[p * n + c])) p = r;
        if (U[p * n + c] == 0.0) return false;
        if (p != c) {
            for (int k = 0; k < n; k++) std::swap(U[c * n + k], U[p * n + k]);
            std::swap(v[c], v[p]);
        }
        for (int r = c + 1; r < n; r++) {
            double f = U[r * n + c] / U[c * n + c];
            for (int k = c; k < n; k++) U[r * n + k] -= f * U[c * n + k];
            v[r] -= f * v[c];
        }
    }
    for (int r = n - 1; r >= 0; r--) {
        double s = v[r];
        for (int k = r + 1; k < n; k++) s -= U[r * n + k] * v[k];
        v[r] = s / U[r * n + r];
    }
    return true;
}

struct AmRun {
    bool active = false;
    pscfg_am_param prm;
    std::vector<AmState> st;
    // graph-driven iterations (prm.graph_check > 0): device state and the
    // per-act-position job arrays the device control kernels write
    bool graph = false;
    int g_ninst = 0;
    AmgInst *g_st = nullptr;
    int *g_act = nullptr, *g_tidx = nullptr;
    double *g_terms = nullptr;
    AmJob *g_aj = nullptr;
    AmFix *g_fx = nullptr;
    AmDot *g_dots = nullptr;
    AmMix *g_mix = nullptr;
    CopyJob *g_hc = nullptr;
    GeomJob *g_geo = nullptr;
    SymJob *g_sym = nullptr;
    int g_maxorb = 0;
    std::vector<int> g_cap;         // instances of the captured iteration
    long g_launches = 0;            // kernel launches per replay
    std::vector<AmgInst> g_host;    // read-back mirror
};

static int am_iterate_graph(Engine &E, AmRun &R, int iters);
static void amg_alloc(Engine &E, AmRun &R);
static void amg_init(Engine &E, AmRun &R);
static void amg_drop_graph(Engine &E);

// Space-group projection of omega for the given instances, in place.
static void symmetrize_omega(Engine &E, const std::vector<int> &which)
{
    std::vector<SymJob> jobs;
    int maxorb = 0;
    for (int i : which) {
        Inst &I = E.inst[i];
        if (I.nops <= 0) continue;
        SymJob j;
        std::memset(&j, 0, sizeof(j));
        j.f = I.omega;
        j.perm = I.d_orb_perm;
        j.start = I.d_orb_start;
        j.norb = I.norb;
        j.M = E.M;
        jobs.push_back(j);
        maxorb = std::max(maxorb, I.norb);
    }
    if (jobs.empty()) return;
    SymJob *dj = E.upload(jobs, E.geom_off + ((size_t)1 << 20));
    dim3 grid((unsigned)std::max(1, std::min((maxorb + 127) / 128, 256)), (unsigned)jobs.size());
    k_symmetrize<<<grid, 128, 0, E.st>>>(dj, E.nr);
    E.launched();
}

static void am_begin(Engine &E, AmRun &R, const pscfg_am_param &prm)
{
    const int H = prm.n_hist;
    if (H < 1 || H > PSCFG_MAXH - 1) throw Err(PSCFG_EINVAL, "n_hist out of range");
    if (prm.max_itr < 0) throw Err(PSCFG_EINVAL, "max_itr must be >= 0");
    if (prm.graph_check < 0) throw Err(PSCFG_EINVAL, "graph_check must be >= 0");
    if (prm.graph_check > 0 && (E.prec != PSCFG_FP64 || E.ckpt))
        throw Err(PSCFG_EINVAL, "graph_check needs an FP64 engine without PSCFG_CHECKPOINT");
    amg_drop_graph(E);
    const int S = H + 1;
    const long fl = (long)E.M * E.nr;
    const int ninst = (int)E.inst.size();
    if (E.n_hist_alloc < S) {
        for (auto &I : E.inst) {
            I.om_hist = (double *)E.dalloc(sizeof(double) * fl * S);
            I.dev_hist = (double *)E.dalloc(sizeof(double) * fl * S);
        }
        E.n_hist_alloc = S;
    }
    R.prm = prm;
    R.st.assign(ninst, AmState());
    for (auto &I : E.inst) I.prec_now = (E.prec == PSCFG_FP64) ? PSCFG_FP64 : PSCFG_FP32;
    std::vector<int> all(ninst);
    for (int i = 0; i < ninst; i++) all[i] = i;
    // symmetric initial guess, then the first density (src/iterate_mod.fp.f90:1123)
    symmetrize_omega(E, all);
    density_all(E, all);
    // uniform component of omega (set_omega_uniform, src/scf_mod.fp.f90:724-750)
    std::vector<double> w(fl);
    for (int i = 0; i < ninst; i++) {
        Inst &I = E.inst[i];
        CK(cudaMemcpyAsync(w.data(), I.omega, sizeof(double) * fl, cudaMemcpyDeviceToHost, E.st));
        CK(cudaStreamSynchronize(E.st));
        double phi_mon[PSCFG_MAXM] = {0};
        for (int c = 0; c < I.sys.n_chain; c++)
            for (int b = 0; b < I.sys.n_block[c]; b++)
                phi_mon[I.sys.block_monomer[c][b]] += I.sys.phi_chain[c] * I.sys.block_length[c][b] / I.length[c];
        for (int sv = 0; sv < I.sys.n_solvent; sv++) phi_mon[I.sys.solvent_monomer[sv]] += I.sys.phi_solvent[sv];
        for (int a = 0; a < E.M && I.sys.ensemble == 0; a++) {
            double w0 = 0;
            for (int b = 0; b < E.M; b++) w0 = w0 + I.sys.chi[a][b] * phi_mon[b];
            double m = 0;
            for (long r = 0; r < E.nr; r++) m += w[a * E.nr + r];
            m /= (double)E.nr;
            for (long r = 0; r < E.nr; r++) w[a * E.nr + r] += w0 - m;
        }
        CK(cudaMemcpyAsync(I.omega, w.data(), sizeof(double) * fl, cudaMemcpyHostToDevice, E.st));
        CK(cudaMemcpyAsync(I.om_hist, I.omega, sizeof(double) * fl, cudaMemcpyDeviceToDevice, E.st));
        AmState &st = R.st[i];
        st.gram.assign((size_t)S * S, 0.0);
        st.devcp.assign(S, std::vector<double>(PSCFG_MAXCP, 0.0));
        st.cph.assign(S, std::vector<double>(PSCFG_MAXCP, 0.0));
        for (int k = 0; k < I.cell.ncp; k++) st.cph[0][k] = I.sys.cell_param[k];
        st.head = 0;
        st.nstore = 0;
    }
    CK(cudaStreamSynchronize(E.st));
    R.graph = prm.graph_check > 0;
    R.g_cap.clear();
    if (R.graph) {
        amg_alloc(E, R);
        amg_init(E, R);
    }
    R.active = true;
}

// Up to `iters` Anderson iterations of every unfinished instance; returns
// the number of instances still iterating.
static int am_iterate(Engine &E, AmRun &R, int iters)
{
    if (!R.active) throw Err(PSCFG_ESTATE, "no Anderson run in progress");
    if (R.graph) return am_iterate_graph(E, R, iters);
    const pscfg_am_param &prm = R.prm;
    const int H = prm.n_hist, S = H + 1;
    const long fl = (long)E.M * E.nr;
    const int ninst = (int)E.inst.size();
    const double large = 100.0;
    std::vector<AmState> &st = R.st;
    std::vector<double> hsmall;
    int remaining = 0;
    for (int it = 0; it < iters; it++) {
        std::vector<int> act;
        for (int i = 0; i < ninst; i++)
            if (!st[i].done) act.push_back(i);
        remaining = (int)act.size();
        if (act.empty()) break;
        const int na = (int)act.size();
        const int nct = red_ctas(E.nr, na);
        for (int i : act) st[i].itr++;

        // density, stress, free-energy terms and the Anderson sums are all
        // enqueued first; their scalars come back through the pinned staging
        // buffer with one synchronisation (below)
        density_all(E, act, false);
        if (prm.domain) stress_all(E, act);
        std::vector<double> fe, pe;
        free_energy_all(E, act, fe, pe, false);
        if (prm.domain) {
            std::vector<CopyJob> sj;
            double *dst = E.dstage + (size_t)E.hpin_inst * 16;
            for (int k = 0; k < na; k++) sj.push_back(CopyJob{E.inst[act[k]].stress_dev, dst + (size_t)k * 8, PSCFG_MAXCP});
            copy_list(E, sj, 8);
            CK(cudaMemcpyAsync(E.hst(0), dst, sizeof(double) * 8 * na, cudaMemcpyDeviceToHost, E.st));
        }
        // deviations into the ring slot of the current omega
        std::vector<AmJob> aj;
        for (int k = 0; k < na; k++) {
            Inst &I = E.inst[act[k]];
            AmJob j;
            std::memset(&j, 0, sizeof(j));
            j.omega = I.omega;
            j.rho = I.rho;
            j.dev = I.dev_hist + (long)st[act[k]].head * fl;
            j.M = E.M;
            for (int a = 0; a < E.M; a++)
                for (int b = 0; b < E.M; b++) j.chi[a][b] = I.sys.chi[a][b];
            aj.push_back(j);
        }
        AmJob *daj = E.upload(aj, 0);
        size_t off = ((aj.size() * sizeof(AmJob) + 255) / 256) * 256;
        double *part = E.part((size_t)nct * na * (PSCFG_MAXM + 1 + PSCFG_MAXH + 1) + 64);
        double *mpart = part + (size_t)nct * na * PSCFG_MAXM;
        double *dpart = mpart + (size_t)nct * na;
        k_am_dev<<<dim3(nct, na), 256, 0, E.st>>>(daj, E.nr, part);
        E.launched();
        k_final_sum<<<(unsigned)((na * PSCFG_MAXM + 127) / 128), 128, 0, E.st>>>(part, nct, (double)E.nr, E.d_small,
                                                                                  na * PSCFG_MAXM);
        E.launched();
        std::vector<AmFix> fx;
        for (int k = 0; k < na; k++) {
            AmFix f;
            f.dev = aj[k].dev;
            f.mean = E.d_small + (size_t)k * PSCFG_MAXM;
            f.M = E.M;
            fx.push_back(f);
        }
        AmFix *dfx = E.upload(fx, off);
        off += ((fx.size() * sizeof(AmFix) + 255) / 256) * 256;
        k_am_fix<<<dim3(nct, na), 256, 0, E.st>>>(dfx, E.nr, mpart);
        E.launched();
        double *emax = E.d_small + (size_t)na * PSCFG_MAXM;
        k_final_max<<<(unsigned)((na + 127) / 128), 128, 0, E.st>>>(mpart, nct, emax, na);
        E.launched();
        std::vector<AmDot> dots;
        for (int k = 0; k < na; k++) {
            int i = act[k];
            AmDot d;
            std::memset(&d, 0, sizeof(d));
            d.cur = aj[k].dev;
            d.len = fl;
            int nst = std::min(st[i].nstore + 1, S);
            d.nh = nst;
            for (int h = 0; h < nst; h++) {
                int slot = ((st[i].head - h) % S + S) % S;
                d.hist[h] = E.inst[i].dev_hist + (long)slot * fl;
            }
            dots.push_back(d);
        }
        AmDot *ddot = E.upload(dots, off);
        off += ((dots.size() * sizeof(AmDot) + 255) / 256) * 256;
        k_am_dots<<<dim3(nct, na), 256, 0, E.st>>>(ddot, dpart);
        E.launched();
        double *dres = E.d_small + (size_t)na * (PSCFG_MAXM + 1);
        k_final_sum<<<(unsigned)((na * (PSCFG_MAXH + 1) + 127) / 128), 128, 0, E.st>>>(dpart, nct, 1.0, dres,
                                                                                       na * (PSCFG_MAXH + 1));
        E.launched();
        double *dstat = dres + (size_t)na * (PSCFG_MAXH + 1);
        k_am_status<<<(unsigned)((na + 127) / 128), 128, 0, E.st>>>(emax, dres, PSCFG_MAXH + 1, 100.0 * large, dstat, na);
        E.launched();
        const size_t nsm = (size_t)na * (PSCFG_MAXM + 1 + PSCFG_MAXH + 2);
        CK(cudaMemcpyAsync(E.hsm(), E.d_small, sizeof(double) * nsm, cudaMemcpyDeviceToHost, E.st));
        CK(cudaStreamSynchronize(E.st));
        density_finish(E, act);
        fe_finish(E, act, fe, pe);
        hsmall.assign(E.hsm(), E.hsm() + nsm);
        std::vector<double> sh((size_t)na * PSCFG_MAXCP, 0.0);
        if (prm.domain)
            for (int k = 0; k < na; k++) std::memcpy(&sh[(size_t)k * PSCFG_MAXCP], E.hst(k), sizeof(double) * PSCFG_MAXCP);

        std::vector<AmMix> mixes;
        std::vector<int> mix_inst;
        for (int k = 0; k < na; k++) {
            const int i = act[k];
            AmState &s = st[i];
            Inst &I = E.inst[i];
            const int ncp = prm.domain ? I.cell.ncp : 0;
            s.f = fe[k];
            s.p = pe[k];
            for (int b = 0; b < PSCFG_MAXCP; b++) s.stress[b] = sh[(size_t)k * PSCFG_MAXCP + b];
            const double *g = &hsmall[(size_t)na * (PSCFG_MAXM + 1) + (size_t)k * (PSCFG_MAXH + 1)];
            int nst = std::min(s.nstore + 1, S);
            for (int h = 0; h < nst; h++) {
                int slot = ((s.head - h) % S + S) % S;
                s.gram[(size_t)s.head * S + slot] = g[h] / (double)E.nr;
                s.gram[(size_t)slot * S + s.head] = g[h] / (double)E.nr;
            }
            for (int b = 0; b < ncp; b++) s.devcp[s.head][b] = -s.stress[b];
            double e1 = hsmall[(size_t)na * PSCFG_MAXM + k];
            double e2 = 0;
            for (int b = 0; b < ncp; b++) e2 = std::max(e2, std::fabs(s.stress[b]));
            s.error = std::max(e1, e2);
            s.nstore = nst;
            const double word = hsmall[(size_t)na * (PSCFG_MAXM + 1 + PSCFG_MAXH + 1) + k];
            if (word == 1.0 || !std::isfinite(s.error)) {
                s.error = NAN;
                s.status = PSCFG_AM_NONFINITE;
                s.done = true;
                continue;
            }
            // mixed precision: an FP32 iteration never counts as converged; the
            // instance moves to FP64 once its error is below the switch error,
            // or once it is within 1000x of it and has not improved by 10% for
            // 10 iterations (the FP32 noise floor), or as soon as its error
            // rises to 10x the best FP32 error or stops being finite, or after
            // 500 FP32 iterations.  (Looser guards let FP32 runs that drift
            // during a large cell change land in a different basin, from which
            // the FP64 iteration may not converge.)
            const bool was32 = I.prec_now == PSCFG_FP32;
            if (was32) {
                s.itr_fp32++;
                const double sw = prm.switch_error > 0 ? prm.switch_error : 1e-3;
                bool go = s.error < sw || s.error < prm.error_max || s.itr_fp32 >= 500 ||
                          !(s.error <= 10.0 * s.best);
                if (s.error < 0.9 * s.best) {
                    s.best = s.error;
                    s.since_best = 0;
                } else if (++s.since_best >= 10 && s.error < 1e3 * sw) {
                    go = true;
                }
                if (go && E.prec == PSCFG_MIXED) I.prec_now = PSCFG_FP64;
            }
            if (!(was32 && E.prec == PSCFG_MIXED) && s.error < prm.error_max) {
                s.converged = true;
                s.status = PSCFG_AM_CONVERGED;
                s.done = true;
                continue;
            }
            if (!(s.error <= 100.0 * large)) { s.status = PSCFG_AM_DIVERGED; s.done = true; continue; }
            if (s.itr > prm.max_itr) { s.status = PSCFG_AM_MAXITER; s.done = true; continue; }

            // optional restart (not in the reference): drop the history and
            // start the lambda ramp again from this iteration
            if (prm.restart > 0 && s.itr - s.k0 > 1 && s.error > prm.restart * s.best_run) {
                s.k0 = s.itr - 1;
                s.nstore = 1;
                s.best_run = s.error;
            }
            s.best_run = std::min(s.best_run, s.error);
            // lambda and history depth (src/iterate_mod.fp.f90:1147-1153),
            // counted from the last restart (the start, by default)
            const int kk = s.itr - s.k0;
            int itr_prev;
            double lam;
            if (kk < H + 1) { itr_prev = kk - 1; lam = am_lambda_ramp(kk); }
            else { itr_prev = H; lam = 1.0; }
            itr_prev = std::min(itr_prev, s.nstore - 1);
            if (prm.mix_max > 0) lam = std::min(lam, prm.mix_max);
            AmMix m;
            std::memset(&m, 0, sizeof(m));
            m.omega = I.omega;
            m.om_cur = I.om_hist + (long)s.head * fl;
            m.d_cur = I.dev_hist + (long)s.head * fl;
            m.len = fl;
            m.lam = lam;
            const int cur = s.head;
            std::vector<double> cp_new(ncp);
            if (itr_prev == 0) {
                m.n = 0;
                for (int b = 0; b < ncp; b++) cp_new[b] = I.sys.cell_param[b] + lam * s.devcp[cur][b];
            } else {
                // U_mn, V_m (src/iterate_mod.fp.f90:1349-1381) from the Gram ring
                const int n = itr_prev;
                std::vector<double> U((size_t)n * n), V(n);
                auto G = [&](int a, int b) { return s.gram[(size_t)a * S + b]; };
                std::vector<int> sl(n);
                for (int mm = 0; mm < n; mm++) sl[mm] = ((cur - 1 - mm) % S + S) % S;
                for (int mm = 0; mm < n; mm++) {
                    for (int nn = mm; nn < n; nn++) {
                        double u = G(cur, cur) - G(cur, sl[nn]) - G(sl[mm], cur) + G(sl[mm], sl[nn]);
                        for (int b = 0; b < ncp; b++)
                            u += (s.devcp[cur][b] - s.devcp[sl[mm]][b]) * (s.devcp[cur][b] - s.devcp[sl[nn]][b]);
                        U[(size_t)mm * n + nn] = u;
                        U[(size_t)nn * n + mm] = u;
                    }
                    double v = G(cur, cur) - G(sl[mm], cur);
                    for (int b = 0; b < ncp; b++) v += (s.devcp[cur][b] - s.devcp[sl[mm]][b]) * s.devcp[cur][b];
                    V[mm] = v;
                }
                if (!solve_dense(n, U, V)) { s.done = true; s.error = INFINITY; s.status = PSCFG_AM_SINGULAR; continue; }
                m.n = n;
                for (int nn = 0; nn < n; nn++) {
                    m.C[nn] = V[nn];
                    m.om[nn] = I.om_hist + (long)sl[nn] * fl;
                    m.d[nn] = I.dev_hist + (long)sl[nn] * fl;
                }
                for (int b = 0; b < ncp; b++) {
                    double ww = I.sys.cell_param[b], dd = s.devcp[cur][b];
                    for (int nn = 0; nn < n; nn++) {
                        ww += V[nn] * (s.cph[sl[nn]][b] - s.cph[cur][b]);
                        dd += V[nn] * (s.devcp[sl[nn]][b] - s.devcp[cur][b]);
                    }
                    cp_new[b] = ww + lam * dd;
                }
            }
            mixes.push_back(m);
            mix_inst.push_back(i);
            for (int b = 0; b < ncp; b++) I.sys.cell_param[b] = cp_new[b];
        }
        if (!mixes.empty()) {
            AmMix *dm = E.upload(mixes, 0);
            k_am_mix<<<dim3(nct, (unsigned)mixes.size()), 256, 0, E.st>>>(dm);
            E.launched();
            std::vector<double *> slots;
            for (int i : mix_inst) {
                AmState &s = st[i];
                s.head = (s.head + 1) % S;
                slots.push_back(E.inst[i].om_hist + (long)s.head * fl);
                for (int b = 0; b < E.inst[i].cell.ncp; b++) s.cph[s.head][b] = E.inst[i].sys.cell_param[b];
            }
            // symmetric omega (the reference's star basis), recorded in the history
            symmetrize_omega(E, mix_inst);
            std::vector<CopyJob> hj;
            for (size_t k = 0; k < mix_inst.size(); k++) hj.push_back(CopyJob{E.inst[mix_inst[k]].omega, slots[k], fl});
            copy_list(E, hj, fl);
            if (prm.domain) update_cells(E, mix_inst);
        }
        remaining = 0;
        for (int i = 0; i < ninst; i++)
            if (!st[i].done) remaining++;
    }
    return remaining;
}

// ---------------------------------------------------------------------
// Graph-driven Anderson iterations (pscfg_am_param.graph_check > 0)
// ---------------------------------------------------------------------
// One iteration of the instances `act` is a fixed sequence of launches
// whose control data live on the device (am_graph.cuh), so it is captured
// once into a CUDA graph and replayed graph_check times between host
// checks.  The graph is rebuilt without the finished instances once the
// running ones are fewer than three quarters of those it holds.

static void amg_alloc(Engine &E, AmRun &R)
{
    const int n = (int)E.inst.size();
    if (R.g_ninst >= n) return;
    R.g_st = (AmgInst *)E.dalloc(sizeof(AmgInst) * n);
    R.g_act = (int *)E.dalloc(sizeof(int) * n);
    R.g_tidx = (int *)E.dalloc(sizeof(int) * n);
    R.g_terms = (double *)E.dalloc(sizeof(double) * n);
    R.g_aj = (AmJob *)E.dalloc(sizeof(AmJob) * n);
    R.g_fx = (AmFix *)E.dalloc(sizeof(AmFix) * n);
    R.g_dots = (AmDot *)E.dalloc(sizeof(AmDot) * n);
    R.g_mix = (AmMix *)E.dalloc(sizeof(AmMix) * n);
    R.g_hc = (CopyJob *)E.dalloc(sizeof(CopyJob) * n);
    R.g_geo = (GeomJob *)E.dalloc(sizeof(GeomJob) * n);
    R.g_sym = (SymJob *)E.dalloc(sizeof(SymJob) * n);
    R.g_ninst = n;
}

// Initial device state of every instance (after am_begin's first density).
static void amg_init(Engine &E, AmRun &R)
{
    const int n = (int)E.inst.size();
    const int S = R.prm.n_hist + 1;
    std::vector<AmgInst> h(n);
    for (int i = 0; i < n; i++) {
        Inst &I = E.inst[i];
        AmgInst &A = h[i];
        std::memset(&A, 0, sizeof(A));
        A.n_chain = I.sys.n_chain;
        A.n_solvent = I.sys.n_solvent;
        A.ensemble = I.sys.ensemble;
        A.ncp = I.cell.ncp;
        A.dim = E.dim;
        A.crystal = I.sys.crystal_system;
        for (int c = 0; c < I.sys.n_chain; c++) {
            A.length[c] = I.length[c];
            A.phi[c] = I.sys.phi_chain[c];
            A.mu[c] = I.sys.mu_chain[c];
            A.Qv[c] = I.Q[c];
        }
        for (int v = 0; v < I.sys.n_solvent; v++) {
            A.solvent_size[v] = I.sys.solvent_size[v];
            A.phis[v] = I.sys.phi_solvent[v];
            A.mus[v] = I.sys.mu_solvent[v];
            A.Qsv[v] = I.Qs[v];
        }
        A.omega = I.omega;
        A.om_hist = I.om_hist;
        A.dev_hist = I.dev_hist;
        A.fl = (long)E.M * E.nr;
        A.Q = I.Qdev;
        A.Qs = I.Qsolv;
        A.stress_dev = I.stress_dev;
        A.status = PSCFG_AM_RUNNING;
        A.best_run = INFINITY;
        for (int b = 0; b < I.cell.ncp; b++) {
            A.cell[b] = I.sys.cell_param[b];
            A.cph[0][b] = I.sys.cell_param[b];
        }
        (void)S;
        if (I.kweight && !I.wdg0) I.wdg0 = (double *)E.dalloc(sizeof(double) * PSCFG_MAXCP * E.nk);
    }
    CK(cudaMemcpyAsync(R.g_st, h.data(), sizeof(AmgInst) * n, cudaMemcpyHostToDevice, E.st));
    CK(cudaStreamSynchronize(E.st));
    R.g_host.assign(n, AmgInst());
}

// The job fields the device does not write, for the act positions.
static void amg_setup(Engine &E, AmRun &R, const std::vector<int> &act)
{
    const int na = (int)act.size();
    std::vector<AmJob> aj(na);
    std::vector<AmFix> fx(na);
    std::vector<GeomJob> geo(na);
    std::vector<SymJob> sym(na);
    std::vector<int> tidx(na);
    std::vector<size_t> pos_plain, pos_w;
    fe_partition(E, act, pos_plain, pos_w);
    for (size_t k = 0; k < pos_plain.size(); k++) tidx[pos_plain[k]] = (int)k;
    for (size_t k = 0; k < pos_w.size(); k++) tidx[pos_w[k]] = (int)(pos_plain.size() + k);
    R.g_maxorb = 0;
    E.amg_G.assign(E.inst.size(), nullptr);
    for (int k = 0; k < na; k++) {
        Inst &I = E.inst[act[k]];
        std::memset(&aj[k], 0, sizeof(AmJob));
        aj[k].omega = I.omega;
        aj[k].rho = I.rho;
        aj[k].M = E.M;
        for (int a = 0; a < E.M; a++)
            for (int b = 0; b < E.M; b++) aj[k].chi[a][b] = I.sys.chi[a][b];
        std::memset(&fx[k], 0, sizeof(AmFix));
        fx[k].mean = E.d_small + (size_t)k * PSCFG_MAXM;
        fx[k].M = E.M;
        GeomJob &g = geo[k];
        std::memset(&g, 0, sizeof(g));
        std::memcpy(g.G, I.cell.G, sizeof(g.G));
        std::memcpy(g.dGG, I.cell.dGG, sizeof(g.dGG));
        g.ncp = I.cell.ncp;
        g.ksq = I.ksq;
        g.wdgsq = I.wdgsq;
        g.kweight = I.kweight;
        g.wdg0 = I.kweight ? I.wdg0 : nullptr;
        g.gate = &R.g_st[act[k]].mixed;
        E.amg_G[act[k]] = (const double *)((const char *)(R.g_geo + k) + offsetof(GeomJob, G));
        SymJob &y = sym[k];
        std::memset(&y, 0, sizeof(y));
        y.f = I.omega;
        y.perm = I.d_orb_perm;
        y.start = I.d_orb_start;
        y.norb = I.nops > 0 ? I.norb : 0;
        y.M = E.M;
        y.gate = &R.g_st[act[k]].mixed;
        R.g_maxorb = std::max(R.g_maxorb, y.norb);
    }
    CK(cudaMemcpyAsync(R.g_act, act.data(), sizeof(int) * na, cudaMemcpyHostToDevice, E.st));
    CK(cudaMemcpyAsync(R.g_tidx, tidx.data(), sizeof(int) * na, cudaMemcpyHostToDevice, E.st));
    CK(cudaMemcpyAsync(R.g_aj, aj.data(), sizeof(AmJob) * na, cudaMemcpyHostToDevice, E.st));
    CK(cudaMemcpyAsync(R.g_fx, fx.data(), sizeof(AmFix) * na, cudaMemcpyHostToDevice, E.st));
    CK(cudaMemcpyAsync(R.g_geo, geo.data(), sizeof(GeomJob) * na, cudaMemcpyHostToDevice, E.st));
    CK(cudaMemcpyAsync(R.g_sym, sym.data(), sizeof(SymJob) * na, cudaMemcpyHostToDevice, E.st));
    CK(cudaStreamSynchronize(E.st));
}

// Enqueue one iteration of the instances `act` (their jobs set up by
// amg_setup): the host iteration's launches with the Anderson step,
// mixing, history and cell update on the device.
static void amg_iteration(Engine &E, AmRun &R, const std::vector<int> &act)
{
    struct Flag {
        bool &f;
        explicit Flag(bool &x) : f(x) { f = true; }
        ~Flag() { f = false; }
    } on(E.amg);
    const pscfg_am_param &prm = R.prm;
    const int na = (int)act.size();
    const int S = prm.n_hist + 1;
    const long fl = (long)E.M * E.nr;
    const int nct = red_ctas(E.nr, na);
    const double large = 100.0;
    const unsigned g1 = (unsigned)((na + 127) / 128);
    density_all(E, act, false);
    if (prm.domain) stress_all(E, act);
    std::vector<double> fe, pe;
    free_energy_all(E, act, fe, pe, false, R.g_terms);
    amg_launch_finish(E.st, R.g_st, R.g_act, na, R.g_terms, R.g_tidx);
    E.launched();
    amg_launch_prep(E.st, R.g_st, R.g_act, na, S, R.g_aj, R.g_fx, R.g_dots);
    E.launched();
    double *part = E.part((size_t)nct * na * (PSCFG_MAXM + 1 + PSCFG_MAXH + 1) + 64);
    double *mpart = part + (size_t)nct * na * PSCFG_MAXM;
    double *dpart = mpart + (size_t)nct * na;
    k_am_dev<<<dim3(nct, na), 256, 0, E.st>>>(R.g_aj, E.nr, part);
    E.launched();
    k_final_sum<<<(unsigned)((na * PSCFG_MAXM + 127) / 128), 128, 0, E.st>>>(part, nct, (double)E.nr, E.d_small,
                                                                              na * PSCFG_MAXM);
    E.launched();
    k_am_fix<<<dim3(nct, na), 256, 0, E.st>>>(R.g_fx, E.nr, mpart);
    E.launched();
    double *emax = E.d_small + (size_t)na * PSCFG_MAXM;
    k_final_max<<<g1, 128, 0, E.st>>>(mpart, nct, emax, na);
    E.launched();
    k_am_dots<<<dim3(nct, na), 256, 0, E.st>>>(R.g_dots, dpart);
    E.launched();
    double *dres = E.d_small + (size_t)na * (PSCFG_MAXM + 1);
    k_final_sum<<<(unsigned)((na * (PSCFG_MAXH + 1) + 127) / 128), 128, 0, E.st>>>(dpart, nct, 1.0, dres,
                                                                                   na * (PSCFG_MAXH + 1));
    E.launched();
    double *dstat = dres + (size_t)na * (PSCFG_MAXH + 1);
    k_am_status<<<g1, 128, 0, E.st>>>(emax, dres, PSCFG_MAXH + 1, 100.0 * large, dstat, na);
    E.launched();
    AmgParam P;
    P.H = prm.n_hist;
    P.max_itr = prm.max_itr;
    P.domain = prm.domain;
    P.error_max = prm.error_max;
    P.mix_max = prm.mix_max;
    P.restart = prm.restart;
    P.large = large;
    P.nr = (double)E.nr;
    amg_launch_update(E.st, P, R.g_st, R.g_act, na, emax, dres, dstat, R.g_mix, R.g_hc, R.g_geo);
    E.launched();
    k_am_mix<<<dim3(nct, na), 256, 0, E.st>>>(R.g_mix);
    E.launched();
    if (R.g_maxorb > 0) {
        dim3 grid((unsigned)std::max(1, std::min((R.g_maxorb + 127) / 128, 256)), (unsigned)na);
        k_symmetrize<<<grid, 128, 0, E.st>>>(R.g_sym, E.nr);
        E.launched();
    }
    const unsigned gx = (unsigned)red_ctas(fl, na);
    k_copy_list<<<dim3(gx, na), 256, 0, E.st>>>(R.g_hc);
    E.launched();
    if (prm.domain) {
        dim3 grid((unsigned)std::min<long>((E.nk + 255) / 256, 512), (unsigned)na);
        k_make_geom<<<grid, 256, 0, E.st>>>(R.g_geo, E.dim, E.n[0], E.n[1], E.n[2]);
        E.launched();
    }
}

// Capture one iteration of `act` into E.amg_exec (the stream is idle).
static void amg_capture(Engine &E, AmRun &R, const std::vector<int> &act)
{
    const bool prof = E.profiling;
    E.profiling = false;
    E.capturing = true;
    const long l0 = E.launches;
    cudaGraph_t graph = nullptr;
    cudaError_t be = cudaStreamBeginCapture(E.st, cudaStreamCaptureModeRelaxed);
    if (be != cudaSuccess) {
        E.capturing = false;
        E.profiling = prof;
        CK(be);
    }
    try {
        amg_iteration(E, R, act);
    } catch (...) {
        cudaStreamEndCapture(E.st, &graph);
        if (graph) cudaGraphDestroy(graph);
        E.capturing = false;
        E.profiling = prof;
        E.launches = l0;
        throw;
    }
    E.capturing = false;
    E.profiling = prof;
    CK(cudaStreamEndCapture(E.st, &graph));
    cudaError_t ie = cudaGraphInstantiate(&E.amg_exec, graph, 0);
    cudaGraphDestroy(graph);
    CK(ie);
    R.g_launches = E.launches - l0;
    E.launches = l0;
    R.g_cap = act;
}

// Host view of the device state: AmState, the chemistry, Q and the cell.
static void amg_readback(Engine &E, AmRun &R)
{
    const int n = (int)E.inst.size();
    const size_t head = offsetof(AmgInst, devcp);
    CK(cudaMemcpy2DAsync(R.g_host.data(), sizeof(AmgInst), R.g_st, sizeof(AmgInst), head, n, cudaMemcpyDeviceToHost,
                         E.st));
    CK(cudaStreamSynchronize(E.st));
    for (int i = 0; i < n; i++) {
        const AmgInst &A = R.g_host[i];
        AmState &s = R.st[i];
        Inst &I = E.inst[i];
        s.itr = A.itr;
        s.status = A.status;
        s.done = A.done != 0;
        s.converged = A.status == PSCFG_AM_CONVERGED;
        s.error = A.error;
        s.f = A.f;
        s.p = A.p;
        for (int b = 0; b < PSCFG_MAXCP; b++) s.stress[b] = A.stress[b];
        for (int c = 0; c < I.sys.n_chain; c++) {
            I.sys.phi_chain[c] = A.phi[c];
            I.sys.mu_chain[c] = A.mu[c];
            I.Q[c] = A.Qv[c];
        }
        for (int v = 0; v < I.sys.n_solvent; v++) {
            I.sys.phi_solvent[v] = A.phis[v];
            I.sys.mu_solvent[v] = A.mus[v];
            I.Qs[v] = A.Qsv[v];
        }
        if (R.prm.domain) {
            for (int b = 0; b < I.cell.ncp; b++) I.sys.cell_param[b] = A.cell[b];
            Cell c;
            if (make_unit_cell(E.dim, I.sys.crystal_system, I.sys.cell_param, c)) I.cell = c;
        }
    }
}

static void amg_drop_graph(Engine &E)
{
    CK(cudaStreamSynchronize(E.st));
    if (E.amg_exec) {
        CK(cudaGraphExecDestroy(E.amg_exec));
        E.amg_exec = nullptr;
    }
    E.cap_free();
}

static int am_iterate_graph(Engine &E, AmRun &R, int iters)
{
    const int ninst = (int)E.inst.size();
    int it = 0;
    while (it < iters) {
        std::vector<int> act;
        for (int i = 0; i < ninst; i++)
            if (!R.st[i].done) act.push_back(i);
        if (act.empty()) break;
        if (!E.amg_exec || act.size() * 4 < R.g_cap.size() * 3) {
            // (re)build: one iteration of the new set launched directly
            // sizes the scratch buffers (their sizes depend on the set), then
            // the same sequence is captured
            amg_drop_graph(E);
            amg_setup(E, R, act);
            amg_iteration(E, R, act);
            it++;
            amg_capture(E, R, act);
            if (it >= iters) {
                amg_readback(E, R);
                break;
            }
        }
        const int n = std::min(R.prm.graph_check, iters - it);
        for (int r = 0; r < n; r++) CK(cudaGraphLaunch(E.amg_exec, E.st));
        E.launches += (long)n * R.g_launches;
        it += n;
        amg_readback(E, R);
    }
    int remaining = 0;
    for (int i = 0; i < ninst; i++)
        if (!R.st[i].done) remaining++;
    return remaining;
}

static void am_results(Engine &E, AmRun &R, std::vector<pscfg_am_result> &res)
{
    if (!R.active) throw Err(PSCFG_ESTATE, "no Anderson run in progress");
    const int ninst = (int)E.inst.size();
    std::vector<int> all(ninst);
    for (int i = 0; i < ninst; i++) all[i] = i;
    std::vector<double> shost((size_t)ninst * PSCFG_MAXCP, 0.0);
    if (!R.prm.domain) {
        stress_all(E, all);
        for (int i = 0; i < ninst; i++)
            CK(cudaMemcpyAsync(&shost[(size_t)i * PSCFG_MAXCP], E.inst[i].stress_dev, sizeof(double) * PSCFG_MAXCP,
                               cudaMemcpyDeviceToHost, E.st));
        CK(cudaStreamSynchronize(E.st));
    }
    res.resize(ninst);
    for (int i = 0; i < ninst; i++) {
        pscfg_am_result &r = res[i];
        std::memset(&r, 0, sizeof(r));
        AmState &s = R.st[i];
        Inst &I = E.inst[i];
        r.itr = s.itr;
        r.itr_fp32 = s.itr_fp32;
        r.converged = s.converged ? 1 : 0;
        r.status = s.status;
        r.error = s.error;
        r.f_helmholtz = s.f;
        r.pressure = s.p;
        for (int b = 0; b < I.cell.ncp; b++) {
            r.stress[b] = R.prm.domain ? s.stress[b] : shost[(size_t)i * PSCFG_MAXCP + b];
            r.cell_param[b] = I.sys.cell_param[b];
        }
        for (int c = 0; c < I.sys.n_chain; c++) {
            r.q[c] = I.Q[c];
            r.mu_chain[c] = I.sys.mu_chain[c];
        }
    }
}

// ---------------------------------------------------------------------
// Adjoint of density() with respect to omega (adjoint.cuh)
// ---------------------------------------------------------------------
// Simpson weights of slice j summed over the blocks that contain it, per
// monomer: wsum_j[m] = sum_{b ∋ j, m_b = m} (ds_b / 3) w_j^b.
static void simpson_weights(const Inst &I, int c, std::vector<double> &w)
{
    const int ns = I.ns[c];
    w.assign((size_t)(ns + 1) * PSCFG_MAXM, 0.0);
    for (int b = 0; b < I.sys.n_block[c]; b++) {
        const int ib = I.bgn[c][b], ie = I.bgn[c][b + 1], m = I.sys.block_monomer[c][b];
        for (int j = ib; j <= ie; j++) {
            double wt = (j == ib || j == ie) ? 1.0 : (((j - ib) % 2 == 1) ? 4.0 : 2.0);
            w[(size_t)j * PSCFG_MAXM + m] += I.bds[c][b] / 3.0 * wt;
        }
    }
}

static int seg_block(const Inst &I, int c, int j)   // block of the segment (j, j+1)
{
    int b = 0;
    while (b < I.sys.n_block[c] - 1 && j >= I.bgn[c][b + 1]) b++;
    return b;
}

// One step of every field in dfl (fields with ns = 1 and in/out overrides),
// on whichever step kernels the grid has.
template <typename T>
static void run_single_steps(Engine &E, const SweepField<T> *dfl, int nf)
{
    const PlaneGeom &g = E.geom();
    const long nr = E.nr;
    if (E.dim <= 2) {
        size_t sm = 2 * (size_t)g.n2 * g.LS * sizeof(cx<T>) + 2 * (size_t)nr * sizeof(T);
        CK(allow_dyn_smem((const void *)k_sweep_plane<T>));
        int threads = (int)std::min<long>(256, std::max<long>(32, ((nr / 2 + 31) / 32) * 32));
        k_sweep_plane<T><<<nf, threads, sm, E.st>>>(dfl, g, 0, 1);
        E.launched();
    } else if (!step3_fixed<T>(E, dfl, nf, 0) && !step3l<T>(E, dfl, nf, 0)) {
        size_t smxy = 2 * (size_t)g.n2 * g.LS * sizeof(cx<T>);
        size_t smz = 2 * (size_t)g.n3 * Z_TILE * sizeof(cx<T>);
        CK(allow_dyn_smem((const void *)k3_fwd_pair<T>));
        CK(allow_dyn_smem((const void *)k3_inv_mid<T>));
        CK(allow_dyn_smem((const void *)k3_inv_final<T>));
        CK(allow_dyn_smem((const void *)k3_zconv<T, Z_TILE>));
        const long P = (long)g.n1h * g.n2;
        const int ntile = (int)((P + Z_TILE - 1) / Z_TILE);
        k3_fwd_pair<T><<<dim3(g.n3, nf), 256, smxy, E.st>>>(dfl, g, 0);
        E.launched();
        k3_zconv<T, Z_TILE><<<dim3(ntile, nf, 2), 256, smz, E.st>>>(dfl, g, 0, 3);
        E.launched();
        k3_inv_mid<T><<<dim3(g.n3, nf), 256, smxy, E.st>>>(dfl, g, 0);
        E.launched();
        k3_zconv<T, Z_TILE><<<dim3(ntile, nf, 1), 256, smz, E.st>>>(dfl, g, 0, 2);
        E.launched();
        k3_inv_final<T><<<dim3(g.n3, nf), 256, smxy, E.st>>>(dfl, g, 0);
        E.launched();
    }
}

template <typename T>
static void adjoint_impl(Engine &E, const std::vector<int> &act, const std::vector<const double *> &G,
                         const std::vector<const double *> &gQ, const std::vector<double *> &grad,
                         const std::vector<double *> &gcell)
{
    const size_t ts = sizeof(T);
    const long nr = E.nr, nk = E.nk;
    struct Sweep {
        int inst, c, d, ns;
        T *lam[2];
        T *p1[2], *h[2], *p2[2], *dummy[2];
        cx<T> *S1[2], *S2[2];
        double *gbuf;
        std::vector<double> coef;   // [ns+1][MAXM] incl. phi/(L Q)
    };
    std::vector<Sweep> sw;
    const int nct = red_ctas(nr);
    // coefficients, overlaps S_c
    std::vector<AdjOverlap> ov;
    std::vector<std::pair<int, int>> ov_ic;
    size_t off = 0;
    for (size_t k = 0; k < act.size(); k++) {
        Inst &I = E.inst[act[k]];
        for (int c = 0; c < I.sys.n_chain; c++) {
            std::vector<double> w;
            simpson_weights(I, c, w);
            const double cphi = (I.sys.ensemble == 0) ? I.sys.phi_chain[c] / (I.length[c] * I.Q[c])
                                                      : std::exp(I.sys.mu_chain[c]) / I.length[c];
            for (auto &x : w) x *= cphi;
            if (!I.adj_coef[c]) I.adj_coef[c] = (double *)E.dalloc(sizeof(double) * w.size());
            CK(cudaMemcpyAsync(I.adj_coef[c], w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice, E.st));
            for (int d = 0; d < 2; d++) {
                if (!I.adj_real[c][d]) {
                    I.adj_real[c][d] = E.dalloc(ts * nr * 10);
                    I.adj_spec[c][d] = E.dalloc(2 * ts * nk * 4);
                    I.adj_grad[c][d] = (double *)E.dalloc(sizeof(double) * E.M * nr);
                }
                Sweep S;
                S.inst = act[k];
                S.c = c;
                S.d = d;
                S.ns = I.ns[c];
                T *R = (T *)I.adj_real[c][d];
                cx<T> *SP = (cx<T> *)I.adj_spec[c][d];
                S.lam[0] = R;
                S.lam[1] = R + nr;
                for (int f = 0; f < 2; f++) {
                    S.p1[f] = R + (2 + 4 * f) * nr;
                    S.h[f] = R + (3 + 4 * f) * nr;
                    S.p2[f] = R + (4 + 4 * f) * nr;
                    S.dummy[f] = R + (5 + 4 * f) * nr;
                    S.S1[f] = SP + (2 * f) * nk;
                    S.S2[f] = SP + (2 * f + 1) * nk;
                }
                S.gbuf = I.adj_grad[c][d];
                S.coef = w;
                k_zero<<<(unsigned)std::min<long>((E.M * nr + 255) / 256, 1024), 256, 0, E.st>>>(S.gbuf, (long)E.M * nr);
                E.launched();
                sw.push_back(S);
            }
            AdjOverlap o;
            o.qf = I.qf[c];
            o.qr = I.qr[c];
            o.G = G[k];
            o.coef = I.adj_coef[c];
            o.nslices = I.ns[c] + 1;
            o.M = E.M;
            ov.push_back(o);
            ov_ic.push_back({(int)k, c});
        }
    }
    if (sw.empty()) return;
    // cell derivative: pair slabs, slice sums and per-instance accumulators
    bool want_cell = false;
    for (double *p : gcell) want_cell = want_cell || p != nullptr;
    CallScratch cscr;
    double *cA = nullptr, *cB = nullptr, *cinc = nullptr, *cg = nullptr;
    if (want_cell) {
        cA = (double *)cscr.get(sizeof(double) * 3 * nr * sw.size());
        cB = (double *)cscr.get(sizeof(double) * 3 * nr * sw.size());
        cinc = (double *)cscr.get(sizeof(double) * 3 * PSCFG_MAXCP * sw.size());
        cg = (double *)cscr.get(sizeof(double) * PSCFG_MAXCP * act.size());
        CK(cudaMemsetAsync(cg, 0, sizeof(double) * PSCFG_MAXCP * act.size(), E.st));
    }
    std::vector<double> Sc(ov.size(), 0.0);
    std::vector<const T *> ekf_of;
    if (E.ckpt) {
        // overlaps segment by segment from the recomputed propagators
        ckpt_tables<T>(E, act, ekf_of);
        std::vector<CkChain> ch;
        int nseg_max = 0;
        for (auto &ic : ov_ic) {
            ch.push_back(CkChain{act[ic.first], ic.second});
            nseg_max = std::max(nseg_max, E.inst[act[ic.first]].nseg[ic.second]);
        }
        const int K = E.ckK;
        for (int j = 0; j < nseg_max; j++) {
            ckpt_segment<T>(E, ch, ekf_of, j, +1, false);
            ckpt_segment<T>(E, ch, ekf_of, j, -1, false);
            std::vector<AdjOverlap> os;
            std::vector<size_t> idx;
            for (size_t q = 0; q < ov.size(); q++) {
                Inst &I = E.inst[ch[q].inst];
                const int c = ch[q].c;
                if (j >= I.nseg[c]) continue;
                AdjOverlap o = ov[q];
                o.qf = I.segA[c];
                o.qr = I.segB[c];
                o.coef = I.adj_coef[c] + (size_t)j * K * PSCFG_MAXM;
                o.nslices = (j == I.nseg[c] - 1) ? I.ns[c] + 1 - j * K : K;
                os.push_back(o);
                idx.push_back(q);
            }
            if (os.empty()) continue;
            AdjOverlap *dov = E.upload(os, 0);
            double *part = E.part((size_t)nct * os.size());
            k_adj_overlap<T><<<dim3(nct, (unsigned)os.size()), 256, 0, E.st>>>(dov, nr, part);
            E.launched();
            k_final_sum<<<(unsigned)((os.size() + 127) / 128), 128, 0, E.st>>>(part, nct, 1.0, E.d_small, (int)os.size());
            E.launched();
            std::vector<double> h(os.size());
            CK(cudaMemcpyAsync(h.data(), E.d_small, sizeof(double) * os.size(), cudaMemcpyDeviceToHost, E.st));
            CK(cudaStreamSynchronize(E.st));
            for (size_t q = 0; q < os.size(); q++) Sc[idx[q]] += h[q];
        }
    } else {
        AdjOverlap *dov = E.upload(ov, off);
        off += ((ov.size() * sizeof(AdjOverlap) + 255) / 256) * 256;
        double *part = E.part((size_t)nct * ov.size());
        k_adj_overlap<T><<<dim3(nct, (unsigned)ov.size()), 256, 0, E.st>>>(dov, nr, part);
        E.launched();
        k_final_sum<<<(unsigned)((ov.size() + 127) / 128), 128, 0, E.st>>>(part, nct, 1.0, E.d_small, (int)ov.size());
        E.launched();
        CK(cudaMemcpyAsync(Sc.data(), E.d_small, sizeof(double) * ov.size(), cudaMemcpyDeviceToHost, E.st));
        CK(cudaStreamSynchronize(E.st));
    }
    // initial adjoint states
    {
        std::vector<AdjInit> ini;
        size_t oi = 0;
        for (auto &S : sw) {
            Inst &I = E.inst[S.inst];
            size_t k = 0;
            while (act[k] != S.inst) k++;
            const int j = (S.d == 0) ? S.ns : 0;
            AdjInit a;
            std::memset(&a, 0, sizeof(a));
            a.lam = S.lam[0];
            a.G = G[k];
            if (E.ckpt)   // the end slices are the checkpoints nseg (qr) and 0 (qf)
                a.other = (S.d == 0) ? (const T *)I.qr[S.c] + (long)I.nseg[S.c] * nr : (const T *)I.qf[S.c];
            else
                a.other = (S.d == 0) ? (const T *)I.qr[S.c] + (long)j * nr : (const T *)I.qf[S.c] + (long)j * nr;
            for (int m = 0; m < E.M; m++) a.coef[m] = S.coef[(size_t)j * PSCFG_MAXM + m];
            a.M = E.M;
            if (S.d == 0) {
                while (!(ov_ic[oi].first == (int)k && ov_ic[oi].second == S.c)) oi++;
                const double g = gQ[k] ? gQ[k][S.c] : 0.0;
                const double sterm = (I.sys.ensemble == 0) ? Sc[oi] : 0.0;
                a.cst = (g - sterm) / (I.Q[S.c] * (double)nr);
                oi = 0;
            }
            ini.push_back(a);
        }
        AdjInit *di = E.upload(ini, 0);
        k_adj_init<T><<<dim3((unsigned)std::min<long>((nr + 255) / 256, 256), (unsigned)ini.size()), 256, 0, E.st>>>(di, nr);
        E.launched();
    }
    int ns_max = 0;
    for (auto &S : sw) ns_max = std::max(ns_max, S.ns);
    const PlaneGeom &g = E.geom();
    // slice s of chain c of instance I: propagator 0 = qf, 1 = qr (stored
    // slabs, or the loaded checkpoint segment j_seg)
    int j_seg = -1;
    auto slice = [&](const Inst &I, int c, int which, int sl) -> const T * {
        if (!E.ckpt) return (const T *)(which == 0 ? I.qf[c] : I.qr[c]) + (long)sl * nr;
        return (const T *)(which == 0 ? I.segA[c] : I.segB[c]) + (long)(sl - j_seg * E.ckK) * nr;
    };
    auto adj_step = [&](int t, const std::vector<size_t> &sel) {
        std::vector<SweepField<T>> fl;
        std::vector<AdjPoint> pts;
        for (size_t si : sel) {
            auto &S = sw[si];
            if (t >= S.ns) continue;
            Inst &I = E.inst[S.inst];
            size_t k = 0;
            while (act[k] != S.inst) k++;
            const int cur = t & 1;
            int qslice, newslice, blk;
            const T *qsrc, *other;
            if (S.d == 0) {
                qslice = S.ns - 1 - t;            // step qf_j -> qf_{j+1}
                newslice = qslice;
                blk = seg_block(I, S.c, qslice);
                qsrc = slice(I, S.c, 0, qslice);
                other = slice(I, S.c, 1, newslice);
            } else {
                qslice = t + 1;                   // step qr_s -> qr_{s-1}
                newslice = qslice;
                blk = seg_block(I, S.c, qslice - 1);
                qsrc = slice(I, S.c, 1, qslice);
                other = slice(I, S.c, 0, newslice);
            }
            for (int f = 0; f < 2; f++) {
                SweepField<T> F;
                std::memset(&F, 0, sizeof(F));
                F.slab = S.dummy[f];
                F.ns = 1;
                F.dir = 1;
                F.nblk = 1;
                F.bgn[0] = 0;
                F.bgn[1] = 1;
                F.eo1[0] = (const T *)I.eo1[S.c][blk];
                F.eo2[0] = (const T *)I.eo2[S.c][blk];
                F.ek1[0] = (const T *)I.ek1[S.c][blk];
                F.ek2[0] = (const T *)I.ek2[S.c][blk];
                F.S1 = S.S1[f];
                F.S2 = S.S2[f];
                F.q1 = S.p1[f];
                F.in = (f == 0) ? S.lam[cur] : qsrc;
                F.out = S.dummy[f];
                F.h_out = S.h[f];
                F.q2_out = S.p2[f];
                fl.push_back(F);
            }
            AdjPoint a;
            std::memset(&a, 0, sizeof(a));
            a.lam = S.lam[cur];
            a.p1l = S.p1[0];
            a.hl = S.h[0];
            a.p2l = S.p2[0];
            a.q = qsrc;
            a.p1q = S.p1[1];
            a.hq = S.h[1];
            a.p2q = S.p2[1];
            a.eo1 = I.eo1[S.c][blk];
            a.ds = I.bds[S.c][blk];
            a.grad = S.gbuf + (long)I.sys.block_monomer[S.c][blk] * nr;
            a.lam_new = S.lam[cur ^ 1];
            a.G = G[k];
            a.other = other;
            for (int m = 0; m < E.M; m++) a.coef[m] = S.coef[(size_t)newslice * PSCFG_MAXM + m];
            a.M = E.M;
            pts.push_back(a);
        }
        SweepField<T> *dfl = E.upload(fl, 0);
        size_t o2 = ((fl.size() * sizeof(SweepField<T>) + 255) / 256) * 256;
        AdjPoint *dpt = E.upload(pts, o2);
        run_single_steps<T>(E, dfl, (int)fl.size());
        k_adj_point<T><<<dim3((unsigned)std::min<long>((nr + 255) / 256, 256), (unsigned)pts.size()), 256, 0, E.st>>>(dpt, nr);
        E.launched();
        if (want_cell) {
            // the step's cell derivative (4/3) d<lam,P2 q> - (1/3) d<lam,P1 q>
            // from three real-field pairs per sweep (adjoint.cuh)
            std::vector<AdjCellPair> cp;
            std::vector<StressJob<double>> cj;
            std::vector<AdjCellAcc> ca;
            int k = 0;
            for (size_t si : sel) {
                auto &S = sw[si];
                if (t >= S.ns) continue;
                Inst &I = E.inst[S.inst];
                size_t kin = 0;
                while (act[kin] != S.inst) kin++;
                const int cur = t & 1;
                const int qslice = (S.d == 0) ? S.ns - 1 - t : t + 1;
                const int blk = (S.d == 0) ? seg_block(I, S.c, qslice) : seg_block(I, S.c, qslice - 1);
                AdjCellPair a;
                a.lam = (const double *)S.lam[cur];
                a.hl = (const double *)S.h[0];
                a.p1q = (const double *)S.p1[1];
                a.hq = (const double *)S.h[1];
                a.p2q = (const double *)S.p2[1];
                a.eo1 = (const double *)I.eo1[S.c][blk];
                a.eo2 = (const double *)I.eo2[S.c][blk];
                a.a = cA + (long)3 * k * nr;
                a.b = cB + (long)3 * k * nr;
                cp.push_back(a);
                StressJob<double> j;
                j.qf = a.a;
                j.qr = a.b;
                j.wdgsq = I.wdg0 ? I.wdg0 : I.wdgsq;
                j.ncp = I.cell.ncp;
                j.nslices = 3;
                j.inc = cinc + (long)3 * k * PSCFG_MAXCP;
                cj.push_back(j);
                const double bb = I.sys.kuhn[I.sys.block_monomer[S.c][blk]];
                const double f = I.bds[S.c][blk] * bb * bb / (double)nr;
                AdjCellAcc acc;
                acc.inc = j.inc;
                acc.coef[0] = f / 18.0;
                acc.coef[1] = -f / 9.0;
                acc.coef[2] = -f / 9.0;
                acc.g = cg + (long)kin * PSCFG_MAXCP;
                acc.ncp = I.cell.ncp;
                ca.push_back(acc);
                k++;
            }
            if (k > 0) {
                AdjCellPair *dcp = E.upload(cp, (size_t)8 << 20);
                k_adj_cellpairs<<<dim3((unsigned)std::min<long>((nr + 255) / 256, 256), (unsigned)k), 256, 0, E.st>>>(dcp, nr);
                E.launched();
                slice_dots<double>(E, cj);
                AdjCellAcc *dca = E.upload(ca, (size_t)9 << 20);
                k_adj_cellacc<<<1, 32, 0, E.st>>>(dca, k);
                E.launched();
            }
        }
    };
    if (!E.ckpt) {
        std::vector<size_t> all(sw.size());
        for (size_t q = 0; q < sw.size(); q++) all[q] = q;
        for (int t = 0; t < ns_max; t++) adj_step(t, all);
    } else {
        // one chain and direction at a time, the segment holding the step's
        // slices recomputed when the step leaves the loaded one
        const int K = E.ckK;
        for (size_t q = 0; q < sw.size(); q++) {
            auto &S = sw[q];
            const std::vector<CkChain> one{CkChain{S.inst, S.c}};
            j_seg = -1;
            for (int t = 0; t < S.ns; t++) {
                const int sl = (S.d == 0) ? S.ns - 1 - t : t + 1;
                const int j = (S.d == 0) ? sl / K : (sl - 1) / K;
                if (j != j_seg) {
                    std::vector<const T *> ekf1;
                    if (!ekf_of.empty()) {
                        size_t pos = 0;
                        for (size_t r = 0; r < ov_ic.size(); r++)
                            if (act[ov_ic[r].first] == S.inst && ov_ic[r].second == S.c) pos = r;
                        ekf1.push_back(ekf_of[pos]);
                    }
                    ckpt_segment<T>(E, one, ekf1, j, +1, false);
                    ckpt_segment<T>(E, one, ekf1, j, -1, false);
                    j_seg = j;
                }
                adj_step(t, std::vector<size_t>{q});
            }
        }
    }
    if (want_cell) {
        std::vector<double> h(PSCFG_MAXCP * act.size());
        CK(cudaMemcpyAsync(h.data(), cg, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, E.st));
        CK(cudaStreamSynchronize(E.st));
        for (size_t k = 0; k < act.size(); k++)
            if (k < gcell.size() && gcell[k])
                for (int b = 0; b < PSCFG_MAXCP; b++) gcell[k][b] = b < E.inst[act[k]].cell.ncp ? h[k * PSCFG_MAXCP + b] : 0.0;
    }
    // grad = sum over sweeps of the instance, fixed order
    for (size_t k = 0; k < act.size(); k++) {
        CK(cudaMemsetAsync(grad[k], 0, sizeof(double) * E.M * nr, E.st));
        std::vector<const double *> parts;
        for (auto &S : sw)
            if (S.inst == act[k]) parts.push_back(S.gbuf);
        for (const double *p : parts) {
            k_axpy<<<(unsigned)std::min<long>((E.M * nr + 255) / 256, 1024), 256, 0, E.st>>>(grad[k], p, (long)E.M * nr);
            E.launched();
        }
    }
}

static void adjoint_all(Engine &E, const std::vector<int> &act, const std::vector<const double *> &G,
                        const std::vector<const double *> &gQ, const std::vector<double *> &grad,
                        const std::vector<double *> &gcell = {})
{
    for (int i : act)
        if (!E.inst[i].have_density) throw Err(PSCFG_ESTATE, "the adjoint requires a preceding density call");
    std::vector<int> a64, a32;
    split_prec(E, act, a64, a32);
    if (!a32.empty()) throw Err(PSCFG_EINVAL, "the adjoint runs on FP64 propagators (use PSCFG_FP64 or PSCFG_MIXED)");
    E.cur = PSCFG_FP64;
    adjoint_impl<double>(E, act, G, gQ, grad, gcell);
}

// ---------------------------------------------------------------------
// Linear response of a periodic state (RESPONSE, src/response_mod.f90)
// ---------------------------------------------------------------------

// Line passes of one complex transform of every job (k_cline).  step: the
// fftc_step E IFFT[K FFT[E x]]; otherwise the forward transform / N.
static void run_cpasses(Engine &E, const CJob *djobs, int njobs, bool step, const LinePlan plans[3])
{
    const int dim = E.dim;
    std::vector<CPass> passes;
    auto mk_pass = [&](int a) {
        CPass P;
        std::memset(&P, 0, sizeof(P));
        P.axis = a;
        P.L = E.n[a];
        P.nl = (int)(E.nr / P.L);
        P.TL = std::max(1, std::min(32, 2048 / P.L));
        P.TL = std::min(P.TL, P.nl);
        P.plan = plans[a];
        return P;
    };
    for (int a = 0; a < dim; a++) {
        CPass P = mk_pass(a);
        P.fwd = 1;
        if (a == 0) P.first = 1;
        if (a == dim - 1) {
            P.kmul = 1;
            if (step) P.inv = 1;
        }
        passes.push_back(P);
    }
    if (step) {
        for (int a = dim - 2; a >= 0; a--) {
            CPass P = mk_pass(a);
            P.inv = 1;
            passes.push_back(P);
        }
        passes.back().last = 1;
    }
    CK(allow_dyn_smem((const void *)k_cline));
    const double inv_n = 1.0 / (double)E.nr;
    for (const CPass &P : passes) {
        const size_t sm = 2 * sizeof(cx<double>) * (size_t)P.TL * P.L;
        const unsigned gx = (unsigned)((P.nl + P.TL - 1) / P.TL);
        for (int j0 = 0; j0 < njobs; j0 += 65535) {
            const int nj = std::min(65535, njobs - j0);
            k_cline<<<dim3(gx, nj), 128, sm, E.st>>>(djobs + j0, P, E.n[0], E.n[1], inv_n);
            E.launched();
        }
    }
}

static void response_impl(Engine &E, int inst, const double kvec[3], double ktrans_sq, int n_pert,
                          const int *pert_monomer, const double *pert_field, int n_read, const int *read_index,
                          const double *read_coef, double *out)
{
    Inst &I = E.inst[inst];
    if (E.ckpt) throw Err(PSCFG_ESTATE, "pscfg_response reads every stored propagator slice (not kept with PSCFG_CHECKPOINT)");
    if (!I.have_density) throw Err(PSCFG_ESTATE, "the response requires a preceding density call");
    if (E.prec == PSCFG_FP32 || I.dens_prec != PSCFG_FP64)
        throw Err(PSCFG_EINVAL, "the response runs on FP64 propagators");
    for (int p = 0; p < n_pert; p++)
        if (pert_monomer[p] < 0 || pert_monomer[p] >= E.M) throw Err(PSCFG_EINVAL, "perturbed monomer out of range");
    for (int k = 0; k < n_read; k++)
        if (read_index[k] < 0 || read_index[k] >= E.nr) throw Err(PSCFG_EINVAL, "readout index out of range");
    E.cur = PSCFG_FP64;
    const long nr = E.nr, nk = E.nk;
    const int M = E.M, nch = I.sys.n_chain;
    const PlaneGeom &g = E.g64;
    CallScratch cs;
    E.desc((size_t)64 << 20);
    const unsigned ngrid = (unsigned)std::min<long>((nr + 255) / 256, 1024);

    // 1. unperturbed step intermediates of every step of both sweeps
    //    (calc_q0): P1 q (chains0 order 0), the half-step midpoint and
    //    P2 q (chains0 order 1), from the stored propagators
    struct Inter { double *q1, *h, *q2; };
    Inter it[PSCFG_MAXC][2];
    for (int c = 0; c < nch; c++) {
        const int ns = I.ns[c];
        for (int d = 0; d < 2; d++) {
            it[c][d].q1 = (double *)cs.get(sizeof(double) * nr * (ns + 1));
            it[c][d].h = (double *)cs.get(sizeof(double) * nr * (ns + 1));
            it[c][d].q2 = (double *)cs.get(sizeof(double) * nr * (ns + 1));
        }
    }
    {
        const int FCH = 64;
        double *dummy = (double *)cs.get(sizeof(double) * nr * FCH);
        cx<double> *S12 = E.dim == 3 ? (cx<double> *)cs.get(sizeof(cx<double>) * nk * 2 * FCH) : nullptr;
        std::vector<SweepField<double>> fl;
        std::vector<CDiv> dv;
        auto flush = [&]() {
            if (fl.empty()) return;
            SweepField<double> *dfl = E.upload(fl, 0);
            run_single_steps<double>(E, dfl, (int)fl.size());
            CDiv *ddv = E.upload(dv, (size_t)4 << 20);
            k_resp_div<<<dim3(ngrid, (unsigned)dv.size()), 256, 0, E.st>>>(ddv, nr);
            E.launched();
            fl.clear();
            dv.clear();
        };
        for (int c = 0; c < nch; c++) {
            const int ns = I.ns[c];
            for (int d = 0; d < 2; d++)
                for (int j = (d == 0 ? 1 : 0); j <= (d == 0 ? ns : ns - 1); j++) {
                    const int blk = seg_block(I, c, d == 0 ? j - 1 : j);
                    const int slot = (int)fl.size();
                    SweepField<double> F;
                    std::memset(&F, 0, sizeof(F));
                    F.slab = dummy + (long)slot * nr;
                    F.ns = 1;
                    F.dir = 1;
                    F.nblk = 1;
                    F.bgn[0] = 0;
                    F.bgn[1] = 1;
                    F.eo1[0] = (const double *)I.eo1[c][blk];
                    F.eo2[0] = (const double *)I.eo2[c][blk];
                    F.ek1[0] = (const double *)I.ek1[c][blk];
                    F.ek2[0] = (const double *)I.ek2[c][blk];
                    if (S12) {
                        F.S1 = S12 + (long)(2 * slot) * nk;
                        F.S2 = S12 + (long)(2 * slot + 1) * nk;
                    }
                    F.in = d == 0 ? (const double *)I.qf[c] + (long)(j - 1) * nr
                                  : (const double *)I.qr[c] + (long)(j + 1) * nr;
                    F.out = dummy + (long)slot * nr;
                    F.q1 = it[c][d].q1 + (long)j * nr;
                    F.h_out = it[c][d].h + (long)j * nr;
                    F.q2_out = it[c][d].q2 + (long)j * nr;
                    fl.push_back(F);
                    CDiv v;
                    v.x = it[c][d].h + (long)j * nr;
                    v.d = (const double *)I.eo2[c][blk];
                    dv.push_back(v);
                    if ((int)fl.size() == FCH) flush();
                }
        }
        flush();
    }

    // 2. |G+k|^2 and the exp tables of levels ds, ds/2, ds/4 per block
    std::vector<double> kq;
    ksq_bloch(E.dim, E.n, I.cell.G, kvec, ktrans_sq, kq);
    double *ksq_new = (double *)cs.get(sizeof(double) * nr);
    CK(cudaMemcpyAsync(ksq_new, kq.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, E.st));
    const double *Et[PSCFG_MAXC][PSCFG_MAXB][3], *Kt[PSCFG_MAXC][PSCFG_MAXB][3];
    {
        std::vector<CTab> tj;
        for (int c = 0; c < nch; c++)
            for (int b = 0; b < I.sys.n_block[c]; b++) {
                const int m = I.sys.block_monomer[c][b];
                double dsl = I.bds[c][b];
                for (int l = 0; l < 3; l++) {
                    CTab t;
                    t.w = I.omega + (long)m * nr;
                    t.ksq = ksq_new;
                    t.E = (double *)cs.get(sizeof(double) * nr);
                    t.K = (double *)cs.get(sizeof(double) * nr);
                    t.ds = dsl;
                    t.b2 = I.sys.kuhn[m] * I.sys.kuhn[m];
                    Et[c][b][l] = t.E;
                    Kt[c][b][l] = t.K;
                    tj.push_back(t);
                    dsl /= 2.0;
                }
            }
        CTab *dtj = E.upload(tj, 0);
        k_resp_tables<<<dim3(ngrid, (unsigned)tj.size()), 256, 0, E.st>>>(dtj, nr);
        E.launched();
    }
    // Simpson coefficients per slice and monomer, times phi/(N Q)
    // (calc_delrho, src/response_mod.f90:1107-1182)
    std::vector<double> coef[PSCFG_MAXC];
    for (int c = 0; c < nch; c++) {
        simpson_weights(I, c, coef[c]);
        const double f = I.sys.phi_chain[c] / (I.length[c] * I.Q[c]);
        for (auto &x : coef[c]) x *= f;
    }
    LinePlan plans[3] = {g.row, g.col, g.zp};
    plans[0].n = E.n[0];
    if (!plan_radices(E.n[0], plans[0].rad, plans[0].nst)) throw Err(PSCFG_EINVAL, "grid size not supported");
    plans[0].tw = g.rtw;

    // 3. perturbations in chunks bounded by memory
    const int nsd = 2 * nch;                       // sweeps per perturbation
    const size_t per = sizeof(cx<double>) * nr * ((size_t)nsd * (7 + M) + 1 + M);
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    const size_t budget = std::min((size_t)8 << 30, fr / 4);
    // the job descriptors of one segment must fit the pre-grown descriptor
    // scratch (an upload that grew it would free descriptors already queued)
    const size_t per_desc = (size_t)nsd * (6 * sizeof(CJob) + sizeof(CCombine)) + 2 * M * sizeof(CJob) + 256;
    const size_t desc_cap = ((size_t)48 << 20) / per_desc;
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>(std::min<size_t>((size_t)n_pert, budget / per), desc_cap));
    double *dout = (double *)cs.get(sizeof(double) * (size_t)chunk * M * std::max(n_read, 1));
    int *didx = (int *)cs.get(sizeof(int) * std::max(n_read, 1));
    double *dcoef = (double *)cs.get(sizeof(double) * 2 * std::max(n_read, 1));
    if (n_read > 0) {
        CK(cudaMemcpyAsync(didx, read_index, sizeof(int) * n_read, cudaMemcpyHostToDevice, E.st));
        CK(cudaMemcpyAsync(dcoef, read_coef, sizeof(double) * 2 * n_read, cudaMemcpyHostToDevice, E.st));
    }
    cx<double> *W = (cx<double> *)cs.get(sizeof(cx<double>) * nr * chunk);
    cx<double> *state = (cx<double> *)cs.get(sizeof(cx<double>) * nr * (size_t)chunk * nsd * (7 + M));
    cx<double> *drho = (cx<double> *)cs.get(sizeof(cx<double>) * nr * (size_t)chunk * M);
    int ns_max = 0;
    for (int c = 0; c < nch; c++) ns_max = std::max(ns_max, I.ns[c]);

    for (int p0 = 0; p0 < n_pert; p0 += chunk) {
        const int np = std::min(chunk, n_pert - p0);
        CK(cudaMemcpyAsync(W, pert_field + (size_t)p0 * 2 * nr, sizeof(cx<double>) * nr * np, cudaMemcpyHostToDevice,
                           E.st));
        CK(cudaMemsetAsync(state, 0, sizeof(cx<double>) * nr * (size_t)np * nsd * (7 + M), E.st));
        auto buf = [&](int p, int sd, int k) { return state + nr * (((size_t)p * nsd + sd) * (7 + M) + k); };
        for (int t = 0; t < ns_max; t++) {
            std::vector<CJob> ja, jb;
            std::vector<CCombine> cb;
            for (int p = 0; p < np; p++) {
                const int pm = pert_monomer[p0 + p];
                for (int c = 0; c < nch; c++) {
                    const int ns = I.ns[c], nblk = I.sys.n_block[c];
                    if (t >= ns) continue;
                    for (int d = 0; d < 2; d++) {
                        const int sd = 2 * c + d;
                        const int jn = d == 0 ? t + 1 : ns - 1 - t;          // new node
                        const int jp = d == 0 ? t : ns - t;                  // previous node
                        const int blk = seg_block(I, c, d == 0 ? t : jn);
                        const int m = I.sys.block_monomer[c][blk];
                        const bool src = m == pm;
                        // no source yet: the perturbed propagator is still zero
                        if (!src && ((d == 0 && blk == 0) || (d == 1 && blk == nblk - 1))) continue;
                        const double ds = I.bds[c][blk];
                        const double *qprev = (const double *)(d == 0 ? I.qf[c] : I.qr[c]) + (long)jp * nr;
                        const double *q1e = it[c][d].q1 + (long)jn * nr;
                        const double *hm = it[c][d].h + (long)jn * nr;
                        const double *q2e = it[c][d].q2 + (long)jn * nr;
                        cx<double> *dq = buf(p, sd, 0), *A1 = buf(p, sd, 1), *A2 = buf(p, sd, 2), *A3 = buf(p, sd, 3);
                        cx<double> *A4 = buf(p, sd, 4), *A5 = buf(p, sd, 5), *B = buf(p, sd, 6);
                        cx<double> *acc = buf(p, sd, 7);
                        const cx<double> *Wp = W + (long)p * nr;
                        auto job = [&](const cx<double> *a, const cx<double> *bb, double cbv, const double *qa,
                                       const double *qb, int l, cx<double> *o) {
                            CJob J;
                            std::memset(&J, 0, sizeof(J));
                            J.A = a;
                            J.ca = 1.0;
                            J.B = bb;
                            J.cb = cbv;
                            if (qa) {
                                J.W = Wp;
                                J.cw = 1.0;
                                J.qa = qa;
                                J.qb = qb;
                            }
                            J.E = Et[c][blk][l];
                            J.K = Kt[c][blk][l];
                            J.out = o;
                            return J;
                        };
                        // ps_propagate order 0 and order 1 (src/response_step_mod.f90:135-151)
                        ja.push_back(job(dq, nullptr, 0.0, nullptr, nullptr, 0, A1));
                        ja.push_back(job(dq, nullptr, 0.0, nullptr, nullptr, 1, A3));
                        if (src) {
                            ja.push_back(job(nullptr, nullptr, 0.0, qprev, q1e, 1, A2));
                            ja.push_back(job(nullptr, nullptr, 0.0, qprev, hm, 2, A4));
                            ja.push_back(job(nullptr, nullptr, 0.0, hm, q2e, 2, A5));
                        }
                        jb.push_back(job(A3, src ? A4 : nullptr, -ds / 2.0, nullptr, nullptr, 1, B));
                        CCombine k;
                        std::memset(&k, 0, sizeof(k));
                        k.dq = dq;
                        k.A1 = A1;
                        k.A2 = src ? A2 : nullptr;
                        k.A5 = src ? A5 : nullptr;
                        k.B = B;
                        k.ds = ds;
                        k.other = (const double *)(d == 0 ? I.qr[c] : I.qf[c]) + (long)jn * nr;
                        k.acc = acc;
                        for (int mm = 0; mm < M; mm++) k.coef[mm] = coef[c][(size_t)jn * PSCFG_MAXM + mm];
                        k.M = M;
                        cb.push_back(k);
                    }
                }
            }
            if (cb.empty()) continue;
            size_t off = 0;
            const CJob *dja = E.upload(ja, off);
            off += ((ja.size() * sizeof(CJob) + 255) / 256) * 256;
            const CJob *djb = E.upload(jb, off);
            off += ((jb.size() * sizeof(CJob) + 255) / 256) * 256;
            const CCombine *dcb = E.upload(cb, off);
            run_cpasses(E, dja, (int)ja.size(), true, plans);
            run_cpasses(E, djb, (int)jb.size(), true, plans);
            for (size_t j0 = 0; j0 < cb.size(); j0 += 65535) {
                const unsigned nj = (unsigned)std::min<size_t>(65535, cb.size() - j0);
                k_resp_combine<<<dim3(ngrid, nj), 256, 0, E.st>>>(dcb + j0, nr);
                E.launched();
            }
        }
        // 4. drho of every perturbation: sum over sweeps, forward transform / N,
        //    basis readout (kgrid_to_basis with no_parity)
        std::vector<CSum> sums;
        for (int p = 0; p < np; p++)
            for (int mm = 0; mm < M; mm++) {
                CSum sj;
                std::memset(&sj, 0, sizeof(sj));
                sj.dst = drho + nr * ((size_t)p * M + mm);
                for (int sd = 0; sd < nsd; sd++) sj.src[sj.n++] = buf(p, sd, 7) + (long)mm * nr;
                sums.push_back(sj);
            }
        const CSum *dsm = E.upload(sums, 0);
        k_csum<<<dim3(ngrid, (unsigned)sums.size()), 256, 0, E.st>>>(dsm, nr);
        E.launched();
        std::vector<CJob> fj;
        std::vector<CRead> rd;
        for (int q = 0; q < np * M; q++) {
            CJob J;
            std::memset(&J, 0, sizeof(J));
            J.A = drho + nr * (size_t)q;
            J.ca = 1.0;
            J.out = drho + nr * (size_t)q;
            fj.push_back(J);
            CRead r;
            r.spec = drho + nr * (size_t)q;
            r.out = dout + (size_t)q * std::max(n_read, 1);
            rd.push_back(r);
        }
        size_t off = ((sums.size() * sizeof(CSum) + 255) / 256) * 256;
        const CJob *dfj = E.upload(fj, off);
        off += ((fj.size() * sizeof(CJob) + 255) / 256) * 256;
        const CRead *drd = E.upload(rd, off);
        run_cpasses(E, dfj, (int)fj.size(), false, plans);
        if (n_read > 0) {
            k_resp_readout<<<dim3((unsigned)std::min(1024, (n_read + 127) / 128), (unsigned)rd.size()), 128, 0, E.st>>>(
                drd, didx, dcoef, n_read);
            E.launched();
            CK(cudaMemcpyAsync(out + (size_t)p0 * M * n_read, dout, sizeof(double) * (size_t)np * M * n_read,
                               cudaMemcpyDeviceToHost, E.st));
        }
        CK(cudaStreamSynchronize(E.st));
    }
}

// ---------------------------------------------------------------------
// Single-field propagation (parity checks of step_exp)
// ---------------------------------------------------------------------
template <typename T>
static void propagate_impl(Engine &E, int inst, const double *omega_m, double b, double ds, const double *qin,
                           double *qout, int nsteps)
{
    Inst &I = E.inst[inst];
    const size_t ts = sizeof(T);
    // scratch: omega, slab [nsteps+1][nr], tables, 3-D scratch
    double *w = nullptr;
    void *slab = nullptr, *eo1 = nullptr, *eo2 = nullptr, *ek1 = nullptr, *ek2 = nullptr;
    void *S1 = nullptr, *S2 = nullptr, *q1 = nullptr;
    auto cleanup = [&]() {
        cudaFree(w); cudaFree(slab); cudaFree(eo1); cudaFree(eo2); cudaFree(ek1); cudaFree(ek2);
        cudaFree(S1); cudaFree(S2); cudaFree(q1);
    };
    try {
        CK(cudaMalloc(&w, sizeof(double) * E.nr));
        CK(cudaMalloc(&slab, ts * E.nr * (nsteps + 1)));
        CK(cudaMalloc(&eo1, ts * E.nr));
        CK(cudaMalloc(&eo2, ts * E.nr));
        CK(cudaMalloc(&ek1, ts * E.nk));
        CK(cudaMalloc(&ek2, ts * E.nk));
        CK(cudaMalloc(&S1, 2 * ts * E.nk));
        CK(cudaMalloc(&S2, 2 * ts * E.nk));
        CK(cudaMalloc(&q1, ts * E.nr));
        CK(cudaMemcpyAsync(w, omega_m, sizeof(double) * E.nr, cudaMemcpyHostToDevice, E.st));
        std::vector<T> h(E.nr);
        for (long r = 0; r < E.nr; r++) h[r] = (T)qin[r];
        CK(cudaMemcpyAsync(slab, h.data(), ts * E.nr, cudaMemcpyHostToDevice, E.st));
        std::vector<TableJob<T>> tj(1);
        tj[0].omega = w;
        tj[0].ksq = I.ksq;
        tj[0].eo1 = (T *)eo1;
        tj[0].eo2 = (T *)eo2;
        tj[0].ek1 = (T *)ek1;
        tj[0].ek2 = (T *)ek2;
        tj[0].ds = ds;
        tj[0].b = b;
        TableJob<T> *dtj = E.upload(tj, 0);
        SweepField<T> f;
        std::memset(&f, 0, sizeof(f));
        f.slab = (T *)slab;
        f.ns = nsteps;
        f.dir = 1;
        f.nblk = 1;
        f.bgn[0] = 0;
        f.bgn[1] = nsteps;
        f.eo1[0] = (T *)eo1;
        f.eo2[0] = (T *)eo2;
        f.ek1[0] = (T *)ek1;
        f.ek2[0] = (T *)ek2;
        f.S1 = (cx<T> *)S1;
        f.S2 = (cx<T> *)S2;
        f.q1 = (T *)q1;
        std::vector<SweepField<T>> fl(1, f);
        SweepField<T> *dfl = E.upload(fl, 1024);
        k_make_tables<T><<<dim3((unsigned)std::min<long>((E.nr + 255) / 256, 256), 1), 256, 0, E.st>>>(dtj, E.nr, E.nk);
        E.launched();
        const PlaneGeom &g = E.geom();
        if (E.dim <= 2) {
            size_t sm = 2 * (size_t)g.n2 * g.LS * sizeof(cx<T>) + 2 * (size_t)E.nr * sizeof(T);
            if (sm > 227 * 1024) throw Err(PSCFG_EINVAL, "grid too large for the single-CTA plane step");
            CK(allow_dyn_smem((const void *)k_sweep_plane<T>));
            int threads = (int)std::min<long>(256, std::max<long>(32, ((E.nr / 2 + 31) / 32) * 32));
            k_sweep_plane<T><<<1, threads, sm, E.st>>>(dfl, g, 0, nsteps);
            E.launched();
        } else {
            size_t smxy = 2 * (size_t)g.n2 * g.LS * sizeof(cx<T>);
            size_t smz = 2 * (size_t)g.n3 * Z_TILE * sizeof(cx<T>);
            CK(allow_dyn_smem((const void *)k3_fwd_pair<T>));
            CK(allow_dyn_smem((const void *)k3_inv_mid<T>));
            CK(allow_dyn_smem((const void *)k3_inv_final<T>));
            CK(allow_dyn_smem((const void *)k3_zconv<T, Z_TILE>));
            const long P = (long)g.n1h * g.n2;
            const int ntile = (int)((P + Z_TILE - 1) / Z_TILE);
            for (int t = 0; t < nsteps; t++) {
                if (step3_fixed<T>(E, dfl, 1, t)) continue;
                k3_fwd_pair<T><<<dim3(g.n3, 1), 256, smxy, E.st>>>(dfl, g, t);
                E.launched();
                k3_zconv<T, Z_TILE><<<dim3(ntile, 1, 2), 256, smz, E.st>>>(dfl, g, t, 3);
                E.launched();
                k3_inv_mid<T><<<dim3(g.n3, 1), 256, smxy, E.st>>>(dfl, g, t);
                E.launched();
                k3_zconv<T, Z_TILE><<<dim3(ntile, 1, 1), 256, smz, E.st>>>(dfl, g, t, 2);
                E.launched();
                k3_inv_final<T><<<dim3(g.n3, 1), 256, smxy, E.st>>>(dfl, g, t);
                E.launched();
            }
        }
        CK(cudaMemcpyAsync(h.data(), (T *)slab + (long)nsteps * E.nr, ts * E.nr, cudaMemcpyDeviceToHost, E.st));
        CK(cudaStreamSynchronize(E.st));
        for (long r = 0; r < E.nr; r++) qout[r] = (double)h[r];
    } catch (...) {
        cudaStreamSynchronize(E.st);
        cleanup();
        throw;
    }
    cleanup();
}

}  // namespace pscfg

// =====================================================================
// C ABI
// =====================================================================
using namespace pscfg;

struct pscfg_engine {
    Engine E;
    AmRun am;
};

#define ABI_BEGIN try {
#define ABI_END(e)                                    \
    }                                                 \
    catch (const Err &x)                              \
    {                                                 \
        if (e) (e)->E.err = x.msg;                    \
        return x.code;                                \
    }                                                 \
    catch (const std::exception &x)                   \
    {                                                 \
        if (e) (e)->E.err = x.what();                 \
        return PSCFG_EINVAL;                          \
    }                                                 \
    return PSCFG_OK;

extern "C" {

int pscfg_create(const pscfg_system *systems, int n_inst, int precision, pscfg_engine **out)
{
    if (!systems || !out) {
        g_create_error = "null argument";
        return PSCFG_EINVAL;
    }
    *out = nullptr;
    pscfg_engine *e = new (std::nothrow) pscfg_engine();
    if (!e) {
        g_create_error = "host allocation failed";
        return PSCFG_ENOMEM;
    }
    try {
        create_engine(e->E, systems, n_inst, precision);
    } catch (const Err &x) {
        g_create_error = x.msg;
        delete e;
        return x.code;
    }
    *out = e;
    return PSCFG_OK;
}

void pscfg_destroy(pscfg_engine *e) { delete e; }

const char *pscfg_last_error(const pscfg_engine *e)
{
    if (!e) return g_create_error.c_str();
    return e->E.err.c_str();
}

int pscfg_set_cell_param(pscfg_engine *e, int inst, const double *cell_param)
{
    if (!e || !cell_param) return PSCFG_EINVAL;
    ABI_BEGIN
    if (inst < 0 || inst >= (int)e->E.inst.size()) throw Err(PSCFG_EINVAL, "instance index out of range");
    Inst &I = e->E.inst[inst];
    for (int k = 0; k < PSCFG_MAXCP; k++) I.sys.cell_param[k] = cell_param[k];
    upload_cell(e->E, I);
    ABI_END(e)
}

int pscfg_get_ksq(pscfg_engine *e, int inst, double *ksq)
{
    if (!e || !ksq) return PSCFG_EINVAL;
    ABI_BEGIN
    if (inst < 0 || inst >= (int)e->E.inst.size()) throw Err(PSCFG_EINVAL, "instance index out of range");
    CK(cudaMemcpyAsync(ksq, e->E.inst[inst].ksq, sizeof(double) * e->E.nk, cudaMemcpyDeviceToHost, e->E.st));
    CK(cudaStreamSynchronize(e->E.st));
    ABI_END(e)
}

static int density_common(pscfg_engine *e, const double *omega, double *rho, double *q, double *qs, bool device)
{
    ABI_BEGIN
    Engine &E = e->E;
    const long fl = (long)E.M * E.nr;
    const int ni = (int)E.inst.size();
    for (int i = 0; i < ni; i++)
        CK(cudaMemcpyAsync(E.inst[i].omega, omega + (long)i * fl, sizeof(double) * fl,
                           device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, E.st));
    std::vector<int> all(ni);
    for (int i = 0; i < ni; i++) all[i] = i;
    density_all(E, all);
    if (rho) {
        for (int i = 0; i < ni; i++)
            CK(cudaMemcpyAsync(rho + (long)i * fl, E.inst[i].rho, sizeof(double) * fl,
                               device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, E.st));
    }
    CK(cudaStreamSynchronize(E.st));
    for (int i = 0; i < ni; i++) {
        if (q)
            for (int c = 0; c < PSCFG_MAXC; c++) q[(long)i * PSCFG_MAXC + c] = (c < E.inst[i].sys.n_chain) ? E.inst[i].Q[c] : 0.0;
        if (qs)
            for (int s = 0; s < PSCFG_MAXS; s++)
                qs[(long)i * PSCFG_MAXS + s] = (s < E.inst[i].sys.n_solvent) ? E.inst[i].Qs[s] : 0.0;
    }
    ABI_END(e)
}

int pscfg_density(pscfg_engine *e, const double *omega, double *rho, double *q, double *q_solvent)
{
    if (!e || !omega) return PSCFG_EINVAL;
    return density_common(e, omega, rho, q, q_solvent, false);
}

int pscfg_density_device(pscfg_engine *e, const double *omega_dev, double *rho_dev, double *q, double *q_solvent)
{
    if (!e || !omega_dev) return PSCFG_EINVAL;
    return density_common(e, omega_dev, rho_dev, q, q_solvent, true);
}

int pscfg_stress(pscfg_engine *e, double *stress)
{
    if (!e || !stress) return PSCFG_EINVAL;
    ABI_BEGIN
    Engine &E = e->E;
    const int ni = (int)E.inst.size();
    std::vector<int> all(ni);
    for (int i = 0; i < ni; i++) all[i] = i;
    stress_all(E, all);
    for (int i = 0; i < ni; i++)
        CK(cudaMemcpyAsync(stress + (long)i * PSCFG_MAXCP, E.inst[i].stress_dev, sizeof(double) * PSCFG_MAXCP,
                           cudaMemcpyDeviceToHost, E.st));
    CK(cudaStreamSynchronize(E.st));
    for (int i = 0; i < ni; i++)
        for (int b = E.inst[i].cell.ncp; b < PSCFG_MAXCP; b++) stress[(long)i * PSCFG_MAXCP + b] = 0.0;
    ABI_END(e)
}

int pscfg_free_energy(pscfg_engine *e, double *out, double *mu_chain)
{
    if (!e || !out) return PSCFG_EINVAL;
    ABI_BEGIN
    Engine &E = e->E;
    const int ni = (int)E.inst.size();
    std::vector<int> all(ni);
    for (int i = 0; i < ni; i++) {
        all[i] = i;
        if (!E.inst[i].have_density) throw Err(PSCFG_ESTATE, "free_energy requires a preceding density call");
    }
    std::vector<double> f, p;
    free_energy_all(E, all, f, p);
    for (int i = 0; i < ni; i++) {
        out[2 * i] = f[i];
        out[2 * i + 1] = p[i];
        if (mu_chain)
            for (int c = 0; c < PSCFG_MAXC; c++)
                mu_chain[(long)i * PSCFG_MAXC + c] = (c < E.inst[i].sys.n_chain) ? E.inst[i].sys.mu_chain[c] : 0.0;
    }
    ABI_END(e)
}

static void load_omega(Engine &E, const double *omega)
{
    const long fl = (long)E.M * E.nr;
    for (size_t i = 0; i < E.inst.size(); i++)
        CK(cudaMemcpyAsync(E.inst[i].omega, omega + (long)i * fl, sizeof(double) * fl, cudaMemcpyHostToDevice, E.st));
}

static void store_fields(Engine &E, double *omega, double *rho)
{
    const long fl = (long)E.M * E.nr;
    for (size_t i = 0; i < E.inst.size(); i++) {
        if (omega) CK(cudaMemcpyAsync(omega + (long)i * fl, E.inst[i].omega, sizeof(double) * fl, cudaMemcpyDeviceToHost, E.st));
        if (rho) CK(cudaMemcpyAsync(rho + (long)i * fl, E.inst[i].rho, sizeof(double) * fl, cudaMemcpyDeviceToHost, E.st));
    }
    CK(cudaStreamSynchronize(E.st));
}

int pscfg_iterate_am(pscfg_engine *e, double *omega, const pscfg_am_param *prm, double *rho, pscfg_am_result *results)
{
    if (!e || !omega || !prm || !results) return PSCFG_EINVAL;
    ABI_BEGIN
    Engine &E = e->E;
    load_omega(E, omega);
    am_begin(E, e->am, *prm);
    while (am_iterate(E, e->am, 1 << 30) > 0) {
    }
    std::vector<pscfg_am_result> res;
    am_results(E, e->am, res);
    e->am.active = false;
    int any_fail = 0;
    for (size_t i = 0; i < res.size(); i++) {
        results[i] = res[i];
        if (!res[i].converged) any_fail = 1;
    }
    store_fields(E, omega, rho);
    if (any_fail) {
        E.err = "at least one instance did not converge";
        return PSCFG_ENOTCONV;
    }
    ABI_END(e)
}

int pscfg_am_begin(pscfg_engine *e, const double *omega, const pscfg_am_param *prm)
{
    if (!e || !prm) return PSCFG_EINVAL;
    ABI_BEGIN
    if (omega) load_omega(e->E, omega);
    am_begin(e->E, e->am, *prm);
    ABI_END(e)
}

int pscfg_am_iterate(pscfg_engine *e, int iters, int *remaining)
{
    if (!e || iters < 0) return PSCFG_EINVAL;
    ABI_BEGIN
    int r = am_iterate(e->E, e->am, iters);
    if (remaining) *remaining = r;
    ABI_END(e)
}

int pscfg_am_results(pscfg_engine *e, double *omega, double *rho, pscfg_am_result *results)
{
    if (!e || !results) return PSCFG_EINVAL;
    ABI_BEGIN
    std::vector<pscfg_am_result> res;
    am_results(e->E, e->am, res);
    for (size_t i = 0; i < res.size(); i++) results[i] = res[i];
    store_fields(e->E, omega, rho);
    ABI_END(e)
}

int pscfg_set_basis(pscfg_engine *e, int inst, int n_star, int n_wave, const int *wave_k, const int *wave_star,
                    const double *coeff)
{
    if (!e || n_star < 0 || n_wave < 0 || (n_wave > 0 && (!wave_k || !wave_star || !coeff))) return PSCFG_EINVAL;
    ABI_BEGIN
    Engine &E = e->E;
    if (inst < 0 || inst >= (int)E.inst.size()) throw Err(PSCFG_EINVAL, "instance index out of range");
    Inst &I = E.inst[inst];
    std::vector<char> seen(E.nk, 0);
    std::vector<int> order(n_wave), count(n_star + 1, 0);
    for (int j = 0; j < n_wave; j++) {
        if (wave_k[j] < 0 || wave_k[j] >= E.nk) throw Err(PSCFG_EINVAL, "wave index outside the half grid");
        if (wave_star[j] < 0 || wave_star[j] >= n_star) throw Err(PSCFG_EINVAL, "star index out of range");
        // at most two functions per wave: the pair of a star and its inverse
        if (seen[wave_k[j]] >= 2) throw Err(PSCFG_EINVAL, "a half-grid wave appears more than twice in the basis");
        seen[wave_k[j]]++;
        count[wave_star[j] + 1]++;
    }
    for (int s2 = 0; s2 < n_star; s2++) count[s2 + 1] += count[s2];
    {   // stable sort by star
        std::vector<int> pos(count.begin(), count.end() - 1);
        for (int j = 0; j < n_wave; j++) order[pos[wave_star[j]]++] = j;
    }
    const size_t a256 = 256;
    auto al = [&](size_t b) { return (b + a256 - 1) / a256 * a256; };
    const size_t o_k = al(sizeof(int) * (n_star + 1)), o_s = o_k + al(sizeof(int) * n_wave),
                 o_c = o_s + al(sizeof(int) * n_wave), total = o_c + sizeof(cx<double>) * std::max(n_wave, 1);
    std::vector<unsigned char> h(total, 0);
    std::memcpy(h.data(), count.data(), sizeof(int) * (n_star + 1));
    for (int j = 0; j < n_wave; j++) {
        const int src = order[j];
        ((int *)(h.data() + o_k))[j] = wave_k[src];
        ((int *)(h.data() + o_s))[j] = wave_star[src];
        ((double *)(h.data() + o_c))[2 * j] = coeff[2 * src];
        ((double *)(h.data() + o_c))[2 * j + 1] = coeff[2 * src + 1];
    }
    if (I.basis_buf) {
        CK(cudaStreamSynchronize(E.st));
        cudaFree(I.basis_buf);
        I.basis_buf = nullptr;
    }
    CK(cudaMalloc(&I.basis_buf, total));
    CK(cudaMemcpy(I.basis_buf, h.data(), total, cudaMemcpyHostToDevice));
    unsigned char *d = (unsigned char *)I.basis_buf;
    I.b_start = (const int *)d;
    I.b_k = (const int *)(d + o_k);
    I.b_star = (const int *)(d + o_s);
    I.b_c = (const cx<double> *)(d + o_c);
    I.n_star = n_star;
    I.n_wave = n_wave;
    ABI_END(e)
}

// Half spectra -> real fields (unnormalised c2r), or real fields -> half
// spectra (unnormalised r2c), for nf fields.
static void field_ffts(Engine &E, const std::vector<const double *> &re_in, const std::vector<double *> &re_out,
                       const std::vector<cx<double> *> &spec, bool inverse)
{
    const PlaneGeom &g = E.g64;
    const int nf = (int)spec.size();
    if (nf == 0) return;
    cx<double> **dspec = E.upload(spec, 0);
    size_t off = ((spec.size() * sizeof(void *) + 255) / 256) * 256;
    const size_t smxy = 2 * (size_t)g.n2 * g.LS * sizeof(cx<double>);
    const long P = (long)g.n1h * g.n2;
    const int ntile = (int)((P + Z_TILE - 1) / Z_TILE);
    const size_t smz = 2 * (size_t)g.n3 * Z_TILE * sizeof(cx<double>);
    if (smxy > 227 * 1024 || (E.dim == 3 && smz > 227 * 1024))
        throw Err(PSCFG_EINVAL, "grid plane too large for the basis maps");
    if (inverse) {
        double **dout = E.upload(re_out, off);
        if (E.dim <= 2) {
            CK(allow_dyn_smem((const void *)k2_ifft_fields));
            const int threads = (int)std::min<long>(256, std::max<long>(32, ((E.nr / 2 + 31) / 32) * 32));
            k2_ifft_fields<<<nf, threads, smxy, E.st>>>((const cx<double> *const *)dspec, dout, g);
            E.launched();
        } else {
            CK(allow_dyn_smem((const void *)k3_ifft_fields_z<Z_TILE>));
            CK(allow_dyn_smem((const void *)k3_ifft_fields_xy));
            k3_ifft_fields_z<Z_TILE><<<dim3(ntile, nf), 256, smz, E.st>>>(dspec, g);
            E.launched();
            k3_ifft_fields_xy<<<dim3(g.n3, nf), 256, smxy, E.st>>>((const cx<double> *const *)dspec, dout, g);
            E.launched();
        }
    } else {
        const double **din = (const double **)E.upload(re_in, off);
        if (E.dim <= 2) {
            CK(allow_dyn_smem((const void *)k2_fft_fields));
            const int threads = (int)std::min<long>(256, std::max<long>(32, ((E.nr / 2 + 31) / 32) * 32));
            k2_fft_fields<<<nf, threads, smxy, E.st>>>(din, dspec, g);
            E.launched();
        } else {
            CK(allow_dyn_smem((const void *)k3_fft_fields_xy));
            CK(allow_dyn_smem((const void *)k3_fft_fields_z<Z_TILE>));
            k3_fft_fields_xy<<<dim3(g.n3, nf), 256, smxy, E.st>>>(din, dspec, g);
            E.launched();
            k3_fft_fields_z<Z_TILE><<<dim3(ntile, nf), 256, smz, E.st>>>(dspec, g);
            E.launched();
        }
    }
}

int pscfg_density_basis(pscfg_engine *e, const double *omega_basis, double *rho_basis, double *q, double *q_solvent)
{
    if (!e || !omega_basis) return PSCFG_EINVAL;
    ABI_BEGIN
    Engine &E = e->E;
    const int ni = (int)E.inst.size(), M = E.M;
    long ncoef = 0, max_star = 0, max_wave = 0;
    for (auto &I : E.inst) {
        if (!I.basis_buf) throw Err(PSCFG_ESTATE, "pscfg_density_basis needs pscfg_set_basis on every instance");
        ncoef += (long)M * I.n_star;
        max_star = std::max<long>(max_star, I.n_star);
        max_wave = std::max<long>(max_wave, I.n_wave);
    }
    // scratch: one half spectrum per (instance, monomer), coefficients in and out
    const size_t spec_bytes = sizeof(cx<double>) * (size_t)E.nk * ni * M;
    const size_t need = spec_bytes + 2 * sizeof(double) * (size_t)std::max<long>(ncoef, 1);
    if (E.basis_scr_bytes < need) {
        if (E.basis_scr) {
            CK(cudaStreamSynchronize(E.st));
            cudaFree(E.basis_scr);
        }
        E.basis_scr = nullptr;
        CK(cudaMalloc(&E.basis_scr, need));
        E.basis_scr_bytes = need;
    }
    cx<double> *spec = (cx<double> *)E.basis_scr;
    double *cin = (double *)((char *)E.basis_scr + spec_bytes), *cout = cin + std::max<long>(ncoef, 1);
    CK(cudaMemcpyAsync(cin, omega_basis, sizeof(double) * ncoef, cudaMemcpyHostToDevice, E.st));
    CK(cudaMemsetAsync(spec, 0, spec_bytes, E.st));
    std::vector<BasisJob> jobs;
    std::vector<cx<double> *> sp;
    std::vector<double *> wout;
    std::vector<const double *> rin;
    long off_c = 0;
    for (int i = 0; i < ni; i++) {
        Inst &I = E.inst[i];
        for (int a = 0; a < M; a++) {
            BasisJob j;
            j.start = I.b_start;
            j.wave_k = I.b_k;
            j.wave_star = I.b_star;
            j.c = I.b_c;
            j.n_star = I.n_star;
            j.n_wave = I.n_wave;
            j.S = spec + ((size_t)i * M + a) * E.nk;
            j.a = cin + off_c;
            j.out = cout + off_c;
            off_c += I.n_star;
            jobs.push_back(j);
            sp.push_back(j.S);
            wout.push_back(I.omega + (long)a * E.nr);
            rin.push_back(I.rho + (long)a * E.nr);
        }
    }
    const int nj = (int)jobs.size();
    // basis_to_kgrid + inverse FFT: omega on the grid
    BasisJob *dj = E.upload(jobs, (size_t)4 << 20);
    k_basis_scatter<<<dim3((unsigned)std::max<long>(1, std::min<long>((max_wave + 255) / 256, 1024)), nj), 256, 0, E.st>>>(dj);
    E.launched();
    field_ffts(E, {}, wout, sp, true);
    std::vector<int> all(ni);
    for (int i = 0; i < ni; i++) all[i] = i;
    density_all(E, all);
    if (rho_basis) {
        // forward FFT + kgrid_to_basis of rho
        field_ffts(E, rin, {}, sp, false);
        dj = E.upload(jobs, (size_t)4 << 20);
        k_basis_gather<<<dim3((unsigned)std::max<long>(1, (max_star + 7) / 8), nj), 256, 0, E.st>>>(dj, E.n[0],
                                                                                                   1.0 / (double)E.nr);
        E.launched();
        CK(cudaMemcpyAsync(rho_basis, cout, sizeof(double) * ncoef, cudaMemcpyDeviceToHost, E.st));
    }
    CK(cudaStreamSynchronize(E.st));
    for (int i = 0; i < ni; i++) {
        if (q)
            for (int c = 0; c < PSCFG_MAXC; c++) q[(long)i * PSCFG_MAXC + c] = (c < E.inst[i].sys.n_chain) ? E.inst[i].Q[c] : 0.0;
        if (q_solvent)
            for (int s2 = 0; s2 < PSCFG_MAXS; s2++)
                q_solvent[(long)i * PSCFG_MAXS + s2] = (s2 < E.inst[i].sys.n_solvent) ? E.inst[i].Qs[s2] : 0.0;
    }
    ABI_END(e)
}

int pscfg_set_symmetry(pscfg_engine *e, int inst, int nops, const int *ops)
{
    if (!e || nops < 0 || (nops > 0 && !ops)) return PSCFG_EINVAL;
    ABI_BEGIN
    Engine &E = e->E;
    if (inst < 0 || inst >= (int)E.inst.size()) throw Err(PSCFG_EINVAL, "instance index out of range");
    Inst &I = E.inst[inst];
    if (nops > 1024) throw Err(PSCFG_EINVAL, "too many group elements");
    if (nops > 0) {
        // real-space orbits r -> M r + t (mod n), grouped for the projection
        {
            std::vector<int> perm, start, img(nops);
            std::vector<char> seen_r(E.nr, 0);
            perm.reserve(E.nr);
            for (long r = 0; r < E.nr; r++) {
                if (seen_r[r]) continue;
                start.push_back((int)perm.size());
                const int i[3] = {(int)(r % E.n[0]), (int)((r / E.n[0]) % E.n[1]), (int)(r / ((long)E.n[0] * E.n[1]))};
                for (int k = 0; k < nops; k++) {
                    const int *o = ops + 12 * k;
                    long j[3];
                    for (int a = 0; a < 3; a++) {
                        long v = o[9 + a] + (long)o[3 * a] * i[0] + (long)o[3 * a + 1] * i[1] + (long)o[3 * a + 2] * i[2];
                        v %= E.n[a];
                        if (v < 0) v += E.n[a];
                        j[a] = v;
                    }
                    const long rr = j[0] + (long)E.n[0] * (j[1] + (long)E.n[1] * j[2]);
                    if (!seen_r[rr]) {
                        seen_r[rr] = 1;
                        perm.push_back((int)rr);
                    }
                }
                if (!seen_r[r]) throw Err(PSCFG_EINVAL, "group elements do not include the identity");
            }
            start.push_back((int)perm.size());
            if (!I.d_orb_perm) I.d_orb_perm = (int *)E.dalloc(sizeof(int) * E.nr);
            if (!I.d_orb_start) I.d_orb_start = (int *)E.dalloc(sizeof(int) * (E.nr + 1));
            I.norb = (int)start.size() - 1;
            CK(cudaMemcpyAsync(I.d_orb_perm, perm.data(), sizeof(int) * E.nr, cudaMemcpyHostToDevice, E.st));
            CK(cudaMemcpyAsync(I.d_orb_start, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice, E.st));
            CK(cudaStreamSynchronize(E.st));
        }
        // Star weights: a star is the orbit of a wave G under the point
        // group (G -> G.m, src/group_mod.f90:77-78) on the FFT grid; the
        // reference normalises its star coefficients with a single-precision
        // sqrt(real(star_N)) (src/basis_mod.f90:920), so its star sums weight
        // a star of N waves by fl32(sqrt(N))^2 / N.
        std::vector<double> kw(E.nk);
        std::vector<long> seen(nops);
        const int n1h = E.n[0] / 2 + 1;
        for (int i3 = 0; i3 < E.n[2]; i3++)
            for (int i2 = 0; i2 < E.n[1]; i2++)
                for (int i1 = 0; i1 < n1h; i1++) {
                    const int G[3] = {i1, i2, i3};
                    int cnt = 0;
                    for (int k = 0; k < nops; k++) {
                        const int *m = ops + 12 * k;
                        long key = 0;
                        for (int j = 0; j < 3; j++) {
                            long v = 0;
                            for (int i = 0; i < 3; i++) v += (long)G[i] * m[3 * i + j];
                            v %= E.n[j];
                            if (v < 0) v += E.n[j];
                            key = key * E.n[j] + v;
                        }
                        bool dup = false;
                        for (int q = 0; q < cnt; q++)
                            if (seen[q] == key) { dup = true; break; }
                        if (!dup) seen[cnt++] = key;
                    }
                    const float sf = std::sqrt((float)cnt);
                    kw[i1 + (long)n1h * (i2 + (long)E.n[1] * i3)] = ((double)sf * (double)sf) / (double)cnt;
                }
        if (!I.kweight) I.kweight = (double *)E.dalloc(sizeof(double) * E.nk);
        CK(cudaMemcpyAsync(I.kweight, kw.data(), sizeof(double) * E.nk, cudaMemcpyHostToDevice, E.st));
        CK(cudaStreamSynchronize(E.st));
    } else {
        I.kweight = nullptr;
    }
    I.nops = nops;
    update_cells(E, std::vector<int>{inst});
    CK(cudaStreamSynchronize(E.st));
    ABI_END(e)
}

void *pscfg_stream(const pscfg_engine *e) { return e ? (void *)e->E.st : nullptr; }

static int adjoint_common(pscfg_engine *e, const double *grad_rho, const double *grad_lnq, double *grad_omega, bool device,
                          double *grad_cell = nullptr)
{
    if (!e || !grad_rho || !grad_omega) return PSCFG_EINVAL;
    ABI_BEGIN
    Engine &E = e->E;
    const int ni = (int)E.inst.size();
    const long fl = (long)E.M * E.nr;
    std::vector<int> all(ni);
    std::vector<const double *> G(ni), gQ(ni);
    std::vector<double *> out(ni);
    double *tmp = nullptr;
    if (!device) {
        // stage host arrays in one device buffer: G then grad
        CK(cudaMalloc(&tmp, sizeof(double) * fl * ni * 2));
    }
    for (int i = 0; i < ni; i++) {
        all[i] = i;
        if (device) {
            G[i] = grad_rho + (long)i * fl;
            out[i] = grad_omega + (long)i * fl;
        } else {
            CK(cudaMemcpyAsync(tmp + (long)i * fl, grad_rho + (long)i * fl, sizeof(double) * fl, cudaMemcpyHostToDevice, E.st));
            G[i] = tmp + (long)i * fl;
            out[i] = tmp + (long)(ni + i) * fl;
        }
        gQ[i] = grad_lnq ? grad_lnq + (long)i * PSCFG_MAXC : nullptr;
    }
    try {
        std::vector<double *> gc;
        if (grad_cell)
            for (int i = 0; i < ni; i++) gc.push_back(grad_cell + (long)i * PSCFG_MAXCP);
        adjoint_all(E, all, G, gQ, out, gc);
        if (!device) {
            for (int i = 0; i < ni; i++)
                CK(cudaMemcpyAsync(grad_omega + (long)i * fl, out[i], sizeof(double) * fl, cudaMemcpyDeviceToHost, E.st));
        }
        CK(cudaStreamSynchronize(E.st));
    } catch (...) {
        if (tmp) cudaFree(tmp);
        throw;
    }
    if (tmp) cudaFree(tmp);
    ABI_END(e)
}

int pscfg_density_adjoint(pscfg_engine *e, const double *grad_rho, const double *grad_lnq, double *grad_omega)
{
    return adjoint_common(e, grad_rho, grad_lnq, grad_omega, false);
}

int pscfg_density_adjoint_device(pscfg_engine *e, const double *grad_rho_dev, const double *grad_lnq,
                                 double *grad_omega_dev)
{
    return adjoint_common(e, grad_rho_dev, grad_lnq, grad_omega_dev, true);
}

int pscfg_density_adjoint_cell(pscfg_engine *e, const double *grad_rho, const double *grad_lnq, double *grad_omega,
                               double *grad_cell)
{
    if (!grad_cell) return PSCFG_EINVAL;
    return adjoint_common(e, grad_rho, grad_lnq, grad_omega, false, grad_cell);
}

int pscfg_response(pscfg_engine *e, int inst, const double *kvec, double ktrans_sq, int n_pert,
                   const int *pert_monomer, const double *pert_field, int n_read, const int *read_index,
                   const double *read_coef, double *out)
{
    if (!e || !kvec || n_pert < 0 || n_read < 0 || (n_pert > 0 && (!pert_monomer || !pert_field)) ||
        (n_read > 0 && (!read_index || !read_coef || !out)))
        return PSCFG_EINVAL;
    ABI_BEGIN
    Engine &E = e->E;
    if (inst < 0 || inst >= (int)E.inst.size()) throw Err(PSCFG_EINVAL, "instance index out of range");
    if (n_pert > 0) response_impl(E, inst, kvec, ktrans_sq, n_pert, pert_monomer, pert_field, n_read, read_index,
                                  read_coef, out);
    ABI_END(e)
}

int pscfg_set_profiling(pscfg_engine *e, int on)
{
    if (!e) return PSCFG_EINVAL;
    ABI_BEGIN
    Engine &E = e->E;
    if (on && !E.ev0) {
        CK(cudaEventCreate(&E.ev0));
        CK(cudaEventCreate(&E.ev1));
    }
    E.profiling = on != 0;
    E.t_sweep = E.t_contour = E.t_stress = E.t_mix = 0;
    E.n_steps_timed = 0;
    E.sweep_launches = 0;
    ABI_END(e)
}

int pscfg_get_profile(const pscfg_engine *e, double *out)
{
    if (!e || !out) return PSCFG_EINVAL;
    const Engine &E = e->E;
    out[0] = E.t_sweep;
    out[1] = E.t_contour;
    out[2] = E.t_stress;
    out[3] = E.t_mix;
    out[4] = (double)E.n_steps_timed;
    out[5] = (double)E.sweep_launches;
    return PSCFG_OK;
}

int pscfg_propagate(pscfg_engine *e, int inst, const double *omega_m, double b, double ds, const double *q_in,
                    double *q_out, int nsteps)
{
    if (!e || !omega_m || !q_in || !q_out || nsteps < 1) return PSCFG_EINVAL;
    ABI_BEGIN
    if (inst < 0 || inst >= (int)e->E.inst.size()) throw Err(PSCFG_EINVAL, "instance index out of range");
    if (e->E.prec == PSCFG_FP32) {
        e->E.cur = PSCFG_FP32;
        propagate_impl<float>(e->E, inst, omega_m, b, ds, q_in, q_out, nsteps);
    } else {
        e->E.cur = PSCFG_FP64;
        propagate_impl<double>(e->E, inst, omega_m, b, ds, q_in, q_out, nsteps);
    }
    ABI_END(e)
}

int pscfg_get_propagators(pscfg_engine *e, int inst, int chain, double *qf, double *qr, int *n_slices)
{
    if (!e) return PSCFG_EINVAL;
    ABI_BEGIN
    Engine &E = e->E;
    if (inst < 0 || inst >= (int)E.inst.size()) throw Err(PSCFG_EINVAL, "instance index out of range");
    Inst &I = E.inst[inst];
    if (chain < 0 || chain >= I.sys.n_chain) throw Err(PSCFG_EINVAL, "chain index out of range");
    const long ns = I.ns[chain] + 1;
    if (n_slices) *n_slices = (int)ns;
    if (E.ckpt && (qf || qr)) {
        // rebuild the slices from the checkpoints, segment by segment
        if (!I.have_density) throw Err(PSCFG_ESTATE, "no propagators before a density call");
        const bool f32 = I.dens_prec == PSCFG_FP32;
        E.cur = f32 ? PSCFG_FP32 : PSCFG_FP64;
        const std::vector<int> one{inst};
        const std::vector<CkChain> ch{CkChain{inst, chain}};
        const int K = E.ckK;
        std::vector<float> hf;
        auto seg_out = [&](const void *seg, int s0, int cnt, double *dst) {
            if (!dst || cnt <= 0) return;
            if (!f32) {
                CK(cudaMemcpyAsync(dst + (long)s0 * E.nr, seg, sizeof(double) * E.nr * cnt, cudaMemcpyDeviceToHost, E.st));
                CK(cudaStreamSynchronize(E.st));
            } else {
                hf.resize((size_t)E.nr * cnt);
                CK(cudaMemcpyAsync(hf.data(), seg, sizeof(float) * E.nr * cnt, cudaMemcpyDeviceToHost, E.st));
                CK(cudaStreamSynchronize(E.st));
                for (long k = 0; k < E.nr * cnt; k++) dst[(long)s0 * E.nr + k] = hf[k];
            }
        };
        for (int j = 0; j < I.nseg[chain]; j++) {
            const int s0 = j * K, cnt = (j == I.nseg[chain] - 1) ? I.ns[chain] + 1 - s0 : K;
            if (f32) {
                std::vector<const float *> ekf;
                ckpt_tables<float>(E, one, ekf);
                ckpt_segment<float>(E, ch, ekf, j, +1, false);
                ckpt_segment<float>(E, ch, ekf, j, -1, false);
            } else {
                std::vector<const double *> ekf;
                ckpt_tables<double>(E, one, ekf);
                ckpt_segment<double>(E, ch, ekf, j, +1, false);
                ckpt_segment<double>(E, ch, ekf, j, -1, false);
            }
            seg_out(I.segA[chain], s0, cnt, qf);
            seg_out(I.segB[chain], s0, cnt, qr);
        }
        return PSCFG_OK;
    }
    for (int d = 0; d < 2; d++) {
        double *dst = d == 0 ? qf : qr;
        if (!dst) continue;
        const void *src = d == 0 ? I.qf[chain] : I.qr[chain];
        if (I.prec_now != PSCFG_FP32) {
            CK(cudaMemcpyAsync(dst, src, sizeof(double) * E.nr * ns, cudaMemcpyDeviceToHost, E.st));
            CK(cudaStreamSynchronize(E.st));
        } else {
            std::vector<float> h(E.nr * ns);
            CK(cudaMemcpyAsync(h.data(), src, sizeof(float) * E.nr * ns, cudaMemcpyDeviceToHost, E.st));
            CK(cudaStreamSynchronize(E.st));
            for (long k = 0; k < E.nr * ns; k++) dst[k] = h[k];
        }
    }
    ABI_END(e)
}

long pscfg_steps_per_density(const pscfg_engine *e)
{
    if (!e) return 0;
    long s = 0;
    for (const Inst &I : e->E.inst)
        for (int c = 0; c < I.sys.n_chain; c++) s += 2L * I.ns[c];
    return s;
}

long pscfg_launch_count(const pscfg_engine *e) { return e ? e->E.launches : 0; }

int pscfg_sweep_planes(const pscfg_engine *e, int n_fields, int fp32)
{
    if (!e || e->E.dim != 3 || e->E.n[0] != e->E.n[1] || e->E.n[1] != e->E.n[2]) return 0;
    const int n3 = e->E.n[2];
    if (n3 != 16 && n3 != 32) return 0;
    const long key = planes_key(n3, fp32 ? 4 : 8, n_fields);
    std::lock_guard<std::mutex> lk(g_planes_mu);
    auto it = g_planes_best.find(key);
    if (it == g_planes_best.end()) return 0;
    return it->second > 0 ? it->second : -1;   // 0 in the cache: the cluster step
}

}  // extern "C"
