// noalloc.cu -- MDE propagation that allocates no device memory.
//
// pscfg_propagate (engine.cu) allocates its scratch with cudaMalloc on every
// call.  Some hosts cannot let a library do that: a program that hands its
// whole device memory budget to its own pool (a Fortran host running many
// solver instances side by side, or a framework whose caching allocator owns
// the device) needs every call to stay inside memory it already knows about.
// pscfg_propagate_noalloc runs the same kernels with all of its scratch in
// one file-scope device array (g_scratch below), sized for grids of at most
// PSCFG_NOALLOC_MAX_NR points; every GPU that loads this library holds that
// array until the process exits.
//
// The array is shared by every call on a device and keeps whatever the last
// call left in it.  Each call writes every scratch entry it later reads
// (tables, spectra, the two working slices), so nothing needs clearing
// between calls, but calls whose work overlaps on the GPU (two host threads,
// or two streams without an ordering between them) race on the array.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/pscf_gpu.h"
#include "host_geom.h"
#include "kernels.cuh"
#include "launch_util.h"

namespace pscfg {
void set_global_error(const std::string &msg);   // engine.cu
}

namespace pscfg_noalloc {

using namespace pscfg;

constexpr long MAX_NR = PSCFG_NOALLOC_MAX_NR;
constexpr int MAX_LINE = PSCFG_NOALLOC_MAX_LINE;
constexpr int Z_TILE = 16;

// Byte layout of the scratch array (each part 256-byte aligned).
constexpr size_t al(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t TW_BYTES = al(sizeof(cx<double>) * MAX_LINE);    // one twiddle table
constexpr size_t OFF_TW = 0;                                        // 4 tables
constexpr size_t OFF_DESC = OFF_TW + 4 * TW_BYTES;                  // TableJob + 4 SweepFields
constexpr size_t DESC_BYTES = al(sizeof(TableJob<double>)) + al(4 * sizeof(SweepField<double>));
constexpr size_t OFF_REAL = OFF_DESC + DESC_BYTES;                  // eo1, eo2, q1, slab[2]: 5 nr
constexpr size_t REAL_BYTES = al(sizeof(double) * MAX_NR);
constexpr size_t OFF_EK = OFF_REAL + 5 * REAL_BYTES;                // ek1, ek2: 2 nk (nk <= nr)
constexpr size_t OFF_SPEC = OFF_EK + 2 * REAL_BYTES;                // S1, S2: 2 nk complex
constexpr size_t SCRATCH_BYTES = OFF_SPEC + 2 * al(sizeof(cx<double>) * MAX_NR);

static __device__ __align__(256) unsigned char g_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
static std::mutex g_mutex;
static unsigned char *g_scratch_addr[MAX_DEVICES] = {};

static int fail(int code, const std::string &msg)
{
    pscfg::set_global_error(msg);   // read back with pscfg_last_error(NULL)
    return code;
}

#define CKN(call)                                                                         \
    do {                                                                                  \
        cudaError_t _e = (call);                                                          \
        if (_e != cudaSuccess) return fail(PSCFG_ECUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
    } while (0)

// Device address of g_scratch on the current device.  In host code the
// symbol g_scratch is only a host-side stand-in; the address a kernel may
// use comes from cudaGetSymbolAddress, looked up once per device (with that
// device current) on the first call made on it.  The same set-up uploads
// the radix-5/7 codelet constants of this translation unit.
static int scratch_address(unsigned char **out)
{
    int dev = 0;
    CKN(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return fail(PSCFG_EINVAL, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p)
            return fail(PSCFG_ECUDA, std::string("cudaGetSymbolAddress(g_scratch): ") + cudaGetErrorString(e));
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
        CKN(cudaMemcpyToSymbol(c_dft5, t5, sizeof(t5)));
        CKN(cudaMemcpyToSymbol(c_dft7, t7, sizeof(t7)));
        g_scratch_addr[dev] = (unsigned char *)p;
    }
    *out = g_scratch_addr[dev];
    return PSCFG_OK;
}

// The descriptors of one call, passed by value to k_setup.  f[0]: first
// step (reads q_in), f[1]: slice 0 -> 1, f[2]: slice 1 -> 0, f[3]: last step
// (writes q_out).
struct Descs {
    TableJob<double> tj;
    SweepField<double> f[4];
};

// Writes the call's descriptors and its four twiddle tables W_n^m (forward
// sign, m < n, n = lens) into the scratch array, so that a call issues
// kernel launches only (no host-to-device copies).
__global__ void k_setup(Descs d, TableJob<double> *dtj, SweepField<double> *dfl, unsigned char *tw0, int4 lens,
                        long tw_stride)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *dtj = d.tj;
        for (int k = 0; k < 4; k++) dfl[k] = d.f[k];
    }
    const int ln[4] = {lens.x, lens.y, lens.z, lens.w};
    for (int k = 0; k < 4; k++) {
        cx<double> *tw = (cx<double> *)(tw0 + k * tw_stride);
        for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < ln[k]; m += gridDim.x * blockDim.x) {
            double sv, cv;
            sincospi(2.0 * (double)m / (double)ln[k], &sv, &cv);
            tw[m].x = cv;
            tw[m].y = -sv;
        }
    }
}

}  // namespace pscfg_noalloc

using namespace pscfg_noalloc;

extern "C" int pscfg_propagate_noalloc(int dim, const int *n, const double *ksq_dev, const double *omega_dev,
                                       double b, double ds, const double *q_in_dev, double *q_out_dev, int nsteps,
                                       void *stream)
{
    // every check comes before any GPU work
    if (!n || !ksq_dev || !omega_dev || !q_in_dev || !q_out_dev || nsteps < 1)
        return fail(PSCFG_EINVAL, "null pointer or nsteps < 1");
    if (dim < 1 || dim > 3) return fail(PSCFG_EINVAL, "dim must be 1, 2 or 3");
    int g3[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) g3[d] = n[d];
    for (int d = 0; d < 3; d++)
        if (g3[d] < 1 || g3[d] > MAX_LINE)
            return fail(PSCFG_EINVAL, "grid extent " + std::to_string(g3[d]) + " outside 1.." +
                                          std::to_string(MAX_LINE) + " (PSCFG_NOALLOC_MAX_LINE)");
    const long nr = (long)g3[0] * g3[1] * g3[2];
    const long nk = (long)(g3[0] / 2 + 1) * g3[1] * g3[2];
    if (nr > MAX_NR)
        return fail(PSCFG_EINVAL, "grid of " + std::to_string(nr) + " points exceeds the no-allocation limit of " +
                                      std::to_string(MAX_NR) + " (PSCFG_NOALLOC_MAX_NR)");
    PlaneGeom g;
    std::memset(&g, 0, sizeof(g));
    g.n1 = g3[0];
    g.n2 = g3[1];
    g.n3 = g3[2];
    g.n1h = g.n1 / 2 + 1;
    g.even = (g.n1 % 2 == 0) ? 1 : 0;
    g.LS = g.even ? g.n1h : g.n1;
    LinePlan *plans[3] = {&g.row, &g.col, &g.zp};
    const int lens[4] = {g.even ? g.n1 / 2 : g.n1, g.n2, g.n3, g.n1};
    for (int k = 0; k < 3; k++) {
        plans[k]->n = lens[k];
        if (!plan_radices(lens[k], plans[k]->rad, plans[k]->nst))
            return fail(PSCFG_EINVAL, "grid size has a prime factor other than 2, 3, 5, 7");
    }
    const long P = (long)g.n1h * g.n2;
    const int ntile = (int)((P + Z_TILE - 1) / Z_TILE);
    const size_t smxy = 2 * (size_t)g.n2 * g.LS * sizeof(cx<double>);
    const size_t smz = 2 * (size_t)g.n3 * Z_TILE * sizeof(cx<double>);
    const size_t smpl = smxy + 2 * (size_t)nr * sizeof(double);
    const size_t smmax = 227 * 1024;
    if (dim <= 2 && smpl > smmax)
        return fail(PSCFG_EINVAL, "no-allocation limit: a grid of dim <= 2 is propagated by one CTA in shared "
                                  "memory and needs " + std::to_string(smpl) + " bytes of it (at most " +
                                  std::to_string(smmax) + ")");
    if (dim == 3 && (smxy > smmax || smz > smmax))
        return fail(PSCFG_EINVAL, "no-allocation limit: an x-y plane spectrum needs " + std::to_string(smxy) +
                                  " bytes of shared memory and a z tile " + std::to_string(smz) + " (at most " +
                                  std::to_string(smmax) + " each)");

    cudaStream_t st = (cudaStream_t)stream;
    unsigned char *base = nullptr;
    int rc = scratch_address(&base);
    if (rc != PSCFG_OK) return rc;
    for (int k = 0; k < 3; k++) plans[k]->tw = base + OFF_TW + k * TW_BYTES;
    g.rtw = base + OFF_TW + 3 * TW_BYTES;

    double *eo1 = (double *)(base + OFF_REAL);
    double *eo2 = (double *)(base + OFF_REAL + REAL_BYTES);
    double *q1 = (double *)(base + OFF_REAL + 2 * REAL_BYTES);
    double *slab = (double *)(base + OFF_REAL + 3 * REAL_BYTES);   // 2 slices, nr apart
    double *ek1 = (double *)(base + OFF_EK);
    double *ek2 = (double *)(base + OFF_EK + REAL_BYTES);
    cx<double> *S1 = (cx<double> *)(base + OFF_SPEC);
    cx<double> *S2 = (cx<double> *)(base + OFF_SPEC + al(sizeof(cx<double>) * MAX_NR));

    Descs d;
    std::memset(&d, 0, sizeof(d));
    d.tj.omega = omega_dev;
    d.tj.ksq = ksq_dev;
    d.tj.eo1 = eo1;
    d.tj.eo2 = eo2;
    d.tj.ek1 = ek1;
    d.tj.ek2 = ek2;
    d.tj.ds = ds;
    d.tj.b = b;
    // one step on a two-slice slab: dir +1 reads slice 0 and writes slice 1,
    // dir -1 the reverse, so that consecutive steps alternate without copies
    SweepField<double> f;
    std::memset(&f, 0, sizeof(f));
    f.slab = slab;
    f.ns = 1;
    f.dir = 1;
    f.nblk = 1;
    f.bgn[0] = 0;
    f.bgn[1] = 1;
    f.eo1[0] = eo1;
    f.eo2[0] = eo2;
    f.ek1[0] = ek1;
    f.ek2[0] = ek2;
    f.S1 = S1;
    f.S2 = S2;
    f.q1 = q1;
    d.f[0] = f;                                   // first step: q_in -> slice 1 (or q_out)
    d.f[0].in = q_in_dev;
    if (nsteps == 1) d.f[0].out = q_out_dev;
    d.f[1] = f;                                   // slice 0 -> slice 1
    d.f[2] = f;                                   // slice 1 -> slice 0
    d.f[2].dir = -1;
    d.f[3] = ((nsteps - 1) % 2 == 1) ? d.f[2] : d.f[1];   // last step (nsteps >= 2) -> q_out
    d.f[3].out = q_out_dev;
    TableJob<double> *dtj = (TableJob<double> *)(base + OFF_DESC);
    SweepField<double> *dfl = (SweepField<double> *)(base + OFF_DESC + al(sizeof(TableJob<double>)));
    k_setup<<<4, 256, 0, st>>>(d, dtj, dfl, base + OFF_TW, make_int4(lens[0], lens[1], lens[2], lens[3]),
                               (long)TW_BYTES);
    CKN(cudaGetLastError());
    k_make_tables<double><<<dim3((unsigned)std::min<long>((nr + 255) / 256, 256), 1), 256, 0, st>>>(dtj, nr, nk);
    CKN(cudaGetLastError());
    if (dim <= 2) {
        CKN(allow_dyn_smem((const void *)k_sweep_plane<double>));
    } else {
        CKN(allow_dyn_smem((const void *)k3_fwd_pair<double>));
        CKN(allow_dyn_smem((const void *)k3_inv_mid<double>));
        CKN(allow_dyn_smem((const void *)k3_inv_final<double>));
        CKN(allow_dyn_smem((const void *)k3_zconv<double, Z_TILE>));
    }
    const int threads = (int)std::min<long>(256, std::max<long>(32, ((nr / 2 + 31) / 32) * 32));
    for (int s = 0; s < nsteps; s++) {
        // step 0 reads q_in, then odd steps slice 1 -> 0 and even steps
        // slice 0 -> 1; the last step writes q_out
        const SweepField<double> *df = dfl + (s == 0 ? 0 : s == nsteps - 1 ? 3 : (s % 2 == 1 ? 2 : 1));
        if (dim <= 2) {
            k_sweep_plane<double><<<1, threads, smpl, st>>>(df, g, 0, 1);
            CKN(cudaGetLastError());
        } else {
            k3_fwd_pair<double><<<dim3(g.n3, 1), 256, smxy, st>>>(df, g, 0);
            k3_zconv<double, Z_TILE><<<dim3(ntile, 1, 2), 256, smz, st>>>(df, g, 0, 3);
            k3_inv_mid<double><<<dim3(g.n3, 1), 256, smxy, st>>>(df, g, 0);
            k3_zconv<double, Z_TILE><<<dim3(ntile, 1, 1), 256, smz, st>>>(df, g, 0, 2);
            k3_inv_final<double><<<dim3(g.n3, 1), 256, smxy, st>>>(df, g, 0);
            CKN(cudaGetLastError());
        }
    }
    return PSCFG_OK;
}
