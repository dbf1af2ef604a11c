// basis.cuh -- fields in a symmetry-adapted (star) basis on the device.
//
// The reference keeps omega and rho as coefficients of real star basis
// functions and converts them on every density() call: basis_to_kgrid
// (src/grid_basis_mod.f90:47-120) writes each star's coefficient times the
// wave's coefficient into the half k-grid, an inverse FFT gives the grid
// field; kgrid_to_basis (:124-200) reads the forward FFT of rho back into
// star coefficients.  Here the star structure of an instance is held as
// device tables sorted by basis function (CSR): the half-grid index k, the
// function and the complex coefficient c of each wave, so both maps are one
// kernel each:
//   scatter  S[k_j] += a[star_j] c_j
//   gather   a_s = sum_{j in s} w_j Re(conj(c_j) S[k_j]) / N
// A half-grid wave belongs to one function, or to the two real functions
// (cosine- and sine-like) of a pair of stars related by inversion in a group
// without inversion (star_invert = +-1, src/grid_basis_mod.f90:82-110); its
// two contributions are added atomically into the zeroed S, and a sum of
// two terms onto zero does not depend on their order.
// with w = 2 for the half-grid waves whose Hermitian partner lies outside the
// half grid (0 < kx < n1/2) and 1 otherwise.  The gather sums each star in a
// fixed order (one warp per star), so results are reproducible.
#pragma once
#include "kernels.cuh"

namespace pscfg {

struct BasisJob {
    const int *start;        // [n_star + 1] first wave of each star
    const int *wave_k;       // [n_wave] half-grid index kx + (n1/2+1)(ky + n2 kz)
    const int *wave_star;    // [n_wave]
    const cx<double> *c;     // [n_wave]
    int n_star, n_wave;
    cx<double> *S;           // half spectrum [nk]
    const double *a;         // scatter: coefficients in [n_star]
    double *out;             // gather: coefficients out [n_star]
};

// grid = (ceil(max n_wave / 256), njobs): S[k_j] += a[star_j] c_j
// (S zeroed beforehand; at most two terms per wave).
static __global__ void k_basis_scatter(const BasisJob *jobs)
{
    const BasisJob &J = jobs[blockIdx.y];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < J.n_wave; j += gridDim.x * blockDim.x) {
        const double a = J.a[J.wave_star[j]];
        const cx<double> c = J.c[j];
        double *S = (double *)(J.S + J.wave_k[j]);
        atomicAdd(S, a * c.x);
        atomicAdd(S + 1, a * c.y);
    }
}

// grid = (ceil(max n_star / 8), njobs), 256 threads: one warp per star.
static __global__ void k_basis_gather(const BasisJob *jobs, int n1, double inv_nr)
{
    const BasisJob &J = jobs[blockIdx.y];
    const int s = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (s >= J.n_star) return;
    const int n1h = n1 / 2 + 1;
    double acc = 0.0;
    for (int j = J.start[s] + lane; j < J.start[s + 1]; j += 32) {
        const int k = J.wave_k[j], kx = k % n1h;
        const double w = (kx == 0 || (n1 % 2 == 0 && kx == n1 / 2)) ? 1.0 : 2.0;
        const cx<double> c = J.c[j], f = J.S[k];
        acc += w * (c.x * f.x + c.y * f.y);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) J.out[s] = acc * inv_nr;
}

// Inverse (c2r, unnormalised) of half spectra [z][y][n1/2+1] into real
// fields, the counterparts of k2_fft_fields / k3_fft_fields_* (scf_kernels.cuh).
static __global__ void k2_ifft_fields(const cx<double> *const *src, double *const *dst, PlaneGeom g)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<double> *A = (cx<double> *)smem_raw;
    cx<double> *B = A + g.n2 * g.LS;
    load_plane<double>(A, src[blockIdx.x], g);
    const cx<double> *Z = plane_inverse<double>(A, B, g);
    double *f = dst[blockIdx.x];
    for (int r = threadIdx.x; r < g.n1 * g.n2; r += blockDim.x) f[r] = unpack_real<double>(Z, g, r);
}

template <int TC>
static __global__ void k3_ifft_fields_z(cx<double> *const *spec, PlaneGeom g)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<double> *A = (cx<double> *)smem_raw;
    cx<double> *B = A + g.n3 * TC;
    cx<double> *S = spec[blockIdx.y];
    const long P = (long)g.n1h * g.n2;
    const long c0 = (long)blockIdx.x * TC;
    const int nc = (int)min((long)TC, P - c0);
    for (int i = threadIdx.x; i < g.n3 * TC; i += blockDim.x) {
        int z = i / TC, c = i - z * TC;
        A[i] = (c < nc) ? S[z * P + c0 + c] : mk<double>(0.0, 0.0);
    }
    cx<double> *F = fft_lines<1, double>(A, B, g.zp, TC, TC, 1, true);
    for (int i = threadIdx.x; i < g.n3 * TC; i += blockDim.x) {
        int z = i / TC, c = i - z * TC;
        if (c < nc) S[z * P + c0 + c] = F[i];
    }
}

static __global__ void k3_ifft_fields_xy(const cx<double> *const *src, double *const *dst, PlaneGeom g)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<double> *A = (cx<double> *)smem_raw;
    cx<double> *B = A + g.n2 * g.LS;
    const int z = blockIdx.x;
    const long np = (long)g.n1 * g.n2, nkp = (long)g.n1h * g.n2;
    load_plane<double>(A, src[blockIdx.y] + z * nkp, g);
    const cx<double> *Z = plane_inverse<double>(A, B, g);
    double *f = dst[blockIdx.y] + z * np;
    for (int r = threadIdx.x; r < np; r += blockDim.x) f[r] = unpack_real<double>(Z, g, r);
}

}  // namespace pscfg
