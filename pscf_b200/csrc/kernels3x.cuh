// kernels3x.cuh -- one-launch MDE step for a 32^3 grid on a thread-block
// cluster (distributed shared memory).
//
// A cluster of CL = 8 CTAs owns one sweep field for one step.  CTA r holds
// z-planes [4r, 4r+4) for the x-y transforms and the spectral columns
// [68r, 68r+68) of every plane (4 of the 32 transposed y rows, all kx) for
// the z transforms.  Between the two layouts each CTA pushes its tiles into
// the owning CTA's shared memory (st.shared::cluster through
// cluster.map_shared_rank); a cluster barrier follows each push.  A step
// (src/step_mod.f90:146-176) is
//   xy-forward(eo1 q, eo2 q) -> push -> z: F, x ek1 / x ek2, F^-1 -> push ->
//   xy-inverse -> q1, h -> xy-forward(h) -> push -> z: F, x ek2, F^-1 ->
//   push -> xy-inverse -> q_out = (4 q2 - q1)/3,
// four cluster barriers; HBM sees q(s), the tables and q(s +- ds) only.
// q1 is kept in shared memory and stored (with h and q2) only when the
// caller asks for the step intermediates (h_out set).
#pragma once
#include <cooperative_groups.h>

#include "kernels3c.cuh"

namespace pscfg {

namespace cgx = cooperative_groups;

template <typename T>
struct Cl32 {
    static constexpr int N = 32, NH = 17, PS = N * NH, CL = 8, ZP = N / CL, NCOL = PS / CL;
    static constexpr size_t smem_bytes()
    {
        return sizeof(cx<T>) * (2 * ZP * PS + 2 * N * NCOL) + sizeof(T) * ZP * N * N;
    }
};

// plane layout [p][y'][kx] (local) -> column layout [z][j] of the owner of
// entry e = y' * NH + kx, j = e - NCOL * owner
template <typename T>
__device__ __forceinline__ void push_planes(cgx::cluster_group &cl, const cx<T> *P, cx<T> *C, int rank)
{
    using K = Cl32<T>;
    for (int i = threadIdx.x; i < K::ZP * K::PS; i += blockDim.x) {
        const int p = i / K::PS, e = i % K::PS;
        const int owner = e / K::NCOL, j = e % K::NCOL;
        cx<T> *dst = cl.map_shared_rank(C, owner);
        dst[(rank * K::ZP + p) * K::NCOL + j] = P[i];
    }
}

// column layout [z][j] (local, entries NCOL*rank + j) -> owner of plane z
template <typename T>
__device__ __forceinline__ void push_cols(cgx::cluster_group &cl, const cx<T> *C, cx<T> *P, int rank)
{
    using K = Cl32<T>;
    for (int i = threadIdx.x; i < K::N * K::NCOL; i += blockDim.x) {
        const int z = i / K::NCOL, j = i % K::NCOL;
        cx<T> *dst = cl.map_shared_rank(P, z / K::ZP);
        dst[(z % K::ZP) * K::PS + K::NCOL * rank + j] = C[i];
    }
}

template <typename T>
__device__ __forceinline__ void zconv_cols(cx<T> *C, const T *__restrict__ ek, const cx<T> *twz, int rank)
{
    using K = Cl32<T>;
    stack_fft<32, -1, T, K::NCOL, K::NCOL, 0, 1, K::NCOL>(C, twz);
    for (int i = threadIdx.x; i < K::N * K::NCOL; i += blockDim.x) {
        const int pz = i / K::NCOL, col = K::NCOL * rank + i % K::NCOL;
        const int py = col / K::NH, kx = col % K::NH;
        const T e = ek[kx + K::NH * (iperm<32>(py) + 32 * iperm<32>(pz))];
        C[i] = mk<T>(e * C[i].x, e * C[i].y);
    }
    stack_fft<32, 1, T, K::NCOL, K::NCOL, 0, 1, K::NCOL>(C, twz);
}

// One step (t) of field f by the cluster.  first: the cluster's first
// step in this launch -- every CTA of the cluster must be running before
// its shared memory is written by a peer, so each arrives on entry and
// waits just before its first push.  Later steps need no such barrier: a
// peer writes this CTA's column buffers only after the last cluster
// barrier of the previous step, past which nothing reads them.
template <typename T>
__device__ __forceinline__ void cl32_step(cgx::cluster_group &cl, const SweepField<T> &f, const PlaneGeom &g,
                                          int blk, int src, int dst, bool first)
{
    using K = Cl32<T>;
    using PSk = PlaneStack<T, 32, 32, K::ZP>;
    const int rank = (int)cl.block_rank();
    if (first) asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *PA = (cx<T> *)smem_raw;
    cx<T> *PB = PA + K::ZP * K::PS;
    cx<T> *CA = PB + K::ZP * K::PS;
    cx<T> *CB = CA + K::N * K::NCOL;
    T *Q1 = (T *)(CB + K::N * K::NCOL);
    const long nr = 32L * 32 * 32;
    const long poff = (long)rank * K::ZP * 32 * 32;
    const T rn = (T)nr;
    const T *q = src_slice(f, src, nr) + poff;
    const T *eo1 = f.eo1[blk] + poff, *eo2 = f.eo2[blk] + poff;
    const cx<T> *twM = (const cx<T> *)g.row.tw, *twN2 = (const cx<T> *)g.col.tw, *twN1 = (const cx<T> *)g.rtw;
    const cx<T> *twz = (const cx<T> *)g.zp.tw;
    constexpr int NP = PSk::NP;

    // full step and first half step share the x-y forward stage
    PSk::pack(PA, [&](int e) { return eo1[e] * q[e]; });
    PSk::pack(PB, [&](int e) { return eo2[e] * q[e]; });
    PSk::forward(PA, twM, twN2, twN1);
    PSk::forward(PB, twM, twN2, twN1);
    if (first) asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory");
    push_planes<T>(cl, PA, CA, rank);
    push_planes<T>(cl, PB, CB, rank);
    cl.sync();
    zconv_cols<T>(CA, f.ek1[blk], twz, rank);
    zconv_cols<T>(CB, f.ek2[blk], twz, rank);
    __syncthreads();
    push_cols<T>(cl, CA, PA, rank);
    push_cols<T>(cl, CB, PB, rank);
    cl.sync();
    PSk::inverse(PA, twM, twN2, twN1);
    PSk::inverse(PB, twM, twN2, twN1);
    T *q1g = f.h_out ? f.q1 + poff : nullptr;
    T *hg = f.h_out ? f.h_out + poff : nullptr;
    for (int e = threadIdx.x; e < K::ZP * NP; e += blockDim.x) {
        const T v = eo1[e] * PSk::real_at(PA, e) / rn;
        Q1[e] = v;
        if (q1g) q1g[e] = v;
    }
    for (int i = threadIdx.x; i < K::ZP * 32 * PSk::M; i += blockDim.x) {
        const int p = i / (32 * PSk::M), r = i % (32 * PSk::M), y = r / PSk::M, m = r % PSk::M;
        const int e = p * NP + y * 32 + 2 * m;
        cx<T> &z = PB[p * K::PS + y * PSk::NH + m];
        z = mk<T>(eo1[e] * z.x / rn, eo1[e + 1] * z.y / rn);
        if (hg) {
            hg[e] = z.x;
            hg[e + 1] = z.y;
        }
    }
    // second half step
    PSk::forward(PB, twM, twN2, twN1);
    push_planes<T>(cl, PB, CB, rank);
    cl.sync();
    zconv_cols<T>(CB, f.ek2[blk], twz, rank);
    __syncthreads();
    push_cols<T>(cl, CB, PB, rank);
    cl.sync();
    PSk::inverse(PB, twM, twN2, twN1);
    T *out = dst_slice(f, dst, nr) + poff;
    T *q2o = f.q2_out ? f.q2_out + poff : nullptr;
    for (int e = threadIdx.x; e < K::ZP * NP; e += blockDim.x) {
        const T q2 = eo2[e] * PSk::real_at(PB, e) / rn;
        out[e] = ((T)4 * q2 - Q1[e]) / (T)3;
        if (q2o) q2o[e] = q2;
    }
}


template <typename T>
__global__ void __cluster_dims__(8, 1, 1) __launch_bounds__(512, 1)
    k3x_step32(const SweepField<T> *fields, PlaneGeom g, int t)
{
    cgx::cluster_group cl = cgx::this_cluster();
    const SweepField<T> &f = fields[blockIdx.x / Cl32<T>::CL];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;   // same for every CTA of the cluster
    cl32_step<T>(cl, f, g, blk, src, dst, true);
}

// Steps [t0, t1) of every field in one launch: a cluster walks its field's
// contour, each CTA reading back the planes of q it wrote the step before.
template <typename T>
__global__ void __cluster_dims__(8, 1, 1) __launch_bounds__(512, 1)
    k3x_sweep32(const SweepField<T> *fields, PlaneGeom g, int t0, int t1)
{
    cgx::cluster_group cl = cgx::this_cluster();
    const SweepField<T> &f = fields[blockIdx.x / Cl32<T>::CL];
    for (int t = t0; t < t1; t++) {
        int blk, src, dst;
        if (!step_slices(f, t, blk, src, dst)) break;   // same for every CTA of the cluster
        cl32_step<T>(cl, f, g, blk, src, dst, t == t0);
        __syncthreads();
    }
}

}  // namespace pscfg
