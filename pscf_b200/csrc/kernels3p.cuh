// kernels3p.cuh -- 3-D MDE step kernels for large grids of compile-time
// shape (64 x 128 x 224, 64 x 64 x 64).
//
// Same four launches per step as the register-column kernels (kernels3c.cuh:
// x-y forward pair, z pass on both spectra, x-y inverse + h + forward, z
// pass, x-y inverse + Richardson fused with the next step's forward pair),
// built for planes and z lines too long for registers:
//   * a CTA of 256 threads holds one x-y plane spectrum (N2 rows of
//     NH = N1/2 + 1 complex values) in shared memory, or a tile of TC z
//     columns;
//   * every 1-D transform is an in-place two-pass (four-step) transform
//     N = P x Q (Split<N>) whose work items are numbered line-fastest, so
//     that consecutive threads touch consecutive lines: with NH odd (row
//     stride) or unit line stride every shared-memory pass is free of bank
//     conflicts, and no radix above 16 is held in registers;
//   * the row (x) transform of a real plane is a half-length complex
//     transform of packed rows z[m] = f(2m) + i f(2m+1) untangled in place
//     at the positions the forward transform leaves its outputs at, and the
//     two real columns kx = 0 and kx = N1/2 are transformed as one complex
//     column and separated by Hermitian symmetry (32 complex column lines
//     per plane, every column pass an exact number of thread rounds).
//
// Spectrum layout ("positions").  Row y' of a plane spectrum holds ky =
// iperm<N2>(y'); entry x' < M (M = N1/2) holds kx = iperm<M>(x'), entry M
// holds kx = M.  A z column is forward transformed in natural z order,
// multiplied by exp(-ds b^2 k^2/6 or /12) in the permuted order z' its
// forward leaves, and inverse transformed back to natural order, so no
// transform ever reorders data.  The k-space tables stay in the natural
// order of make_propg (src/step_mod.f90:109-129).
//
// The algebra is step_exp (src/step_mod.f90:146-176), as in kernels.cuh.
#pragma once
#include "kernels3c.cuh"

namespace pscfg {

template <> struct Split<224> { static constexpr int P = 16, Q = 14; };

// W_N^m = exp(-2 pi i m / N), m < N, for the line lengths of these kernels,
// in constant memory: every index used below is the same for all lanes of a
// warp (the line index varies fastest across lanes), so each read is one
// broadcast from the constant cache instead of a global load that streaming
// plane data would evict from L1.  Filled by the host (upload_p_twiddles).
__constant__ double c_ptw32[2][32], c_ptw64[2][64], c_ptw128[2][128], c_ptw224[2][224];
__constant__ float c_ptw32f[2][32], c_ptw64f[2][64], c_ptw128f[2][128], c_ptw224f[2][224];

template <typename T, int N> struct PTw;
#define PSCFG_PTW(N)                                                                                         \
    template <> struct PTw<double, N> {                                                                      \
        __device__ __forceinline__ static cx<double> at(int m) { return mk<double>(c_ptw##N[0][m], c_ptw##N[1][m]); } \
    };                                                                                                       \
    template <> struct PTw<float, N> {                                                                       \
        __device__ __forceinline__ static cx<float> at(int m) { return mk<float>(c_ptw##N##f[0][m], c_ptw##N##f[1][m]); } \
    };
PSCFG_PTW(32)
PSCFG_PTW(64)
PSCFG_PTW(128)
PSCFG_PTW(224)
#undef PSCFG_PTW

// Pass A of a forward (S < 0) or the second pass of an inverse (S > 0)
// transform of NL lines of length N: element e of line l at
// buf[l * LSTR + e * ESTR].
template <int N, int S, typename T, int NL, int LSTR, int ESTR>
__device__ __forceinline__ void lf_passA(cx<T> *buf)
{
    constexpr int P = Split<N>::P, Q = Split<N>::Q;
    for (int w = threadIdx.x; w < NL * Q; w += blockDim.x) {
        const int l = w % NL, n2 = w / NL;
        cx<T> *b = buf + l * LSTR;
        cx<T> v[P];
        if (S < 0) {
#pragma unroll
            for (int n1 = 0; n1 < P; n1++) v[n1] = b[(Q * n1 + n2) * ESTR];
            Dft<P, S, T>::run(v);
            if (Q > 1) {
#pragma unroll
                for (int k1 = 1; k1 < P; k1++) v[k1] = cmul(v[k1], PTw<T, N>::at(n2 * k1));
            }
#pragma unroll
            for (int k1 = 0; k1 < P; k1++) b[(Q * k1 + n2) * ESTR] = v[k1];
        } else {
#pragma unroll
            for (int k1 = 0; k1 < P; k1++) v[k1] = b[(Q * k1 + n2) * ESTR];
            if (Q > 1) {
#pragma unroll
                for (int k1 = 1; k1 < P; k1++) v[k1] = cmul(v[k1], conjg(PTw<T, N>::at(n2 * k1)));
            }
            Dft<P, S, T>::run(v);
#pragma unroll
            for (int n1 = 0; n1 < P; n1++) b[(Q * n1 + n2) * ESTR] = v[n1];
        }
    }
}

// Pass B: length-Q transforms of the Q contiguous (stride ESTR) values at
// Q k1 of each line.
template <int N, int S, typename T, int NL, int LSTR, int ESTR>
__device__ __forceinline__ void lf_passB(cx<T> *buf)
{
    constexpr int P = Split<N>::P, Q = Split<N>::Q;
    if (Q == 1) return;
    for (int w = threadIdx.x; w < NL * P; w += blockDim.x) {
        const int l = w % NL, k1 = w / NL;
        cx<T> *b = buf + l * LSTR + Q * k1 * ESTR;
        cx<T> v[Q];
#pragma unroll
        for (int j = 0; j < Q; j++) v[j] = b[j * ESTR];
        Dft<Q, S, T>::run(v);
#pragma unroll
        for (int j = 0; j < Q; j++) b[j * ESTR] = v[j];
    }
}

// Forward (natural in, permuted out) or inverse (permuted in, natural out)
// of NL lines; begins and ends with __syncthreads.
template <int N, int S, typename T, int NL, int LSTR, int ESTR>
__device__ __forceinline__ void lf_fft(cx<T> *buf)
{
    __syncthreads();
    if (S < 0) {
        lf_passA<N, S, T, NL, LSTR, ESTR>(buf);
        if (Split<N>::Q > 1) {
            __syncthreads();
            lf_passB<N, S, T, NL, LSTR, ESTR>(buf);
        }
    } else {
        if (Split<N>::Q > 1) {
            lf_passB<N, S, T, NL, LSTR, ESTR>(buf);
            __syncthreads();
        }
        lf_passA<N, S, T, NL, LSTR, ESTR>(buf);
    }
    __syncthreads();
}

// 16-byte asynchronous global -> shared copies (cp.async): every copy of a
// tile is in flight at once and none holds a register.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// bytes (a multiple of 16, both addresses 16-byte aligned) from global to
// shared memory by all threads of the CTA; the caller synchronises
template <int BYTES>
__device__ __forceinline__ void copy_in(void *smem, const void *gmem)
{
    static_assert(BYTES % 16 == 0, "16-byte chunks");
#pragma unroll 8
    for (int c = threadIdx.x; c < BYTES / 16; c += blockDim.x)
        cp_async16((char *)smem + 16 * c, (const char *)gmem + 16 * c);
    cp_async_wait_all();
}

// Bulk prefetch of `bytes` (a multiple of 16, 16-byte aligned) into L2 by
// one thread: planes that a kernel reads only after its transforms are in
// L2 by then, so the pointwise passes wait for L2 instead of DRAM.
__device__ __forceinline__ void prefetch_l2(const void *p, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}

template <typename T> struct Pair;
template <> struct Pair<double> { using V = double2; };
template <> struct Pair<float> { using V = float2; };

// two consecutive reals at an even offset (16- or 8-byte aligned)
template <typename T>
__device__ __forceinline__ cx<T> ld_pair(const T *p)
{
    const typename Pair<T>::V v = *(const typename Pair<T>::V *)p;
    return mk<T>(v.x, v.y);
}
template <typename T>
__device__ __forceinline__ void st_pair(T *p, T a, T b)
{
    typename Pair<T>::V v;
    v.x = a;
    v.y = b;
    *(typename Pair<T>::V *)p = v;
}

// One x-y plane (N1 even, M = N1/2 a power of two >= 8, N2 a power of two).
template <typename T, int N1, int N2>
struct PlaneP {
    static constexpr int M = N1 / 2, NH = M + 1, PS = N2 * NH, NP = N1 * N2, H = M / 2;
    static constexpr int KT = 256;   // threads per CTA of every kernel below
    static_assert((N2 * M) % KT == 0, "packed-row loops in whole rounds");

    // kx of row position x'
    __device__ __forceinline__ static int kx_of(int xp) { return xp < M ? iperm<M>(xp) : M; }

    // packed natural rows: buf[y*NH + m] = pair(e) with pair(e) = (f(e), f(e+1)), e = y N1 + 2m
    template <typename F>
    __device__ __forceinline__ static void pack(cx<T> *buf, F pair)
    {
#pragma unroll 4
        for (int r = 0; r < N2 * M / KT; r++) {
            const int i = threadIdx.x + r * KT, y = i / M, m = i % M;
            buf[y * NH + m] = pair(y * N1 + 2 * m);
        }
    }

    // element loop over the packed rows in the same thread mapping as pack():
    // fn(slot, e) with slot = packed pair of reals e, e+1
    template <typename F>
    __device__ __forceinline__ static void each_pair(cx<T> *buf, F fn)
    {
#pragma unroll 4
        for (int r = 0; r < N2 * M / KT; r++) {
            const int i = threadIdx.x + r * KT, y = i / M, m = i % M;
            fn(buf[y * NH + m], y * N1 + 2 * m);
        }
    }

    // (asynchronous copies; the transform that follows begins with a barrier)
    __device__ __forceinline__ static void load(cx<T> *buf, const cx<T> *src)
    {
        copy_in<PS * (int)sizeof(cx<T>)>(buf, src);
    }
    __device__ __forceinline__ static void store(cx<T> *dst, const cx<T> *buf)
    {
#pragma unroll 4
        for (int i = threadIdx.x; i < PS; i += blockDim.x) dst[i] = buf[i];
    }

    // packed natural rows -> plane spectrum (positions).  Ends synchronised.
    __device__ static void forward(cx<T> *buf)
    {
        lf_fft<M, -1, T, N2, NH, 1>(buf);   // rows: permuted kx out
        // untangle in place (each item reads and writes only the positions
        // of kx = k and M - k); X[0] and X[M] are real and share position 0
        for (int i = threadIdx.x; i < N2 * (H + 1); i += blockDim.x) {
            const int k = i / N2, y = i % N2;   // lanes across rows: conflict-free, uniform twiddles
            cx<T> *b = buf + y * NH;
            if (k == 0) {
                const cx<T> z0 = b[0];
                b[0] = mk<T>(z0.x + z0.y, z0.x - z0.y);
            } else if (k == H) {
                const int p = perm<M>(H);
                b[p] = conjg(b[p]);
            } else {
                const int p = perm<M>(k), pm = perm<M>(M - k);
                const cx<T> zk = b[p], zm = b[pm];
                const cx<T> wk = PTw<T, N1>::at(k), wm = PTw<T, N1>::at(M - k);
                const cx<T> ak = zk + conjg(zm), dk = zk - conjg(zm);
                const cx<T> am = zm + conjg(zk), dm = zm - conjg(zk);
                b[p] = scale(ak + mul_si<-1>(cmul(wk, dk)), (T)0.5);
                b[pm] = scale(am + mul_si<-1>(cmul(wm, dm)), (T)0.5);
            }
        }
        lf_fft<N2, -1, T, M, 1, NH>(buf);  // columns x' < M: permuted ky out
        // separate column 0 = X0 + i XM into kx = 0 (position 0) and kx = M
        for (int ky = threadIdx.x; ky <= N2 / 2; ky += blockDim.x) {
            const int p = perm<N2>(ky);
            if (ky == 0 || ky == N2 / 2) {
                const cx<T> c = buf[p * NH];
                buf[p * NH] = mk<T>(c.x, (T)0);
                buf[p * NH + M] = mk<T>(c.y, (T)0);
            } else {
                const int pm = perm<N2>(N2 - ky);
                const cx<T> ck = buf[p * NH], cm = conjg(buf[pm * NH]);
                const cx<T> a = scale(ck + cm, (T)0.5);
                const cx<T> b = scale(mul_si<-1>(ck - cm), (T)0.5);
                buf[p * NH] = a;
                buf[pm * NH] = conjg(a);
                buf[p * NH + M] = b;
                buf[pm * NH + M] = conjg(b);
            }
        }
        __syncthreads();
    }

    // plane spectrum (positions) -> packed natural rows of the unnormalised
    // c2r.  Ends synchronised.
    __device__ static void inverse(cx<T> *buf)
    {
        __syncthreads();
        for (int r = threadIdx.x; r < N2; r += blockDim.x) {
            const cx<T> a = buf[r * NH], b = buf[r * NH + M];
            buf[r * NH] = mk<T>(a.x - b.y, a.y + b.x);   // a + i b
        }
        lf_fft<N2, 1, T, M, 1, NH>(buf);   // columns: natural y out
        for (int i = threadIdx.x; i < N2 * (H + 1); i += blockDim.x) {
            const int k = i / N2, y = i % N2;
            cx<T> *b = buf + y * NH;
            if (k == 0) {
                const cx<T> c = b[0];   // (X0, XM), both real
                b[0] = mk<T>(c.x + c.y, c.x - c.y);
            } else if (k == H) {
                const int p = perm<M>(H);
                b[p] = scale(conjg(b[p]), (T)2);
            } else {
                const int p = perm<M>(k), pm = perm<M>(M - k);
                const cx<T> xk = b[p], xm = b[pm];
                const cx<T> wk = conjg(PTw<T, N1>::at(k)), wm = conjg(PTw<T, N1>::at(M - k));
                b[p] = (xk + conjg(xm)) + mul_si<1>(cmul(wk, xk - conjg(xm)));
                b[pm] = (xm + conjg(xk)) + mul_si<1>(cmul(wm, xm - conjg(xk)));
            }
        }
        lf_fft<M, 1, T, N2, NH, 1>(buf);    // rows: natural packed out
    }
};

// K1 (first step of a sweep): S1 = Fxy[eo1 q], S2 = Fxy[eo2 q], with
// eo1 = eo2^2.  grid = (N3, nfields), 256 threads.
template <typename T, int N1, int N2, int N3>
__global__ void __launch_bounds__(256, 2) k3p_fwd_pair(const SweepField<T> *fields, PlaneGeom g, int t)
{
    using PL = PlaneP<T, N1, N2>;
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const long nr = (long)N1 * N2 * N3;
    const int z = blockIdx.x;
    const T *q = src_slice(f, src, nr) + (long)z * PL::NP;
    const T *eo2 = f.eo2[blk] + (long)z * PL::NP;
    PL::pack(buf, [&](int e) {
        const cx<T> a = ld_pair(eo2 + e), v = ld_pair(q + e);
        return mk<T>(a.x * (a.x * v.x), a.y * (a.y * v.y));
    });
    PL::forward(buf);
    PL::store(f.S1 + (long)z * PL::PS, buf);
    __syncthreads();
    PL::pack(buf, [&](int e) {
        const cx<T> a = ld_pair(eo2 + e), v = ld_pair(q + e);
        return mk<T>(a.x * v.x, a.y * v.y);
    });
    PL::forward(buf);
    PL::store(f.S2 + (long)z * PL::PS, buf);
}

// K2/K4: S <- Fz^-1[ek . Fz[S]] on a tile of TC columns (positions c =
// y' NH + x').  which: 1 = S1/ek1, 2 = S2/ek2, 3 = both (grid.z selects).
// grid = (N2 NH / TC, nfields, 1 or 2), 256 threads.  pf_stride > 0: the
// first warp also prefetches into L2 the tile of CTA blockIdx.x + pf_stride
// (the CTA that runs one resident wave later, on the same spectrum).
template <typename T, int N1, int N2, int N3, int TC>
__global__ void __launch_bounds__(256, 2) k3p_zconv(const SweepField<T> *fields, PlaneGeom g, int t, int which,
                                                    int pf_stride)
{
    using PL = PlaneP<T, N1, N2>;
    constexpr int NH = PL::NH, P = PL::PS;
    static_assert(P % TC == 0, "column tiles must divide the plane");
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    const int sel = which == 3 ? (int)blockIdx.z + 1 : which;
    cx<T> *S = (sel == 1) ? f.S1 : f.S2;
    const T *ek = (sel == 1) ? f.ek1[blk] : f.ek2[blk];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const int c0 = blockIdx.x * TC;
    if (pf_stride > 0 && threadIdx.x < 32 && blockIdx.x + pf_stride < gridDim.x) {
        const cx<T> *nx = S + (long)(blockIdx.x + pf_stride) * TC;
        for (int z = threadIdx.x; z < N3; z += 32) prefetch_l2(nx + (long)z * P, TC * (unsigned)sizeof(cx<T>));
    }
    {
        // TC consecutive columns of each z row: RB 16-byte chunks per row
        constexpr int RB = TC * (int)sizeof(cx<T>) / 16;
        static_assert(RB * 16 == TC * (int)sizeof(cx<T>), "tile rows in 16-byte chunks");
#pragma unroll 8
        for (int c = threadIdx.x; c < N3 * RB; c += blockDim.x) {
            const int z = c / RB, j = c % RB;
            cp_async16((char *)(buf + z * TC) + 16 * j, (const char *)(S + (long)z * P + c0) + 16 * j);
        }
        cp_async_wait_all();
    }
    lf_fft<N3, -1, T, TC, 1, TC>(buf);
    const T *ekf = f.ekf[blk];
    if (ekf) {
        // orthogonal cell: ek = fx[x'] fy[y'] fz[z'] in spectrum positions
        // (each thread keeps one column: blockDim.x is a multiple of TC)
        const T *fx = ekf + (sel == 1 ? 0 : NH + N2 + N3), *fy = fx + NH, *fz = fy + N2;
        const int c = c0 + threadIdx.x % TC;
        const T exy = fx[c % NH] * fy[c / NH];
#pragma unroll 7
        for (int i = threadIdx.x; i < N3 * TC; i += blockDim.x) buf[i] = scale(buf[i], exy * fz[i / TC]);
    } else {
#pragma unroll 7
        for (int i = threadIdx.x; i < N3 * TC; i += blockDim.x) {
            const int pz = i / TC, c = c0 + i % TC;
            const int yp = c / NH, xp = c % NH;
            const long kidx = PL::kx_of(xp) + (long)NH * (iperm<N2>(yp) + (long)N2 * iperm<N3>(pz));
            buf[i] = scale(buf[i], __ldg(ek + kidx));
        }
    }
    lf_fft<N3, 1, T, TC, 1, TC>(buf);
#pragma unroll 7
    for (int i = threadIdx.x; i < N3 * TC; i += blockDim.x) {
        const int z = i / TC, c = i % TC;
        S[(long)z * P + c0 + c] = buf[i];
    }
}

// K3: role 0 (grid.z = 0): q1 = eo1 . Fxy^-1[S1] / N.  Role 1: S2 <-
// Fxy[eo2 . (eo2 . Fxy^-1[S2] / N)], the second half step's input.
// grid = (N3, nfields, 2).
template <typename T, int N1, int N2, int N3>
__global__ void __launch_bounds__(256, 2) k3p_mid(const SweepField<T> *fields, PlaneGeom g, int t)
{
    using PL = PlaneP<T, N1, N2>;
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const T rn = (T)((long)N1 * N2 * N3);
    const int z = blockIdx.x;
    const T *eo2 = f.eo2[blk] + (long)z * PL::NP;
    if (threadIdx.x == 0) prefetch_l2(eo2, PL::NP * (unsigned)sizeof(T));
    if (blockIdx.z == 0) {
        T *q1 = f.q1 + (long)z * PL::NP;
        PL::load(buf, f.S1 + (long)z * PL::PS);
        PL::inverse(buf);
        PL::each_pair(buf, [&](cx<T> &s, int e) {
            const cx<T> a = ld_pair(eo2 + e);
            st_pair(q1 + e, (a.x * a.x) * s.x / rn, (a.y * a.y) * s.y / rn);
        });
    } else {
        PL::load(buf, f.S2 + (long)z * PL::PS);
        PL::inverse(buf);
        PL::each_pair(buf, [&](cx<T> &s, int e) {
            const cx<T> a = ld_pair(eo2 + e);
            s = mk<T>((a.x * a.x) * s.x / rn, (a.y * a.y) * s.y / rn);
        });
        PL::forward(buf);
        PL::store(f.S2 + (long)z * PL::PS, buf);
    }
}

// K5 fused with the next step's K1: q_out = (4 eo2 . Fxy^-1[S2]/N - q1)/3,
// then (if step t + 1 exists) S1 = Fxy[eo1' q_out], S2 = Fxy[eo2' q_out]
// with the tables of step t + 1's block.  grid = (N3, nfields).
template <typename T, int N1, int N2, int N3>
__global__ void __launch_bounds__(256, 2) k3p_final_fwd(const SweepField<T> *fields, PlaneGeom g, int t)
{
    using PL = PlaneP<T, N1, N2>;
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const long nr = (long)N1 * N2 * N3;
    const T rn = (T)nr;
    const int z = blockIdx.x;
    const T *eo2 = f.eo2[blk] + (long)z * PL::NP;
    const T *q1 = f.q1 + (long)z * PL::NP;
    T *out = dst_slice(f, dst, nr) + (long)z * PL::NP;
    int blk2, src2, dst2;
    const bool next = step_slices(f, t + 1, blk2, src2, dst2);   // the same for the whole CTA
    const T *n2 = f.eo2[next ? blk2 : blk] + (long)z * PL::NP;
    if (threadIdx.x == 0) {
        prefetch_l2(eo2, PL::NP * (unsigned)sizeof(T));
        prefetch_l2(q1, PL::NP * (unsigned)sizeof(T));
        if (n2 != eo2) prefetch_l2(n2, PL::NP * (unsigned)sizeof(T));
    }
    PL::load(buf, f.S2 + (long)z * PL::PS);
    PL::inverse(buf);
    PL::each_pair(buf, [&](cx<T> &s, int e) {
        const cx<T> a = ld_pair(eo2 + e), p = ld_pair(q1 + e);
        const T o0 = ((T)4 * (a.x * s.x / rn) - p.x) / (T)3;
        const T o1 = ((T)4 * (a.y * s.y / rn) - p.y) / (T)3;
        st_pair(out + e, o0, o1);
        const cx<T> b = ld_pair(n2 + e);
        s = mk<T>((b.x * b.x) * o0, (b.y * b.y) * o1);
    });
    if (!next) return;
    PL::forward(buf);
    PL::store(f.S1 + (long)z * PL::PS, buf);
    __syncthreads();
    // out was written above by the same threads in the same element mapping
    PL::pack(buf, [&](int e) {
        const cx<T> b = ld_pair(n2 + e), o = ld_pair((const T *)out + e);
        return mk<T>(b.x * o.x, b.y * o.y);
    });
    PL::forward(buf);
    PL::store(f.S2 + (long)z * PL::PS, buf);
}

// Stress pass (scf_stress, src/scf_mod.fp.f90:451-550), pass 1: x-y
// forward of slices [s0, s0 + cs) of qf (grid.z = 0) and qr (grid.z = 1)
// into spec[(s - s0) * 2 + dir][z][positions].  grid = (N3, cs, 2).
template <typename T, int N1, int N2, int N3>
__global__ void __launch_bounds__(256, 2) k3p_stress_xy(const StressJob<T> *job, int s0, cx<T> *spec)
{
    using PL = PlaneP<T, N1, N2>;
    const StressJob<T> &J = *job;
    const int s = s0 + blockIdx.y;
    if (s >= J.nslices) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const long nr = (long)N1 * N2 * N3, nk = (long)PL::PS * N3;
    const int z = blockIdx.x;
    const T *q = (blockIdx.z == 0 ? J.qf : J.qr) + (long)s * nr + (long)z * PL::NP;
    PL::pack(buf, [&](int e) { return ld_pair(q + e); });
    PL::forward(buf);
    PL::store(spec + ((long)blockIdx.y * 2 + blockIdx.z) * nk + (long)z * PL::PS, buf);
}

// Pass 2: z forward of a tile of TC columns of both spectra of a slice and
// the partial sums sum_k wdgsq_b(k) Re(F_qf(k) conj F_qr(k)) of every cell
// parameter b in one sweep over the tile, into
// part[((s - s0) * gridDim.x + tile) * PSCFG_MAXCP + b].  grid = (N2 NH / TC, cs).
template <typename T, int N1, int N2, int N3, int TC>
__global__ void __launch_bounds__(256, 2) k3p_stress_z(const StressJob<T> *job, int s0, const cx<T> *spec, double *part)
{
    using PL = PlaneP<T, N1, N2>;
    constexpr int NH = PL::NH, P = PL::PS;
    static_assert(P % TC == 0, "column tiles must divide the plane");
    const StressJob<T> &J = *job;
    const int s = s0 + blockIdx.y;
    if (s >= J.nslices) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *F = (cx<T> *)smem_raw, *R = F + N3 * TC;
    __shared__ double red[32];
    const long nk = (long)P * N3;
    const int c0 = blockIdx.x * TC;
    const cx<T> *sf = spec + ((long)blockIdx.y * 2) * nk, *sr = sf + nk;
    {
        constexpr int RB = TC * (int)sizeof(cx<T>) / 16;
        static_assert(RB * 16 == TC * (int)sizeof(cx<T>), "tile rows in 16-byte chunks");
#pragma unroll 8
        for (int c = threadIdx.x; c < N3 * RB; c += blockDim.x) {
            const int z = c / RB, j = c % RB;
            cp_async16((char *)(F + z * TC) + 16 * j, (const char *)(sf + (long)z * P + c0) + 16 * j);
            cp_async16((char *)(R + z * TC) + 16 * j, (const char *)(sr + (long)z * P + c0) + 16 * j);
        }
        cp_async_wait_all();
    }
    lf_fft<N3, -1, T, TC, 1, TC>(F);
    lf_fft<N3, -1, T, TC, 1, TC>(R);
    double acc[PSCFG_MAXCP] = {0, 0, 0, 0, 0, 0};
    const int ncp = J.ncp;
    for (int i = threadIdx.x; i < N3 * TC; i += blockDim.x) {
        const int pz = i / TC, c = c0 + i % TC;
        const int yp = c / NH, xp = c % NH;
        const long k = PL::kx_of(xp) + (long)NH * (iperm<N2>(yp) + (long)N2 * iperm<N3>(pz));
        const cx<T> f = F[i], r = R[i];
        const double pr = (double)f.x * (double)r.x + (double)f.y * (double)r.y;
#pragma unroll
        for (int b = 0; b < PSCFG_MAXCP; b++)
            if (b < ncp) acc[b] += __ldg(J.wdgsq + (long)b * nk + k) * pr;
    }
#pragma unroll
    for (int b = 0; b < PSCFG_MAXCP; b++) {
        if (b >= ncp) break;   // uniform across the CTA
        const double tot = block_sum(acc[b], red);
        if (threadIdx.x == 0) part[((long)blockIdx.y * gridDim.x + blockIdx.x) * PSCFG_MAXCP + b] = tot;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------
// Whole 2-D sweep (dim = 2, the grid is one N1 x N2 plane) of one field per
// CTA, for the small-batch case where a field's steps are latency bound:
// the current block's tables (eo1, eo2 on the grid, ek1, ek2 on the half
// spectrum [ky][kx]) and q, q1 stay in shared memory, and every transform
// is PlaneP::forward / inverse in place (constant twiddles, conflict-free
// line passes).  A step is the reference's step_exp
// (src/step_mod.f90:146-176): q1 = eo1 F^-1[ek1 F[eo1 q]], two half steps
// with eo2 / ek2, q <- (4 q2 - q1) / 3.  Optional per-step outputs as in
// k_sweep_plane: f.q1, f.h_out (eo1 x first half step), f.q2_out.
// grid = nfields, 256 threads.
template <typename T, int N1, int N2>
struct Sweep2P {
    using PL = PlaneP<T, N1, N2>;
    static constexpr int NP = PL::NP, PS = PL::PS, NH = PL::NH, NK = NH * N2;
    static constexpr size_t smem_bytes() { return sizeof(cx<T>) * PS + sizeof(T) * (4 * NP + 2 * NK); }
};

template <typename T, int N1, int N2>
__device__ __forceinline__ void k2p_mul(cx<T> *A, const T *ek)
{
    using PL = PlaneP<T, N1, N2>;
    for (int i = threadIdx.x; i < PL::PS; i += blockDim.x) {
        const int py = i / PL::NH, xp = i - py * PL::NH;
        const T e = ek[PL::kx_of(xp) + PL::NH * iperm<N2>(py)];
        A[i] = mk<T>(e * A[i].x, e * A[i].y);
    }
}

template <typename T, int N1, int N2>
__global__ void __launch_bounds__(256, 1) k2p_sweep(const SweepField<T> *fields, int t0, int t1)
{
    using K = Sweep2P<T, N1, N2>;
    using PL = typename K::PL;
    constexpr int NP = K::NP, NK = K::NK;
    const SweepField<T> &f = fields[blockIdx.x];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *A = (cx<T> *)smem_raw;
    T *q = (T *)(A + K::PS);
    T *q1 = q + NP;
    T *eo1 = q1 + NP, *eo2 = eo1 + NP;
    T *ek1 = eo2 + NP, *ek2 = ek1 + NK;
    const T rn = (T)NP;
    int blk, src, dst;
    if (!step_slices(f, t0, blk, src, dst)) return;
    {
        const T *qs = src_slice(f, src, NP);
        for (int i = threadIdx.x; i < NP; i += blockDim.x) q[i] = qs[i];
    }
    int cur = -1;
    for (int t = t0; t < t1; t++) {
        if (!step_slices(f, t, blk, src, dst)) break;
        if (blk != cur) {
            __syncthreads();
            for (int i = threadIdx.x; i < NP; i += blockDim.x) {
                eo1[i] = f.eo1[blk][i];
                eo2[i] = f.eo2[blk][i];
            }
            for (int i = threadIdx.x; i < NK; i += blockDim.x) {
                ek1[i] = f.ek1[blk][i];
                ek2[i] = f.ek2[blk][i];
            }
            cur = blk;
        }
        __syncthreads();
        // full step
        PL::pack(A, [&](int e) { return mk<T>(eo1[e] * q[e], eo1[e + 1] * q[e + 1]); });
        PL::forward(A);
        k2p_mul<T, N1, N2>(A, ek1);
        PL::inverse(A);
        PL::each_pair(A, [&](cx<T> &z, int e) {
            const T a = eo1[e] * z.x / rn, b = eo1[e + 1] * z.y / rn;
            q1[e] = a;
            q1[e + 1] = b;
            if (f.q1) {
                f.q1[e] = a;
                f.q1[e + 1] = b;
            }
        });
        __syncthreads();
        // two half steps
        PL::pack(A, [&](int e) { return mk<T>(eo2[e] * q[e], eo2[e + 1] * q[e + 1]); });
        PL::forward(A);
        k2p_mul<T, N1, N2>(A, ek2);
        PL::inverse(A);
        PL::each_pair(A, [&](cx<T> &z, int e) {
            const T a = eo1[e] * z.x / rn, b = eo1[e + 1] * z.y / rn;
            if (f.h_out) {
                f.h_out[e] = a;
                f.h_out[e + 1] = b;
            }
            z = mk<T>(a, b);
        });
        PL::forward(A);
        k2p_mul<T, N1, N2>(A, ek2);
        PL::inverse(A);
        T *out = dst_slice(f, dst, NP);
        PL::each_pair(A, [&](cx<T> &z, int e) {
            const T qa = eo2[e] * z.x / rn, qb = eo2[e + 1] * z.y / rn;
            const T va = ((T)4 * qa - q1[e]) / (T)3, vb = ((T)4 * qb - q1[e + 1]) / (T)3;
            q[e] = va;
            q[e + 1] = vb;
            out[e] = va;
            out[e + 1] = vb;
            if (f.q2_out) {
                f.q2_out[e] = qa;
                f.q2_out[e + 1] = qb;
            }
        });
    }
}

}  // namespace pscfg
