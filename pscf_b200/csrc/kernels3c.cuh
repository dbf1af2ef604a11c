// kernels3c.cuh -- 3-D MDE step kernels for power-of-two grids with the
// grid shape fixed at compile time (fft_ct.cuh transforms).
//
// Same five launches per step and the same algebra as the run-time sized
// k3_* kernels (kernels.cuh), but each CTA owns PPC z-planes, every
// transform is in place (no ping-pong buffer), and all index arithmetic is
// constant.  Global spectra S1/S2 are stored [z][y'][kx] with y' the
// transposed order a forward y-transform leaves (perm<N2>).
#pragma once
#include "fft_ct.cuh"
#include "kernels.cuh"

namespace pscfg {

template <int N> __device__ __forceinline__ int iperm(int p)
{
    constexpr int P = Split<N>::P, Q = Split<N>::Q;
    return p / Q + P * (p % Q);
}

// Lines of a stack of planes: line l of the stack lies at
// (l / LPP) * PSTR + (l % LPP) * LSTR, elements ESTR apart.
template <int N, int S, typename T, int NL, int LPP, int PSTR, int LSTR, int ESTR>
__device__ __forceinline__ void stack_passA(cx<T> *buf, const cx<T> *__restrict__ tw)
{
    constexpr int P = Split<N>::P, Q = Split<N>::Q;
    constexpr bool LF = LSTR < ESTR;   // consecutive threads take consecutive lines
    for (int w = threadIdx.x; w < NL * Q; w += blockDim.x) {
        const int l = LF ? w % NL : w / Q, n2 = LF ? w / NL : w % Q;
        cx<T> *b = buf + (l / LPP) * PSTR + (l % LPP) * LSTR;
        cx<T> v[P];
        if (S < 0) {
#pragma unroll
            for (int n1 = 0; n1 < P; n1++) v[n1] = b[(Q * n1 + n2) * ESTR];
            Dft<P, S, T>::run(v);
            if (Q > 1) {
#pragma unroll
                for (int k1 = 1; k1 < P; k1++) v[k1] = cmul(v[k1], __ldg_cx(tw + n2 * k1));
            }
#pragma unroll
            for (int k1 = 0; k1 < P; k1++) b[(Q * k1 + n2) * ESTR] = v[k1];
        } else {
#pragma unroll
            for (int k1 = 0; k1 < P; k1++) v[k1] = b[(Q * k1 + n2) * ESTR];
            if (Q > 1) {
#pragma unroll
                for (int k1 = 1; k1 < P; k1++) v[k1] = cmul(v[k1], conjg(__ldg_cx(tw + n2 * k1)));
            }
            Dft<P, S, T>::run(v);
#pragma unroll
            for (int n1 = 0; n1 < P; n1++) b[(Q * n1 + n2) * ESTR] = v[n1];
        }
    }
}

template <int N, int S, typename T, int NL, int LPP, int PSTR, int LSTR, int ESTR>
__device__ __forceinline__ void stack_passB(cx<T> *buf)
{
    constexpr int P = Split<N>::P, Q = Split<N>::Q;
    constexpr bool LF = LSTR < ESTR;
    if (Q == 1) return;
    for (int w = threadIdx.x; w < NL * P; w += blockDim.x) {
        const int l = LF ? w % NL : w / P, k1 = LF ? w / NL : w % P;
        cx<T> *b = buf + (l / LPP) * PSTR + (l % LPP) * LSTR + Q * k1 * ESTR;
        cx<T> v[Q];
#pragma unroll
        for (int j = 0; j < Q; j++) v[j] = b[j * ESTR];
        Dft<Q, S, T>::run(v);
#pragma unroll
        for (int j = 0; j < Q; j++) b[j * ESTR] = v[j];
    }
}

template <int N, int S, typename T, int NL, int LPP, int PSTR, int LSTR, int ESTR>
__device__ __forceinline__ void stack_fft(cx<T> *buf, const cx<T> *__restrict__ tw)
{
    __syncthreads();
    if (S < 0) {
        stack_passA<N, S, T, NL, LPP, PSTR, LSTR, ESTR>(buf, tw);
        if (Split<N>::Q > 1) {
            __syncthreads();
            stack_passB<N, S, T, NL, LPP, PSTR, LSTR, ESTR>(buf);
        }
    } else {
        if (Split<N>::Q > 1) {
            stack_passB<N, S, T, NL, LPP, PSTR, LSTR, ESTR>(buf);
            __syncthreads();
        }
        stack_passA<N, S, T, NL, LPP, PSTR, LSTR, ESTR>(buf, tw);
    }
    __syncthreads();
}

// A stack of PPC x-y planes of an N1 x N2 real grid (N1 even).  Buffer
// layout: plane p, row y, entry j at buf[p*PS + y*NH + j], NH = N1/2 + 1.
template <typename T, int N1, int N2, int PPC>
struct PlaneStack {
    static constexpr int M = N1 / 2, NH = M + 1, PS = N2 * NH, NP = N1 * N2;

    // packed rows: z[m] = f(2m) + i f(2m+1), natural order
    template <typename F>
    __device__ __forceinline__ static void pack(cx<T> *buf, F value)
    {
        for (int i = threadIdx.x; i < PPC * N2 * M; i += blockDim.x) {
            const int p = i / (N2 * M), r = i % (N2 * M), y = r / M, m = r % M;
            const int e = p * NP + y * N1 + 2 * m;
            buf[p * PS + y * NH + m] = mk<T>(value(e), value(e + 1));
        }
    }

    // natural packed rows -> spectrum [plane][y'][kx].  Each row is
    // transformed by one thread in registers (length M, natural order) and
    // untangled there; only the column transform goes through shared memory.
    __device__ __forceinline__ static void forward(cx<T> *buf, const cx<T> *twM, const cx<T> *twN2, const cx<T> *twN1)
    {
        (void)twM;
        __syncthreads();
        for (int row = threadIdx.x; row < PPC * N2; row += blockDim.x) {
            cx<T> *b = buf + row * NH;
            cx<T> z[M];
#pragma unroll
            for (int m = 0; m < M; m++) z[m] = b[m];
            RegDft<M, -1, T>::run(z);
            cx<T> x[M + 1];
#pragma unroll
            for (int k = 0; k <= M; k++) {
                const cx<T> zk = z[k % M], zm = conjg(z[(M - k) % M]);
                const cx<T> w = twc<T>(N1, k);
                x[k] = scale((zk + zm) + mul_si<-1>(cmul(w, zk - zm)), (T)0.5);
            }
#pragma unroll
            for (int k = 0; k <= M; k++) b[k] = x[k];
        }
        stack_fft<N2, -1, T, PPC * NH, NH, PS, 1, NH>(buf, twN2);        // columns (y permuted out)
    }

    // spectrum [plane][y'][kx] -> natural packed rows of the unnormalised c2r
    __device__ __forceinline__ static void inverse(cx<T> *buf, const cx<T> *twM, const cx<T> *twN2, const cx<T> *twN1)
    {
        (void)twM;
        stack_fft<N2, 1, T, PPC * NH, NH, PS, 1, NH>(buf, twN2);         // columns (natural y out)
        for (int row = threadIdx.x; row < PPC * N2; row += blockDim.x) {
            cx<T> *b = buf + row * NH;
            cx<T> x[M + 1];
#pragma unroll
            for (int k = 0; k <= M; k++) x[k] = b[k];
            cx<T> z[M];
#pragma unroll
            for (int k = 0; k < M; k++) {
                const cx<T> xk = x[k], xm = conjg(x[M - k]);
                const cx<T> w = conjg(twc<T>(N1, k));
                z[k] = (xk + xm) + mul_si<1>(cmul(w, xk - xm));
            }
            RegDft<M, 1, T>::run(z);
#pragma unroll
            for (int m = 0; m < M; m++) b[m] = z[m];
        }
        __syncthreads();
    }

    // real value at plane-stack index e (plane p, x fastest) from packed rows
    __device__ __forceinline__ static T real_at(const cx<T> *buf, int e)
    {
        const int p = e / NP, r = e % NP, y = r / N1, x = r % N1;
        const cx<T> z = buf[p * PS + y * NH + (x >> 1)];
        return (x & 1) ? z.y : z.x;
    }

    __device__ __forceinline__ static void store(cx<T> *dst, const cx<T> *buf)
    {
        for (int i = threadIdx.x; i < PPC * PS; i += blockDim.x) dst[i] = buf[i];
    }
    __device__ __forceinline__ static void load(cx<T> *buf, const cx<T> *src)
    {
        for (int i = threadIdx.x; i < PPC * PS; i += blockDim.x) buf[i] = src[i];
    }
};

// K2/K4 with a z column shared by two threads (half the registers of
// k3r_zconv): lanes c and c+16 of a warp own column col.  Forward by
// decimation in time: lane half h transforms the samples z = 2j + h
// (length N3/2, registers), the odd half applies W_N^k, the halves meet in
// shared memory and each lane forms one half of the spectrum, X[k + h N3/2].
// After the ek multiply the inverse runs by decimation in frequency: the
// spectrum halves meet again, lane half h forms (A + B) or (A - B) w^k,
// transforms it and owns the samples z = 2m + h.  Natural order in and out.
// 128 threads = 4 warps x 16 columns; grid = (ceil(P/64), nfields, 1 or 2).
template <typename T, int N1, int N2, int N3, bool YNAT>
__global__ void __launch_bounds__(128) k3s_zconv(const SweepField<T> *fields, int t, int which)
{
    constexpr int NH = N1 / 2 + 1, P = N2 * NH, H = N3 / 2;
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    __shared__ __align__(16) cx<T> X[4][N3][16];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, h = lane >> 4, c = lane & 15;
    const int col = (blockIdx.x * 4 + w) * 16 + c;
    const bool ok = col < P;
    const int sel = which == 3 ? (int)blockIdx.z + 1 : which;
    cx<T> *S = ((sel == 1) ? f.S1 : f.S2) + (ok ? col : 0);
    cx<T> v[H];
#pragma unroll
    for (int j = 0; j < H; j++) v[j] = ok ? S[(long)(2 * j + h) * P] : mk<T>((T)0, (T)0);
    RegDft<H, -1, T>::run(v);
#pragma unroll
    for (int k = 0; k < H; k++) X[w][h * H + k][c] = (h && k) ? cmul(v[k], twc<T>(N3, k)) : v[k];
    __syncwarp();
    const T *ek = ((sel == 1) ? f.ek1[blk] : f.ek2[blk]) + (ok ? (col % NH) + NH * (YNAT ? col / NH : iperm<N2>(col / NH)) : 0);
#pragma unroll
    for (int k = 0; k < H; k++) {
        const cx<T> a = X[w][k][c], b = X[w][H + k][c];
        const cx<T> x = h ? a - b : a + b;
        const T e = ok ? __ldg(ek + (long)(k + h * H) * P) : (T)0;
        v[k] = mk<T>(e * x.x, e * x.y);
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < H; k++) X[w][h * H + k][c] = v[k];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < H; k++) {
        const cx<T> a = X[w][k][c], b = X[w][H + k][c];
        v[k] = h ? ((k == 0) ? a - b : cmul(a - b, conjg(twc<T>(N3, k)))) : a + b;
    }
    RegDft<H, 1, T>::run(v);
    if (ok) {
#pragma unroll
        for (int m = 0; m < H; m++) S[(long)(2 * m + h) * P] = v[m];
    }
}

// A stack of PPC x-y planes like PlaneStack, with the column (y)
// transforms in registers: two lanes of a warp share a (plane, kx) column
// and hold half of its N2 values each (decimation in time forward, in
// frequency inverse, the halves meeting in place in the plane buffer), so
// a transform is one shared-memory pass for the rows and one for the
// columns, and spectra are in natural y order.  The forward transform
// writes the columns straight to global memory, the inverse reads them
// from there.  Kernels using it run blockDim = KT (128) threads.
template <typename T, int N1, int N2, int PPC>
struct PlaneStackR {
    static constexpr int M = N1 / 2, NH = M + 1, PS = N2 * NH, NP = N1 * N2;
    using Base = PlaneStack<T, N1, N2, PPC>;

    static constexpr int KT = 128;   // threads per CTA of the kernels using this stack
    // column passes: 16 columns per warp (two lanes each).  Columns kx = 0
    // and kx = M are real after the row pass and can be transformed together
    // as one complex column; that is done where it saves a round of the
    // warps (4 planes of 32 x 32: 68 -> 64 columns), not where it only
    // adds the separation step.  FP64 only: the FP32 transforms keep the
    // plain layout, whose rounding the mixed-precision switch was tuned on
    // (with packed FP32 columns one of 64 BCC solves left its basin).
    static constexpr int WARPS = KT / 32;
    static constexpr bool PACK = sizeof(T) == 8 &&
        ((PPC * NH + 15) / 16 + WARPS - 1) / WARPS > ((PPC * M + 15) / 16 + WARPS - 1) / WARPS;
    static constexpr int CW = PACK ? M : NH;   // column tasks per plane
    static_assert(!PACK || 16 % M == 0, "packed column tasks must tile the 16-task warp blocks");

    // packed rows z[m] = f(2m) + i f(2m+1); compile-time stride so that the
    // loads of several iterations are in flight together
    template <typename F>
    __device__ __forceinline__ static void pack(cx<T> *buf, F value)
    {
#pragma unroll 16
        for (int i = threadIdx.x; i < PPC * N2 * M; i += KT) {
            const int p = i / (N2 * M), r = i % (N2 * M), y = r / M, m = r % M;
            const int e = p * NP + y * N1 + 2 * m;
            buf[p * PS + y * NH + m] = mk<T>(value(e), value(e + 1));
        }
    }
    __device__ __forceinline__ static T real_at(const cx<T> *buf, int e) { return Base::real_at(buf, e); }
    // the slot real_at reads, for writing a real value back in place
    __device__ __forceinline__ static T &real_ref(cx<T> *buf, int e)
    {
        const int p = e / NP, r = e % NP, y = r / N1, x = r % N1;
        cx<T> &z = buf[p * PS + y * NH + (x >> 1)];
        return (x & 1) ? z.y : z.x;
    }

    // natural packed rows in buf -> spectrum [plane][y][kx] in dst (global)
    __device__ __forceinline__ static void forward_to(cx<T> *buf, cx<T> *__restrict__ dst)
    {
        __syncthreads();
        for (int row = threadIdx.x; row < PPC * N2; row += blockDim.x) {
            cx<T> *b = buf + row * NH;
            cx<T> z[M];
#pragma unroll
            for (int m = 0; m < M; m++) z[m] = b[m];
            RegDft<M, -1, T>::run(z);
#pragma unroll
            for (int k = 0; k <= M; k++) {
                const cx<T> zk = z[k % M], zm = conjg(z[(M - k) % M]);
                const cx<T> w = twc<T>(N1, k);
                b[k] = scale((zk + zm) + mul_si<-1>(cmul(w, zk - zm)), (T)0.5);
            }
        }
        __syncthreads();
        // columns, two lanes per column (lanes c and c+16 of a warp):
        // decimation in time, the halves meet in place in buf.  With PACK,
        // task kx = 0 transforms x0 + i xM and separates the two columns
        // afterwards by Hermitian symmetry.
        constexpr int H = N2 / 2, NC = PPC * CW, NCB = (NC + 15) / 16;
        const int h = (threadIdx.x >> 4) & 1, cl = threadIdx.x & 15;
        for (int cb = threadIdx.x >> 5; cb < NCB; cb += KT >> 5) {
            const int c = cb * 16 + cl;
            const bool ok = c < NC;
            const int kx = ok ? c % CW : 1;
            const int off = ok ? (c / CW) * PS + kx : 0;
            const bool pk = PACK && ok && kx == 0;
            cx<T> v[H];
            if (ok) {
#pragma unroll
                for (int j = 0; j < H; j++) {
                    v[j] = buf[off + (2 * j + h) * NH];
                    if (pk) v[j] = mk<T>(v[j].x, buf[off + M + (2 * j + h) * NH].x);
                }
                RegDft<H, -1, T>::run(v);
#pragma unroll
                for (int k = 0; k < H; k++) buf[off + (2 * k + h) * NH] = (h && k) ? cmul(v[k], twc<T>(N2, k)) : v[k];
            }
            __syncwarp();
            if (ok) {
                // the packed task parks its transform in column M (read by
                // both of its lanes before the previous __syncwarp)
#pragma unroll
                for (int k = 0; k < H; k++) {
                    const cx<T> a = buf[off + 2 * k * NH], b = buf[off + (2 * k + 1) * NH];
                    const cx<T> r = h ? a - b : a + b;
                    if (pk)
                        buf[off + M + (k + h * H) * NH] = r;
                    else
                        dst[off + (k + h * H) * NH] = r;
                }
            }
            __syncwarp();
            if (PACK) {
                // separation of the block's packed columns, one (column, ky)
                // per lane: X0[ky] = (Z[ky] + conj Z[-ky]) / 2,
                // XM[ky] = (Z[ky] - conj Z[-ky]) / 2i
                constexpr int PB = 16 / M;   // packed columns per block of 16 tasks
                for (int l = threadIdx.x & 31; l < PB * N2; l += 32) {
                    const int p = (cb * 16) / M + l / N2, ky = l % N2;
                    if (p < PPC) {
                        const int o = p * PS;
                        const cx<T> z = buf[o + M + ky * NH], zm = conjg(buf[o + M + ((N2 - ky) % N2) * NH]);
                        dst[o + ky * NH] = scale(z + zm, (T)0.5);
                        dst[o + M + ky * NH] = scale(mul_si<-1>(z - zm), (T)0.5);
                    }
                }
            }
            __syncwarp();
        }
    }

    // spectrum [plane][y][kx] in src (global) -> natural packed rows of the
    // unnormalised c2r in buf
    __device__ __forceinline__ static void inverse_from(const cx<T> *__restrict__ src, cx<T> *buf)
    {
        __syncthreads();
        // columns, two lanes per column: each lane brings its spectrum half
        // into buf, then decimation in frequency; lane half h ends with the
        // samples y = 2m + h
        // (with PACK, columns kx = 0 and M, Hermitian in ky, go together as
        // one complex column X0 + i XM whose transform is x0 + i xM)
        constexpr int H = N2 / 2, NC = PPC * CW, NCB = (NC + 15) / 16;
        const int h = (threadIdx.x >> 4) & 1, cl = threadIdx.x & 15;
        for (int cb = threadIdx.x >> 5; cb < NCB; cb += KT >> 5) {
            const int c = cb * 16 + cl;
            const bool ok = c < NC;
            const int kx = ok ? c % CW : 1;
            const int off = ok ? (c / CW) * PS + kx : 0;
            const bool pk = PACK && ok && kx == 0;
            cx<T> v[H];
            if (ok) {
#pragma unroll
                for (int k = 0; k < H; k++) {
                    const int e = off + (k + h * H) * NH;
                    buf[e] = pk ? src[e] + mul_si<1>(src[e + M]) : src[e];
                }
            }
            __syncwarp();
            if (ok) {
#pragma unroll
                for (int k = 0; k < H; k++) {
                    const cx<T> a = buf[off + k * NH], b = buf[off + (k + H) * NH];
                    v[k] = h ? ((k == 0) ? a - b : cmul(a - b, conjg(twc<T>(N2, k)))) : a + b;
                }
            }
            __syncwarp();
            if (ok) {
                RegDft<H, 1, T>::run(v);
#pragma unroll
                for (int m = 0; m < H; m++) {
                    if (pk) {
                        buf[off + (2 * m + h) * NH] = mk<T>(v[m].x, (T)0);
                        buf[off + M + (2 * m + h) * NH] = mk<T>(v[m].y, (T)0);
                    } else {
                        buf[off + (2 * m + h) * NH] = v[m];
                    }
                }
            }
        }
        __syncthreads();
        for (int row = threadIdx.x; row < PPC * N2; row += blockDim.x) {
            cx<T> *b = buf + row * NH;
            cx<T> z[M];
#pragma unroll
            for (int k = 0; k < M; k++) {
                const cx<T> xk = b[k], xm = conjg(b[M - k]);
                const cx<T> w = conjg(twc<T>(N1, k));
                z[k] = (xk + xm) + mul_si<1>(cmul(w, xk - xm));
            }
            RegDft<M, 1, T>::run(z);
#pragma unroll
            for (int m = 0; m < M; m++) b[m] = z[m];
        }
        __syncthreads();
    }
};

// The step kernels of the register-column variant (same algebra as
// k3c_fwd_pair / k3c_inv_mid / k3c_inv_final; spectra in natural y order,
// z pass k3s_zconv<..., true>).  128 threads, PPC planes per CTA.  They read
// only exp(-w ds/4) and square it for exp(-w ds/2) (one table load less
// per grid point; within an ulp of the tabulated value).
template <typename T, int N1, int N2, int N3, int PPC>
__global__ void __launch_bounds__(128, 4) k3r_fwd_pair(const SweepField<T> *fields, int t)
{
    using PSk = PlaneStackR<T, N1, N2, PPC>;
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const long nr = (long)N1 * N2 * N3;
    const int z0 = blockIdx.x * PPC;
    const T *q = src_slice(f, src, nr) + (long)z0 * PSk::NP;
    const T *eo2 = f.eo2[blk] + (long)z0 * PSk::NP;
    PSk::pack(buf, [&](int e) { const T a = eo2[e]; return a * (a * q[e]); });
    PSk::forward_to(buf, f.S1 + (long)z0 * PSk::PS);
    __syncthreads();
    PSk::pack(buf, [&](int e) { return eo2[e] * q[e]; });
    PSk::forward_to(buf, f.S2 + (long)z0 * PSk::PS);
}

template <typename T, int N1, int N2, int N3, int PPC>
__global__ void __launch_bounds__(128, 4) k3r_inv_mid(const SweepField<T> *fields, int t)
{
    using PSk = PlaneStackR<T, N1, N2, PPC>;
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const T rn = (T)((long)N1 * N2 * N3);
    const int z0 = blockIdx.x * PPC;
    const T *eo2 = f.eo2[blk] + (long)z0 * PSk::NP;
    T *q1 = f.q1 + (long)z0 * PSk::NP;
    PSk::inverse_from(f.S1 + (long)z0 * PSk::PS, buf);
#pragma unroll 16
    for (int e = threadIdx.x; e < PPC * PSk::NP; e += PSk::KT) { const T a = eo2[e]; q1[e] = (a * a) * PSk::real_at(buf, e) / rn; }
    PSk::inverse_from(f.S2 + (long)z0 * PSk::PS, buf);
    T *hout = f.h_out ? f.h_out + (long)z0 * PSk::NP : nullptr;

#pragma unroll 16
    for (int i = threadIdx.x; i < PPC * N2 * PSk::M; i += PSk::KT) {
        const int p = i / (N2 * PSk::M), r = i % (N2 * PSk::M), y = r / PSk::M, m = r % PSk::M;
        const int e = p * PSk::NP + y * N1 + 2 * m;
        cx<T> &z = buf[p * PSk::PS + y * PSk::NH + m];
        { const T a = eo2[e], c = eo2[e + 1]; z = mk<T>((a * a) * z.x / rn, (c * c) * z.y / rn); }
        if (hout) {
            hout[e] = z.x;
            hout[e + 1] = z.y;
        }
    }
    PSk::forward_to(buf, f.S2 + (long)z0 * PSk::PS);
}

template <typename T, int N1, int N2, int N3, int PPC>
__global__ void __launch_bounds__(128, 4) k3r_inv_final(const SweepField<T> *fields, int t)
{
    using PSk = PlaneStackR<T, N1, N2, PPC>;
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const long nr = (long)N1 * N2 * N3;
    const T rn = (T)nr;
    const int z0 = blockIdx.x * PPC;
    const T *eo2 = f.eo2[blk] + (long)z0 * PSk::NP;
    const T *q1 = f.q1 + (long)z0 * PSk::NP;
    T *out = dst_slice(f, dst, nr) + (long)z0 * PSk::NP;
    T *q2o = f.q2_out ? f.q2_out + (long)z0 * PSk::NP : nullptr;
    PSk::inverse_from(f.S2 + (long)z0 * PSk::PS, buf);

#pragma unroll 16
    for (int e = threadIdx.x; e < PPC * PSk::NP; e += PSk::KT) {
        const T q2 = eo2[e] * PSk::real_at(buf, e) / rn;
        out[e] = ((T)4 * q2 - q1[e]) / (T)3;
        if (q2o) q2o[e] = q2;
    }
}

// K1: S1 = Fxy[eo1 q], S2 = Fxy[eo2 q]   grid = (N3/PPC, nfields)
template <typename T, int N1, int N2, int N3, int PPC>
__global__ void __launch_bounds__(256) k3c_fwd_pair(const SweepField<T> *fields, PlaneGeom g, int t)
{
    using PSk = PlaneStack<T, N1, N2, PPC>;
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const long nr = (long)N1 * N2 * N3;
    const int z0 = blockIdx.x * PPC;
    const T *q = src_slice(f, src, nr) + (long)z0 * PSk::NP;
    const T *eo1 = f.eo1[blk] + (long)z0 * PSk::NP, *eo2 = f.eo2[blk] + (long)z0 * PSk::NP;
    const cx<T> *twM = (const cx<T> *)g.row.tw, *twN2 = (const cx<T> *)g.col.tw, *twN1 = (const cx<T> *)g.rtw;
    PSk::pack(buf, [&](int e) { return eo1[e] * q[e]; });
    PSk::forward(buf, twM, twN2, twN1);
    PSk::store(f.S1 + (long)z0 * PSk::PS, buf);
    __syncthreads();
    PSk::pack(buf, [&](int e) { return eo2[e] * q[e]; });
    PSk::forward(buf, twM, twN2, twN1);
    PSk::store(f.S2 + (long)z0 * PSk::PS, buf);
}

// K2/K4: along z on a tile of TC columns: S <- Fz^-1[ek . Fz[S]]
// which: 1 = S1/ek1, 2 = S2/ek2, 3 = both (grid.z selects)
template <typename T, int N1, int N2, int N3, int TC>
__global__ void __launch_bounds__(256) k3c_zconv(const SweepField<T> *fields, PlaneGeom g, int t, int which)
{
    constexpr int NH = N1 / 2 + 1, P = N2 * NH;
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    const int sel = which == 3 ? (int)blockIdx.z + 1 : which;
    cx<T> *S = (sel == 1) ? f.S1 : f.S2;
    const T *ek = (sel == 1) ? f.ek1[blk] : f.ek2[blk];
    __shared__ __align__(16) cx<T> buf[N3 * TC];
    const int c0 = blockIdx.x * TC;
    for (int i = threadIdx.x; i < N3 * TC; i += blockDim.x) {
        const int z = i / TC, c = i % TC;
        buf[i] = (c0 + c < P) ? S[(long)z * P + c0 + c] : mk<T>((T)0, (T)0);
    }
    const cx<T> *twz = (const cx<T> *)g.zp.tw;
    stack_fft<N3, -1, T, TC, TC, 0, 1, TC>(buf, twz);
    for (int i = threadIdx.x; i < N3 * TC; i += blockDim.x) {
        const int pz = i / TC, c = i % TC;
        const int col = c0 + c;
        if (col < P) {
            const int py = col / NH, kx = col % NH;
            const int kz = iperm<N3>(pz), ky = iperm<N2>(py);
            const T e = ek[kx + NH * (ky + N2 * kz)];
            buf[i] = mk<T>(e * buf[i].x, e * buf[i].y);
        }
    }
    stack_fft<N3, 1, T, TC, TC, 0, 1, TC>(buf, twz);
    for (int i = threadIdx.x; i < N3 * TC; i += blockDim.x) {
        const int z = i / TC, c = i % TC;
        if (c0 + c < P) S[(long)z * P + c0 + c] = buf[i];
    }
}

// K2/K4 with register columns: one thread owns a whole z column of the
// spectrum (N3 values, loaded coalesced across the warp: consecutive threads
// take consecutive columns), transforms it in registers in natural order,
// multiplies by ek and transforms back.  No shared memory, no barriers.
// grid = (ceil(P / 128), nfields, 1 or 2); which as in k3c_zconv.
template <typename T, int N1, int N2, int N3, bool YNAT = false>
__global__ void __launch_bounds__(128) k3r_zconv(const SweepField<T> *fields, int t, int which)
{
    constexpr int NH = N1 / 2 + 1, P = N2 * NH;
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= P) return;
    const int sel = which == 3 ? (int)blockIdx.z + 1 : which;
    cx<T> *S = ((sel == 1) ? f.S1 : f.S2) + col;
    const T *ek = ((sel == 1) ? f.ek1[blk] : f.ek2[blk]) + (col % NH) + NH * (YNAT ? col / NH : iperm<N2>(col / NH));
    cx<T> v[N3];
#pragma unroll
    for (int z = 0; z < N3; z++) v[z] = S[(long)z * P];
    RegDft<N3, -1, T>::run(v);
#pragma unroll
    for (int k = 0; k < N3; k++) {
        const T e = __ldg(ek + (long)k * P);
        v[k] = mk<T>(e * v[k].x, e * v[k].y);
    }
    RegDft<N3, 1, T>::run(v);
#pragma unroll
    for (int z = 0; z < N3; z++) S[(long)z * P] = v[z];
}

// K3: q1 = eo1 Fxy^-1[S1]/N ; S2 <- Fxy[eo1 Fxy^-1[S2]/N]
template <typename T, int N1, int N2, int N3, int PPC>
__global__ void __launch_bounds__(256) k3c_inv_mid(const SweepField<T> *fields, PlaneGeom g, int t)
{
    using PSk = PlaneStack<T, N1, N2, PPC>;
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const T rn = (T)((long)N1 * N2 * N3);
    const int z0 = blockIdx.x * PPC;
    const T *eo1 = f.eo1[blk] + (long)z0 * PSk::NP;
    T *q1 = f.q1 + (long)z0 * PSk::NP;
    const cx<T> *twM = (const cx<T> *)g.row.tw, *twN2 = (const cx<T> *)g.col.tw, *twN1 = (const cx<T> *)g.rtw;
    PSk::load(buf, f.S1 + (long)z0 * PSk::PS);
    PSk::inverse(buf, twM, twN2, twN1);
    for (int e = threadIdx.x; e < PPC * PSk::NP; e += blockDim.x) q1[e] = eo1[e] * PSk::real_at(buf, e) / rn;
    __syncthreads();
    PSk::load(buf, f.S2 + (long)z0 * PSk::PS);
    PSk::inverse(buf, twM, twN2, twN1);
    // h = eo1 y / N, packed in place: entry (p, y, m) <- (h(2m), h(2m+1))
    T *hout = f.h_out ? f.h_out + (long)z0 * PSk::NP : nullptr;
    for (int i = threadIdx.x; i < PPC * N2 * PSk::M; i += blockDim.x) {
        const int p = i / (N2 * PSk::M), r = i % (N2 * PSk::M), y = r / PSk::M, m = r % PSk::M;
        const int e = p * PSk::NP + y * N1 + 2 * m;
        cx<T> &z = buf[p * PSk::PS + y * PSk::NH + m];
        z = mk<T>(eo1[e] * z.x / rn, eo1[e + 1] * z.y / rn);
        if (hout) {
            hout[e] = z.x;
            hout[e + 1] = z.y;
        }
    }
    PSk::forward(buf, twM, twN2, twN1);
    PSk::store(f.S2 + (long)z0 * PSk::PS, buf);
}

// K5: q_out = (4 eo2 Fxy^-1[S2]/N - q1)/3
template <typename T, int N1, int N2, int N3, int PPC>
__global__ void __launch_bounds__(256) k3c_inv_final(const SweepField<T> *fields, PlaneGeom g, int t)
{
    using PSk = PlaneStack<T, N1, N2, PPC>;
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const long nr = (long)N1 * N2 * N3;
    const T rn = (T)nr;
    const int z0 = blockIdx.x * PPC;
    const T *eo2 = f.eo2[blk] + (long)z0 * PSk::NP;
    const T *q1 = f.q1 + (long)z0 * PSk::NP;
    T *out = dst_slice(f, dst, nr) + (long)z0 * PSk::NP;
    T *q2o = f.q2_out ? f.q2_out + (long)z0 * PSk::NP : nullptr;
    const cx<T> *twM = (const cx<T> *)g.row.tw, *twN2 = (const cx<T> *)g.col.tw, *twN1 = (const cx<T> *)g.rtw;
    PSk::load(buf, f.S2 + (long)z0 * PSk::PS);
    PSk::inverse(buf, twM, twN2, twN1);
    for (int e = threadIdx.x; e < PPC * PSk::NP; e += blockDim.x) {
        const T q2 = eo2[e] * PSk::real_at(buf, e) / rn;
        out[e] = ((T)4 * q2 - q1[e]) / (T)3;
        if (q2o) q2o[e] = q2;
    }
}

}  // namespace pscfg

namespace pscfg {

// Stress slice sums with compile-time-shaped transforms (same contract as
// k3_stress_xy / k3_stress_z / k3_stress_sum in scf_kernels.cuh).
// Pass 1: xy-forward of PPC planes of slice s (qf or qr) into
// spec[((s - s0) * 2 + fr)][z][y'][kx].  grid = (N3/PPC, cs, 2).
template <typename T, int N1, int N2, int N3, int PPC>
__global__ void __launch_bounds__(256) k3c_stress_xy(const StressJob<T> *job, PlaneGeom g, int s0, cx<T> *spec)
{
    using PSk = PlaneStack<T, N1, N2, PPC>;
    const StressJob<T> &J = *job;
    const int s = s0 + blockIdx.y;
    if (s >= J.nslices) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const long nr = (long)N1 * N2 * N3, nk = (long)PSk::PS * N3;
    const int z0 = blockIdx.x * PPC;
    const T *q = (blockIdx.z == 0 ? J.qf : J.qr) + (long)s * nr + (long)z0 * PSk::NP;
    PSk::pack(buf, [&](int e) { return q[e]; });
    PSk::forward(buf, (const cx<T> *)g.row.tw, (const cx<T> *)g.col.tw, (const cx<T> *)g.rtw);
    PSk::store(spec + ((long)blockIdx.y * 2 + blockIdx.z) * nk + (long)z0 * PSk::PS, buf);
}

// K5 of step t fused with K1 of step t+1 (sweeps only): q_out as in
// k3r_inv_final, kept in the plane buffer, then, if the field has a step
// t+1, its x-y forward transforms of exp(-w ds/2) q_out and
// exp(-w ds/4) q_out with the tables of step t+1's block.
template <typename T, int N1, int N2, int N3, int PPC>
__global__ void __launch_bounds__(128, 4) k3r_final_fwd(const SweepField<T> *fields, int t)
{
    using PSk = PlaneStackR<T, N1, N2, PPC>;
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const long nr = (long)N1 * N2 * N3;
    const T rn = (T)nr;
    const int z0 = blockIdx.x * PPC;
    const T *eo2 = f.eo2[blk] + (long)z0 * PSk::NP;
    const T *q1 = f.q1 + (long)z0 * PSk::NP;
    T *out = dst_slice(f, dst, nr) + (long)z0 * PSk::NP;
    PSk::inverse_from(f.S2 + (long)z0 * PSk::PS, buf);

#pragma unroll 16
    for (int e = threadIdx.x; e < PPC * PSk::NP; e += PSk::KT) {
        T &slot = PSk::real_ref(buf, e);
        const T q2 = eo2[e] * slot / rn;
        const T o = ((T)4 * q2 - q1[e]) / (T)3;
        out[e] = o;
        slot = o;
    }
    int blk2, src2, dst2;
    if (!step_slices(f, t + 1, blk2, src2, dst2)) return;   // the same for the whole CTA
    __syncthreads();
    const T *n2 = f.eo2[blk2] + (long)z0 * PSk::NP;

#pragma unroll 16
    for (int e = threadIdx.x; e < PPC * PSk::NP; e += PSk::KT) {
        T &slot = PSk::real_ref(buf, e);
        { const T a = n2[e]; slot = (a * a) * slot; }
    }
    PSk::forward_to(buf, f.S1 + (long)z0 * PSk::PS);
    __syncthreads();
    const T *qn = out;   // written above by this CTA; visible after the barrier
    PSk::pack(buf, [&](int e) { return n2[e] * qn[e]; });
    PSk::forward_to(buf, f.S2 + (long)z0 * PSk::PS);
}

// Register-column variant of the stress pass.  Pass 1: x-y forward of PPC
// planes of slice s (qf or qr) with PlaneStackR (natural y order), 128
// threads.  grid = (N3/PPC, cs, 2).
template <typename T, int N1, int N2, int N3, int PPC>
__global__ void __launch_bounds__(128, 4) k3r_stress_xy(const StressJob<T> *job, int s0, cx<T> *spec)
{
    using PSk = PlaneStackR<T, N1, N2, PPC>;
    const StressJob<T> &J = *job;
    const int s = s0 + blockIdx.y;
    if (s >= J.nslices) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const long nr = (long)N1 * N2 * N3, nk = (long)PSk::PS * N3;
    const int z0 = blockIdx.x * PPC;
    const T *q = (blockIdx.z == 0 ? J.qf : J.qr) + (long)s * nr + (long)z0 * PSk::NP;
    PSk::pack(buf, [&](int e) { return q[e]; });
    PSk::forward_to(buf, spec + ((long)blockIdx.y * 2 + blockIdx.z) * nk + (long)z0 * PSk::PS);
}

// Pass 2: one thread per z column: z-forward of the qf spectrum in
// registers (written back in place), then of the qr spectrum, and the
// weighted products sum_k wdgsq_b(k) Re(F conj R) of its column; block
// sums per tile of 128 columns.  grid = (ceil(P/128), cs).
template <typename T, int N1, int N2, int N3>
__global__ void __launch_bounds__(128) k3r_stress_z(const StressJob<T> *job, int s0, cx<T> *spec, double *part)
{
    constexpr int NH = N1 / 2 + 1, P = N2 * NH;
    const StressJob<T> &J = *job;
    const int s = s0 + blockIdx.y;
    if (s >= J.nslices) return;
    __shared__ double red[32];
    const long nk = (long)P * N3;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[PSCFG_MAXCP] = {0, 0, 0, 0, 0, 0};
    if (col < P) {
        cx<T> *sf = spec + ((long)blockIdx.y * 2) * nk + col;
        const cx<T> *sr = sf + nk;
        cx<T> v[N3];
#pragma unroll
        for (int z = 0; z < N3; z++) v[z] = sf[(long)z * P];
        RegDft<N3, -1, T>::run(v);
#pragma unroll
        for (int k = 0; k < N3; k++) sf[(long)k * P] = v[k];
        // re-read the stored spectrum below instead of keeping it live in
        // registers next to the second column (which would spill)
        asm volatile("" ::: "memory");
#pragma unroll
        for (int z = 0; z < N3; z++) v[z] = sr[(long)z * P];
        RegDft<N3, -1, T>::run(v);
        double d[N3];
#pragma unroll
        for (int k = 0; k < N3; k++) {
            const cx<T> f = sf[(long)k * P];
            d[k] = (double)f.x * (double)v[k].x + (double)f.y * (double)v[k].y;
        }
        const double *w = J.wdgsq + col;
#pragma unroll 1
        for (int b = 0; b < J.ncp; b++) {
            double a = 0.0;
#pragma unroll
            for (int k = 0; k < N3; k++) a += __ldg(w + (long)b * nk + (long)k * P) * d[k];
            acc[b] = a;
        }
    }
    for (int b = 0; b < J.ncp; b++) {
        const double tot = block_sum(acc[b], red);
        if (threadIdx.x == 0) part[((long)blockIdx.y * gridDim.x + blockIdx.x) * PSCFG_MAXCP + b] = tot;
        __syncthreads();
    }
}

// Stress pass 2 with two lanes per z column (as k3s_zconv): each lane ends
// with half of the qf spectrum and the same half of the qr spectrum in
// registers and forms its products sum_k wdgsq_b(k) Re(F conj R) there;
// block sums per tile of 64 columns.  grid = (ceil(P/64), cs).
template <typename T, int N1, int N2, int N3>
__global__ void __launch_bounds__(128) k3s_stress_z(const StressJob<T> *job, int s0, const cx<T> *spec, double *part)
{
    constexpr int NH = N1 / 2 + 1, P = N2 * NH, H = N3 / 2;
    const StressJob<T> &J = *job;
    const int s = s0 + blockIdx.y;
    if (s >= J.nslices) return;
    __shared__ __align__(16) cx<T> X[4][N3][16];
    __shared__ double red[32];
    const long nk = (long)P * N3;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, h = lane >> 4, c = lane & 15;
    const int col = (blockIdx.x * 4 + w) * 16 + c;
    const bool ok = col < P;
    const cx<T> *sf = spec + ((long)blockIdx.y * 2) * nk + (ok ? col : 0), *sr = sf + nk;
    // forward z transform of one column half (decimation in time); returns
    // the spectrum entries k + h H, k < H, in v
    auto ztrans = [&](const cx<T> *src, cx<T> *v) {
#pragma unroll
        for (int j = 0; j < H; j++) v[j] = ok ? src[(long)(2 * j + h) * P] : mk<T>((T)0, (T)0);
        RegDft<H, -1, T>::run(v);
#pragma unroll
        for (int k = 0; k < H; k++) X[w][h * H + k][c] = (h && k) ? cmul(v[k], twc<T>(N3, k)) : v[k];
        __syncwarp();
#pragma unroll
        for (int k = 0; k < H; k++) {
            const cx<T> a = X[w][k][c], b = X[w][H + k][c];
            v[k] = h ? a - b : a + b;
        }
        __syncwarp();
    };
    cx<T> fv[H], rv[H];
    ztrans(sf, fv);
    ztrans(sr, rv);
    double acc[PSCFG_MAXCP] = {0, 0, 0, 0, 0, 0};
    if (ok) {
        const double *wp = J.wdgsq + col + (long)h * H * P;
#pragma unroll 1
        for (int b = 0; b < J.ncp; b++) {
            double a = 0.0;
#pragma unroll
            for (int k = 0; k < H; k++)
                a += __ldg(wp + (long)b * nk + (long)k * P) *
                     ((double)fv[k].x * (double)rv[k].x + (double)fv[k].y * (double)rv[k].y);
            acc[b] = a;
        }
    }
    for (int b = 0; b < J.ncp; b++) {
        const double tot = block_sum(acc[b], red);
        if (threadIdx.x == 0) part[((long)blockIdx.y * gridDim.x + blockIdx.x) * PSCFG_MAXCP + b] = tot;
        __syncthreads();
    }
}

// Batched forms of the register-column stress pass: all jobs of a call in
// one launch per pass (job = blockIdx.z [/ 2]), cs slices from s0 each;
// spectra at ((job cs + slice) 2 + which) nk, partial sums at
// ((job cs + slice) ntiles + tile) PSCFG_MAXCP.
template <typename T, int N1, int N2, int N3, int PPC>
__global__ void __launch_bounds__(128, 4) k3r_stress_xy_b(const StressJob<T> *jobs, int s0, int cs, cx<T> *spec)
{
    using PSk = PlaneStackR<T, N1, N2, PPC>;
    const int job = blockIdx.z >> 1, which = blockIdx.z & 1;
    const StressJob<T> &J = jobs[job];
    const int s = s0 + blockIdx.y;
    if (s >= J.nslices) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *buf = (cx<T> *)smem_raw;
    const long nr = (long)N1 * N2 * N3, nk = (long)PSk::PS * N3;
    const int z0 = blockIdx.x * PPC;
    const T *q = (which == 0 ? J.qf : J.qr) + (long)s * nr + (long)z0 * PSk::NP;
    PSk::pack(buf, [&](int e) { return q[e]; });
    PSk::forward_to(buf, spec + (((long)job * cs + blockIdx.y) * 2 + which) * nk + (long)z0 * PSk::PS);
}

template <typename T, int N1, int N2, int N3>
__global__ void __launch_bounds__(128) k3s_stress_z_b(const StressJob<T> *jobs, int s0, int cs, const cx<T> *spec,
                                                      double *part)
{
    constexpr int NH = N1 / 2 + 1, P = N2 * NH, H = N3 / 2;
    const int job = blockIdx.z;
    const StressJob<T> &J = jobs[job];
    const int s = s0 + blockIdx.y;
    if (s >= J.nslices) return;
    __shared__ __align__(16) cx<T> X[4][N3][16];
    __shared__ double red[32];
    const long nk = (long)P * N3;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, h = lane >> 4, c = lane & 15;
    const int col = (blockIdx.x * 4 + w) * 16 + c;
    const bool ok = col < P;
    const cx<T> *sf = spec + (((long)job * cs + blockIdx.y) * 2) * nk + (ok ? col : 0), *sr = sf + nk;
    auto ztrans = [&](const cx<T> *src, cx<T> *v) {
#pragma unroll
        for (int j = 0; j < H; j++) v[j] = ok ? src[(long)(2 * j + h) * P] : mk<T>((T)0, (T)0);
        RegDft<H, -1, T>::run(v);
#pragma unroll
        for (int k = 0; k < H; k++) X[w][h * H + k][c] = (h && k) ? cmul(v[k], twc<T>(N3, k)) : v[k];
        __syncwarp();
#pragma unroll
        for (int k = 0; k < H; k++) {
            const cx<T> a = X[w][k][c], b = X[w][H + k][c];
            v[k] = h ? a - b : a + b;
        }
        __syncwarp();
    };
    cx<T> fv[H], rv[H];
    ztrans(sf, fv);
    ztrans(sr, rv);
    double acc[PSCFG_MAXCP] = {0, 0, 0, 0, 0, 0};
    if (ok) {
        const double *wp = J.wdgsq + col + (long)h * H * P;
#pragma unroll 1
        for (int b = 0; b < J.ncp; b++) {
            double a = 0.0;
#pragma unroll
            for (int k = 0; k < H; k++)
                a += __ldg(wp + (long)b * nk + (long)k * P) *
                     ((double)fv[k].x * (double)rv[k].x + (double)fv[k].y * (double)rv[k].y);
            acc[b] = a;
        }
    }
    for (int b = 0; b < J.ncp; b++) {
        const double tot = block_sum(acc[b], red);
        if (threadIdx.x == 0)
            part[(((long)job * cs + blockIdx.y) * gridDim.x + blockIdx.x) * PSCFG_MAXCP + b] = tot;
        __syncthreads();
    }
}

template <typename T>
__global__ void k3_stress_sum_b(const StressJob<T> *jobs, int s0, int cs, int ntiles, const double *part)
{
    const int job = blockIdx.y;
    const StressJob<T> &J = jobs[job];
    const int s = s0 + blockIdx.x;
    if (s >= J.nslices || threadIdx.x >= J.ncp) return;
    const int b = threadIdx.x;
    double acc = 0.0;
    for (int t = 0; t < ntiles; t++) acc += part[(((long)job * cs + blockIdx.x) * ntiles + t) * PSCFG_MAXCP + b];
    J.inc[(long)s * PSCFG_MAXCP + b] = acc;
}

// Pass 2: z-forward of both spectra on TC columns and the weighted dot
// products sum_k wdgsq_b(k) Re(F conj R).  grid = (ntiles, cs).
template <typename T, int N1, int N2, int N3, int TC>
__global__ void __launch_bounds__(256) k3c_stress_z(const StressJob<T> *job, PlaneGeom g, int s0, const cx<T> *spec,
                                                    double *part)
{
    constexpr int NH = N1 / 2 + 1, P = N2 * NH;
    const StressJob<T> &J = *job;
    const int s = s0 + blockIdx.y;
    if (s >= J.nslices) return;
    __shared__ __align__(16) cx<T> F[N3 * TC];
    __shared__ __align__(16) cx<T> R[N3 * TC];
    __shared__ double red[32];
    const long nk = (long)P * N3;
    const int c0 = blockIdx.x * TC;
    const cx<T> *sf = spec + ((long)blockIdx.y * 2) * nk, *sr = sf + nk;
    for (int i = threadIdx.x; i < N3 * TC; i += blockDim.x) {
        const int z = i / TC, c = i % TC;
        const bool ok = c0 + c < P;
        F[i] = ok ? sf[(long)z * P + c0 + c] : mk<T>((T)0, (T)0);
        R[i] = ok ? sr[(long)z * P + c0 + c] : mk<T>((T)0, (T)0);
    }
    const cx<T> *twz = (const cx<T> *)g.zp.tw;
    stack_fft<N3, -1, T, TC, TC, 0, 1, TC>(F, twz);
    stack_fft<N3, -1, T, TC, TC, 0, 1, TC>(R, twz);
    for (int b = 0; b < J.ncp; b++) {
        double acc = 0.0;
        for (int i = threadIdx.x; i < N3 * TC; i += blockDim.x) {
            const int pz = i / TC, c = i % TC, col = c0 + c;
            if (col < P) {
                const int py = col / NH, kx = col % NH;
                const long k = kx + NH * (iperm<N2>(py) + (long)N2 * iperm<N3>(pz));
                const cx<T> f = F[i], r = R[i];
                acc += J.wdgsq[(long)b * nk + k] * ((double)f.x * (double)r.x + (double)f.y * (double)r.y);
            }
        }
        const double tot = block_sum(acc, red);
        if (threadIdx.x == 0) part[((long)blockIdx.y * gridDim.x + blockIdx.x) * PSCFG_MAXCP + b] = tot;
        __syncthreads();
    }
}

}  // namespace pscfg
