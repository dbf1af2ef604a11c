// fft_ct.cuh -- compile-time-sized in-place FFTs for power-of-two lines.
//
// A line of length N = P*Q is transformed in place in shared memory by the
// four-step split n = Q*n1 + n2, k = k1 + P*k2:
//   pass A (one work item per n2): length-P DFT over n1 of x[Q n1 + n2],
//           times W_N^(n2 k1), stored back at Q k1 + n2;
//   pass B (one work item per k1): length-Q DFT over the Q contiguous
//           values at Q k1 + n2, stored back at Q k1 + k2.
// The forward result X[k1 + P k2] therefore sits at position Q k1 + k2
// (perm(k) below).  The inverse runs the passes in reverse order with
// conjugate twiddles, consumes that permuted order and returns natural
// order, so a forward/multiply/inverse chain never reorders data.  Every
// thread reads and writes only its own positions within a pass, so one
// __syncthreads separates the passes.  All sizes are template constants:
// the index arithmetic is shifts and masks.
#pragma once
#include "fft_dev.cuh"

namespace pscfg {

template <int N> struct Split;
template <> struct Split<2> { static constexpr int P = 2, Q = 1; };
template <> struct Split<4> { static constexpr int P = 4, Q = 1; };
template <> struct Split<8> { static constexpr int P = 8, Q = 1; };
template <> struct Split<16> { static constexpr int P = 4, Q = 4; };
template <> struct Split<32> { static constexpr int P = 4, Q = 8; };
template <> struct Split<64> { static constexpr int P = 8, Q = 8; };
template <> struct Split<128> { static constexpr int P = 8, Q = 16; };

// Length-16 DFT in registers as 4 x 4.
template <int S, typename T> struct Dft<16, S, T> {
    __device__ __forceinline__ static void run(cx<T> *v)
    {
        // n = 4 n1 + n2; k = k1 + 4 k2
        cx<T> y[16];
#pragma unroll
        for (int n2 = 0; n2 < 4; n2++) {
            cx<T> a[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
            Dft<4, S, T>::run(a);
#pragma unroll
            for (int k1 = 0; k1 < 4; k1++) y[4 * k1 + n2] = a[k1];
        }
        // twiddles W16^(n2 k1)
        const T c1 = (T)0.92387953251128675612818318939678828682;   // cos(pi/8)
        const T s1 = (T)0.38268343236508977172845998403039886676;   // sin(pi/8)
        const T h = (T)0.70710678118654752440084436210484903928;
        const cx<T> w1 = mk<T>(c1, (T)S * s1), w2 = mk<T>(h, (T)S * h), w3 = mk<T>(s1, (T)S * c1);
        const cx<T> w4 = mk<T>((T)0, (T)S), w6 = mk<T>(-h, (T)S * h), w9 = mk<T>(-c1, -(T)S * s1);
        y[4 * 1 + 1] = cmul(y[5], w1);
        y[4 * 1 + 2] = cmul(y[6], w2);
        y[4 * 1 + 3] = cmul(y[7], w3);
        y[4 * 2 + 1] = cmul(y[9], w2);
        y[4 * 2 + 2] = cmul(y[10], w4);
        y[4 * 2 + 3] = cmul(y[11], w6);
        y[4 * 3 + 1] = cmul(y[13], w3);
        y[4 * 3 + 2] = cmul(y[14], w6);
        y[4 * 3 + 3] = cmul(y[15], w9);
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++) {
            cx<T> a[4] = {y[4 * k1], y[4 * k1 + 1], y[4 * k1 + 2], y[4 * k1 + 3]};
            Dft<4, S, T>::run(a);
#pragma unroll
            for (int k2 = 0; k2 < 4; k2++) v[k1 + 4 * k2] = a[k2];
        }
    }
};

template <int S, typename T> struct Dft<1, S, T> {
    __device__ __forceinline__ static void run(cx<T> *) {}
};

// W_64^m = exp(-2 pi i m / 64), m in [0, 64): twiddles of the register
// transforms (uniform across a warp, so constant-cache broadcasts).
__constant__ double c_w64[2][64];

template <typename T>
__device__ __forceinline__ cx<T> twc(int n, int k)
{
    const int m = (k * (64 / n)) & 63;
    return mk<T>((T)c_w64[0][m], (T)c_w64[1][m]);
}

// Register DFT of power-of-two length N <= 64, natural order in and out:
// four-step N = 4 x (N/4) with the inner transforms recursive.
template <int N, int S, typename T> struct RegDft {
    __device__ __forceinline__ static void run(cx<T> *v)
    {
        constexpr int P = 4, Q = N / 4;
        cx<T> y[N];
#pragma unroll
        for (int n2 = 0; n2 < Q; n2++) {
            cx<T> a[P];
#pragma unroll
            for (int n1 = 0; n1 < P; n1++) a[n1] = v[Q * n1 + n2];
            Dft<P, S, T>::run(a);
#pragma unroll
            for (int k1 = 0; k1 < P; k1++) {
                cx<T> w = twc<T>(N, n2 * k1);
                if (S > 0) w = conjg(w);
                y[Q * k1 + n2] = (n2 * k1 == 0) ? a[k1] : cmul(a[k1], w);
            }
        }
#pragma unroll
        for (int k1 = 0; k1 < P; k1++) {
            cx<T> b[Q];
#pragma unroll
            for (int n2 = 0; n2 < Q; n2++) b[n2] = y[Q * k1 + n2];
            RegDft<Q, S, T>::run(b);
#pragma unroll
            for (int k2 = 0; k2 < Q; k2++) v[k1 + P * k2] = b[k2];
        }
    }
};
template <int S, typename T> struct RegDft<4, S, T> {
    __device__ __forceinline__ static void run(cx<T> *v) { Dft<4, S, T>::run(v); }
};
template <int S, typename T> struct RegDft<8, S, T> {
    __device__ __forceinline__ static void run(cx<T> *v) { Dft<8, S, T>::run(v); }
};
template <int S, typename T> struct RegDft<2, S, T> {
    __device__ __forceinline__ static void run(cx<T> *v) { Dft<2, S, T>::run(v); }
};
template <int S, typename T> struct RegDft<1, S, T> {
    __device__ __forceinline__ static void run(cx<T> *) {}
};

// Position of frequency k after a forward transform of length N.
template <int N>
__device__ __forceinline__ int perm(int k)
{
    constexpr int P = Split<N>::P, Q = Split<N>::Q;
    return Q * (k % P) + k / P;
}

// Lines: element e of line l at buf[l*LS + e*ES].  NL lines.  tw = W_N^m
// table (forward sign) in shared or global memory.
template <int N, int S, typename T, int NL, int ES, int LS>
__device__ __forceinline__ void fft_ct_passA(cx<T> *buf, const cx<T> *__restrict__ tw)
{
    constexpr int P = Split<N>::P, Q = Split<N>::Q;
    // work items (line, n2)
    for (int w = threadIdx.x; w < NL * Q; w += blockDim.x) {
        const int l = w / Q, n2 = w % Q;
        cx<T> *b = buf + l * LS;
        cx<T> v[P];
        if (S > 0) {
            // inverse: this is the second pass; twiddle first (conjugate)
#pragma unroll
            for (int k1 = 0; k1 < P; k1++) v[k1] = b[(Q * k1 + n2) * ES];
            if (Q > 1) {
#pragma unroll
                for (int k1 = 1; k1 < P; k1++) {
                    cx<T> t = tw[(n2 * k1) % N];
                    v[k1] = cmul(v[k1], conjg(t));
                }
            }
            Dft<P, S, T>::run(v);
#pragma unroll
            for (int n1 = 0; n1 < P; n1++) b[(Q * n1 + n2) * ES] = v[n1];
        } else {
#pragma unroll
            for (int n1 = 0; n1 < P; n1++) v[n1] = b[(Q * n1 + n2) * ES];
            Dft<P, S, T>::run(v);
            if (Q > 1) {
#pragma unroll
                for (int k1 = 1; k1 < P; k1++) v[k1] = cmul(v[k1], tw[(n2 * k1) % N]);
            }
#pragma unroll
            for (int k1 = 0; k1 < P; k1++) b[(Q * k1 + n2) * ES] = v[k1];
        }
    }
}

template <int N, int S, typename T, int NL, int ES, int LS>
__device__ __forceinline__ void fft_ct_passB(cx<T> *buf)
{
    constexpr int P = Split<N>::P, Q = Split<N>::Q;
    if (Q == 1) return;
    for (int w = threadIdx.x; w < NL * P; w += blockDim.x) {
        const int l = w / P, k1 = w % P;
        cx<T> *b = buf + l * LS + Q * k1 * ES;
        cx<T> v[Q];
#pragma unroll
        for (int j = 0; j < Q; j++) v[j] = b[j * ES];
        Dft<Q, S, T>::run(v);
#pragma unroll
        for (int j = 0; j < Q; j++) b[j * ES] = v[j];
    }
}

// Forward (S = -1): natural in, permuted out.  Inverse (S = +1): permuted
// in, natural out.  Begins and ends with __syncthreads.
template <int N, int S, typename T, int NL, int ES, int LS>
__device__ __forceinline__ void fft_ct(cx<T> *buf, const cx<T> *__restrict__ tw)
{
    __syncthreads();
    if (S < 0) {
        fft_ct_passA<N, S, T, NL, ES, LS>(buf, tw);
        __syncthreads();
        fft_ct_passB<N, S, T, NL, ES, LS>(buf);
    } else {
        fft_ct_passB<N, S, T, NL, ES, LS>(buf);
        __syncthreads();
        fft_ct_passA<N, S, T, NL, ES, LS>(buf, tw);
    }
    __syncthreads();
}

}  // namespace pscfg
