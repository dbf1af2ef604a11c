// fft_dev.cuh -- shared-memory FFT building blocks for the MDE step kernels.
//
// Replaces the FFTW calls of the reference (src/fft3_mod.f90:85-157):
//   fft  : r2c forward, unnormalised  (dfftw_plan_dft_r2c_3d)
//   ifft : c2r inverse, unnormalised  (dfftw_plan_dft_c2r_3d)
// with FFTW's sign convention (forward e^{-i}).  Transforms run entirely in
// shared memory: mixed-radix Stockham stages (radix 8,4,2,3,5,7) ping-pong
// between two buffers, all threads of the CTA cooperating, one __syncthreads
// per stage.  A real row of even length n is transformed as n/2 packed
// complex values plus an untangling pass (the standard even/odd split), so
// r2c costs one half-length complex FFT per row.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pscfg {

template <typename T>
struct __align__(2 * sizeof(T)) cx {
    T x, y;
};

template <typename T> __device__ __forceinline__ cx<T> mk(T a, T b) { cx<T> r; r.x = a; r.y = b; return r; }
template <typename T> __device__ __forceinline__ cx<T> operator+(cx<T> a, cx<T> b) { return mk(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ cx<T> operator-(cx<T> a, cx<T> b) { return mk(a.x - b.x, a.y - b.y); }
template <typename T> __device__ __forceinline__ cx<T> cmul(cx<T> a, cx<T> b)
{
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T> __device__ __forceinline__ cx<T> conjg(cx<T> a) { return mk(a.x, -a.y); }
template <typename T> __device__ __forceinline__ cx<T> scale(cx<T> a, T s) { return mk(a.x * s, a.y * s); }
__device__ __forceinline__ cx<double> __ldg_cx(const cx<double> *p)
{
    double2 v = __ldg((const double2 *)p);
    return mk<double>(v.x, v.y);
}
__device__ __forceinline__ cx<float> __ldg_cx(const cx<float> *p)
{
    float2 v = __ldg((const float2 *)p);
    return mk<float>(v.x, v.y);
}

// multiply by (S * i), S = +1 or -1
template <int S, typename T> __device__ __forceinline__ cx<T> mul_si(cx<T> a)
{
    return (S > 0) ? mk(-a.y, a.x) : mk(a.y, -a.x);
}

// cos/sin(2 pi m / R) for R = 5 and 7 (m = 0..R-1), filled by the host from
// long-double evaluations.
__constant__ double c_dft5[2][5];
__constant__ double c_dft7[2][7];

// ---------------------------------------------------------------------
// DFT codelets, in registers.  S = -1 forward, +1 inverse.
// ---------------------------------------------------------------------
template <int R, int S, typename T> struct Dft;

template <int S, typename T> struct Dft<2, S, T> {
    __device__ __forceinline__ static void run(cx<T> *v)
    {
        cx<T> a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    }
};

template <int S, typename T> struct Dft<4, S, T> {
    __device__ __forceinline__ static void run(cx<T> *v)
    {
        cx<T> t0 = v[0] + v[2], t1 = v[0] - v[2];
        cx<T> t2 = v[1] + v[3], t3 = mul_si<S>(v[1] - v[3]);
        v[0] = t0 + t2;
        v[1] = t1 + t3;
        v[2] = t0 - t2;
        v[3] = t1 - t3;
    }
};

template <int S, typename T> struct Dft<8, S, T> {
    __device__ __forceinline__ static void run(cx<T> *v)
    {
        const T h = (T)0.70710678118654752440084436210484903928;
        cx<T> e[4] = {v[0], v[2], v[4], v[6]};
        cx<T> o[4] = {v[1], v[3], v[5], v[7]};
        Dft<4, S, T>::run(e);
        Dft<4, S, T>::run(o);
        // W8^1 = (h, S h), W8^2 = (0, S), W8^3 = (-h, S h)
        cx<T> o1 = cmul(o[1], mk<T>(h, (T)S * h));
        cx<T> o2 = mul_si<S>(o[2]);
        cx<T> o3 = cmul(o[3], mk<T>(-h, (T)S * h));
        v[0] = e[0] + o[0];
        v[4] = e[0] - o[0];
        v[1] = e[1] + o1;
        v[5] = e[1] - o1;
        v[2] = e[2] + o2;
        v[6] = e[2] - o2;
        v[3] = e[3] + o3;
        v[7] = e[3] - o3;
    }
};

template <int S, typename T> struct Dft<3, S, T> {
    __device__ __forceinline__ static void run(cx<T> *v)
    {
        const T s3 = (T)0.86602540378443864676372317075293618347;  // sqrt(3)/2
        cx<T> t1 = v[1] + v[2];
        cx<T> m = mk<T>(v[0].x - (T)0.5 * t1.x, v[0].y - (T)0.5 * t1.y);
        cx<T> d = scale(mul_si<S>(v[1] - v[2]), s3);
        v[0] = v[0] + t1;
        v[1] = m + d;
        v[2] = m - d;
    }
};

template <int R, int S, typename T> struct DftGeneric {
    __device__ __forceinline__ static void run(cx<T> *v)
    {
        const double(*tab)[R] = (R == 5) ? (const double(*)[R])c_dft5 : (const double(*)[R])c_dft7;
        cx<T> out[R];
#pragma unroll
        for (int q = 0; q < R; q++) {
            cx<T> s = v[0];
#pragma unroll
            for (int r = 1; r < R; r++) {
                int m = (r * q) % R;
                cx<T> w = mk<T>((T)tab[0][m], (T)S * (T)tab[1][m]);
                s = s + cmul(v[r], w);
            }
            out[q] = s;
        }
#pragma unroll
        for (int q = 0; q < R; q++) v[q] = out[q];
    }
};
template <int S, typename T> struct Dft<5, S, T> : DftGeneric<5, S, T> {};

// Length-7 DFT from the symmetric pairs t_j = x_j + x_{7-j}, d_j = x_j - x_{7-j}:
// X_k = x_0 + sum_j cos(2 pi jk/7) t_j + S i sum_j sin(2 pi jk/7) d_j and
// X_{7-k} the same with -S (k = 1, 2, 3): 66 real operations.
template <int S, typename T> struct Dft<7, S, T> {
    __device__ __forceinline__ static void run(cx<T> *v)
    {
        const T c1 = (T)0.623489801858733530525004884004239811;    // cos(2 pi/7)
        const T c2 = (T)-0.222520933956314404288902564496794759;   // cos(4 pi/7)
        const T c3 = (T)-0.900968867902419126236102319507445051;   // cos(6 pi/7)
        const T s1 = (T)0.78183148246802980870844452667405775;     // sin(2 pi/7)
        const T s2 = (T)0.974927912181823607018131682993931217;    // sin(4 pi/7)
        const T s3 = (T)0.433883739117558120475768332848358755;    // sin(6 pi/7)
        const cx<T> x0 = v[0];
        const cx<T> t1 = v[1] + v[6], t2 = v[2] + v[5], t3 = v[3] + v[4];
        const cx<T> d1 = v[1] - v[6], d2 = v[2] - v[5], d3 = v[3] - v[4];
        v[0] = x0 + t1 + t2 + t3;
        const cx<T> a1 = mk<T>(x0.x + c1 * t1.x + c2 * t2.x + c3 * t3.x, x0.y + c1 * t1.y + c2 * t2.y + c3 * t3.y);
        const cx<T> a2 = mk<T>(x0.x + c2 * t1.x + c3 * t2.x + c1 * t3.x, x0.y + c2 * t1.y + c3 * t2.y + c1 * t3.y);
        const cx<T> a3 = mk<T>(x0.x + c3 * t1.x + c1 * t2.x + c2 * t3.x, x0.y + c3 * t1.y + c1 * t2.y + c2 * t3.y);
        const cx<T> b1 = mul_si<S>(mk<T>(s1 * d1.x + s2 * d2.x + s3 * d3.x, s1 * d1.y + s2 * d2.y + s3 * d3.y));
        const cx<T> b2 = mul_si<S>(mk<T>(s2 * d1.x - s3 * d2.x - s1 * d3.x, s2 * d1.y - s3 * d2.y - s1 * d3.y));
        const cx<T> b3 = mul_si<S>(mk<T>(s3 * d1.x - s1 * d2.x + s2 * d3.x, s3 * d1.y - s1 * d2.y + s2 * d3.y));
        v[1] = a1 + b1;
        v[6] = a1 - b1;
        v[2] = a2 + b2;
        v[5] = a2 - b2;
        v[3] = a3 + b3;
        v[4] = a3 - b3;
    }
};

// Length-14 DFT as 2 x 7: n = 7 n1 + n2, k = k1 + 2 k2.
template <int S, typename T> struct Dft<14, S, T> {
    __device__ __forceinline__ static void run(cx<T> *v)
    {
        // W_14^m = cos(pi m/7) + S i sin(pi m/7), m = 1..6
        const T c[7] = {(T)1, (T)0.900968867902419126236102319507445051, (T)0.623489801858733530525004884004239811,
                        (T)0.222520933956314404288902564496794759, (T)-0.222520933956314404288902564496794759,
                        (T)-0.623489801858733530525004884004239811, (T)-0.900968867902419126236102319507445051};
        const T s[7] = {(T)0, (T)0.433883739117558120475768332848358755, (T)0.78183148246802980870844452667405775,
                        (T)0.974927912181823607018131682993931217, (T)0.974927912181823607018131682993931217,
                        (T)0.78183148246802980870844452667405775, (T)0.433883739117558120475768332848358755};
        cx<T> a[7], b[7];
#pragma unroll
        for (int n2 = 0; n2 < 7; n2++) {
            a[n2] = v[n2] + v[7 + n2];
            const cx<T> d = v[n2] - v[7 + n2];
            b[n2] = (n2 == 0) ? d : cmul(d, mk<T>(c[n2], (T)S * s[n2]));
        }
        Dft<7, S, T>::run(a);
        Dft<7, S, T>::run(b);
#pragma unroll
        for (int k2 = 0; k2 < 7; k2++) {
            v[2 * k2] = a[k2];
            v[2 * k2 + 1] = b[k2];
        }
    }
};

// ---------------------------------------------------------------------
// Line plan: length n = prod(rad[0..nst)), twiddle table tw[m] = W_n^m
// (forward sign) for m in [0, n).
// ---------------------------------------------------------------------
struct LinePlan {
    int n;
    int nst;
    int rad[10];
    const void *tw;   // cx<T>[n] on device
};

// One Stockham stage over `nlines` lines.  Element e of line l is at
// buf[l*ls + e*es].  line_fast chooses which index varies fastest across
// threads (pick the one with unit shared-memory stride).
template <int R, int S, typename T>
__device__ __forceinline__ void stockham_stage(const cx<T> *__restrict__ src, cx<T> *__restrict__ dst,
                                               int n, int Ns, int nlines, int es, int ls, bool line_fast,
                                               const cx<T> *__restrict__ tw)
{
    const int nb = n / R;
    const int total = nlines * nb;
    const int tstride = n / (Ns * R);
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
        int l, j;
        if (line_fast) { l = b % nlines; j = b / nlines; }
        else { j = b % nb; l = b / nb; }
        const cx<T> *s = src + (long)l * ls;
        cx<T> *d = dst + (long)l * ls;
        const int k = j % Ns;
        cx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = s[(j + r * nb) * es];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                cx<T> w = tw[r * k * tstride];
                if (S > 0) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        Dft<R, S, T>::run(v);
        const int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) d[(base + r * Ns) * es] = v[r];
    }
}

// Full transform of `nlines` lines, ping-ponging between a and b.  Returns
// the buffer that holds the result.  Starts and ends with __syncthreads.
template <int S, typename T>
__device__ cx<T> *fft_lines(cx<T> *a, cx<T> *b, const LinePlan &p, int nlines, int es, int ls, bool line_fast)
{
    __syncthreads();
    const cx<T> *tw = (const cx<T> *)p.tw;
    cx<T> *src = a, *dst = b;
    int Ns = 1;
    for (int st = 0; st < p.nst; st++) {
        const int R = p.rad[st];
        switch (R) {
        case 8: stockham_stage<8, S, T>(src, dst, p.n, Ns, nlines, es, ls, line_fast, tw); break;
        case 4: stockham_stage<4, S, T>(src, dst, p.n, Ns, nlines, es, ls, line_fast, tw); break;
        case 2: stockham_stage<2, S, T>(src, dst, p.n, Ns, nlines, es, ls, line_fast, tw); break;
        case 3: stockham_stage<3, S, T>(src, dst, p.n, Ns, nlines, es, ls, line_fast, tw); break;
        case 5: stockham_stage<5, S, T>(src, dst, p.n, Ns, nlines, es, ls, line_fast, tw); break;
        case 7: stockham_stage<7, S, T>(src, dst, p.n, Ns, nlines, es, ls, line_fast, tw); break;
        default: break;
        }
        Ns *= R;
        __syncthreads();
        cx<T> *t = src; src = dst; dst = t;
    }
    return src;
}

// ---------------------------------------------------------------------
// Plane geometry shared by all step kernels of one grid shape.
// A "plane" is the x-y plane (the whole grid for dim <= 2).  Its spectrum
// is stored as n2 rows of LS complex values, LS = n1/2+1 (n1 even) or n1
// (n1 odd, full-length rows).
// ---------------------------------------------------------------------
struct PlaneGeom {
    int n1, n2, n3;
    int n1h;          // n1/2 + 1
    int LS;           // row stride of spectral plane buffers (complex units)
    int even;         // n1 even -> packed real rows
    LinePlan row;     // length n1/2 (even) or n1 (odd)
    LinePlan col;     // length n2
    LinePlan zp;      // length n3
    const void *rtw;  // W_{n1}^k, k in [0, n1): untangling twiddles (cx<T>)
};

// Load eo*q for a real plane (n1 x n2, x fastest) into buffer P as packed
// rows.  `src` and `eo` may be shared or global.  Returns nothing; caller syncs.
template <typename T, typename F>
__device__ __forceinline__ void pack_rows(cx<T> *P, const PlaneGeom &g, F value)
{
    if (g.even) {
        const int M = g.n1 / 2;
        for (int i = threadIdx.x; i < M * g.n2; i += blockDim.x) {
            int y = i / M, m = i - y * M;
            int r0 = y * g.n1 + 2 * m;
            P[y * g.LS + m] = mk<T>(value(r0), value(r0 + 1));
        }
    } else {
        for (int i = threadIdx.x; i < g.n1 * g.n2; i += blockDim.x) {
            int y = i / g.n1, x = i - y * g.n1;
            P[y * g.LS + x] = mk<T>(value(i), (T)0);
        }
    }
}

// Row spectrum Z of packed rows -> r2c row spectrum X[0..n1/2] (even n1).
template <typename T>
__device__ __forceinline__ void untangle_rows(const cx<T> *Z, cx<T> *X, const PlaneGeom &g)
{
    const cx<T> *W = (const cx<T> *)g.rtw;
    if (g.even) {
        const int M = g.n1 / 2;
        const int nh = M + 1;
        for (int i = threadIdx.x; i < nh * g.n2; i += blockDim.x) {
            int y = i / nh, k = i - y * nh;
            cx<T> zk = Z[y * g.LS + (k == M ? 0 : k)];
            cx<T> zc = conjg(Z[y * g.LS + (k == 0 ? 0 : M - k)]);
            cx<T> e = scale(zk + zc, (T)0.5);
            cx<T> o = scale(mul_si<-1>(zk - zc), (T)0.5);   // (zk - zc)/(2i)
            X[y * g.LS + k] = e + cmul(W[k], o);
        }
    } else {
        // full-length complex rows: spectrum is already X; nothing to do but copy
        for (int i = threadIdx.x; i < g.LS * g.n2; i += blockDim.x) X[i] = Z[i];
    }
}

// r2c row spectrum X[0..n1/2] -> packed complex input Z of the inverse
// half-length FFT (even n1), or a full Hermitian row (odd n1).
template <typename T>
__device__ __forceinline__ void tangle_rows(const cx<T> *X, cx<T> *Z, const PlaneGeom &g)
{
    const cx<T> *W = (const cx<T> *)g.rtw;
    if (g.even) {
        const int M = g.n1 / 2;
        for (int i = threadIdx.x; i < M * g.n2; i += blockDim.x) {
            int y = i / M, k = i - y * M;
            cx<T> xk = X[y * g.LS + k];
            cx<T> xc = conjg(X[y * g.LS + M - k]);
            cx<T> w = conjg(W[k]);                       // W_n1^{-k}
            Z[y * g.LS + k] = (xk + xc) + mul_si<1>(cmul(w, xk - xc));
        }
    } else {
        const int n1 = g.n1, nh = g.n1h;
        for (int i = threadIdx.x; i < n1 * g.n2; i += blockDim.x) {
            int y = i / n1, k = i - y * n1;
            Z[y * g.LS + k] = (k < nh) ? X[y * g.LS + k] : conjg(X[y * g.LS + (n1 - k)]);
        }
    }
}

// Forward 2-D r2c of packed rows held in P (Q is scratch).  Returns the
// buffer holding the spectral plane [n2][LS].
template <typename T>
__device__ cx<T> *plane_forward(cx<T> *P, cx<T> *Q, const PlaneGeom &g)
{
    cx<T> *r = fft_lines<-1, T>(P, Q, g.row, g.n2, 1, g.LS, false);
    cx<T> *o = (r == P) ? Q : P;
    untangle_rows<T>(r, o, g);
    if (g.n2 > 1) return fft_lines<-1, T>(o, r, g.col, g.n1h, g.LS, 1, true);
    __syncthreads();
    return o;
}

// Inverse 2-D of a spectral plane held in S (Q scratch).  Returns the
// buffer holding packed rows z[m] = y[2m] + i y[2m+1] (even n1) or
// z[m] = y[m] + i*(junk) (odd n1), y the unnormalised c2r output.
template <typename T>
__device__ cx<T> *plane_inverse(cx<T> *S, cx<T> *Q, const PlaneGeom &g)
{
    cx<T> *r = S;
    if (g.n2 > 1) r = fft_lines<1, T>(S, Q, g.col, g.n1h, g.LS, 1, true);
    else __syncthreads();
    cx<T> *o = (r == S) ? Q : S;
    tangle_rows<T>(r, o, g);
    return fft_lines<1, T>(o, r, g.row, g.n2, 1, g.LS, false);
}

// Real value at plane index i (x fastest) from the packed inverse output.
template <typename T>
__device__ __forceinline__ T unpack_real(const cx<T> *Z, const PlaneGeom &g, int i)
{
    if (g.even) {
        int y = i / g.n1, x = i - y * g.n1;
        cx<T> z = Z[y * g.LS + (x >> 1)];
        return (x & 1) ? z.y : z.x;
    } else {
        int y = i / g.n1, x = i - y * g.n1;
        return Z[y * g.LS + x].x;
    }
}

}  // namespace pscfg
