// kernels3l.cuh -- 3-D MDE step as line passes, for any grid shape with an
// even n1 and 2,3,5,7-smooth extents.
//
// The whole-plane kernels (kernels.cuh k3_*) keep an n2 x (n1/2+1) spectral
// plane and its ping-pong copy in shared memory, which for large planes
// (64 x 128: 135 KB) leaves one CTA per SM.  Here every kernel works on a
// few lines only:
//   k3l_rows   x transforms of TL rows (real <-> half spectrum through the
//              packed half-length complex FFT), with the step's pointwise
//              work fused in (exp(-w ds/2) q, q1, h and its forward, the
//              Richardson combination);
//   k3l_lines  complex transforms of TL lines of the half spectrum along y
//              or z; along z the k-space filter is applied between the
//              forward and the inverse transform.
// One step (src/step_mod.f90:146-176) is nine launches:
//   rows fwd (E1 q -> S1, E2 q -> S2) | y fwd | z conv (ek1, ek2) | y inv |
//   rows mid (q1; h -> S2) | y fwd | z conv (ek2) | y inv | rows final.
// Spectra are stored [z][y][kx] in natural order, unnormalised; 1/N is
// applied in the row inverses.  Same SweepField contract as the other step
// kernels (in/out overrides, q1, h_out, q2_out).
#pragma once
#include "kernels.cuh"

namespace pscfg {

static constexpr int L3_THREADS = 128;

// rows per CTA so that the two row buffers take about 32 KB
template <typename T>
__host__ __device__ inline int l3_rows_per_cta(int M)
{
    const int tl = (int)(32768 / (2 * (M + 1) * (int)sizeof(cx<T>)));
    return tl < 1 ? 1 : (tl > 64 ? 64 : tl);
}

// MODE 0: forward of exp(-w ds/2) q (blockIdx.z = 0 -> S1) and
//         exp(-w ds/4) q (blockIdx.z = 1 -> S2);
// MODE 1: blockIdx.z = 0: inverse of S1 -> q1 = E1 x / N;
//         blockIdx.z = 1: inverse of S2 -> h = E1 x / N (h_out), forward of h -> S2;
// MODE 2: inverse of S2 -> q2 = E2 x / N, q_out = (4 q2 - q1) / 3 (q2_out).
// grid = (ceil(n2 n3 / TL), nfields, 2 or 1); dynamic smem
// 2 * TL * (n1/2 + 1) complex.
template <typename T, int MODE>
__global__ void __launch_bounds__(L3_THREADS) k3l_rows(const SweepField<T> *fields, PlaneGeom g, int t, int TL)
{
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    const int n1 = g.n1, M = n1 / 2, NH = M + 1;
    const long nrow = (long)g.n2 * g.n3, nr = nrow * n1;
    const long r0 = (long)blockIdx.x * TL;
    const int nl = (int)min((long)TL, nrow - r0);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *a = (cx<T> *)smem_raw;
    cx<T> *b = a + (long)TL * NH;
    const cx<T> *W = (const cx<T> *)g.rtw;
    const T rn = (T)nr;
    const int z = (MODE == 2) ? 0 : (int)blockIdx.z;
    cx<T> *S = (MODE == 0) ? (z == 0 ? f.S1 : f.S2) : (MODE == 1 ? (z == 0 ? f.S1 : f.S2) : f.S2);
    const long soff = r0 * NH, roff = r0 * n1;

    // forward x transform of the packed rows in buffer p (line-major,
    // stride M) into S rows: FFT, untangle, store
    auto forward = [&](cx<T> *p, cx<T> *q) {
        cx<T> *res = fft_lines<-1, T>(p, q, g.row, nl, 1, M, false);
        for (int i = threadIdx.x; i < nl * NH; i += blockDim.x) {
            const int li = i / NH, k = i % NH;
            const cx<T> zk = res[li * M + (k % M)], zm = conjg(res[li * M + ((M - k) % M)]);
            S[soff + (long)li * NH + k] = scale((zk + zm) + mul_si<-1>(cmul(W[k], zk - zm)), (T)0.5);
        }
        __syncthreads();
    };
    // inverse: S rows -> tangle into q -> inverse FFT; returns the buffer of
    // the packed real rows (unnormalised)
    auto inverse = [&](cx<T> *p, cx<T> *q) -> cx<T> * {
        for (int i = threadIdx.x; i < nl * NH; i += blockDim.x) p[i] = S[soff + i];
        __syncthreads();
        for (int i = threadIdx.x; i < nl * M; i += blockDim.x) {
            const int li = i / M, k = i % M;
            const cx<T> xk = p[li * NH + k], xm = conjg(p[li * NH + M - k]);
            q[li * M + k] = (xk + xm) + mul_si<1>(cmul(conjg(W[k]), xk - xm));
        }
        return fft_lines<1, T>(q, p, g.row, nl, 1, M, false);
    };

    if (MODE == 0) {
        const T *qs = src_slice(f, src, nr) + roff;
        const T *eo = (z == 0 ? f.eo1[blk] : f.eo2[blk]) + roff;
        for (int i = threadIdx.x; i < nl * M; i += blockDim.x) {
            const int e = 2 * i;   // rows are contiguous: packed entry i holds e, e+1
            a[i] = mk<T>(eo[e] * qs[e], eo[e + 1] * qs[e + 1]);
        }
        forward(a, b);
    } else if (MODE == 1) {
        const T *eo1 = f.eo1[blk] + roff;
        cx<T> *x = inverse(a, b);
        if (z == 0) {
            T *q1 = f.q1 + roff;
            for (int i = threadIdx.x; i < nl * M; i += blockDim.x) {
                const int e = 2 * i;
                q1[e] = eo1[e] * x[i].x / rn;
                q1[e + 1] = eo1[e + 1] * x[i].y / rn;
            }
        } else {
            T *hg = f.h_out ? f.h_out + roff : nullptr;
            for (int i = threadIdx.x; i < nl * M; i += blockDim.x) {
                const int e = 2 * i;
                const cx<T> v = mk<T>(eo1[e] * x[i].x / rn, eo1[e + 1] * x[i].y / rn);
                x[i] = v;
                if (hg) {
                    hg[e] = v.x;
                    hg[e + 1] = v.y;
                }
            }
            forward(x, x == a ? b : a);
        }
    } else {
        const T *eo2 = f.eo2[blk] + roff;
        const T *q1 = f.q1 + roff;
        T *out = dst_slice(f, dst, nr) + roff;
        T *q2o = f.q2_out ? f.q2_out + roff : nullptr;
        cx<T> *x = inverse(a, b);
        for (int i = threadIdx.x; i < nl * M; i += blockDim.x) {
            const int e = 2 * i;
            const T q2a = eo2[e] * x[i].x / rn, q2b = eo2[e + 1] * x[i].y / rn;
            out[e] = ((T)4 * q2a - q1[e]) / (T)3;
            out[e + 1] = ((T)4 * q2b - q1[e + 1]) / (T)3;
            if (q2o) {
                q2o[e] = q2a;
                q2o[e + 1] = q2b;
            }
        }
    }
}

// Lines of the half spectrum (row length NH = n1/2+1): axis 1 = y (stride
// NH, lines (kx, z)), axis 2 = z (stride NH n2, lines (kx, y)).  op 0
// forward, 1 inverse, 2 forward, times ek, inverse.  which: 1 = S1/ek1,
// 2 = S2/ek2, 3 = both (blockIdx.z selects).  grid = (ceil(nlines / TL),
// nfields, 1 or 2); dynamic smem 2 * TL * L complex.
template <typename T>
__global__ void __launch_bounds__(L3_THREADS) k3l_lines(const SweepField<T> *fields, PlaneGeom g, int t, int axis,
                                                        int op, int which, int TL)
{
    const SweepField<T> &f = fields[blockIdx.y];
    int blk, src, dst;
    if (!step_slices(f, t, blk, src, dst)) return;
    const int NH = g.n1 / 2 + 1;
    const int L = axis == 1 ? g.n2 : g.n3;
    const long nlines = axis == 1 ? (long)NH * g.n3 : (long)NH * g.n2;
    const long es = axis == 1 ? NH : (long)NH * g.n2;
    const LinePlan &plan = axis == 1 ? g.col : g.zp;
    const int sel = which == 3 ? (int)blockIdx.z + 1 : which;
    cx<T> *S = sel == 1 ? f.S1 : f.S2;
    const T *ek = sel == 1 ? f.ek1[blk] : f.ek2[blk];
    const long l0 = (long)blockIdx.x * TL;
    const int nl = (int)min((long)TL, nlines - l0);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T> *a = (cx<T> *)smem_raw;
    cx<T> *b = a + (long)TL * L;
    // element-major: consecutive threads take consecutive lines (kx)
    auto base = [&](long l) -> long {
        return axis == 1 ? (l % NH) + (l / NH) * (long)NH * g.n2 : l;
    };
    const int tot = nl * L;
    for (int i = threadIdx.x; i < tot; i += blockDim.x) {
        const int li = i % nl, e = i / nl;
        a[e * TL + li] = S[base(l0 + li) + e * es];
    }
    cx<T> *res = a;
    if (op != 1) res = fft_lines<-1, T>(a, b, plan, nl, TL, 1, true);
    if (op == 2) {
        for (int i = threadIdx.x; i < tot; i += blockDim.x) {
            const int li = i % nl, e = i / nl;
            const T k = ek[base(l0 + li) + e * es];
            cx<T> &v = res[e * TL + li];
            v = mk<T>(k * v.x, k * v.y);
        }
    }
    if (op != 0) res = fft_lines<1, T>(res, res == a ? b : a, plan, nl, TL, 1, true);
    __syncthreads();
    for (int i = threadIdx.x; i < tot; i += blockDim.x) {
        const int li = i % nl, e = i / nl;
        S[base(l0 + li) + e * es] = res[e * TL + li];
    }
}

}  // namespace pscfg
