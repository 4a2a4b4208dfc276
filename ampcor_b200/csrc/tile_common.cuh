// Device helpers shared by the FP32 kernels of the plain and spectral forms (512-thread CTAs):
// amplitudes, fixed-order block reductions, the reference's first-maximum order and the FP64
// placement statistics.
#pragma once

#include "kernels.cuh"

#include <limits.h>
#include <math.h>

namespace ampcor_b200 {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// |z| as the reference CPU path computes it (float std::abs of complex<float>): the FP64
// square root of the exactly formed FP64 sum of squares, rounded to float
__device__ __forceinline__ float amp_of(float2 z)
{
    const double re = z.x, im = z.y;
    return (float)sqrt(re * re + im * im);
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// block-wide FP64 sum in a fixed order; every thread gets the same value
__device__ double block_sum(double v, double* red)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) s += red[w];
    __syncthreads();
    return s;
}

// (value, index) order of the reference argmax (maxcor.cu:114-126): the first cell, in row-major
// order, holding the largest value
__device__ __forceinline__ void better(float& bv, int& bi, float v, int i)
{
    if (v > bv || (v == bv && i < bi)) {
        bv = v;
        bi = i;
    }
}

__device__ void block_argmax(float& bv, int& bi, float* redf, int* redi)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(kFull, bv, o);
        const int oi = __shfl_xor_sync(kFull, bi, o);
        better(bv, bi, ov, oi);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        redf[warp] = bv;
        redi[warp] = bi;
    }
    __syncthreads();
    bv = redf[0];
    bi = redi[0];
    for (int w = 1; w < kWarps; ++w) better(bv, bi, redf[w], redi[w]);
    __syncthreads();
}

template <int NT>
__device__ void block_argmax_n(float& bv, int& bi, float* redf, int* redi)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(kFull, bv, o);
        const int oi = __shfl_xor_sync(kFull, bi, o);
        better(bv, bi, ov, oi);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        redf[warp] = bv;
        redi[warp] = bi;
    }
    __syncthreads();
    bv = redf[0];
    bi = redi[0];
    for (int w = 1; w < NT / 32; ++w) better(bv, bi, redf[w], redi[w]);
    __syncthreads();
}

// exclusive prefix sum of row[0..n) written in place, with the total in row[n] (one warp)
__device__ void warp_prefix(double* row, int n)
{
    const int lane = threadIdx.x & 31;
    const int per = (n + 31) / 32;
    const int beg = min(lane * per, n), end = min(beg + per, n);
    double local = 0.0;
    for (int k = beg; k < end; ++k) local += row[k];
    double incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    double run = __shfl_up_sync(kFull, incl, 1);
    if (lane == 0) run = 0.0;
    for (int k = beg; k < end; ++k) {
        const double v = row[k];
        row[k] = run;
        run += v;
    }
    if (end == n && beg < n) row[n] = run;
}

// 1/sqrt(sum_box t^2 - (sum_box t)^2 / R^2) for every placement, 0 for a flat box.
// FP64 column sums slide down the window; each chunk of kStatRows placement rows is turned into
// box sums by a prefix sum along the row (the FP64 summed-area table of tgtStats.cu:139-162 and
// sat.cu:81-149, evaluated in slices so that it fits beside the tiles).
// (XS: the column stride of the window in floats; S: its row stride)
template <int XS>
__device__ void window_stats_xs(const float* win, int S, int W, int R, int C, int SR, float* inv,
                                double* vbuf)
{
    const int tid = threadIdx.x, warp = tid >> 5;
    double* V1 = vbuf;
    double* V2 = vbuf + SR * (W + 1);
    double s1 = 0.0, s2 = 0.0;
    if (tid < W) {
        for (int i = 0; i < R; ++i) {
            const double t = win[i * S + tid * XS];
            s1 += t;
            s2 += t * t;
        }
    }
    const double cells = (double)R * (double)R;
    for (int u0 = 0; u0 < C; u0 += SR) {
        const int nrows = min(SR, C - u0);
        if (tid < W) {
            for (int r = 0; r < nrows; ++r) {
                const int u = u0 + r;
                V1[r * (W + 1) + tid] = s1;
                V2[r * (W + 1) + tid] = s2;
                if (u + 1 < C) {
                    const double a = win[(u + R) * S + tid * XS], b = win[u * S + tid * XS];
                    s1 += a - b;
                    s2 += a * a - b * b;
                }
            }
        }
        __syncthreads();
        if (warp < nrows) {
            warp_prefix(V1 + warp * (W + 1), W);
            warp_prefix(V2 + warp * (W + 1), W);
        }
        __syncthreads();
        for (int idx = tid; idx < nrows * C; idx += kThreads) {
            const int r = idx / C, v = idx - r * C;
            const double* p1 = V1 + r * (W + 1);
            const double* p2 = V2 + r * (W + 1);
            const double b1 = p1[v + R] - p1[v];
            const double b2 = p2[v + R] - p2[v];
            const double var = b2 - b1 * b1 / cells;
            inv[(u0 + r) * C + v] = var > 0.0 ? (float)(1.0 / sqrt(var)) : 0.0f;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void window_stats(const float* win, const NccGeom& g, float* inv,
                                             double* vbuf)
{
    window_stats_xs<1>(win, g.S, g.W, g.R, g.C, g.stat_rows, inv, vbuf);
}

}  // namespace

// Removes the linear phase ramp of an n x n complex tile in shared memory (rows `stride` samples
// apart) before it is interpolated: phi_s = arg sum z(y, x + 1) conj z(y, x) and
// phi_l = arg sum z(y + 1, x) conj z(y, x) (lag-one autocorrelations along samples and lines,
// whose phases are the ramp's steps), then z(y, x) *= exp(-i (phi_s x + phi_l y)).  A Doppler
// ramp moves the tile's spectrum off baseband, where the zero padding of a band-limited
// interpolation would cut through it.  One block of kThreads threads; red holds 4 kWarps
// doubles; ends with a barrier.
__device__ inline void deramp_tile(float2* t, int stride, int n, double* red)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float sr = 0.0f, si = 0.0f, lr = 0.0f, li = 0.0f;
    for (int k = tid; k < n * n; k += kThreads) {
        const int y = k / n, x = k - y * n;
        const float2 z = t[y * stride + x];
        if (x + 1 < n) {
            const float2 w = t[y * stride + x + 1];
            sr = fmaf(w.x, z.x, fmaf(w.y, z.y, sr));
            si = fmaf(w.y, z.x, fmaf(-w.x, z.y, si));
        }
        if (y + 1 < n) {
            const float2 w = t[(y + 1) * stride + x];
            lr = fmaf(w.x, z.x, fmaf(w.y, z.y, lr));
            li = fmaf(w.y, z.x, fmaf(-w.x, z.y, li));
        }
    }
    double v[4] = {sr, si, lr, li};
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) red[4 * warp + k] = v[k];
    __syncthreads();
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (int w = 0; w < kWarps; ++w)
#pragma unroll
        for (int k = 0; k < 4; ++k) a[k] += red[4 * w + k];
    const float ps = (float)atan2(a[1], a[0]), pl = (float)atan2(a[3], a[2]);
    __syncthreads();
    for (int k = tid; k < n * n; k += kThreads) {
        const int y = k / n, x = k - y * n;
        float s, c;
        sincosf(fmaf(ps, (float)x, pl * (float)y), &s, &c);
        const float2 z = t[y * stride + x];
        t[y * stride + x] = make_float2(fmaf(z.x, c, z.y * s), fmaf(z.y, c, -z.x * s));
    }
    __syncthreads();
}

// The mean of an n x n complex tile (rows `stride` apart; in shared memory, or in global memory
// when GLOBAL), with the linear phase ramp (ps, pl) of deramp_tile taken off each sample first
// when DERAMP.  Band-limited upsampling keeps a constant as it is, so a caller that takes the
// mean off the tile before its transforms and adds it back to every output gets the same
// interpolation, with the transforms rounding on the tile's variation instead of on a strong
// steady return.  FP32 sums per thread, FP64 across the block.  red: 2 kWarps doubles; ends with
// a barrier.
template <bool GLOBAL, bool DERAMP>
__device__ inline float2 tile_mean(const float2* t, long long stride, int n, float ps, float pl, double* red)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float sx = 0.0f, sy = 0.0f;
    for (int k = tid; k < n * n; k += kThreads) {
        const int y = k / n, x = k - y * n;
        float2 z = GLOBAL ? __ldg(t + y * stride + x) : t[y * stride + x];
        if (DERAMP) {
            float s, c;
            sincosf(fmaf(ps, (float)x, pl * (float)y), &s, &c);
            z = make_float2(fmaf(z.x, c, z.y * s), fmaf(z.y, c, -z.x * s));
        }
        sx += z.x;
        sy += z.y;
    }
    double a = warp_sum((double)sx), b = warp_sum((double)sy);
    if (lane == 0) {
        red[2 * warp] = a;
        red[2 * warp + 1] = b;
    }
    __syncthreads();
    a = 0.0;
    b = 0.0;
    for (int w = 0; w < kWarps; ++w) {
        a += red[2 * w];
        b += red[2 * w + 1];
    }
    __syncthreads();
    const double cells = (double)n * (double)n;
    return make_float2((float)(a / cells), (float)(b / cells));
}

}  // namespace ampcor_b200
