// sm_100a kernels of the spectral correlation form.
//
// The numerator surface of a tile pair, sum_ij r'(i, j) t(u + i, v + j) over every placement, is
// a 2-D correlation; the reference evaluates it as a direct sum (correlate.cu:69-135), which costs
// C^2 R^2 multiply-adds per pair.  Here one CTA per pair does it with FFTs in shared memory:
// the window t (real parts) and the zero-mean chip r' (imaginary parts) share one N x N complex
// tile (N >= W, so no placement wraps around), one forward 2-D transform gives both spectra, their
// product T conj(R) is formed in place and one inverse transform (pruned to the C placement rows)
// returns the numerators.  About 20x fewer operations than the direct sum at the production
// geometry (64^2 chips, 128^2 windows).
//
// Around it: the amplitudes of each raster are detected once (detect_kernel; neighbouring
// windows overlap, so every sample is shared by many pairs) and the correlation kernel takes float
// amplitudes through asynchronous copies.  The placement statistics (1/sigma of every window box)
// come from the window while it sits in shared memory (spec_box_stats), or, for the coarse stage
// of windows that tile a raster, from FP64 sums over the whole raster (box_vsum_kernel,
// box_inv_kernel).
//
// Accuracy.  The window is centred on its mean before the transform (sum r' = 0, so the
// numerators keep their value) and the twiddles are correctly rounded, which keeps the transform
// error of a normalised correlation near 1e-7; the plain form's FP32 direct sums land in the same
// range.  Where a nearly flat box would magnify the transform error, the numerator is recomputed
// as a direct sum (spec_surface).
#include <algorithm>

#include <cuda.h>

#include "fft.cuh"
#include "kernels.cuh"
#include "tcgen05.cuh"
#include "tile_common.cuh"

namespace ampcor_b200 {

namespace {

struct BlockSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

__device__ __forceinline__ void cp_async4(void* dst, const void* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async8_g(void* dst, const void* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}

// two block-wide FP64 sums in a fixed order (one pair of barriers) over a CTA of NW warps; every
// thread gets both; red holds 2 NW doubles
template <int NW>
__device__ void block_sum2(double& a, double& b, double* red)
{
    a = warp_sum(a);
    b = warp_sum(b);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        red[2 * warp] = a;
        red[2 * warp + 1] = b;
    }
    __syncthreads();
    a = 0.0;
    b = 0.0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        a += red[2 * w];
        b += red[2 * w + 1];
    }
    __syncthreads();
}

// one warp: the positions of fft::half_positions (one member of every Hermitian pair of the
// permuted spectrum, increasing), 32 candidates per ballot
template <int N1, int N2>
__device__ void build_half(int* half)
{
    constexpr int N = N1 * N2;
    const int lane = threadIdx.x & 31;
    int base = 0;
    for (int p0 = 0; p0 < N; p0 += 32) {
        const int p = p0 + lane;
        const bool in = p < N && fft::in_half<N1, N2>(p);
        const unsigned m = __ballot_sync(0xffffffffu, in);
        if (in) half[base + __popc(m & ((1u << lane) - 1u))] = p;
        base += __popc(m);
    }
}

__device__ __forceinline__ const float* spec_chip(const SpecSource& s, long long pair0, int b)
{
    return s.chip + (s.chip_off ? s.chip_off[pair0 + b] : (long long)b * s.chip_step);
}

__device__ __forceinline__ const float* spec_win(const SpecSource& s, long long pair0, int b)
{
    return s.win + (s.win_off ? s.win_off[pair0 + b] : (long long)b * s.win_step);
}

// The transform's error on a numerator is a small multiple of eps |r'| |t'| (|.|: Euclidean norms
// of the zero-mean chip and the centred window; below 1.4e-7 |r'| |t'| over the compiled lengths
// in host runs against FP64 sums), so its error on gamma is bounded by kSpecErr |t'| / sigma_box.
// Where a box is nearly flat that bound grows; a placement whose bound exceeds kSpecTol (half the
// 2e-5 surface tolerance the parity tests hold every form to) has its numerator recomputed as a
// direct FP32 sum whenever its value matters (it could be the maximum, or the surface is
// returned).  On speckle the bound is about kSpecErr W / R (|t'| / sigma_box is about W / R, the
// chip blocks of a blocked stage add theirs), 5e-6 for a 32 px chip in a +-64 px search
// (W / R = 5), while the errors measured there stay below 3e-7; zero-padded or masked windows
// exceed it.
constexpr float kSpecErr = 1e-6f;
constexpr float kSpecTol = 1e-5f;

// Scratch of the placement statistics: slot k is z[st k] for k below nz (the imaginary parts of
// the tile while the chip waits in registers, st = 2; or a free stretch of the tile, st = 1), and
// past them it continues in the tail buffer.
struct StatSlots {
    float* z;  // slot 0
    float* tail;
    int nz;
    int st;    // slot stride (floats)
    __device__ __forceinline__ float* at(int k) const { return k < nz ? z + st * k : tail + (k - nz); }
};

__device__ __forceinline__ float box_inv_of(double b1, double b2, double rcells)
{
    const float var = (float)(b2 - b1 * b1 * rcells);
    return var > 0.0f ? __frsqrt_rn(var) : 0.0f;
}

// 1/sigma_box of every placement from the window (win(y, x): the tile's real parts, or a staged
// copy of the window), the values shifted by sx (the window mean: the box variance does not
// change and the column sums keep their digits).  sigma^2 = S2 - S1^2 / R^2 over the R x R box, its sum of squared deviations
// from its mean: the target variance of correlate.cu:196-309, whose box mean comes from the
// summed-area table (tgtStats.cu).
//
// Column sums V(u, x) over window rows [u, u + R), nseg threads per column: thread s sums band s
// of the first placement's rows (FP32 runs of 8 rows added in FP64) and the slides
// delta(i) = t(i + R) - t(i) of its share of the placement rows (FP32: a slide is small next to a
// column sum); after one exchange (part, FP64) each thread starts its share at V(0) plus the
// earlier shares' slides (as a float pair) and adds the FP32 sum of its own slides so far, and
// writes V(u, x) of its rows as floats into the slots (V1 at slot u W + x, V2 at C W + u W + x).
// Then one warp per placement row (three rows at a time) forms the box sums
// S(v) = sum_{x in [v, v + R)} V(x): S(0) as an FP64 warp sum, the others as S(0) plus an FP32 scan
// of V(v + R) - V(v) across the lanes.  The phases are bound by instruction issue, so the FP64
// work and the float-double conversions are kept to a few per column.  Ends with a barrier.
template <int NT, class Win>
__device__ void spec_box_stats(Win win, const SpecGeom& g, float sx, StatSlots vs, double* part,
                               float* invs)
{
    const int R = g.R, W = g.W, C = g.C, nseg = g.nseg, D = C - 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int x = tid % W, s = tid / W;
    auto tv = [&](int y) { return win(y, x) - sx; };
    constexpr int kRun = 8;
    if (s < nseg) {
        double b1 = 0.0, b2 = 0.0;
        const int ya = s * R / nseg, yb = (s + 1) * R / nseg;
        for (int y0 = ya; y0 < yb; y0 += kRun) {
            float r1 = 0.0f, r2 = 0.0f;
#pragma unroll
            for (int k = 0; k < kRun; ++k)
                if (y0 + k < yb) {
                    const float t = tv(y0 + k);
                    r1 += t;
                    r2 = fmaf(t, t, r2);
                }
            b1 += (double)r1;
            b2 += (double)r2;
        }
        float e1 = 0.0f, e2 = 0.0f;
        constexpr int kA = 4;  // window rows read ahead of the sums
        for (int i0 = s * D / nseg, i1 = (s + 1) * D / nseg; i0 < i1; i0 += kA) {
            float a[kA], b[kA];
#pragma unroll
            for (int k = 0; k < kA; ++k) {
                const int i = min(i0 + k, i1 - 1);
                a[k] = win(i + R, x);
                b[k] = win(i, x);
            }
#pragma unroll
            for (int k = 0; k < kA; ++k)
                if (i0 + k < i1) {
                    const float d = a[k] - b[k];
                    e1 += d;
                    e2 = fmaf(d, (a[k] + b[k]) - 2.0f * sx, e2);
                }
        }
        part[(0 * nseg + s) * W + x] = b1;
        part[(1 * nseg + s) * W + x] = b2;
        part[(2 * nseg + s) * W + x] = (double)e1;
        part[(3 * nseg + s) * W + x] = (double)e2;
    }
    __syncthreads();
    if (s < nseg) {
        double v1 = 0.0, v2 = 0.0;
        for (int q = 0; q < nseg; ++q) {
            v1 += part[(0 * nseg + q) * W + x];
            v2 += part[(1 * nseg + q) * W + x];
        }
        for (int q = 0; q < s; ++q) {
            v1 += part[(2 * nseg + q) * W + x];
            v2 += part[(3 * nseg + q) * W + x];
        }
        // V(u) = V(start) + P(u), P the FP32 sum of this share's slides so far (small next to
        // V); V(start) as a float pair
        const float h1 = (float)v1, l1 = (float)(v1 - (double)h1);
        const float h2 = (float)v2, l2 = (float)(v2 - (double)h2);
        float p1 = 0.0f, p2 = 0.0f;
        const int i1 = (s + 1) * D / nseg;
        constexpr int kB = 4;  // window rows read ahead of the running sums
        for (int i0 = s * D / nseg; i0 < i1; i0 += kB) {
            float a[kB], b[kB];
#pragma unroll
            for (int k = 0; k < kB; ++k) {
                const int i = min(i0 + k, i1 - 1);
                a[k] = win(i + R, x);
                b[k] = win(i, x);
            }
#pragma unroll
            for (int k = 0; k < kB; ++k)
                if (i0 + k < i1) {
                    *vs.at((i0 + k) * W + x) = h1 + (l1 + p1);
                    *vs.at((C + i0 + k) * W + x) = h2 + (l2 + p2);
                    const float d = a[k] - b[k];
                    p1 += d;
                    p2 = fmaf(d, (a[k] + b[k]) - 2.0f * sx, p2);
                }
        }
        if (s == nseg - 1) {
            *vs.at(D * W + x) = h1 + (l1 + p1);
            *vs.at((C + D) * W + x) = h2 + (l2 + p2);
        }
    }
    __syncthreads();
    const double rcells = 1.0 / ((double)R * (double)R);
    // KR placement rows per warp at a time, u0, u0 + NW, ...; rows past the end repeat row C - 1
    // (not stored), so that every warp runs one pass for C <= KR NW
    constexpr int NW = NT / 32, KR = 3;
    for (int u0 = warp; u0 < C; u0 += KR * NW) {
        int uu[KR];
        bool keep[KR];
#pragma unroll
        for (int r = 0; r < KR; ++r) {
            uu[r] = min(u0 + r * NW, C - 1);
            keep[r] = u0 + r * NW < C;
        }
        double s1[KR], s2[KR];
#pragma unroll
        for (int r = 0; r < KR; ++r) {
            float f1 = 0.0f, f2 = 0.0f;
            for (int c = lane; c < R; c += 32) {
                f1 += *vs.at(uu[r] * W + c);
                f2 += *vs.at((C + uu[r]) * W + c);
            }
            s1[r] = (double)f1;
            s2[r] = (double)f2;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int r = 0; r < KR; ++r) {
                s1[r] += __shfl_xor_sync(kFull, s1[r], o);
                s2[r] += __shfl_xor_sync(kFull, s2[r], o);
            }
        if (lane == 0)
#pragma unroll
            for (int r = 0; r < KR; ++r)
                if (keep[r]) invs[uu[r] * C] = box_inv_of(s1[r], s2[r], rcells);
        for (int j0 = 0; j0 < D; j0 += 32) {
            const int j = j0 + lane;
            float i1[KR], i2[KR];
#pragma unroll
            for (int r = 0; r < KR; ++r) {
                i1[r] = 0.0f;
                i2[r] = 0.0f;
                if (j < D) {
                    i1[r] = *vs.at(uu[r] * W + j + R) - *vs.at(uu[r] * W + j);
                    i2[r] = *vs.at((C + uu[r]) * W + j + R) - *vs.at((C + uu[r]) * W + j);
                }
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1)
#pragma unroll
                for (int r = 0; r < KR; ++r) {
                    const float y1 = __shfl_up_sync(kFull, i1[r], o);
                    const float y2 = __shfl_up_sync(kFull, i2[r], o);
                    if (lane >= o) {
                        i1[r] += y1;
                        i2[r] += y2;
                    }
                }
            if (j < D)
#pragma unroll
                for (int r = 0; r < KR; ++r)
                    if (keep[r])
                        invs[uu[r] * C + j + 1] = box_inv_of(s1[r] + (double)i1[r], s2[r] + (double)i2[r], rcells);
#pragma unroll
            for (int r = 0; r < KR; ++r) {
                s1[r] += (double)__shfl_sync(kFull, i1[r], 31);
                s2[r] += (double)__shfl_sync(kFull, i2[r], 31);
            }
        }
    }
    __syncthreads();
}

// The normalised surface G (C x C in shared memory, formed by the last transform step) -> its
// first maximum (valid in every thread) and optional copies; a CTA of NT threads, red holding
// NT / 32 floats and as many ints.  On entry every thread holds the
// maximum of the placements it formed whose transform bound is tight, and whether it formed any
// whose bound is loose (flagged); inv holds 1/sigma_box of the placements (row stride C).
template <int NT>
__device__ void spec_surface(float* G, double* red, const SpecGeom& g, const float* inv,
                             float inv_sigma, double mean_c, float ebox, const float* chip,
                             long long cs, const float* win, long long ws, float* out1, float* out2,
                             float& bv, int& bi, int flagged)
{
    const int C = g.C, R = g.R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    block_argmax_n<NT>(bv, bi, reinterpret_cast<float*>(red), reinterpret_cast<int*>(red) + NT / 32);
    if (__syncthreads_or(flagged)) {
        // direct FP32 numerators where the transform's bound is loose and the value matters: one
        // warp per placement, lanes across the chip columns
        const bool all = out1 || out2;
        float wv = -INFINITY;
        int wi = INT_MAX;
        for (int idx = warp; idx < C * C; idx += NT / 32) {
            const int u = idx / C, v = idx - u * C;
            const float inv_box = inv[idx];
            const float e = ebox * inv_box;
            if (!(e > kSpecTol) || !(all || G[idx] + e >= bv)) continue;
            // the window less the box's own mean (sum r' (t - c) = sum r' t for any constant c):
            // the FP32 sums round on the box's variation, not on its level, and an all-zero box
            // keeps a numerator of exactly zero
            float sb = 0.0f;
            for (int i = 0; i < R; ++i)
                for (int j = lane; j < R; j += 32) sb += __ldg(win + (u + i) * ws + v + j);
            const float wsh = (float)(warp_sum((double)sb) / ((double)R * (double)R));
            float acc = 0.0f;
            for (int i = 0; i < R; ++i)
                for (int j = lane; j < R; j += 32) {
                    const float rp = (float)((double)__ldg(chip + i * cs + j) - mean_c);
                    acc = fmaf(rp, __ldg(win + (u + i) * ws + v + j) - wsh, acc);
                }
            const double num = warp_sum((double)acc);
            const float gv = (float)num * inv_box * inv_sigma;
            __syncwarp();
            if (lane == 0) G[idx] = gv;
            better(wv, wi, gv, idx);
        }
        // every flagged placement that could win has its exact value now; the others stay below
        // the unflagged maximum
        better(bv, bi, wv, wi);
        block_argmax_n<NT>(bv, bi, reinterpret_cast<float*>(red), reinterpret_cast<int*>(red) + NT / 32);
    }
    if (out1 || out2) {
        for (int idx = threadIdx.x; idx < C * C; idx += NT) {
            const float gv = G[idx];
            if (out1) out1[idx] = gv;
            if (out2) out2[idx] = gv;
        }
    }
}

// the stage's result of pair p from the first maximum bv at placement bi: the coarse cell and its
// nudged refinement corners (stage 0), or the refined cell and peak (stage 1)
__device__ void spec_result(const SpecOut& out, long long p, int R, int W, int C, float bv, int bi)
{
    const int u = bi / C, v = bi - u * C;
    if (out.stage == 0) {
        // nudge.cu:107-140 (argument roles from nudge.cu:57: old = W, new = R + 2m)
        const int m = out.m;
        const int E = R + 2 * m;
        int left = v - m;
        if (left < 0) left = 0;
        if (left + E > W) left = W - E;
        int top = u - m;
        if (top < 0) top = 0;
        if (top + E > W) top = W - E;
        out.coarse[p] = CoarseOut{u, v, top, left};
        out.coarse_peak[p] = bv;
    } else {
        out.fine[p] = FineOut{u, v, bv, 0.0f};
    }
}

template <int N1, int N2>
__global__ void __launch_bounds__(kSpecThreads, 1)
spec_kernel(SpecSource src, long long pair0, long long pairs, const long long* valid, SpecGeom g,
            InvSource inv, const float2* tw_g, SpecOut out)
{
    extern __shared__ __align__(16) unsigned char ssm[];
    if (blockIdx.x >= pairs) return;
    const long long p = pair0 + blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (valid[p] < 0) {
        if (out.stage == 0 && tid == 0) {
            out.coarse[p] = CoarseOut{-1, -1, -1, -1};
            out.coarse_peak[p] = NAN;
        }
        return;
    }
    constexpr int N = N1 * N2;
    // the tile's row stride is always N + 1 (odd); as a constant every element offset of a row or
    // column walk is an immediate
    constexpr int RS = N + 1;
    const int W = g.W, R = g.R, C = g.C;
    float2* Z = reinterpret_cast<float2*>(ssm + g.off_z);
    float2* tw = reinterpret_cast<float2*>(ssm + g.off_tw);
    int* neg = reinterpret_cast<int*>(ssm + g.off_neg);
    int* half = reinterpret_cast<int*>(ssm + g.off_half);
    double* red = reinterpret_cast<double*>(ssm + g.off_red);
    float* invs = reinterpret_cast<float*>(ssm + g.off_inv);
    float* G = reinterpret_cast<float*>(ssm + g.off_gam);
    float* Zf = reinterpret_cast<float*>(Z);
    // placement statistics: given (inv.base), else computed here from the window
    const float* inv_b = !inv.base ? nullptr : inv.off ? inv.base + inv.off[p] : inv.base + (long long)blockIdx.x * C * C;
    const long long is = inv.off ? inv.stride : C;
    const float* chip = spec_chip(src, pair0, blockIdx.x);
    const float* win = spec_win(src, pair0, blockIdx.x);
    const long long cs = src.chip_stride, ws = src.win_stride;

    // The chip goes to registers (its loads in flight with the window's), the window amplitudes
    // to the real parts of the tile by 4-byte asynchronous copies, zeros to the other real parts.
    // The imaginary parts are the placement statistics' scratch until the chip is stored there.
    constexpr int JN = (N + kSpecWarps - 1) / kSpecWarps, IN = (N + 31) / 32;
    float cr[JN][IN];
#pragma unroll
    for (int j = 0; j < JN; ++j)
#pragma unroll
        for (int i = 0; i < IN; ++i) {
            const int y = warp + kSpecWarps * j, x = lane + 32 * i;
            cr[j][i] = y < R && x < R ? __ldg(chip + y * cs + x) : 0.0f;
        }
    for (int y = warp; y < N; y += kSpecWarps) {
        float* zr = Zf + 2 * y * RS;
        for (int x = lane; x < N; x += 32) {
            if (y < W && x < W)
                cp_async4(zr + 2 * x, win + y * ws + x);
            else
                zr[2 * x] = 0.0f;
        }
    }
    // given placement statistics land in shared memory with the window
    if (inv_b)
        for (int u = warp; u < C; u += kSpecWarps)
            for (int v = lane; v < C; v += 32) cp_async4(invs + u * C + v, inv_b + u * is + v);
    for (int k = tid; k < N; k += kSpecThreads) {
        tw[k] = __ldg(tw_g + k);
        neg[k] = fft::neg_pos<N1, N2>(k);
    }
    if (warp == 0) build_half<N1, N2>(half);
    cp_async_wait_all();
    __syncthreads();

    // Two sweeps of sums, each combined across the block in FP64 (refStats.cu:118-302).  The first
    // takes the chip's sum (compensated) and, about a pivot k (the window's first sample), the
    // window's sums of t - k and (t - k)^2; the second the chip's sum of squares with its FP64
    // mean off (two floats, so that r' carries the FP64 mean; r' stays in the registers): |r'|
    // exactly, where squares of the uncentred amplitudes would cancel in proportion to the squared
    // level of a strong steady return.  The window mean comes off as the first transform pass reads
    // the tile; it only conditions the transform.  |t'|^2 only scales the transform's error bound,
    // so it is taken as an upper bound: sum (t - k)^2 - (sum (t - k))^2 / W^2 plus 1e-5 sum (t - k)^2,
    // more than the FP32 rounding of the per-thread sums (at most 50 terms each, 3e-6 relative).
    double acc4[4];
    const float pk = Z[0].x;
    {
        float sw = 0.0f, sw2 = 0.0f, sc = 0.0f, cc = 0.0f;
        for (int y = warp; y < W; y += kSpecWarps) {
            const float2* zr = Z + y * RS;
            for (int x = lane; x < W; x += 32) {
                const float t = zr[x].x - pk;
                sw += t;
                sw2 = fmaf(t, t, sw2);
            }
        }
        // register slots past the chip hold zeros in every lane: skipped (warp-uniform tests)
#pragma unroll
        for (int j = 0; j < JN; ++j)
            if (warp + kSpecWarps * j < R)
#pragma unroll
                for (int i = 0; i < IN; ++i)
                    if (32 * i < R) {
                        const float yk = cr[j][i] - cc;
                        const float tk = sc + yk;
                        cc = (tk - sc) - yk;
                        sc = tk;
                    }
        acc4[0] = (double)sc - (double)cc;
        acc4[1] = sw;
        acc4[3] = sw2;
        block_sum2<kSpecWarps>(acc4[0], acc4[1], red);
    }
    const double cells_c = (double)R * (double)R, cells_w = (double)W * (double)W;
    const double mean_c = acc4[0] / cells_c;
    const double mean_w = (double)pk + acc4[1] / cells_w;
    const float mc_hi = (float)mean_c, mc_lo = (float)(mean_c - (double)mc_hi);
    const fft::Centre centre{(float)mean_w, W};
    {
        float sc2 = 0.0f;
#pragma unroll
        for (int j = 0; j < JN; ++j)
#pragma unroll
            for (int i = 0; i < IN; ++i)
                if (warp + kSpecWarps * j < R && lane + 32 * i < R) {
                    const float r = (cr[j][i] - mc_hi) - mc_lo;
                    cr[j][i] = r;
                    sc2 = fmaf(r, r, sc2);
                }
        acc4[2] = sc2;
        block_sum2<kSpecWarps>(acc4[2], acc4[3], red);
    }
    const double ss = acc4[2];
    const double st = fmax(acc4[3] - acc4[1] * acc4[1] / cells_w, 0.0) + 1e-5 * acc4[3];
    const float inv_sigma = ss > 0.0 ? (float)(1.0 / sqrt(ss)) : 0.0f;
    if (!inv_b) {
        double* part = reinterpret_cast<double*>(ssm + g.off_gam);
        const StatSlots vs{Zf + 1, reinterpret_cast<float*>(part + 4 * g.nseg * W), N * RS, 2};
        spec_box_stats<kSpecThreads>([&](int y, int x) { return Z[y * RS + x].x; }, g, centre.sx, vs,
                                     part, invs);
    }
    // the zero-mean chip into the imaginary parts, zeros around it
#pragma unroll
    for (int j = 0; j < JN; ++j)
#pragma unroll
        for (int i = 0; i < IN; ++i) {
            const int y = warp + kSpecWarps * j, x = lane + 32 * i;
            if (y < N && x < N) Zf[2 * (y * RS + x) + 1] = y < R && x < R ? cr[j][i] : 0.0f;
        }
    __syncthreads();

    // the last transform step forms gamma of every placement straight from its outputs and keeps
    // this thread's maximum of those whose transform bound is tight
    const float scale = (float)(1.0 / (4.0 * (double)N * (double)N));
    const float ebox = kSpecErr * (float)sqrt(st);
    float bv = -INFINITY;
    int bi = INT_MAX;
    int flagged = 0;
    fft::correlate_tile<N1, N2>(Z, RS, W, C, tw, neg, half, centre, tid, kSpecThreads, BlockSync{},
                                [&](int u, int v, float2 val) {
                                    if (v < C) {
                                        const int idx = u * C + v;
                                        const float inv_box = invs[idx];
                                        const float gv = val.x * scale * inv_box * inv_sigma;
                                        G[idx] = gv;
                                        if (ebox * inv_box > kSpecTol)
                                            flagged = 1;
                                        else
                                            better(bv, bi, gv, idx);
                                    }
                                });

    float* surf = out.surfaces ? out.surfaces + (size_t)p * C * C : nullptr;
    float* gam = out.stage == 1 ? out.gam + (long long)blockIdx.x * C * C : nullptr;
    spec_surface<kSpecThreads>(G, red, g, invs, inv_sigma, mean_c, ebox, chip, cs, win, ws, gam, surf, bv, bi, flagged);
    if (tid == 0) spec_result(out, p, R, W, C, bv, bi);
}

// ------------------------------------------------------------------------------------------
// staged spectral correlation: one resident CTA per SM walks the pairs of a chunk
// ------------------------------------------------------------------------------------------
//
// spec_kernel holds one CTA per SM (its tile fills the shared memory), so nothing hides the wait
// for its tiles or the two sweeps of block sums that precede the transform; clock stamps put them
// at a third of the fine stage.  Here a CTA stays resident and walks pairs blockIdx.x,
// blockIdx.x + gridDim.x, ...: once a pair's inverse column pass is done (from then on its
// correlation touches only the tile's first rows) the bulk-copy engine brings the next pair's
// window (W x W dense floats, one cp.async.bulk completing on an mbarrier) into the tile's last
// bytes, and the chip's bytes are sent toward L2.  A pair then starts with its window in shared
// memory: the window's sums and placement statistics read from the staged copy (the tile's first
// bytes are the statistics' scratch), then one pass that writes the window and the chip (loaded
// from L2 meanwhile) into the tile and takes the chip's FP64 sums; the first transform pass takes
// both means off.  The numerics are spec_kernel's.  Every wait is bounded; one that
// runs out is counted in errs, the CTA lets the copy in flight land (again bounded) and returns.

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes)
                 : "memory");
}

// bytes (a multiple of 16) from global src to shared dst, both 16-byte aligned; completes on bar
__device__ __forceinline__ void bulk_to_smem(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     saddr(dst)),
                 "l"(src), "r"(bytes), "r"(saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void bulk_prefetch_l2(const void* src, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// the box of a 2-D tensor map at (x, y) (x a multiple of 4 floats) into shared dst; completes on bar
__device__ __forceinline__ void tensor_to_smem(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(saddr(bar))
        : "memory");
}

__device__ __forceinline__ void tensor_prefetch_l2(const CUtensorMap* map, int x, int y)
{
    asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y)
                 : "memory");
}

// RASTER false: the refined tiles, every pair's window W x W dense floats on a 16-byte boundary
// (one copy), its statistics formed here; RASTER true: windows cut from a raster, copied as the
// box of wmap (stage_rs x W floats) whose first column is the 16-byte boundary at or before the
// window's first sample, with the box of the raster's statistics (imap, inv_rs x C floats) at the
// same corner, the chip's box of cmap sent toward L2
template <int N1, int N2, bool RASTER>
__global__ void __launch_bounds__(kSpecThreads, 1)
spec_staged_kernel(SpecSource src, long long pair0, long long pairs, const long long* valid, SpecGeom g,
                   InvSource inv, const float2* tw_g, SpecOut out, unsigned int* errs,
                   const __grid_constant__ CUtensorMap wmap, const __grid_constant__ CUtensorMap cmap,
                   const __grid_constant__ CUtensorMap imap, int stall)
{
    extern __shared__ __align__(16) unsigned char ssm[];
    constexpr int N = N1 * N2;
    constexpr int RS = N + 1;
    constexpr int JN = (N + kSpecWarps - 1) / kSpecWarps, IN = (N + 31) / 32;
    constexpr int PJ = 5;  // row groups of a piece read whole before it is written
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int W = g.W, R = g.R, C = g.C, SW = g.stage_rs;
    float2* Z = reinterpret_cast<float2*>(ssm + g.off_z);
    float* Zf = reinterpret_cast<float*>(Z);
    float2* tw = reinterpret_cast<float2*>(ssm + g.off_tw);
    int* neg = reinterpret_cast<int*>(ssm + g.off_neg);
    int* half = reinterpret_cast<int*>(ssm + g.off_half);
    double* red = reinterpret_cast<double*>(ssm + g.off_red);
    float* invs = reinterpret_cast<float*>(ssm + g.off_inv);
    float* G = reinterpret_cast<float*>(ssm + g.off_gam);
    float* stage = reinterpret_cast<float*>(ssm + g.off_stage);
    float* inv_raw = reinterpret_cast<float*>(ssm + g.off_inv_raw);
    uint64_t* bar = reinterpret_cast<uint64_t*>(ssm + g.off_bar);
    int& s_err = *reinterpret_cast<int*>(ssm + g.off_bar + 8);  // a wait ran out (CTA-wide)
    const long long cs = src.chip_stride, ws = src.win_stride;
    const int jA = g.stage_y0 / kSpecWarps;

    for (int k = tid; k < N; k += kSpecThreads) {
        tw[k] = __ldg(tw_g + k);
        neg[k] = fft::neg_pos<N1, N2>(k);
    }
    if (warp == 0) build_half<N1, N2>(half);
    if (tid == 0) {
        s_err = 0;
        mbar_init(bar, 1);
        mbar_init(bar + 2, 1);  // completed by nothing: the wait of a failure-detection test
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // a failure-detection test: before any copy is issued, every thread waits on a barrier that
    // nothing completes; the bounded wait runs out, sets the error flag, and the CTA skips its
    // pairs and reports the time-out like any other expired wait
    if (stall) {
        mbar_wait(bar + 2, 0u, &s_err, kStallCycles);
        __syncthreads();
    }
    // warp 0: the window rows of chunk pair b into the staging bytes, the chip rows toward L2; a
    // pair without tiles (its offsets are -1) copies nothing and completes the phase at once
    auto issue = [&](long long b) {
        if (valid[pair0 + b] < 0) {
            if (lane == 0) mbar_arrive(bar);
            return;
        }
        const float* w = spec_win(src, pair0, b);
        const float* c = spec_chip(src, pair0, b);
        if constexpr (!RASTER) {
            if (lane == 0) {
                const unsigned bytes = (unsigned)W * (unsigned)W * 4u;
                mbar_expect_tx(bar, bytes);
                bulk_to_smem(stage, w, bytes, bar);
                bulk_prefetch_l2(c, (unsigned)R * (unsigned)cs * 4u);
            }
        } else {
            if (lane == 0) {
                const long long wo = src.win_off[pair0 + b], co = src.chip_off[pair0 + b];
                const int wy = (int)(wo / ws), wx = (int)(wo - (long long)wy * ws);
                const int cy = (int)(co / cs), cx = (int)(co - (long long)cy * cs);
                mbar_expect_tx(bar, ((unsigned)W * (unsigned)SW + (unsigned)C * (unsigned)g.inv_rs) * 4u);
                tensor_to_smem(stage, &wmap, wx & ~3, wy, bar);
                tensor_to_smem(inv_raw, &imap, wx & ~3, wy, bar);
                tensor_prefetch_l2(&cmap, cx & ~3, cy);
            }
        }
    };
    const bool run = !stall || !s_err;
    if (warp == 0 && blockIdx.x < pairs && run) issue(blockIdx.x);
    uint32_t parity = 0;
    bool inflight = blockIdx.x < pairs && run;
    long long b_left = blockIdx.x;  // (raster windows) the first pair left without a result
    for (long long b = blockIdx.x; b < pairs && run; b += gridDim.x) {
        const long long p = pair0 + b;
        const long long bn = b + gridDim.x;
        const bool ok = valid[p] >= 0;
        const float* chip = spec_chip(src, pair0, b);
        const float* win = spec_win(src, pair0, b);
        const bool landed = mbar_wait(bar, parity, &s_err);
        if (__syncthreads_or(!landed)) {
            if constexpr (RASTER) b_left = b;
            break;
        }
        parity ^= 1u;
        inflight = false;
        if (!ok) {
            if (out.stage == 0 && tid == 0) {
                out.coarse[p] = CoarseOut{-1, -1, -1, -1};
                out.coarse_peak[p] = NAN;
            }
            if (bn < pairs) {
                fence_async_smem();
                __syncthreads();
                if (warp == 0) issue(bn);
                inflight = true;
            }
            continue;
        }
        // window sample (y, x) in the staging bytes: the box starts xo samples before the window
        const int xo = RASTER ? (int)((src.win_off[p] % ws) & 3) : 0;
        // the chip to registers: for a raster window at once (its loads in flight while the
        // statistics are moved and its sum taken before the tile is written), for the refined
        // tiles after the statistics (registers are short there)
        float cr[JN][IN];
        auto load_chip = [&]() {
#pragma unroll
            for (int j = 0; j < JN; ++j)
#pragma unroll
                for (int i = 0; i < IN; ++i) {
                    const int y = warp + kSpecWarps * j, x = lane + 32 * i;
                    cr[j][i] = y < R && x < R ? __ldg(chip + y * cs + x) : 0.0f;
                }
        };
        double mean_c = 0.0;
        if constexpr (RASTER) {
            load_chip();
            // the raster's placement statistics, copied with the window, into their C x C layout
            for (int u = warp; u < C; u += kSpecWarps)
                for (int v = lane; v < C; v += 32) invs[u * C + v] = inv_raw[u * g.inv_rs + xo + v];
            // the chip's FP64 mean (spec_kernel's first sweep)
            double c1 = 0.0;
#pragma unroll
            for (int j = 0; j < JN; ++j)
#pragma unroll
                for (int i = 0; i < IN; ++i) c1 += (double)cr[j][i];
            c1 = warp_sum(c1);
            if (lane == 0) red[warp] = c1;
            __syncthreads();
            double t1 = 0.0;
            for (int w = 0; w < kSpecWarps; ++w) t1 += red[w];
            mean_c = t1 / ((double)R * (double)R);
            __syncthreads();
        }
        auto wat = [&](int y, int x) {
            if constexpr (RASTER)
                return stage[y * SW + xo + x];
            else
                return stage[y * W + x];
        };

        // the window's sums of t - k and (t - k)^2 about a pivot k (its first sample), as
        // spec_kernel takes them (in another order): here for the refined window, whose
        // statistics are centred on its mean; as the tile is written for a raster window
        const float pk = wat(0, 0);
        double wsum[2] = {0.0, 0.0};
        if constexpr (!RASTER) {
            float sw = 0.0f, sw2 = 0.0f;
            // four samples a load
            const float4* s4 = reinterpret_cast<const float4*>(stage);
            const int n4 = (W * W) >> 2;
#pragma unroll 4
            for (int k = tid; k < n4; k += kSpecThreads) {
                const float4 v = s4[k];
                const float t[4] = {v.x - pk, v.y - pk, v.z - pk, v.w - pk};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    sw += t[q];
                    sw2 = fmaf(t[q], t[q], sw2);
                }
            }
            wsum[0] = sw;
            wsum[1] = sw2;
            block_sum2<kSpecWarps>(wsum[0], wsum[1], red);
        }
        const double cells_c = (double)R * (double)R, cells_w = (double)W * (double)W;
        double mean_w = (double)pk + wsum[0] / cells_w;
        double st = fmax(wsum[1] - wsum[0] * wsum[0] / cells_w, 0.0) + 1e-5 * wsum[1];
        float sx = (float)mean_w;

        // placement statistics from the staged window where none are given; their scratch is the
        // tile's first bytes
        if constexpr (!RASTER) {
            double* part = reinterpret_cast<double*>(ssm + g.off_gam);
            const StatSlots vs{Zf, reinterpret_cast<float*>(part + 4 * g.nseg * W), g.off_stage / 4, 1};
            spec_box_stats<kSpecThreads>(wat, g, sx, vs, part, invs);
        }

        // window (real parts) and chip (imaginary parts; its bytes were sent toward L2 with the
        // window) into the tile, zeros around them.  Raster windows: the chip goes in zero-mean
        // and |r'|^2 is summed as spec_kernel sums it, the window's sums are taken on the way.
        // Refined tiles: the chip goes in as it is, its FP64 sum and sum of squares taken on the
        // way (every product of two floats is exact in FP64), and the first transform pass takes
        // its mean off.
        if constexpr (!RASTER) load_chip();
        const float mc_hi = (float)mean_c, mc_lo = (float)(mean_c - (double)mc_hi);
        double c1 = 0.0, c2 = 0.0;
        float sw = 0.0f, sw2 = 0.0f, sc2 = 0.0f;
        auto put = [&](int j, int i, float t) {
            const int y = warp + kSpecWarps * j, x = lane + 32 * i;
            if (y < N && x < N) {
                float c = cr[j][i];
                if constexpr (RASTER) {
                    if (y < R && x < R) {
                        c = (c - mc_hi) - mc_lo;
                        sc2 = fmaf(c, c, sc2);
                    }
                    if (y < W && x < W) {
                        const float d = t - pk;
                        sw += d;
                        sw2 = fmaf(d, d, sw2);
                    }
                } else {
                    c1 += (double)c;
                    c2 = fma((double)c, (double)c, c2);
                }
                Z[y * RS + x] = make_float2(t, c);
            }
        };
        auto staged = [&](int j, int i) {
            const int y = warp + kSpecWarps * j, x = lane + 32 * i;
            return y < W && x < W ? wat(y, x) : 0.0f;
        };
        // rows below stage_y0 lie below the staged bytes: written as they are read
#pragma unroll
        for (int j = 0; j < JN; ++j)
            if (j < jA)
#pragma unroll
                for (int i = 0; i < IN; ++i) put(j, i, staged(j, i));
        __syncthreads();
        // the others cover staged bytes: each piece is read whole, then written (a piece's rows
        // never reach the staged rows of a later piece)
#pragma unroll
        for (int j0 = 0; j0 < JN; j0 += PJ) {
            if (j0 + PJ <= jA) continue;
            float v[PJ][IN];
#pragma unroll
            for (int q = 0; q < PJ; ++q)
#pragma unroll
                for (int i = 0; i < IN; ++i) v[q][i] = j0 + q < JN && j0 + q >= jA ? staged(j0 + q, i) : 0.0f;
            __syncthreads();
#pragma unroll
            for (int q = 0; q < PJ; ++q)
                if (j0 + q < JN && j0 + q >= jA)
#pragma unroll
                    for (int i = 0; i < IN; ++i) put(j0 + q, i, v[q][i]);
        }
        double ss;
        fft::Centre centre{sx, W};
        if constexpr (RASTER) {
            const double d0 = warp_sum((double)sc2), d1 = warp_sum((double)sw), d2 = warp_sum((double)sw2);
            if (lane == 0) {
                red[3 * warp] = d0;
                red[3 * warp + 1] = d1;
                red[3 * warp + 2] = d2;
            }
            __syncthreads();
            ss = 0.0;
            for (int w = 0; w < kSpecWarps; ++w) {
                ss += red[3 * w];
                wsum[0] += red[3 * w + 1];
                wsum[1] += red[3 * w + 2];
            }
            mean_w = (double)pk + wsum[0] / cells_w;
            st = fmax(wsum[1] - wsum[0] * wsum[0] / cells_w, 0.0) + 1e-5 * wsum[1];
            centre.sx = (float)mean_w;
        } else {
            c1 = warp_sum(c1);
            c2 = warp_sum(c2);
            if (lane == 0) {
                red[2 * warp] = c1;
                red[2 * warp + 1] = c2;
            }
            __syncthreads();
            double s1 = 0.0, s2 = 0.0;
            for (int w = 0; w < kSpecWarps; ++w) {
                s1 += red[2 * w];
                s2 += red[2 * w + 1];
            }
            // |r'|^2 = S2 - S1^2 / R^2 of the zero-mean chip; a chip flat to within its own
            // rounding (a constant: its zero-mean values are exactly 0) gets 0, as the sum of the
            // squared zero-mean values gives it
            mean_c = s1 / cells_c;
            ss = s2 - s1 * mean_c;
            if (!(ss > 1e-14 * s2)) ss = 0.0;
            const float hi = (float)mean_c;
            centre.ci_hi = hi;
            centre.ci_lo = (float)(mean_c - (double)hi);
            centre.ci = R;
        }
        const float inv_sigma = ss > 0.0 ? (float)(1.0 / sqrt(ss)) : 0.0f;

        const float scale = (float)(1.0 / (4.0 * (double)N * (double)N));
        const float ebox = kSpecErr * (float)sqrt(st);
        float bv = -INFINITY;
        int bi = INT_MAX;
        int flagged = 0;
        fft::correlate_tile<N1, N2, RASTER ? 2 : 0>(
            Z, RS, W, C, tw, neg, half, centre, tid, kSpecThreads, BlockSync{},
            [&](int u, int v, float2 val) {
                if (v < C) {
                    const int idx = u * C + v;
                    const float inv_box = invs[idx];
                    const float gv = val.x * scale * inv_box * inv_sigma;
                    G[idx] = gv;
                    if (ebox * inv_box > kSpecTol)
                        flagged = 1;
                    else
                        better(bv, bi, gv, idx);
                }
            },
            [&]() {
                // the staged bytes are free from here on: the next pair's window comes in
                fence_async_smem();
                __syncthreads();
                if (bn < pairs) {
                    if (warp == 0) issue(bn);
                    inflight = true;
                }
            });

        float* surf = out.surfaces ? out.surfaces + (size_t)p * C * C : nullptr;
        float* gam = out.stage == 1 ? out.gam + b * C * C : nullptr;
        spec_surface<kSpecThreads>(G, red, g, invs, inv_sigma, mean_c, ebox, chip, cs, win, ws, gam, surf, bv, bi,
                                   flagged);
        if (tid == 0) spec_result(out, p, R, W, C, bv, bi);
    }
    if (s_err) {
        // a wait ran out: count it once per CTA, give the pairs left a coarse result whose
        // refinement corners stay inside their windows, and let the copy in flight land before
        // the shared memory is given up
        if (tid == 0) {
            atomicAdd(errs, 1u);
            if constexpr (RASTER)
                for (long long q = b_left; q < pairs; q += gridDim.x) {
                    out.coarse[pair0 + q] = CoarseOut{-1, -1, 0, 0};
                    out.coarse_peak[pair0 + q] = NAN;
                }
            if (inflight) {
                const long long t0 = clock64();
                while (!mbar_try(bar, parity) && clock64() - t0 < kSpinCycles) {
                }
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------------
// refinement by zero-padded FFT (the reference's band-limited upsampling, refine.cu / cuFFT)
// ------------------------------------------------------------------------------------------

// Upsample the N x N complex tile at src (rows stride apart) by F / N and write its amplitudes
// (F x F, dense, row stride F) to out: the tile's 2-D forward transform (N-point FFTs along the
// rows, then down the N columns), F-point inverses down the N columns that pad each column's
// spectrum on the fly (F x N), then CB rows at a time the F-point inverses along the rows, again
// padding on the fly, and the amplitudes out.  Scaled by 1 / N^2.  Transforming both axes forward
// before padding either costs N + N + N + F transforms, against N + N + F + F when the rows are
// upsampled first.
template <int N1, int N2, int F1, int F2>
struct UpsampleGeom {
    static constexpr int N = N1 * N2, F = F1 * F2;
    static constexpr int RSN = N + 1, RSY = N + 1, RSB = F + 1;
    // output rows per block: the block buffer reuses the tile's space
    static constexpr int CBX = N * RSN / RSB;
    static constexpr int CB = CBX < 32 ? CBX : 32;
    static constexpr int smem = (N * RSN + F * RSY + N + F) * 8;
    static_assert(CB >= 1, "the row block must fit in the tile's space");
    // staged form (spec_refine_staged_kernel): the tile as copied from the raster, N rows of SWS
    // floats (2 N + 2 from the 16-byte boundary at or before its first sample), then the copy's
    // mbarrier and the CTA's wait-failure flag
    static constexpr int SWS = (2 * N + 5) & ~3;
    static constexpr int off_stage = (smem + 127) / 128 * 128;
    static constexpr int off_bar = off_stage + N * SWS * 4;
    static constexpr int smem_staged = off_bar + 16;
};

template <int N1, int N2, int F1, int F2>
__device__ void upsample_core(unsigned char* sm, float2 mu, float* __restrict__ out);

template <int N1, int N2, int F1, int F2, bool DERAMP>
__device__ void fft_upsample(const float2* __restrict__ src, long long stride, unsigned char* sm,
                             const float2* __restrict__ twn_g, const float2* __restrict__ twf_g,
                             float* __restrict__ out)
{
    using G = UpsampleGeom<N1, N2, F1, F2>;
    constexpr int N = G::N, F = G::F, RSN = G::RSN, RSY = G::RSY, RSB = G::RSB, CB = G::CB;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float2* X = reinterpret_cast<float2*>(sm);   // the tile, later a block of F-point rows
    float2* Y = X + N * RSN;                     // columns upsampled: F x N
    float2* twn = Y + F * RSY;
    float2* twf = twn + N;
    for (int k = tid; k < N; k += kThreads) twn[k] = __ldg(twn_g + k);
    for (int k = tid; k < F; k += kThreads) twf[k] = __ldg(twf_g + k);
    float2 mu;
    if constexpr (DERAMP) {
        for (int y = warp; y < N; y += kWarps)
            for (int x = lane; x < N; x += 32) cp_async8_g(X + y * RSN + x, src + y * stride + x);
        cp_async_wait_all();
        __syncthreads();
        // the upsampled-columns buffer is free until the columns are written: the deramp's scratch
        deramp_tile(X, RSN, N, reinterpret_cast<double*>(Y));
        // the tile's mean comes off as the rows are read and back on with the amplitudes
        mu = tile_mean<false, false>(X, RSN, N, 0.0f, 0.0f, reinterpret_cast<double*>(Y));
    } else {
        // the tile through registers, its sum taken on the way (tile_mean's order: FP32 sums per
        // thread over samples tid, tid + kThreads, ..., FP64 across the block); the mean comes
        // off as the rows are read and back on with the amplitudes
        constexpr int KT = (N * N + kThreads - 1) / kThreads;
        float2 v[KT];
#pragma unroll
        for (int q = 0; q < KT; ++q) {
            const int k = tid + q * kThreads;
            v[q] = k < N * N ? __ldg(src + (k / N) * stride + k % N) : make_float2(0.0f, 0.0f);
        }
        float sx = 0.0f, sy = 0.0f;
#pragma unroll
        for (int q = 0; q < KT; ++q) {
            const int k = tid + q * kThreads;
            if (k < N * N) {
                X[(k / N) * RSN + k % N] = v[q];
                sx += v[q].x;
                sy += v[q].y;
            }
        }
        double* red = reinterpret_cast<double*>(Y);
        const double a = warp_sum((double)sx), b = warp_sum((double)sy);
        if (lane == 0) {
            red[2 * warp] = a;
            red[2 * warp + 1] = b;
        }
        __syncthreads();
        double ta = 0.0, tb = 0.0;
        for (int w = 0; w < kWarps; ++w) {
            ta += red[2 * w];
            tb += red[2 * w + 1];
        }
        const double cells = (double)N * (double)N;
        mu = make_float2((float)(ta / cells), (float)(tb / cells));
    }
    upsample_core<N1, N2, F1, F2>(sm, mu, out);
}

// the transforms of fft_upsample and the amplitudes out, from the tile in place (X) with its mean
// mu and the twiddles in shared memory
template <int N1, int N2, int F1, int F2>
__device__ void upsample_core(unsigned char* sm, float2 mu, float* __restrict__ out)
{
    using G = UpsampleGeom<N1, N2, F1, F2>;
    constexpr int N = G::N, F = G::F, RSN = G::RSN, RSY = G::RSY, RSB = G::RSB, CB = G::CB;
    const int tid = threadIdx.x;
    float2* X = reinterpret_cast<float2*>(sm);
    float2* Y = X + N * RSN;
    const float2* twn = Y + F * RSY;
    const float2* twf = twn + N;
    // rows: forward N
    for (int t = tid; t < N * N2; t += kThreads) fft::fwd_a_minus<N1, N2>(X + (t % N) * RSN, 1, t / N, twn, mu);
    __syncthreads();
    for (int t = tid; t < N * N1; t += kThreads) fft::step_b<N1, N2, -1>(X + (t % N) * RSN, 1, t / N);
    __syncthreads();
    // columns: forward N
    for (int t = tid; t < N * N2; t += kThreads) fft::fwd_a<N1, N2>(X + t % N, RSN, t / N, twn);
    __syncthreads();
    for (int t = tid; t < N * N1; t += kThreads) fft::step_b<N1, N2, -1>(X + t % N, RSN, t / N);
    __syncthreads();
    // columns: inverse F, the first step padding each column's spectrum as it reads it
    for (int t = tid; t < N * F1; t += kThreads)
        fft::step_b_pad<N1, N2, F1, F2>(X + t % N, RSN, Y + t % N, RSY, t / N);
    __syncthreads();
    for (int t = tid; t < N * F2; t += kThreads) fft::inv_a<F1, F2>(Y + t % N, RSY, t / N, twf);
    __syncthreads();
    const float scale = 1.0f / ((float)N * (float)N);
    for (int r0 = 0; r0 < F; r0 += CB) {
        const int nr = F - r0 < CB ? F - r0 : CB;
        // a block of rows: inverse F (padding on the fly), amplitudes out
        for (int t = tid; t < CB * F1; t += kThreads) {
            const int r = t % CB;
            if (r < nr) fft::step_b_pad<N1, N2, F1, F2>(Y + (r0 + r) * RSY, 1, X + r * RSB, 1, t / CB);
        }
        __syncthreads();
        // the last step writes the amplitudes of its outputs straight to global memory; lanes take
        // consecutive outputs of a row, so the stores coalesce
        for (int t = tid; t < CB * F2; t += kThreads) {
            const int r = t / F2, n2 = t - r * F2;
            if (r < nr) {
                float* row = out + (long long)(r0 + r) * F;
                fft::inv_a_store<F1, F2>(X + r * RSB, 1, n2, twf, [&](int n, float2 v) {
                    const float re = fmaf(v.x, scale, mu.x), im = fmaf(v.y, scale, mu.y);
                    row[n] = sqrtf(re * re + im * im);
                });
            }
        }
        __syncthreads();
    }
}

// one tile of every pair of a chunk: the chip (coarse == nullptr) or the nudged window; two CTAs
// per SM where their shared memory allows
template <int N1, int N2, int F1, int F2, bool DERAMP>
__global__ void __launch_bounds__(kThreads, UpsampleGeom<N1, N2, F1, F2>::smem <= 113 * 1024 ? 2 : 1)
spec_refine_kernel(const float2* base, const long long* off, long long stride,
                   const CoarseOut* coarse, long long pair0, long long pairs, const long long* valid,
                   const float2* twn, const float2* twf, float* refined, long long refined_stride,
                   long long out_off)
{
    extern __shared__ __align__(16) unsigned char rsm[];
    if (blockIdx.x >= pairs) return;
    const long long p = pair0 + blockIdx.x;
    if (valid[p] < 0) return;
    const float2* src = base + off[p];
    if (coarse) {
        const CoarseOut co = coarse[p];
        src += co.top * stride + co.left;
    }
    fft_upsample<N1, N2, F1, F2, DERAMP>(
        src, stride, rsm, twn, twf, refined + (long long)blockIdx.x * refined_stride + out_off);
}

// Refinement of the windows of a raster job, staged: one resident CTA per SM walks the pairs of
// the chunk, and the copy engine brings the next pair's tile (the box of the secondary raster,
// as floats, at the nudged corner of its coarse result) into a buffer of its own while this
// pair's transforms run.  The tile goes from that buffer into place with its sum taken in
// fft_upsample's order, so the amplitudes are fft_upsample's bit for bit.  Every wait is
// bounded; one that runs out is counted in errs, the CTA lets its copy land (bounded) and returns.
template <int N1, int N2, int F1, int F2>
__global__ void __launch_bounds__(kThreads, 1)
spec_refine_staged_kernel(const __grid_constant__ CUtensorMap tmap, const long long* off, long long stride,
                          const CoarseOut* coarse, long long pair0, long long pairs, const long long* valid,
                          const float2* twn_g, const float2* twf_g, float* refined, long long refined_stride,
                          long long out_off, unsigned int* errs)
{
    extern __shared__ __align__(16) unsigned char rsm[];
    using G = UpsampleGeom<N1, N2, F1, F2>;
    constexpr int N = G::N, F = G::F, RSN = G::RSN, RSY = G::RSY, SWS = G::SWS;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float2* X = reinterpret_cast<float2*>(rsm);
    float2* Y = X + N * RSN;
    float2* twn = Y + F * RSY;
    float2* twf = twn + N;
    float* stage = reinterpret_cast<float*>(rsm + G::off_stage);
    uint64_t* bar = reinterpret_cast<uint64_t*>(rsm + G::off_bar);
    int& s_err = *reinterpret_cast<int*>(rsm + G::off_bar + 8);
    for (int k = tid; k < N; k += kThreads) twn[k] = __ldg(twn_g + k);
    for (int k = tid; k < F; k += kThreads) twf[k] = __ldg(twf_g + k);
    if (tid == 0) {
        s_err = 0;
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // first sample of chunk pair b's tile: line y, sample x of the raster
    auto corner = [&](long long b, int& x, int& y) {
        const long long p = pair0 + b;
        const CoarseOut co = coarse[p];
        const long long o = off[p] + co.top * stride + co.left;
        const long long yy = o / stride;
        y = (int)yy;
        x = (int)(o - yy * stride);
    };
    // thread 0: chunk pair b's tile into the staging buffer; a pair without tiles copies nothing
    auto issue = [&](long long b) {
        if (valid[pair0 + b] < 0) {
            mbar_arrive(bar);
            return;
        }
        int x, y;
        corner(b, x, y);
        mbar_expect_tx(bar, (unsigned)(N * SWS * 4));
        tensor_to_smem(stage, &tmap, (2 * x) & ~3, y, bar);
    };
    if (tid == 0 && blockIdx.x < pairs) issue(blockIdx.x);
    uint32_t parity = 0;
    bool inflight = blockIdx.x < pairs;
    for (long long b = blockIdx.x; b < pairs; b += gridDim.x) {
        const long long p = pair0 + b;
        const long long bn = b + gridDim.x;
        const bool ok = valid[p] >= 0;
        int of = 0;
        if (ok) {
            int x, y;
            corner(b, x, y);
            of = (2 * x) & 3;
        }
        const bool landed = mbar_wait(bar, parity, &s_err);
        if (__syncthreads_or(!landed)) break;
        parity ^= 1u;
        inflight = false;
        if (!ok) {
            if (bn < pairs) {
                fence_async_smem();
                __syncthreads();
                if (tid == 0) issue(bn);
                inflight = true;
            }
            continue;
        }
        // the tile into place, its sum taken on the way (fft_upsample's order)
        constexpr int KT = (N * N + kThreads - 1) / kThreads;
        float sx = 0.0f, sy = 0.0f;
#pragma unroll
        for (int q = 0; q < KT; ++q) {
            const int k = tid + q * kThreads;
            if (k < N * N) {
                const int y = k / N, x = k % N;
                const float2 v = *reinterpret_cast<const float2*>(stage + y * SWS + of + 2 * x);
                X[y * RSN + x] = v;
                sx += v.x;
                sy += v.y;
            }
        }
        double* red = reinterpret_cast<double*>(Y);
        const double a = warp_sum((double)sx), c = warp_sum((double)sy);
        if (lane == 0) {
            red[2 * warp] = a;
            red[2 * warp + 1] = c;
        }
        // the staging buffer is read: the next pair's tile comes in while this one is transformed
        fence_async_smem();
        __syncthreads();
        if (bn < pairs) {
            if (tid == 0) issue(bn);
            inflight = true;
        }
        double ta = 0.0, tb = 0.0;
        for (int w = 0; w < kWarps; ++w) {
            ta += red[2 * w];
            tb += red[2 * w + 1];
        }
        const double cells = (double)N * (double)N;
        const float2 mu = make_float2((float)(ta / cells), (float)(tb / cells));
        upsample_core<N1, N2, F1, F2>(rsm, mu, refined + b * refined_stride + out_off);
    }
    if (s_err) {
        // a wait ran out: count it once per CTA and let the copy in flight land before the shared
        // memory is given up
        if (tid == 0) {
            atomicAdd(errs, 1u);
            if (inflight) {
                const long long t0 = clock64();
                while (!mbar_try(bar, parity) && clock64() - t0 < kSpinCycles) {
                }
            }
        }
        __syncthreads();
    }
}

// refinement (N, F = 2 N) pairs that are compiled: N, N1, N2, F1, F2
#define AMPCOR_REFINE_PAIRS(X) \
    X(16, 4, 4, 4, 8)          \
    X(24, 4, 6, 6, 8)          \
    X(32, 4, 8, 8, 8)          \
    X(40, 5, 8, 8, 10)         \
    X(48, 6, 8, 8, 12)         \
    X(64, 8, 8, 8, 16)         \
    X(80, 8, 10, 10, 16)

// transform lengths: N, N1, N2 (N1 N2 = N)
#define AMPCOR_SPEC_LENGTHS(X) \
    X(16, 4, 4)                \
    X(24, 4, 6)                \
    X(32, 4, 8)                \
    X(40, 5, 8)                \
    X(48, 6, 8)                \
    X(64, 8, 8)                \
    X(80, 8, 10)               \
    X(96, 8, 12)               \
    X(120, 8, 15)              \
    X(128, 8, 16)              \
    X(144, 12, 12)             \
    X(160, 10, 16)

// ------------------------------------------------------------------------------------------
// blocked spectral correlation: tiles beyond one CTA's shared memory
// ------------------------------------------------------------------------------------------
//
// The numerator surface is a sum over the chip's pixels, so it splits over square blocks of the
// chip: block k (rows [i0, i0 + B), columns [j0, j0 + B)) meets the sub-window of rows
// [i0, i0 + B + C - 1), columns [j0, j0 + B + C - 1), and its placements are those of the whole
// window.  spec_block_kernel runs the in-shared-memory FFT correlation of one block (one CTA per
// pair and block) and writes its partial numerators; spec_reduce_kernel sums a pair's partials in
// a fixed order, normalises them, bounds the transform error and takes the first maximum, as
// spec_kernel does for a tile that fits.  The chip is centred on the whole chip's mean
// (spec_chip_stats_kernel), each sub-window on its own mean s_k: the block then computes
// sum c (t - s_k), and the pair's numerator is the sum over blocks plus sum_k s_k sum_k c, c the
// centred chip values the block placed in its tile.

// one CTA of 256 threads per pair: FP64 mean and 1/|r - mean| of the R x R chip
__global__ void __launch_bounds__(256)
spec_chip_stats_kernel(SpecSource src, long long pair0, long long pairs, const long long* valid, int R,
                       ChipStat* out)
{
    __shared__ double red[16];
    if (blockIdx.x >= pairs) return;
    const long long p = pair0 + blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (valid[p] < 0) {
        if (tid == 0) out[blockIdx.x] = ChipStat{0.0, 0.0};
        return;
    }
    const float* chip = spec_chip(src, pair0, blockIdx.x);
    const long long cs = src.chip_stride;
    double s1 = 0.0, s2 = 0.0;
    for (int y = warp; y < R; y += 8)
        for (int x = lane; x < R; x += 32) {
            const double v = __ldg(chip + y * cs + x);
            s1 += v;
            s2 += v * v;
        }
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    if (lane == 0) {
        red[2 * warp] = s1;
        red[2 * warp + 1] = s2;
    }
    __syncthreads();
    if (tid == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < 8; ++w) {
            a += red[2 * w];
            b += red[2 * w + 1];
        }
        const double cells = (double)R * (double)R;
        const double mean = a / cells;
        const double ss = b - cells * mean * mean;
        out[blockIdx.x] = ChipStat{mean, ss > 0.0 ? 1.0 / sqrt(ss) : 0.0};
    }
}

// 1/sigma of every placement box of a window read straight from global memory (windows larger
// than a CTA stages): FP64 column sums sliding down the window, FP64 prefix sums along the rows,
// SR placement rows at a time (window_stats_xs); inv: C^2 floats per chunk-local pair.  W <= kThreads.
__global__ void __launch_bounds__(kThreads, 2)
spec_tile_stats_kernel(SpecSource src, long long pair0, long long pairs, const long long* valid, int R, int W,
                       int SR, float* inv)
{
    extern __shared__ __align__(16) double tsm[];
    if (blockIdx.x >= pairs) return;
    const long long p = pair0 + blockIdx.x;
    if (valid[p] < 0) return;
    const int C = W - R + 1;
    window_stats_xs<1>(spec_win(src, pair0, blockIdx.x), (int)src.win_stride, W, R, C, SR,
                       inv + (long long)blockIdx.x * C * C, tsm);
}

// The partial numerators of one chip block of one pair (CTA b K + k): g is the tile of a block
// (g.R = B, g.W = B + C - 1, g.C = C), nb blocks per axis.  part: C^2 floats per (pair, block),
// already scaled; scal: two doubles per (pair, block), s_k sum_k c and |c| |t - s_k|.
template <int N1, int N2>
__global__ void __launch_bounds__(kSpecThreads, 1)
spec_block_kernel(SpecSource src, long long pair0, long long pairs, const long long* valid, SpecGeom g,
                  int nb, const ChipStat* cstat, const float2* tw_g, float* part, double* scal)
{
    extern __shared__ __align__(16) unsigned char ssm[];
    const int K = nb * nb;
    const int b = blockIdx.x / K, k = blockIdx.x - b * K;
    if (b >= pairs) return;
    const long long p = pair0 + b;
    if (valid[p] < 0) return;
    constexpr int N = N1 * N2;
    constexpr int RS = N + 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int B = g.R, S = g.W, C = g.C;
    const int i0 = (k / nb) * B, j0 = (k - (k / nb) * nb) * B;
    float2* Z = reinterpret_cast<float2*>(ssm + g.off_z);
    float2* tw = reinterpret_cast<float2*>(ssm + g.off_tw);
    int* neg = reinterpret_cast<int*>(ssm + g.off_neg);
    int* half = reinterpret_cast<int*>(ssm + g.off_half);
    double* red = reinterpret_cast<double*>(ssm + g.off_red);
    float* Zf = reinterpret_cast<float*>(Z);
    const long long cs = src.chip_stride, ws = src.win_stride;
    const float* chip = spec_chip(src, pair0, b) + i0 * cs + j0;
    const float* win = spec_win(src, pair0, b) + i0 * ws + j0;
    const ChipStat cst = cstat[b];
    const float mc_hi = (float)cst.mean, mc_lo = (float)(cst.mean - (double)mc_hi);

    // the block of the chip, centred on the whole chip's mean, to registers; the sub-window to the
    // tile's real parts by asynchronous copies, zeros around it
    constexpr int JN = (N + kSpecWarps - 1) / kSpecWarps, IN = (N + 31) / 32;
    float cr[JN][IN];
#pragma unroll
    for (int j = 0; j < JN; ++j)
#pragma unroll
        for (int i = 0; i < IN; ++i) {
            const int y = warp + kSpecWarps * j, x = lane + 32 * i;
            cr[j][i] = y < B && x < B ? (__ldg(chip + y * cs + x) - mc_hi) - mc_lo : 0.0f;
        }
    for (int y = warp; y < N; y += kSpecWarps) {
        float* zr = Zf + 2 * y * RS;
        for (int x = lane; x < N; x += 32) {
            if (y < S && x < S)
                cp_async4(zr + 2 * x, win + y * ws + x);
            else
                zr[2 * x] = 0.0f;
        }
    }
    for (int q = tid; q < N; q += kSpecThreads) {
        tw[q] = __ldg(tw_g + q);
        neg[q] = fft::neg_pos<N1, N2>(q);
    }
    if (warp == 0) build_half<N1, N2>(half);
    cp_async_wait_all();
    __syncthreads();

    // FP64 sums of the centred chip block (its sum and sum of squares) and of the sub-window about
    // a pivot k (its first sample): the sums of t - k and (t - k)^2 give its mean and an upper bound
    // of |t'|^2 (which only scales the error bound), as in spec_kernel
    double a0 = 0.0, a1 = 0.0, a2, a3;
    const float pk = Z[0].x;
    {
        float sw = 0.0f, sw2 = 0.0f;
        for (int y = warp; y < S; y += kSpecWarps) {
            const float2* zr = Z + y * RS;
            for (int x = lane; x < S; x += 32) {
                const float t = zr[x].x - pk;
                sw += t;
                sw2 = fmaf(t, t, sw2);
            }
        }
#pragma unroll
        for (int j = 0; j < JN; ++j)
#pragma unroll
            for (int i = 0; i < IN; ++i) {
                const double c = cr[j][i];
                a0 += c;
                a1 += c * c;
            }
        a2 = sw;
        a3 = sw2;
        block_sum2<kSpecWarps>(a0, a1, red);
        block_sum2<kSpecWarps>(a2, a3, red);
    }
    const double cells_w = (double)S * (double)S;
    const double mean_w = (double)pk + a2 / cells_w;
    const double st = fmax(a3 - a2 * a2 / cells_w, 0.0) + 1e-5 * a3;
    const fft::Centre centre{(float)mean_w, S};
#pragma unroll
    for (int j = 0; j < JN; ++j)
#pragma unroll
        for (int i = 0; i < IN; ++i) {
            const int y = warp + kSpecWarps * j, x = lane + 32 * i;
            if (y < N && x < N) Zf[2 * (y * RS + x) + 1] = cr[j][i];
        }
    __syncthreads();
    // the last inverse step hands placement row u to the store, which puts it in tile row u (no
    // later step reads those rows), so the numerators need no buffer beside the tile
    fft::correlate_tile<N1, N2>(Z, RS, S, C, tw, neg, half, centre, tid, kSpecThreads, BlockSync{},
                                [&](int u, int v, float2 val) { Z[u * RS + v] = val; });
    const float scale = (float)(1.0 / (4.0 * (double)N * (double)N));
    float* out = part + ((long long)b * K + k) * C * C;
    for (int idx = tid; idx < C * C; idx += kSpecThreads) {
        const int u = idx / C, v = idx - u * C;
        out[idx] = Z[u * RS + v].x * scale;
    }
    if (tid == 0) {
        scal[2 * ((long long)b * K + k)] = (double)centre.sx * a0;
        scal[2 * ((long long)b * K + k) + 1] = sqrt(a1 * st);
    }
}

// One CTA per pair: the sum of the K partial numerators of every placement (FP64, in block order,
// plus the centring corrections), normalised by the chip's 1/|r'| and the placement's 1/sigma_box,
// then the direct FP32 recomputation where the transform's bound is loose (spec_surface) and the
// stage's outputs, as in spec_kernel.  g: the whole stage (R, W, C).  Shared memory: the
// placement statistics and the surface (C^2 floats each) and a reduction scratch.
__global__ void __launch_bounds__(kThreads, 1)
spec_reduce_kernel(SpecSource src, long long pair0, long long pairs, const long long* valid, SpecGeom g,
                   int K, const ChipStat* cstat, InvSource inv, const float* part, const double* scal,
                   SpecOut out)
{
    extern __shared__ __align__(16) unsigned char ssm[];
    if (blockIdx.x >= pairs) return;
    const long long p = pair0 + blockIdx.x;
    const int tid = threadIdx.x;
    if (valid[p] < 0) {
        if (out.stage == 0 && tid == 0) {
            out.coarse[p] = CoarseOut{-1, -1, -1, -1};
            out.coarse_peak[p] = NAN;
        }
        return;
    }
    const int R = g.R, W = g.W, C = g.C, CC = C * C;
    float* invs = reinterpret_cast<float*>(ssm);
    float* G = invs + ((CC + 3) & ~3);
    double* red = reinterpret_cast<double*>(G + ((CC + 3) & ~3));
    const float* inv_b = inv.off ? inv.base + inv.off[p] : inv.base + (long long)blockIdx.x * CC;
    const long long is = inv.off ? inv.stride : C;
    for (int idx = tid; idx < CC; idx += kThreads) {
        const int u = idx / C, v = idx - u * C;
        invs[idx] = __ldg(inv_b + u * is + v);
    }
    const double* sc = scal + 2 * (long long)blockIdx.x * K;
    double corr = 0.0, errs = 0.0;
    for (int k = 0; k < K; ++k) {
        corr += sc[2 * k];
        errs += sc[2 * k + 1];
    }
    const ChipStat cst = cstat[blockIdx.x];
    const float inv_sigma = (float)cst.inv_sigma;
    const float ebox = kSpecErr * (float)errs * inv_sigma;
    __syncthreads();
    float bv = -INFINITY;
    int bi = INT_MAX;
    int flagged = 0;
    const float* pp = part + (long long)blockIdx.x * K * CC;
    for (int idx = tid; idx < CC; idx += kThreads) {
        double num = corr;
        for (int k = 0; k < K; ++k) num += (double)__ldg(pp + (long long)k * CC + idx);
        const float inv_box = invs[idx];
        const float gv = (float)num * inv_box * inv_sigma;
        G[idx] = gv;
        if (ebox * inv_box > kSpecTol)
            flagged = 1;
        else
            better(bv, bi, gv, idx);
    }
    __syncthreads();
    const float* chip = spec_chip(src, pair0, blockIdx.x);
    const float* win = spec_win(src, pair0, blockIdx.x);
    float* surf = out.surfaces ? out.surfaces + (size_t)p * CC : nullptr;
    float* gam = out.stage == 1 ? out.gam + (long long)blockIdx.x * CC : nullptr;
    spec_surface<kThreads>(G, red, g, invs, inv_sigma, cst.mean, ebox, chip, src.chip_stride, win,
                           src.win_stride, gam, surf, bv, bi, flagged);
    if (tid == 0) {
        const int u = bi / C, v = bi - u * C;
        if (out.stage == 0) {
            // nudge.cu:107-140 (argument roles from nudge.cu:57: old = W, new = R + 2m)
            const int E = R + 2 * out.m;
            int left = v - out.m;
            if (left < 0) left = 0;
            if (left + E > W) left = W - E;
            int top = u - out.m;
            if (top < 0) top = 0;
            if (top + E > W) top = W - E;
            out.coarse[p] = CoarseOut{u, v, top, left};
            out.coarse_peak[p] = bv;
        } else {
            out.fine[p] = FineOut{u, v, bv, 0.0f};
        }
    }
}

// The linear-phase steps of an n x n complex tile in global memory (rows `stride` apart), as
// deramp_tile measures them: the phases of the lag-one autocorrelations along samples and lines.
// red: 4 kWarps doubles; every thread gets both phases; ends with a barrier.
__device__ void deramp_phases_global(const float2* t, long long stride, int n, double* red, float& ps, float& pl)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float sr = 0.0f, si = 0.0f, lr = 0.0f, li = 0.0f;
    for (int k = tid; k < n * n; k += kThreads) {
        const int y = k / n, x = k - y * n;
        const float2 z = __ldg(t + y * stride + x);
        if (x + 1 < n) {
            const float2 w = __ldg(t + y * stride + x + 1);
            sr = fmaf(w.x, z.x, fmaf(w.y, z.y, sr));
            si = fmaf(w.y, z.x, fmaf(-w.x, z.y, si));
        }
        if (y + 1 < n) {
            const float2 w = __ldg(t + (y + 1) * stride + x);
            lr = fmaf(w.x, z.x, fmaf(w.y, z.y, lr));
            li = fmaf(w.y, z.x, fmaf(-w.x, z.y, li));
        }
    }
    double v[4] = {sr, si, lr, li};
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = warp_sum(v[q]);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q) red[4 * warp + q] = v[q];
    __syncthreads();
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (int w = 0; w < kWarps; ++w)
#pragma unroll
        for (int q = 0; q < 4; ++q) a[q] += red[4 * w + q];
    ps = (float)atan2(a[1], a[0]);
    pl = (float)atan2(a[3], a[2]);
    __syncthreads();
}

// Band-limited upsampling of tiles too large to stage whole (N up to 160, F = 2 N): the transforms
// of fft_upsample in the rows-first order (the mean off as there), a strip of ST rows at a time (N-point FFTs, F-point
// padded inverses) into a per-pair buffer in global memory (N x F complex, row-major), then the
// columns of that buffer CB at a time (N-point FFTs, F-point padded inverses, amplitudes out).
template <int N1, int N2, int F1, int F2>
struct BigUpsampleGeom {
    static constexpr int N = N1 * N2, F = F1 * F2, ST = 32, CB = 32;
    static constexpr int XS = ST * (N + 1) > N * (CB + 1) ? ST * (N + 1) : N * (CB + 1);  // float2
    static constexpr int YS = ST * (F + 1) > F * (CB + 1) ? ST * (F + 1) : F * (CB + 1);
    static constexpr int smem = (XS + YS + N + F) * 8 + 4 * kWarps * 8;
};

template <int N1, int N2, int F1, int F2, bool DERAMP>
__global__ void __launch_bounds__(kThreads, BigUpsampleGeom<N1, N2, F1, F2>::smem <= 113 * 1024 ? 2 : 1)
spec_refine_big_kernel(const float2* base, const long long* off, long long stride, const CoarseOut* coarse,
                       long long pair0, long long pairs, const long long* valid, const float2* twn_g,
                       const float2* twf_g, float2* ybuf, float* refined, long long refined_stride,
                       long long out_off)
{
    using G = BigUpsampleGeom<N1, N2, F1, F2>;
    constexpr int N = G::N, F = G::F, ST = G::ST, CB = G::CB;
    constexpr int RSN = N + 1, RSF = F + 1, CBS = CB + 1;
    extern __shared__ __align__(16) unsigned char rsm[];
    if (blockIdx.x >= pairs) return;
    const long long p = pair0 + blockIdx.x;
    if (valid[p] < 0) return;
    const float2* src = base + off[p];
    if (coarse) {
        const CoarseOut co = coarse[p];
        src += co.top * stride + co.left;
    }
    float2* X = reinterpret_cast<float2*>(rsm);
    float2* Y = X + G::XS;
    float2* twn = Y + G::YS;
    float2* twf = twn + N;
    double* red = reinterpret_cast<double*>(twf + F);
    float2* yg = ybuf + (long long)blockIdx.x * N * F;
    float* out = refined + (long long)blockIdx.x * refined_stride + out_off;
    const int tid = threadIdx.x;
    for (int q = tid; q < N; q += kThreads) twn[q] = __ldg(twn_g + q);
    for (int q = tid; q < F; q += kThreads) twf[q] = __ldg(twf_g + q);
    float ps = 0.0f, pl = 0.0f;
    if (DERAMP) deramp_phases_global(src, stride, N, red, ps, pl);
    // the tile's mean comes off as the strips are read and back on with the amplitudes
    const float2 mu = tile_mean<true, DERAMP>(src, stride, N, ps, pl, red);
    // rows, a strip at a time, into the buffer
    for (int r0 = 0; r0 < N; r0 += ST) {
        const int nr = N - r0 < ST ? N - r0 : ST;
        for (int t = tid; t < nr * N; t += kThreads) {
            const int y = t / N, x = t - y * N;
            float2 z = __ldg(src + (long long)(r0 + y) * stride + x);
            if (DERAMP) {
                float s, c;
                sincosf(fmaf(ps, (float)x, pl * (float)(r0 + y)), &s, &c);
                z = make_float2(fmaf(z.x, c, z.y * s), fmaf(z.y, c, -z.x * s));
            }
            X[y * RSN + x] = make_float2(z.x - mu.x, z.y - mu.y);
        }
        __syncthreads();
        for (int t = tid; t < nr * N2; t += kThreads) fft::fwd_a<N1, N2>(X + (t % nr) * RSN, 1, t / nr, twn);
        __syncthreads();
        for (int t = tid; t < nr * N1; t += kThreads) fft::step_b<N1, N2, -1>(X + (t % nr) * RSN, 1, t / nr);
        __syncthreads();
        for (int t = tid; t < nr * F1; t += kThreads)
            fft::step_b_pad<N1, N2, F1, F2>(X + (t % nr) * RSN, 1, Y + (t % nr) * RSF, 1, t / nr);
        __syncthreads();
        for (int t = tid; t < nr * F2; t += kThreads) fft::inv_a<F1, F2>(Y + (t % nr) * RSF, 1, t / nr, twf);
        __syncthreads();
        for (int t = tid; t < nr * F; t += kThreads) {
            const int y = t / F, x = t - y * F;
            yg[(long long)(r0 + y) * F + x] = Y[y * RSF + x];
        }
        __syncthreads();
    }
    // columns of the buffer, CB at a time
    const float scale = 1.0f / ((float)N * (float)N);
    for (int c0 = 0; c0 < F; c0 += CB) {
        const int nc = F - c0 < CB ? F - c0 : CB;
        for (int t = tid; t < N * CB; t += kThreads) {
            const int y = t / CB, cc = t - y * CB;
            if (cc < nc) X[y * CBS + cc] = yg[(long long)y * F + c0 + cc];
        }
        __syncthreads();
        for (int t = tid; t < CB * N2; t += kThreads) {
            const int cc = t % CB;
            if (cc < nc) fft::fwd_a<N1, N2>(X + cc, CBS, t / CB, twn);
        }
        __syncthreads();
        for (int t = tid; t < CB * N1; t += kThreads) {
            const int cc = t % CB;
            if (cc < nc) fft::step_b<N1, N2, -1>(X + cc, CBS, t / CB);
        }
        __syncthreads();
        for (int t = tid; t < CB * F1; t += kThreads) {
            const int cc = t % CB;
            if (cc < nc) fft::step_b_pad<N1, N2, F1, F2>(X + cc, CBS, Y + cc, CBS, t / CB);
        }
        __syncthreads();
        for (int t = tid; t < CB * F2; t += kThreads) {
            const int cc = t % CB;
            if (cc < nc) {
                float* col = out + c0 + cc;
                fft::inv_a_store<F1, F2>(Y + cc, CBS, t / CB, twf, [&](int n, float2 v) {
                    const float re = fmaf(v.x, scale, mu.x), im = fmaf(v.y, scale, mu.y);
                    col[(long long)n * F] = sqrtf(re * re + im * im);
                });
            }
        }
        __syncthreads();
    }
}

// refinement lengths of the strip kernel: N, N1, N2, F1, F2 (F = 2 N); 96 and up are too large for
// fft_upsample, the shorter ones may run either way (AMPCOR_REFINE_STRIPS)
#define AMPCOR_REFINE_BIG(X) \
    X(32, 4, 8, 8, 8)        \
    X(48, 6, 8, 8, 12)       \
    X(64, 8, 8, 8, 16)       \
    X(80, 8, 10, 10, 16)     \
    X(96, 8, 12, 12, 16)     \
    X(120, 8, 15, 15, 16)    \
    X(128, 8, 16, 16, 16)    \
    X(144, 12, 12, 12, 24)   \
    X(160, 10, 16, 16, 20)

}  // namespace

__global__ void detect_kernel(const float2* __restrict__ src, long long n, float* __restrict__ dst)
{
    const long long step = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += 4 * step) {
        float2 z[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const long long j = i + k * step;
            z[k] = j < n ? __ldg(src + j) : make_float2(0.0f, 0.0f);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const long long j = i + k * step;
            if (j < n) dst[j] = amp_of(z[k]);
        }
    }
}

__global__ void __launch_bounds__(256)
box_vsum_kernel(const float* __restrict__ a, long long samples, int R, long long row_lo,
                long long row_hi, double* __restrict__ v1, double* __restrict__ v2)
{
    const long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long y0 = row_lo + (long long)blockIdx.y * kVBlock;
    if (x >= samples || y0 >= row_hi) return;
    const long long y1 = y0 + kVBlock < row_hi ? y0 + kVBlock : row_hi;
    const float* col = a + x;
    double a1[4] = {0.0, 0.0, 0.0, 0.0}, a2[4] = {0.0, 0.0, 0.0, 0.0};
    int i = 0;
    for (; i + 4 <= R; i += 4) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double tv = __ldg(col + (y0 + i + k) * samples);
            a1[k] += tv;
            a2[k] += tv * tv;
        }
    }
    for (; i < R; ++i) {
        const double tv = __ldg(col + (y0 + i) * samples);
        a1[0] += tv;
        a2[0] += tv * tv;
    }
    double s1 = (a1[0] + a1[1]) + (a1[2] + a1[3]);
    double s2 = (a2[0] + a2[1]) + (a2[2] + a2[3]);
    for (long long y = y0; y < y1; ++y) {
        v1[y * samples + x] = s1;
        v2[y * samples + x] = s2;
        if (y + 1 < y1) {
            const double p = __ldg(col + (y + R) * samples), q = __ldg(col + y * samples);
            s1 += p - q;
            s2 += p * p - q * q;
        }
    }
}

// one CTA per box row: FP64 exclusive prefix sums of the row's column sums (in chunks of four per
// thread, a fixed order), then the box of every x from two prefix differences; two CTAs per SM,
// so that one row's loads overlap another's scan
__global__ void __launch_bounds__(kThreads, 2)
box_inv_kernel(const double* __restrict__ v1, const double* __restrict__ v2, long long row_lo,
               long long row_hi, long long samples, int R, float* __restrict__ inv)
{
    extern __shared__ __align__(16) double psm[];
    const long long y = row_lo + blockIdx.x;
    if (y >= row_hi) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* P1 = psm;
    double* P2 = psm + samples + 1;
    double* red = P2 + samples + 1;  // 2 x kWarps
    const double* r1 = v1 + y * samples;
    const double* r2 = v2 + y * samples;
    double carry1 = 0.0, carry2 = 0.0;
    constexpr int kPer = 4;  // consecutive samples per thread and chunk
    for (long long c0 = 0; c0 < samples; c0 += kThreads * kPer) {
        const long long b0 = c0 + (long long)tid * kPer;
        double l1[kPer], l2[kPer], s1 = 0.0, s2 = 0.0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const long long i = b0 + k;
            const double p = i < samples ? __ldg(r1 + i) : 0.0;
            const double q = i < samples ? __ldg(r2 + i) : 0.0;
            l1[k] = s1;
            l2[k] = s2;
            s1 += p;
            s2 += q;
        }
        // exclusive scan of the thread totals: within the warp, then across warps
        double i1 = s1, i2 = s2;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double u1 = __shfl_up_sync(kFull, i1, o), u2 = __shfl_up_sync(kFull, i2, o);
            if (lane >= o) {
                i1 += u1;
                i2 += u2;
            }
        }
        if (lane == 31) {
            red[warp] = i1;
            red[kWarps + warp] = i2;
        }
        __syncthreads();
        double w1 = 0.0, w2 = 0.0, t1 = 0.0, t2 = 0.0;
        for (int w = 0; w < kWarps; ++w) {
            if (w < warp) {
                w1 += red[w];
                w2 += red[kWarps + w];
            }
            t1 += red[w];
            t2 += red[kWarps + w];
        }
        const double o1 = carry1 + w1 + (i1 - s1), o2 = carry2 + w2 + (i2 - s2);
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const long long i = b0 + k;
            if (i < samples) {
                P1[i] = o1 + l1[k];
                P2[i] = o2 + l2[k];
            }
        }
        carry1 += t1;
        carry2 += t2;
        __syncthreads();
    }
    if (tid == 0) {
        P1[samples] = carry1;
        P2[samples] = carry2;
    }
    __syncthreads();
    const double cells = (double)R * (double)R;
    for (long long x = tid; x + R <= samples; x += kThreads) {
        const double b1 = P1[x + R] - P1[x];
        const double b2 = P2[x + R] - P2[x];
        const float var = (float)(b2 - b1 * b1 / cells);
        inv[y * samples + x] = var > 0.0f ? __frsqrt_rn(var) : 0.0f;
    }
}

bool spec_radices(int n, int& n1, int& n2)
{
#define AMPCOR_SPEC_CASE(NN, A, B) \
    if (n == NN) {                 \
        n1 = A;                    \
        n2 = B;                    \
        return true;               \
    }
    AMPCOR_SPEC_LENGTHS(AMPCOR_SPEC_CASE)
#undef AMPCOR_SPEC_CASE
    return false;
}

int spec_next_length(int w)
{
#define AMPCOR_SPEC_CASE(NN, A, B) \
    if (w <= NN) return NN;
    AMPCOR_SPEC_LENGTHS(AMPCOR_SPEC_CASE)
#undef AMPCOR_SPEC_CASE
    return 0;
}

bool spec_refine_supported(int n, int f, int& smem)
{
    if (f != 2) return false;
#define AMPCOR_REFINE_CASE(NN, A, B, C, D)                \
    if (n == NN) {                                        \
        smem = UpsampleGeom<A, B, C, D>::smem;           \
        return smem <= 227 * 1024;                        \
    }
    AMPCOR_REFINE_PAIRS(AMPCOR_REFINE_CASE)
#undef AMPCOR_REFINE_CASE
    return false;
}

bool spec_refine_big_supported(int n, int f, int& smem)
{
    if (f != 2) return false;
#define AMPCOR_REFINE_CASE(NN, A, B, C, D)              \
    if (n == NN) {                                      \
        smem = BigUpsampleGeom<A, B, C, D>::smem;       \
        return smem <= 227 * 1024;                      \
    }
    AMPCOR_REFINE_BIG(AMPCOR_REFINE_CASE)
#undef AMPCOR_REFINE_CASE
    return false;
}

cudaError_t launch_spec_refine(int n, unsigned blocks, cudaStream_t st, const float2* base,
                               const long long* off, long long stride, const CoarseOut* coarse,
                               long long pair0, long long pairs, const long long* valid,
                               const float2* twn, const float2* twf, float* refined,
                               long long refined_stride, long long out_off, int deramp,
                               float2* ybuf, bool strips)
{
    int small_smem = 0;
    if ((strips || !spec_refine_supported(n, 2, small_smem)) && ybuf) {
#define AMPCOR_REFINE_CASE(NN, A, B, C, D)                                                              \
        if (n == NN) {                                                                                  \
            if (deramp)                                                                                 \
                spec_refine_big_kernel<A, B, C, D, true><<<blocks, kThreads, BigUpsampleGeom<A, B, C, D>::smem, st>>>( \
                    base, off, stride, coarse, pair0, pairs, valid, twn, twf, ybuf, refined, refined_stride, out_off); \
            else                                                                                        \
                spec_refine_big_kernel<A, B, C, D, false><<<blocks, kThreads, BigUpsampleGeom<A, B, C, D>::smem, st>>>( \
                    base, off, stride, coarse, pair0, pairs, valid, twn, twf, ybuf, refined, refined_stride, out_off); \
            return cudaGetLastError();                                                                  \
        }
        AMPCOR_REFINE_BIG(AMPCOR_REFINE_CASE)
#undef AMPCOR_REFINE_CASE
        return cudaErrorInvalidValue;
    }
#define AMPCOR_REFINE_CASE(NN, A, B, C, D)                                                           \
    if (n == NN) {                                                                                   \
        constexpr int smem = UpsampleGeom<A, B, C, D>::smem;                                         \
        if (deramp)                                                                                  \
            spec_refine_kernel<A, B, C, D, true><<<blocks, kThreads, smem, st>>>(                    \
                base, off, stride, coarse, pair0, pairs, valid, twn, twf, refined, refined_stride, out_off); \
        else                                                                                         \
            spec_refine_kernel<A, B, C, D, false><<<blocks, kThreads, smem, st>>>(                   \
                base, off, stride, coarse, pair0, pairs, valid, twn, twf, refined, refined_stride, out_off); \
        return cudaGetLastError();                                                                   \
    }
    AMPCOR_REFINE_PAIRS(AMPCOR_REFINE_CASE)
#undef AMPCOR_REFINE_CASE
    return cudaErrorInvalidValue;
}

bool spec_refine_staged_supported(int n, int f, int& smem, int& box_x)
{
    smem = box_x = 0;
    if (f != 2) return false;
#define AMPCOR_REFINE_CASE(NN, A, B, C, D)                        \
    if (n == NN) {                                                \
        smem = UpsampleGeom<A, B, C, D>::smem_staged;             \
        box_x = UpsampleGeom<A, B, C, D>::SWS;                    \
        return smem <= 227 * 1024 && box_x <= 256;                \
    }
    AMPCOR_REFINE_PAIRS(AMPCOR_REFINE_CASE)
#undef AMPCOR_REFINE_CASE
    return false;
}

cudaError_t launch_spec_refine_staged(int n, unsigned sms, cudaStream_t st, const CUtensorMap* tmap,
                                      const long long* off, long long stride, const CoarseOut* coarse,
                                      long long pair0, long long pairs, const long long* valid,
                                      const float2* twn, const float2* twf, float* refined,
                                      long long refined_stride, long long out_off, unsigned int* errs)
{
    if (pairs <= 0) return cudaSuccess;
    const unsigned blocks = (unsigned)std::min<long long>(pairs, std::max(1u, sms));
#define AMPCOR_REFINE_CASE(NN, A, B, C, D)                                                           \
    if (n == NN) {                                                                                   \
        spec_refine_staged_kernel<A, B, C, D><<<blocks, kThreads, UpsampleGeom<A, B, C, D>::smem_staged, st>>>( \
            *tmap, off, stride, coarse, pair0, pairs, valid, twn, twf, refined, refined_stride, out_off, errs); \
        return cudaGetLastError();                                                                   \
    }
    AMPCOR_REFINE_PAIRS(AMPCOR_REFINE_CASE)
#undef AMPCOR_REFINE_CASE
    return cudaErrorInvalidValue;
}

cudaError_t spec_set_smem_limits()
{
    const int limit = 227 * 1024;
    cudaError_t e = cudaFuncSetAttribute(box_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
#define AMPCOR_REFINE_CASE(NN, A, B, C, D) \
    if (e == cudaSuccess)                  \
        e = cudaFuncSetAttribute(spec_refine_kernel<A, B, C, D, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit); \
    if (e == cudaSuccess)                  \
        e = cudaFuncSetAttribute(spec_refine_kernel<A, B, C, D, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit); \
    if (e == cudaSuccess && UpsampleGeom<A, B, C, D>::smem_staged <= limit) \
        e = cudaFuncSetAttribute(spec_refine_staged_kernel<A, B, C, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
    AMPCOR_REFINE_PAIRS(AMPCOR_REFINE_CASE)
#undef AMPCOR_REFINE_CASE
#define AMPCOR_SPEC_CASE(NN, A, B) \
    if (e == cudaSuccess)          \
        e = cudaFuncSetAttribute(spec_kernel<A, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit); \
    if (e == cudaSuccess)          \
        e = cudaFuncSetAttribute(spec_staged_kernel<A, B, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit); \
    if (e == cudaSuccess)          \
        e = cudaFuncSetAttribute(spec_staged_kernel<A, B, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit); \
    if (e == cudaSuccess)          \
        e = cudaFuncSetAttribute(spec_block_kernel<A, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
    AMPCOR_SPEC_LENGTHS(AMPCOR_SPEC_CASE)
#undef AMPCOR_SPEC_CASE
#define AMPCOR_REFINE_CASE(NN, A, B, C, D) \
    if (e == cudaSuccess)                  \
        e = cudaFuncSetAttribute(spec_refine_big_kernel<A, B, C, D, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit); \
    if (e == cudaSuccess)                  \
        e = cudaFuncSetAttribute(spec_refine_big_kernel<A, B, C, D, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
    AMPCOR_REFINE_BIG(AMPCOR_REFINE_CASE)
#undef AMPCOR_REFINE_CASE
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(spec_reduce_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(spec_tile_stats_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
    return e;
}

cudaError_t launch_spec_chip_stats(unsigned blocks, cudaStream_t st, SpecSource src, long long pair0,
                                   long long pairs, const long long* valid, int R, ChipStat* out)
{
    spec_chip_stats_kernel<<<blocks, 256, 0, st>>>(src, pair0, pairs, valid, R, out);
    return cudaGetLastError();
}

// placement rows per pass of the tile statistics (two CTAs per SM where the window allows) and
// the shared memory that takes; 0 when the window is wider than a CTA has threads
int spec_tile_stats_rows(int W, int C, int& smem)
{
    smem = 0;
    if (W > kThreads || C < 1) return 0;
    // window_stats_xs hands each placement row of a pass to one warp
    int sr = C < kWarps ? C : kWarps;
    while (sr > 1 && 2L * sr * (W + 1) * 8 > 110L * 1024) --sr;
    smem = (int)(2L * sr * (W + 1) * 8);
    return smem <= 227 * 1024 ? sr : 0;
}

cudaError_t launch_spec_tile_stats(unsigned blocks, cudaStream_t st, SpecSource src, long long pair0,
                                   long long pairs, const long long* valid, int R, int W, float* inv)
{
    int smem = 0;
    const int sr = spec_tile_stats_rows(W, W - R + 1, smem);
    if (!sr) return cudaErrorInvalidValue;
    spec_tile_stats_kernel<<<blocks, kThreads, smem, st>>>(src, pair0, pairs, valid, R, W, sr, inv);
    return cudaGetLastError();
}

cudaError_t launch_spec_block(const SpecGeom& tile, int nb, unsigned blocks, cudaStream_t st,
                              SpecSource src, long long pair0, long long pairs,
                              const long long* valid, const ChipStat* cstat, const float2* tw,
                              float* part, double* scal)
{
#define AMPCOR_SPEC_CASE(NN, A, B)                                                                   \
    if (tile.N == NN) {                                                                              \
        spec_block_kernel<A, B><<<blocks, kSpecThreads, tile.smem_bytes, st>>>(src, pair0, pairs, valid, \
                                                                           tile, nb, cstat, tw, part, scal); \
        return cudaGetLastError();                                                                   \
    }
    AMPCOR_SPEC_LENGTHS(AMPCOR_SPEC_CASE)
#undef AMPCOR_SPEC_CASE
    return cudaErrorInvalidValue;
}

int spec_reduce_smem(int C)
{
    return 2 * ((C * C + 3) & ~3) * 4 + 256;
}

cudaError_t launch_spec_reduce(const SpecGeom& full, int K, unsigned blocks, cudaStream_t st,
                               SpecSource src, long long pair0, long long pairs,
                               const long long* valid, const ChipStat* cstat, InvSource inv,
                               const float* part, const double* scal, SpecOut out)
{
    spec_reduce_kernel<<<blocks, kThreads, spec_reduce_smem(full.C), st>>>(src, pair0, pairs, valid, full, K,
                                                                           cstat, inv, part, scal, out);
    return cudaGetLastError();
}


cudaError_t launch_spec(const SpecGeom& g, unsigned blocks, cudaStream_t st, SpecSource src,
                        long long pair0, long long pairs, const long long* valid, InvSource inv,
                        const float2* tw, SpecOut out)
{
#define AMPCOR_SPEC_CASE(NN, A, B)                                                               \
    if (g.N == NN) {                                                                             \
        spec_kernel<A, B><<<blocks, kSpecThreads, g.smem_bytes, st>>>(src, pair0, pairs, valid, g,  \
                                                                  inv, tw, out);                 \
        return cudaGetLastError();                                                               \
    }
    AMPCOR_SPEC_LENGTHS(AMPCOR_SPEC_CASE)
#undef AMPCOR_SPEC_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_spec_staged(const SpecGeom& g, unsigned sms, cudaStream_t st, SpecSource src,
                               long long pair0, long long pairs, const long long* valid, InvSource inv,
                               const float2* tw, SpecOut out, unsigned int* errs, const CUtensorMap* wmap,
                               const CUtensorMap* cmap, const CUtensorMap* imap, int stall)
{
    if (pairs <= 0) return cudaSuccess;
    const unsigned blocks = (unsigned)std::min<long long>(pairs, std::max(1u, sms));
#define AMPCOR_SPEC_CASE(NN, A, B)                                                                      \
    if (g.N == NN) {                                                                                    \
        if (wmap)                                                                                       \
            spec_staged_kernel<A, B, true><<<blocks, kSpecThreads, g.smem_staged, st>>>(                      \
                src, pair0, pairs, valid, g, inv, tw, out, errs, *wmap, *cmap, *imap, stall);               \
        else                                                                                            \
            spec_staged_kernel<A, B, false><<<blocks, kSpecThreads, g.smem_staged, st>>>(                     \
                src, pair0, pairs, valid, g, inv, tw, out, errs, CUtensorMap{}, CUtensorMap{}, CUtensorMap{},  \
                stall);                                                                             \
        return cudaGetLastError();                                                                      \
    }
    AMPCOR_SPEC_LENGTHS(AMPCOR_SPEC_CASE)
#undef AMPCOR_SPEC_CASE
    return cudaErrorInvalidValue;
}

}  // namespace ampcor_b200
