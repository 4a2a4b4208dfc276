// sm_100a kernels of the batched tile correlator (plain FP32 form).
//
// One CTA of 512 threads owns one tile pair at a time and keeps both of its tiles resident in
// shared memory; nothing but the tile sources, the per-pair results and (between the refine and
// fine kernels) the refined amplitudes travels through HBM.  The reference instead stages every
// intermediate (amplitudes, SATs, means, correlation surfaces, a zero-padded complex copy of every
// surface for the zoom) in managed memory and correlates with one kernel launch per placement
// (lib/libampcor_cuda/correlators/correlate.cu:69-135).
//
// Correlation numerator.  For a placement (u, v) the numerator is sum_ij r'(i,j) t(u+i, v+j),
// with r' the zero-mean chip.  The reference subtracts the placement mean from t inside the sum
// (correlate.cu:213-225); because sum r' = 0 that term vanishes and the mean only enters the
// denominator, which is computed from FP64 box sums of t and t^2.  A thread owns one placement
// row u and a block of NV consecutive placement columns; it walks the chip row by row and, along a
// row, slides a register window of NV window samples, so every shared-memory load of a window
// sample feeds NV fused multiply-adds and the chip value is a broadcast load.  Placement rows come
// in blocks of 32 (one per lane, "main" tasks, chip rows split over warps); the odd rows left
// over (C = 2M+1 is odd) are "leftover" tasks where the lanes split the chip rows instead and a
// butterfly sums them.  Shared-memory row strides are odd so that both lane layouts are free of
// bank conflicts.  Partial sums are combined in a fixed order, so every result is bitwise
// independent of what else runs on the device.
#include "kernels.cuh"
#include "tile_common.cuh"

#include <float.h>
#include <limits.h>
#include <math.h>

namespace ampcor_b200 {

namespace {

// ------------------------------------------------------------------------------------------
// correlation numerator: register sliding window along one chip row
// ------------------------------------------------------------------------------------------

// acc[k] += sum_j c[j] * w[j + k] for k < NV and j < steps*NV; c is zero past the chip width.
// x is a ring: at inner step jj of a stride, slot (jj+k) % NV holds w[s*NV + jj + k].
template <int NV>
__device__ __forceinline__ void accum_row(const float* __restrict__ w, const float* __restrict__ c,
                                          int steps, float (&acc)[kSlot])
{
    float x[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) x[k] = w[k];
    for (int s = 0; s < steps; ++s) {
        const float* wn = w + s * NV + NV;
        const float* cs = c + s * NV;
#pragma unroll
        for (int jj = 0; jj < NV; ++jj) {
            const float cv = cs[jj];
#pragma unroll
            for (int k = 0; k < NV; ++k) acc[k] = fmaf(cv, x[(jj + k) % NV], acc[k]);
            x[jj] = wn[jj];
        }
    }
}

template <int NV>
__device__ __forceinline__ void accum_rows(const float* w, int S, const float* c, int CS, int i0,
                                           int i1, int steps, float (&acc)[kSlot])
{
    for (int i = i0; i < i1; ++i) accum_row<NV>(w + i * S, c + i * CS, steps, acc);
}

// the register block widths that are compiled; the planner rounds block widths up to one
__device__ __forceinline__ void accum_dispatch(int nv, const float* w, int S, const float* c,
                                               int CS, int i0, int i1, int steps,
                                               float (&acc)[kSlot])
{
    switch (nv) {
        case 33: accum_rows<33>(w, S, c, CS, i0, i1, steps, acc); break;
        case 32: accum_rows<32>(w, S, c, CS, i0, i1, steps, acc); break;
        case 17: accum_rows<17>(w, S, c, CS, i0, i1, steps, acc); break;
        case 16: accum_rows<16>(w, S, c, CS, i0, i1, steps, acc); break;
        case 9: accum_rows<9>(w, S, c, CS, i0, i1, steps, acc); break;
        default: break;
    }
}

// ------------------------------------------------------------------------------------------
// tile staging and statistics
// ------------------------------------------------------------------------------------------

// rows x cols complex64 tile -> amplitudes, row stride sstride floats, zero past the tile width
__device__ void stage_cplx(float* dst, int rows, int cols, int sstride,
                           const float2* __restrict__ src, long long src_stride)
{
    const int total = rows * sstride;
    for (int idx = threadIdx.x; idx < total; idx += kThreads) {
        const int r = idx / sstride, c = idx - r * sstride;
        dst[idx] = (c < cols) ? amp_of(__ldg(src + r * src_stride + c)) : 0.0f;
    }
}

// rows x cols amplitude tile (dense, row stride cols) -> shared memory, zero past the width
__device__ void stage_real(float* dst, int rows, int cols, int sstride,
                           const float* __restrict__ src)
{
    const int total = rows * sstride;
    for (int idx = threadIdx.x; idx < total; idx += kThreads) {
        const int r = idx / sstride, c = idx - r * sstride;
        dst[idx] = (c < cols) ? __ldg(src + r * cols + c) : 0.0f;
    }
}

// chip amplitudes (already staged, padded with zeros) -> zero mean in place; returns 1/|r'|
// (refStats.cu:118-302, with FP64 accumulation)
__device__ double chip_stats(float* chip, const NccGeom& g, double* red)
{
    const int total = g.R * g.CS;
    double s = 0.0;
    for (int idx = threadIdx.x; idx < total; idx += kThreads) s += chip[idx];
    s = block_sum(s, red);
    const double mean = s / ((double)g.R * (double)g.R);
    double ss = 0.0;
    for (int idx = threadIdx.x; idx < total; idx += kThreads) {
        const int c = idx % g.CS;
        if (c < g.R) {
            const float rp = (float)((double)chip[idx] - mean);
            chip[idx] = rp;
            ss += (double)rp * (double)rp;
        }
    }
    ss = block_sum(ss, red);
    return ss > 0.0 ? 1.0 / sqrt(ss) : 0.0;
}

// The staged window less its smallest sample c: sum r' (t - c) = sum r' t since sum r' = 0.
// Amplitudes are non-negative, so 0 <= t - c <= t: no term grows, a window that holds a zero
// sample is left as it is (an all-zero box keeps a numerator of exactly zero), and under a strong
// steady return the FP32 numerators round on the window's variation, not on its level.  red:
// kWarps doubles; ends with a barrier.
__device__ void shift_window(float* win, const NccGeom& g, double* red)
{
    float m = INFINITY;
    for (int idx = threadIdx.x; idx < g.W * g.W; idx += kThreads) {
        const int r = idx / g.W, col = idx - r * g.W;
        m = fminf(m, win[r * g.S + col]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(kFull, m, o));
    float* rf = reinterpret_cast<float*>(red);
    if ((threadIdx.x & 31) == 0) rf[threadIdx.x >> 5] = m;
    __syncthreads();
    float c = rf[0];
    for (int w = 1; w < kWarps; ++w) c = fminf(c, rf[w]);
    __syncthreads();
    for (int idx = threadIdx.x; idx < g.W * g.W; idx += kThreads) {
        const int r = idx / g.W, col = idx - r * g.W;
        win[r * g.S + col] -= c;
    }
    __syncthreads();
}

// the correlation surface gamma (C x C) from the staged window, the zero-mean chip and the
// placement statistics; the window region is reused for the partial sums
__device__ void ncc_surface(const NccGeom& g, float* smem, float inv_sigma)
{
    const float* win = smem + g.off_win;
    const float* chip = smem + g.off_chip;
    const float* inv = smem + g.off_inv;
    float* gam = smem + g.off_gam;
    float* trans = smem + g.off_trans;
    float* part = smem + g.off_win;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int C = g.C, S = g.S, CS = g.CS;

    // leftover placement rows: lanes split the chip rows, a butterfly sums them
    for (int t = warp; t < g.n_trans; t += kWarps) {
        const int kc = t % g.n_tkc;
        const int rest = t / g.n_tkc;
        const int vb = rest % g.n_vb;
        const int u = 32 * g.n_ub + rest / g.n_vb;
        const int i = kc * 32 + lane;
        float acc[kSlot];
#pragma unroll
        for (int k = 0; k < kSlot; ++k) acc[k] = 0.0f;
        if (i < g.R)
            accum_dispatch(g.vb_nv[vb], win + u * S + g.vb_v0[vb], S, chip, CS, i, i + 1,
                           g.vb_steps[vb], acc);
#pragma unroll
        for (int k = 0; k < kSlot; ++k) {
            float v = acc[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
            if (lane == 0) trans[t * kSlot + k] = v;
        }
    }

    // main tasks: one placement row per lane, the chip rows of one chunk
    float acc[kSlot];
#pragma unroll
    for (int k = 0; k < kSlot; ++k) acc[k] = 0.0f;
    if (warp < g.n_main) {
        const int kc = warp % g.n_kc;
        const int rest = warp / g.n_kc;
        const int vb = rest % g.n_vb;
        const int ub = rest / g.n_vb;
        const int u = ub * 32 + lane;
        const int i0 = kc * g.R / g.n_kc, i1 = (kc + 1) * g.R / g.n_kc;
        accum_dispatch(g.vb_nv[vb], win + u * S + g.vb_v0[vb], S, chip, CS, i0, i1,
                       g.vb_steps[vb], acc);
    }
    __syncthreads();  // the window is dead from here on: its space takes the partial sums
    if (warp < g.n_main) {
        float* slot = part + (warp * 32 + lane) * kSlot;
#pragma unroll
        for (int k = 0; k < kSlot; ++k) slot[k] = acc[k];
    }
    __syncthreads();

    // combine the partial sums in a fixed order and normalise
    for (int idx = threadIdx.x; idx < C * C; idx += kThreads) {
        const int u = idx / C, v = idx - u * C;
        int vb = 0;
        while (vb + 1 < g.n_vb && v >= g.vb_v0[vb + 1]) ++vb;
        const int k = v - g.vb_v0[vb];
        float num = 0.0f;
        if (u < 32 * g.n_ub) {
            const int base = ((u >> 5) * g.n_vb + vb) * g.n_kc;
            const int ln = u & 31;
            for (int kc = 0; kc < g.n_kc; ++kc) num += part[((base + kc) * 32 + ln) * kSlot + k];
        } else {
            const int base = ((u - 32 * g.n_ub) * g.n_vb + vb) * g.n_tkc;
            for (int kc = 0; kc < g.n_tkc; ++kc) num += trans[(base + kc) * kSlot + k];
        }
        gam[idx] = num * inv[idx] * inv_sigma;
    }
    __syncthreads();
}

__device__ void surface_argmax(const float* gam, int n, float* smem_red, float& bv, int& bi)
{
    bv = -INFINITY;
    bi = INT_MAX;
    for (int idx = threadIdx.x; idx < n; idx += kThreads) better(bv, bi, gam[idx], idx);
    block_argmax(bv, bi, smem_red, reinterpret_cast<int*>(smem_red + kWarps));
}

// ------------------------------------------------------------------------------------------
// band-limited interpolation by matrix: out[q] = sum_k' taps[q + k'] in[N-1-k'] for a block of
// kQB consecutive outputs (the taps slide through a register ring, the samples are per lane)
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ void interp_ring(const float* __restrict__ tp,
                                            const float2* __restrict__ xb, int xstride, int N,
                                            float (&ar)[kQB], float (&ai)[kQB])
{
    float t[kQB];
#pragma unroll
    for (int q = 0; q < kQB; ++q) t[q] = tp[q];
    for (int s = 0; s < N / kQB; ++s) {
        const float* tn = tp + s * kQB + kQB;
        const float2* xs = xb + (long long)(s * kQB) * xstride;
#pragma unroll
        for (int jj = 0; jj < kQB; ++jj) {
            const float2 xv = xs[jj * xstride];
#pragma unroll
            for (int q = 0; q < kQB; ++q) {
                ar[q] = fmaf(t[(jj + q) % kQB], xv.x, ar[q]);
                ai[q] = fmaf(t[(jj + q) % kQB], xv.y, ai[q]);
            }
            t[jj] = tn[jj];
        }
    }
}

// upsample the complex N x N tile at src by f and write the amplitudes (F x F, dense) to out
__device__ void interp_tile(const float2* __restrict__ src, long long src_stride,
                            const InterpGeom& ig, const float* __restrict__ taps_g, float* smem,
                            float* __restrict__ out, int deramp)
{
    float2* X = reinterpret_cast<float2*>(smem + ig.off_x);
    float2* Y = reinterpret_cast<float2*>(smem + ig.off_y);
    float* taps = smem + ig.off_taps;
    const int N = ig.N, f = ig.f, F = ig.F, NS = ig.NS, YS = ig.YS;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    for (int idx = threadIdx.x; idx < (f - 1) * ig.taps_len; idx += kThreads)
        taps[idx] = __ldg(taps_g + idx);
    for (int idx = threadIdx.x; idx < N * N; idx += kThreads) {
        const int r = idx / N, c = idx - r * N;
        X[r * NS + c] = __ldg(src + r * src_stride + c);
    }
    __syncthreads();
    // the row-interpolated buffer is free until the rows are written: the deramp's scratch
    if (deramp) deramp_tile(X, NS, N, reinterpret_cast<double*>(Y));
    // the tile's mean off before the interpolation (which keeps a constant as it is), back on
    // with the amplitudes, so that the FP32 sums round on the tile's variation
    const float2 mu = tile_mean<false, false>(X, NS, N, 0.0f, 0.0f, reinterpret_cast<double*>(Y));
    for (int idx = threadIdx.x; idx < N * N; idx += kThreads) {
        const int r = idx / N, c = idx - r * N;
        const float2 z = X[r * NS + c];
        X[r * NS + c] = make_float2(z.x - mu.x, z.y - mu.y);
    }
    __syncthreads();

    // rows: Y[e][f q] = X[e][q], Y[e][f q + s] interpolated
    for (int idx = threadIdx.x; idx < N * N; idx += kThreads) {
        const int e = idx / N, q = idx - e * N;
        Y[e * YS + f * q] = X[e * NS + q];
    }
    const int nqb = N / kQB, neb = (N + 31) / 32;
    for (int t = warp; t < (f - 1) * nqb * neb; t += kWarps) {
        const int eb = t % neb;
        const int rest = t / neb;
        const int q0 = (rest % nqb) * kQB;
        const int s = 1 + rest / nqb;
        const int e = eb * 32 + lane;
        if (e < N) {
            float ar[kQB], ai[kQB];
#pragma unroll
            for (int q = 0; q < kQB; ++q) ar[q] = ai[q] = 0.0f;
            interp_ring(taps + (s - 1) * ig.taps_len + q0, X + e * NS + (N - 1), -1, N, ar, ai);
#pragma unroll
            for (int q = 0; q < kQB; ++q) Y[e * YS + f * (q0 + q) + s] = make_float2(ar[q], ai[q]);
        }
    }
    __syncthreads();

    // columns: out[f q][p] = |Y[q][p]|, out[f q + s][p] interpolated
    for (int idx = threadIdx.x; idx < N * F; idx += kThreads) {
        const int q = idx / F, p = idx - q * F;
        const float2 y = Y[q * YS + p];
        const float re = y.x + mu.x, im = y.y + mu.y;
        out[(long long)(f * q) * F + p] = sqrtf(re * re + im * im);
    }
    const int npb = (F + 31) / 32;
    for (int t = warp; t < (f - 1) * nqb * npb; t += kWarps) {
        const int pb = t % npb;
        const int rest = t / npb;
        const int q0 = (rest % nqb) * kQB;
        const int s = 1 + rest / nqb;
        const int p = pb * 32 + lane;
        if (p < F) {
            float ar[kQB], ai[kQB];
#pragma unroll
            for (int q = 0; q < kQB; ++q) ar[q] = ai[q] = 0.0f;
            interp_ring(taps + (s - 1) * ig.taps_len + q0, Y + (N - 1) * YS + p, -YS, N, ar, ai);
#pragma unroll
            for (int q = 0; q < kQB; ++q) {
                const float re = ar[q] + mu.x, im = ai[q] + mu.y;
                out[(long long)(f * (q0 + q) + s) * F + p] = sqrtf(re * re + im * im);
            }
        }
    }
    __syncthreads();
}

// ------------------------------------------------------------------------------------------
// zoom: Z x Z band-limited interpolation of the Cf x Cf refined surface, reduced straight to its
// first maximum (the surface itself is never stored)
// ------------------------------------------------------------------------------------------

template <int CB>
__device__ __forceinline__ void zoom_rows(const float* __restrict__ tp, const float* __restrict__ tcol,
                                          int Z, int Cf, float (&acc)[CB])
{
    float t[CB];
#pragma unroll
    for (int c = 0; c < CB; ++c) t[c] = tp[c];
    for (int s = 0; s < Cf / CB; ++s) {
        const float* tn = tp + s * CB + CB;
#pragma unroll
        for (int jj = 0; jj < CB; ++jj) {
            const float xv = tcol[-(s * CB + jj) * Z];
#pragma unroll
            for (int c = 0; c < CB; ++c) acc[c] = fmaf(t[(jj + c) % CB], xv, acc[c]);
            t[jj] = tn[jj];
        }
    }
}

template <int CB>
__device__ void zoom_argmax_cb(const float* T, const float* taps, const ZoomGeom& zg, float& bv,
                               int& bi)
{
    const int Cf = zg.Cf, z = zg.z, Z = zg.Z;
    const int ncb = Cf / CB;
    const int items = z * ncb * Z;
    for (int it = threadIdx.x; it < items; it += kThreads) {
        const int q = it % Z;
        const int rest = it / Z;
        const int c0 = (rest % ncb) * CB;
        const int s = rest / ncb;
        if (s == 0) {
#pragma unroll
            for (int c = 0; c < CB; ++c) better(bv, bi, T[(c0 + c) * Z + q], (z * (c0 + c)) * Z + q);
        } else {
            float acc[CB];
#pragma unroll
            for (int c = 0; c < CB; ++c) acc[c] = 0.0f;
            zoom_rows<CB>(taps + s * zg.taps_len + c0, T + (Cf - 1) * Z + q, Z, Cf, acc);
#pragma unroll
            for (int c = 0; c < CB; ++c) better(bv, bi, acc[c], (z * (c0 + c) + s) * Z + q);
        }
    }
}

__device__ void zoom_argmax(const float* G, float* T, const float* taps, const ZoomGeom& zg,
                            float& bv, int& bi)
{
    const int Cf = zg.Cf, z = zg.z, Z = zg.Z;
    // T[a][z b + s] = sum_l D(b + s/z - l) G[a][l]
    for (int idx = threadIdx.x; idx < Cf * Z; idx += kThreads) {
        const int a = idx / Z, q = idx - a * Z;
        const int b = q / z, s = q - b * z;
        if (s == 0) {
            T[idx] = G[a * Cf + b];
        } else {
            const float* tp = taps + s * zg.taps_len + b + Cf - 1;
            const float* gr = G + a * Cf;
            float acc = 0.0f;
            for (int l = 0; l < Cf; ++l) acc = fmaf(tp[-l], gr[l], acc);
            T[idx] = acc;
        }
    }
    __syncthreads();
    bv = -INFINITY;
    bi = INT_MAX;
    switch (zg.cb) {
        case 17: zoom_argmax_cb<17>(T, taps, zg, bv, bi); break;
        case 13: zoom_argmax_cb<13>(T, taps, zg, bv, bi); break;
        case 11: zoom_argmax_cb<11>(T, taps, zg, bv, bi); break;
        case 5: zoom_argmax_cb<5>(T, taps, zg, bv, bi); break;
        case 3: zoom_argmax_cb<3>(T, taps, zg, bv, bi); break;
        default: zoom_argmax_cb<1>(T, taps, zg, bv, bi); break;
    }
}

}  // namespace

// ------------------------------------------------------------------------------------------
// kernels
// ------------------------------------------------------------------------------------------

// tile offsets of every pair from the upper-left corners of chip and window in two rasters;
// pairs whose tiles leave their raster get offset -1 (skipped downstream) and are counted
__global__ void pair_offsets_kernel(const int* ulhc, long long pairs, long long ref_lines,
                                    long long ref_samples, long long tgt_lines,
                                    long long tgt_samples, int R, int W, long long* ref_off,
                                    long long* tgt_off, unsigned int* bad)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pairs) return;
    const long long rl = ulhc[4 * p], rs = ulhc[4 * p + 1];
    const long long tl = ulhc[4 * p + 2], ts = ulhc[4 * p + 3];
    const bool ok = rl >= 0 && rs >= 0 && rl + R <= ref_lines && rs + R <= ref_samples &&
                    tl >= 0 && ts >= 0 && tl + W <= tgt_lines && ts + W <= tgt_samples;
    ref_off[p] = ok ? rl * ref_samples + rs : -1;
    tgt_off[p] = ok ? tl * tgt_samples + ts : -1;
    if (!ok) atomicAdd(bad, 1u);
}

// tile offsets in the arena of the reference worker: pair p holds [chip R^2 | window W^2]
// (lib/libampcor_cuda/correlators/Sequential.icc:15-44)
__global__ void arena_offsets_kernel(long long pairs, long long ref_cells, long long tgt_cells,
                                     long long* ref_off, long long* tgt_off)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pairs) return;
    ref_off[p] = p * (ref_cells + tgt_cells);
    tgt_off[p] = p * (ref_cells + tgt_cells) + ref_cells;
}

__global__ void __launch_bounds__(kThreads, 1)
coarse_kernel(PairSource src, long long pair0, long long pairs, NccGeom g, int m, CoarseOut* out,
              float* coarse_peak, float* surfaces)
{
    extern __shared__ __align__(16) float smem[];
    const long long p = pair0 + blockIdx.x;
    if (blockIdx.x >= pairs) return;
    const long long roff = src.ref_off[p], toff = src.tgt_off[p];
    if (roff < 0 || toff < 0) {
        if (threadIdx.x == 0) {
            out[p] = CoarseOut{-1, -1, -1, -1};
            coarse_peak[p] = NAN;
        }
        return;
    }
    float* win = smem + g.off_win;
    float* chip = smem + g.off_chip;
    float* inv = smem + g.off_inv;
    float* gam = smem + g.off_gam;
    double* red = reinterpret_cast<double*>(smem + g.off_red);

    stage_cplx(win, g.W, g.W, g.S, src.tgt_base + toff, src.tgt_stride);
    __syncthreads();
    window_stats(win, g, inv, reinterpret_cast<double*>(chip));
    stage_cplx(chip, g.R, g.R, g.CS, src.ref_base + roff, src.ref_stride);
    const double inv_sigma = chip_stats(chip, g, red);
    shift_window(win, g, red);
    ncc_surface(g, smem, (float)inv_sigma);

    if (surfaces) {
        float* dst = surfaces + (size_t)p * g.C * g.C;
        for (int idx = threadIdx.x; idx < g.C * g.C; idx += kThreads) dst[idx] = gam[idx];
    }
    float bv;
    int bi;
    surface_argmax(gam, g.C * g.C, smem + g.off_red, bv, bi);
    if (threadIdx.x == 0) {
        // nudge.cu:107-140 (argument roles from nudge.cu:57: old = W, new = R + 2m)
        const int u = bi / g.C, v = bi - u * g.C;
        const int E = g.R + 2 * m;
        int left = v - m;
        if (left < 0) left = 0;
        if (left + E > g.W) left = g.W - E;
        int top = u - m;
        if (top < 0) top = 0;
        if (top + E > g.W) top = g.W - E;
        out[p] = CoarseOut{u, v, top, left};
        coarse_peak[p] = bv;
    }
}

__global__ void __launch_bounds__(kThreads, 1)
refine_kernel(PairSource src, long long pair0, long long pairs, const CoarseOut* coarse,
              InterpGeom chip_g, InterpGeom win_g, const float* chip_taps, const float* win_taps,
              float* refined, long long refined_stride, int deramp)
{
    extern __shared__ __align__(16) float smem[];
    if (blockIdx.x >= pairs) return;
    const long long p = pair0 + blockIdx.x;
    const long long roff = src.ref_off[p], toff = src.tgt_off[p];
    if (roff < 0 || toff < 0) return;
    float* out = refined + (long long)blockIdx.x * refined_stride;
    interp_tile(src.ref_base + roff, src.ref_stride, chip_g, chip_taps, smem, out, deramp);
    const CoarseOut co = coarse[p];
    interp_tile(src.tgt_base + toff + co.top * src.tgt_stride + co.left, src.tgt_stride, win_g,
                win_taps, smem, out + (long long)chip_g.F * chip_g.F, deramp);
}

__global__ void __launch_bounds__(kThreads, 1)
fine_kernel(const float* refined, long long refined_stride, long long pair0, long long pairs,
            const long long* ref_off, NccGeom g, ZoomGeom zg, const float* zoom_taps,
            const CoarseOut* coarse, const float* coarse_peak, int margin, int refine_factor,
            int refine_margin, int ref_compat, float2* offsets, PairDiag* diag, float* surfaces)
{
    extern __shared__ __align__(16) float smem[];
    if (blockIdx.x >= pairs) return;
    const long long p = pair0 + blockIdx.x;
    if (ref_off[p] < 0) {
        if (threadIdx.x == 0) {
            offsets[p] = make_float2(NAN, NAN);
            if (diag) diag[p] = PairDiag{-1, -1, -1, -1, -1, -1, -1, -1, NAN, NAN, NAN, 0.0f};
        }
        return;
    }
    const float* rchip = refined + (long long)blockIdx.x * refined_stride;
    const float* rwin = rchip + (long long)g.R * g.R;
    float* win = smem + g.off_win;
    float* chip = smem + g.off_chip;
    float* inv = smem + g.off_inv;
    float* gam = smem + g.off_gam;
    double* red = reinterpret_cast<double*>(smem + g.off_red);

    stage_real(win, g.W, g.W, g.S, rwin);
    __syncthreads();
    window_stats(win, g, inv, reinterpret_cast<double*>(chip));
    stage_real(chip, g.R, g.R, g.CS, rchip);
    const double inv_sigma = chip_stats(chip, g, red);
    shift_window(win, g, red);
    ncc_surface(g, smem, (float)inv_sigma);

    if (surfaces) {
        float* dst = surfaces + (size_t)p * g.C * g.C;
        for (int idx = threadIdx.x; idx < g.C * g.C; idx += kThreads) dst[idx] = gam[idx];
    }
    float rv;
    int ri;
    surface_argmax(gam, g.C * g.C, smem + g.off_red, rv, ri);

    // zoom: the window region holds the row-interpolated surface, the chip region the taps
    float* T = smem + g.off_win;
    float* taps = smem + g.off_chip;
    for (int idx = threadIdx.x; idx < zg.z * zg.taps_len; idx += kThreads)
        taps[idx] = __ldg(zoom_taps + idx);
    __syncthreads();
    float zv;
    int zi;
    zoom_argmax(gam, T, taps, zg, zv, zi);
    block_argmax(zv, zi, smem + g.off_red, reinterpret_cast<int*>(smem + g.off_red + kWarps));

    if (threadIdx.x == 0) {
        const CoarseOut co = coarse[p];
        const int fp = zi / zg.Z, fq = zi - fp * zg.Z;
        const float zoom = (float)(refine_factor * zg.z);
        float dy, dx;
        if (ref_compat) {
            // offsets.cu:124-125, refine margin subtracted from the nudged corner once more
            dy = ((float)co.top - (float)margin) + ((float)fp / zoom - (float)refine_margin);
            dx = ((float)co.left - (float)margin) + ((float)fq / zoom - (float)refine_margin);
        } else {
            dy = (float)(co.top - margin) + (float)fp / zoom;
            dx = (float)(co.left - margin) + (float)fq / zoom;
        }
        offsets[p] = make_float2(dy, dx);
        if (diag) {
            diag[p] = PairDiag{co.u, co.v, co.top, co.left, ri / g.C, ri % g.C, fp, fq,
                               coarse_peak[p], rv, zv, 0.0f};
        }
    }
}

// ------------------------------------------------------------------------------------------
// helpers of the tensor-core form: placement statistics and the zoom, as separate kernels
// ------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(kThreads, 2)
window_stats_cplx_kernel(PairSource src, long long pair0, long long pairs, NccGeom g, float* inv)
{
    extern __shared__ __align__(16) float smem[];
    if (blockIdx.x >= pairs) return;
    const long long p = pair0 + blockIdx.x;
    const long long toff = src.tgt_off[p];
    if (toff < 0 || src.ref_off[p] < 0) return;
    float* win = smem + g.off_win;
    stage_cplx(win, g.W, g.W, g.S, src.tgt_base + toff, src.tgt_stride);
    __syncthreads();
    window_stats(win, g, inv + (long long)blockIdx.x * g.C * g.C,
                 reinterpret_cast<double*>(smem + g.off_chip));
}

__global__ void __launch_bounds__(kThreads, 2)
window_stats_real_kernel(RealTiles t, long long pairs, NccGeom g, float* inv)
{
    extern __shared__ __align__(16) float smem[];
    if (blockIdx.x >= pairs) return;
    float* win = smem + g.off_win;
    stage_real(win, g.W, g.W, g.S, t.base + (long long)blockIdx.x * t.stride + t.win_off);
    __syncthreads();
    window_stats(win, g, inv + (long long)blockIdx.x * g.C * g.C,
                 reinterpret_cast<double*>(smem + g.off_chip));
}

// zoom of the refined surfaces for the tensor-core form: Zm = U G U^T (U = the Z x Cf
// band-limited interpolation matrix) as two register-tiled products on the FP32 pipes, each
// thread owning an 8 x 8 block of outputs (64 FMAs per four 128-bit shared loads), the zoomed
// surface reduced straight to its first maximum.  Zp = Z rounded up to 8; padded rows/columns
// of U are zero and never win the maximum.
constexpr int kZoomThreads = 256;

__global__ void __launch_bounds__(kZoomThreads, 2)
zoom_kernel(const float* gam, long long pair0, long long pairs, const long long* ref_off,
            ZoomGeom zg, const float* zoom_ut, const CoarseOut* coarse, const float* coarse_peak,
            const FineOut* fout, int margin, int refine_factor, int refine_margin, int ref_compat,
            float2* offsets, PairDiag* diag)
{
    extern __shared__ __align__(16) float smem[];
    if (blockIdx.x >= pairs) return;
    const long long p = pair0 + blockIdx.x;
    if (ref_off[p] < 0) {
        if (threadIdx.x == 0) {
            offsets[p] = make_float2(NAN, NAN);
            if (diag) diag[p] = PairDiag{-1, -1, -1, -1, -1, -1, -1, -1, NAN, NAN, NAN, 0.0f};
        }
        return;
    }
    const int Cf = zg.Cf, Z = zg.Z, Zp = (Z + 7) & ~7, nt = Zp / 8;
    float* G = smem;                          // Cf x Cf
    float* Ut = G + ((Cf * Cf + 3) & ~3);     // Cf x Zp: Ut[l][q] = U[q][l]
    float* T = Ut + Cf * Zp;                  // Cf x Zp: T[a][q] = sum_l G[a][l] U[q][l]
    float* red = T + Cf * Zp;
    const float* src = gam + (long long)blockIdx.x * Cf * Cf;
    for (int idx = threadIdx.x; idx < Cf * Cf; idx += kZoomThreads) G[idx] = src[idx];
    for (int idx = threadIdx.x; idx < Cf * Zp / 4; idx += kZoomThreads)
        reinterpret_cast<float4*>(Ut)[idx] = __ldg(reinterpret_cast<const float4*>(zoom_ut) + idx);
    __syncthreads();
    // T: Cf x (Zp/8) strips of 8 outputs
    for (int t = threadIdx.x; t < Cf * nt; t += kZoomThreads) {
        const int a = t / nt, q0 = (t - a * nt) * 8;
        float acc[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = 0.0f;
        for (int l = 0; l < Cf; ++l) {
            const float gv = G[a * Cf + l];
            const float4 u0 = *reinterpret_cast<const float4*>(Ut + l * Zp + q0);
            const float4 u1 = *reinterpret_cast<const float4*>(Ut + l * Zp + q0 + 4);
            acc[0] = fmaf(gv, u0.x, acc[0]); acc[1] = fmaf(gv, u0.y, acc[1]);
            acc[2] = fmaf(gv, u0.z, acc[2]); acc[3] = fmaf(gv, u0.w, acc[3]);
            acc[4] = fmaf(gv, u1.x, acc[4]); acc[5] = fmaf(gv, u1.y, acc[5]);
            acc[6] = fmaf(gv, u1.z, acc[6]); acc[7] = fmaf(gv, u1.w, acc[7]);
        }
        *reinterpret_cast<float4*>(T + a * Zp + q0) = make_float4(acc[0], acc[1], acc[2], acc[3]);
        *reinterpret_cast<float4*>(T + a * Zp + q0 + 4) = make_float4(acc[4], acc[5], acc[6], acc[7]);
    }
    __syncthreads();
    // Zm: (Zp/8)^2 blocks of 8 x 8
    float bv = -INFINITY;
    int bi = INT_MAX;
    for (int t = threadIdx.x; t < nt * nt; t += kZoomThreads) {
        const int p0 = (t / nt) * 8, q0 = (t % nt) * 8;
        float acc[8][8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[i][k] = 0.0f;
        for (int a = 0; a < Cf; ++a) {
            const float4 ua = *reinterpret_cast<const float4*>(Ut + a * Zp + p0);
            const float4 ub = *reinterpret_cast<const float4*>(Ut + a * Zp + p0 + 4);
            const float4 ta = *reinterpret_cast<const float4*>(T + a * Zp + q0);
            const float4 tb = *reinterpret_cast<const float4*>(T + a * Zp + q0 + 4);
            const float uu[8] = {ua.x, ua.y, ua.z, ua.w, ub.x, ub.y, ub.z, ub.w};
            const float tt[8] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int k = 0; k < 8; ++k) acc[i][k] = fmaf(uu[i], tt[k], acc[i][k]);
        }
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if (p0 + i < Z && q0 + k < Z) better(bv, bi, acc[i][k], (p0 + i) * Z + q0 + k);
    }
    block_argmax_n<kZoomThreads>(bv, bi, red, reinterpret_cast<int*>(red + kZoomThreads / 32));
    if (threadIdx.x == 0) {
        const CoarseOut co = coarse[p];
        const FineOut fo = fout[p];
        const int fp = bi / Z, fq = bi - fp * Z;
        const float zoom = (float)(refine_factor * zg.z);
        float dy, dx;
        if (ref_compat) {
            dy = ((float)co.top - (float)margin) + ((float)fp / zoom - (float)refine_margin);
            dx = ((float)co.left - (float)margin) + ((float)fq / zoom - (float)refine_margin);
        } else {
            dy = (float)(co.top - margin) + (float)fp / zoom;
            dx = (float)(co.left - margin) + (float)fq / zoom;
        }
        offsets[p] = make_float2(dy, dx);
        if (diag) {
            diag[p] = PairDiag{co.u, co.v, co.top, co.left, fo.u, fo.v, fp, fq, coarse_peak[p],
                               fo.peak, bv, 0.0f};
        }
    }
}

}  // namespace ampcor_b200
