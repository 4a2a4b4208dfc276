// Tensor-core form of the correlation numerator (sm_100a tcgen05, bf16x3 split products, FP32
// accumulation in tensor memory).
//
// For one tile pair the numerator of every placement is
//     N(u, v) = sum_i sum_j r'(i, j) t(u + i, v + j),
// r' the zero-mean chip (R x R), t the window (W x W), (u, v) in [0, C)^2.  Indexing the sum by
// the window row w = u + i instead of the chip row turns it into one matrix product accumulated
// over w and over the chip columns j:
//     D[v][u] = sum_w sum_j A_w[v][j] B_w[j][u],   A_w[v][j] = t(w, v + j),
//                                                  B_w[j][u] = r'(w - u, j)  (0 outside the chip),
// so D[v][u] = N(u, v) collects in tensor memory (M = 64 or 128 accumulator rows for v, N >= C
// columns for u) with no per-placement bookkeeping.  Both operands are read by the tensor core
// through K-major shared-memory descriptors without building the Hankel or sheared matrices:
//   * A_w: window row w is written once as overlapping 16-byte rows X[p] = t(w, p .. p+7); row v
//     of the K-slice [16s, 16s+16) is X[v + 16s] and its second half X[v + 16s + 8], so the
//     descriptor is (start = X + 16s rows, 8-row groups 128 B apart, K halves 128 B apart);
//   * B_w: the chip is stored once with its rows reversed, Crev[kc][q] = r'(W-1-q, 8kc .. 8kc+7);
//     column u of B_w is Crev row q = W-1-w+u, so B_w is the window of that buffer starting at
//     row W-1-w: one descriptor whose start moves by 16 bytes per window row.
// The fp32 operands are split as x = hi + lo in bf16 and three products (hi.hi + hi.lo + lo.hi)
// accumulate in FP32, a relative error near 2^-16 per product, below the FP32 summation error of
// the plain form on these surfaces.
//
// A CTA of 256 threads owns one pair: warps 1-7 stream the window rows, two per stage, into a
// ring of operand stages, lane 0 of warp 0 issues the MMAs and commits each stage back to its
// producers, warps 0-3 read the accumulators and reduce the normalised surface to its first
// maximum.  Every wait on an
// mbarrier is bounded in time; on expiry the kernel records an error, drains the MMAs it issued
// and frees its tensor memory before returning.
#include "kernels.cuh"
#include "tcgen05.cuh"

#include <cuda_bf16.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>

namespace ampcor_b200 {

namespace {

constexpr int kTcThreads = 256;
constexpr int kTcWarps = kTcThreads / 32;
constexpr int kProducers = 224;               // warps 1-7 stream the window rows
constexpr int kRowsPerStage = 2;             // window rows per operand stage
constexpr unsigned kFull = 0xffffffffu;

// instruction descriptor: bf16 A and B, both K-major, FP32 accumulator, M x N
__device__ __forceinline__ uint32_t instr_desc(int m, int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ float amp_of(float2 z)
{
    const double re = z.x, im = z.y;
    return (float)sqrt(re * re + im * im);
}

// 8 floats -> 8 bf16 (hi) and 8 bf16 residuals (lo), packed as two 16-byte words
__device__ __forceinline__ void split8(const float (&x)[8], uint4& hi, uint4& lo)
{
    uint32_t h[4], l[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const __nv_bfloat16 h0 = __float2bfloat16_rn(x[2 * k]);
        const __nv_bfloat16 h1 = __float2bfloat16_rn(x[2 * k + 1]);
        const __nv_bfloat16 l0 = __float2bfloat16_rn(x[2 * k] - __bfloat162float(h0));
        const __nv_bfloat16 l1 = __float2bfloat16_rn(x[2 * k + 1] - __bfloat162float(h1));
        h[k] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
        l[k] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ double block_sum(double v, double* red)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kTcWarps; ++w) s += red[w];
    __syncthreads();
    return s;
}

// block-wide minimum; every thread gets the same value
__device__ float block_min(float v, double* red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(kFull, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* r = reinterpret_cast<float*>(red);
    if (lane == 0) r[warp] = v;
    __syncthreads();
    float m = r[0];
#pragma unroll
    for (int w = 1; w < kTcWarps; ++w) m = fminf(m, r[w]);
    __syncthreads();
    return m;
}

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
    for (int w = 1; w < kTcWarps; ++w) better(bv, bi, redf[w], redi[w]);
    __syncthreads();
}

__device__ __forceinline__ void cp_async8(void* dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(saddr(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async4(void* dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(saddr(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// tile access: complex64 rasters (coarse) or dense fp32 amplitude tiles (refined); window rows
// are fetched raw into shared memory ahead of use (cp.async), amplitudes taken when consumed
struct CplxTiles {
    using Raw = float2;
    const float2* chip;
    long long chip_stride;
    const float2* win;
    long long win_stride;
    __device__ float chip_at(int i, int j) const { return amp_of(__ldg(chip + i * chip_stride + j)); }
    __device__ float win_at(int w, int x) const { return amp_of(__ldg(win + w * win_stride + x)); }
    __device__ void fetch(Raw* dst, int w, int x) const { cp_async8(dst, win + w * win_stride + x); }
    __device__ static float amp(const Raw& r) { return amp_of(r); }
};

struct DenseTiles {
    using Raw = float;
    const float* chip;
    const float* win;
    int R, W;
    __device__ float chip_at(int i, int j) const { return __ldg(chip + i * R + j); }
    __device__ float win_at(int w, int x) const { return __ldg(win + w * W + x); }
    __device__ void fetch(Raw* dst, int w, int x) const { cp_async4(dst, win + w * W + x); }
    __device__ static float amp(const Raw& r) { return r; }
};

constexpr int kPrefetch = 2 * kRowsPerStage;  // window rows fetched ahead of the producers

struct SurfaceMax {
    float v;
    int i;
    float inv_sigma;
    double mean;
};

// the numerator of one placement (u, v) as an FP32 dot product (FP64 across threads): the value
// reported for the maximum, free of the tensor cores' accumulation bias.  The window samples go in
// less the box's own mean (sum r' (t - c) = sum r' t for any constant c): the FP32 sums round on
// the box's variation, not on its level, and an all-zero box keeps a numerator of exactly zero.
template <typename Tiles>
__device__ float placement_gamma(const Tiles& tl, const TcGeom& g, int u, int v, double mean,
                                 float inv_box, float inv_sigma, double* red)
{
    float st = 0.0f;
    for (int idx = threadIdx.x; idx < g.R * g.R; idx += kTcThreads) {
        const int i = idx / g.R, j = idx - i * g.R;
        st += tl.win_at(u + i, v + j);
    }
    const float shift = (float)(block_sum((double)st, red) / ((double)g.R * (double)g.R));
    float acc = 0.0f;
    for (int idx = threadIdx.x; idx < g.R * g.R; idx += kTcThreads) {
        const int i = idx / g.R, j = idx - i * g.R;
        const float rp = (float)((double)tl.chip_at(i, j) - mean);
        acc = fmaf(rp, tl.win_at(u + i, v + j) - shift, acc);
    }
    const double num = block_sum((double)acc, red);
    return (float)num * inv_box * inv_sigma;
}

// the correlation surface of one pair on the tensor cores; returns the first maximum of the
// normalised surface (valid in every thread) and writes the surface to gam / surf if given
// (exact_peak: re-evaluate the reported maximum in FP32 on the CUDA cores)
template <typename Tiles>
__device__ SurfaceMax tc_surface(const Tiles& tl, const TcGeom& g, const float* __restrict__ inv,
                                 bool exact_peak, float* gam, float* surf, unsigned int* err_out)
{
    extern __shared__ __align__(1024) unsigned char tsm[];
    unsigned char* crev = tsm + g.off_crev;
    unsigned char* xst = tsm + g.off_x;
    float* rowbuf = reinterpret_cast<float*>(tsm + g.off_row);
    uint64_t* bars = reinterpret_cast<uint64_t*>(tsm + g.off_bar);
    uint64_t* full = bars;
    uint64_t* empty = bars + g.nst;
    uint64_t* done = bars + 2 * g.nst;
    uint64_t* crev_free = bars + 2 * g.nst + 1;
    unsigned char* misc = tsm + g.off_misc;
    uint32_t* tmem_base_s = reinterpret_cast<uint32_t*>(misc);
    volatile int* err = reinterpret_cast<volatile int*>(misc + 8);
    volatile int* stop = reinterpret_cast<volatile int*>(misc + 12);
    double* red = reinterpret_cast<double*>(misc + 16);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int R = g.R, W = g.W, C = g.C, Q = g.Q, KH = g.JC / 8, XR = g.XR;
    const uint32_t xstage_bytes = (uint32_t)kRowsPerStage * 2u * XR * 16u;

    if (tid == 0) {
        *err = 0;
        for (int s = 0; s < g.nst; ++s) {
            mbar_init(&full[s], kProducers);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        mbar_init(crev_free, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        tmem_alloc(tmem_base_s, (uint32_t)g.tmem_cols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_base_s;

    // chip statistics in FP64 (refStats.cu:118-302): mean, then 1 / |r'|
    double s1 = 0.0;
    for (int idx = tid; idx < R * R; idx += kTcThreads) s1 += tl.chip_at(idx / R, idx % R);
    const double mean = block_sum(s1, red) / ((double)R * (double)R);
    double s2 = 0.0;
    for (int idx = tid; idx < R * R; idx += kTcThreads) {
        const float rp = (float)((double)tl.chip_at(idx / R, idx % R) - mean);
        s2 += (double)rp * (double)rp;
    }
    s2 = block_sum(s2, red);
    const float inv_sigma = s2 > 0.0 ? (float)(1.0 / sqrt(s2)) : 0.0f;

    // the window goes into the split less its smallest sample c: sum r' (t - c) = sum r' t for any
    // constant c since sum r' = 0.  Amplitudes are non-negative, so 0 <= t - c <= t: no term grows,
    // a window that holds a zero sample is left as it is (an all-zero box keeps a numerator of
    // exactly zero), and under a strong steady return the bf16 split rounds on the window's
    // variation, not on its level
    float wmin = INFINITY;
    for (int idx = tid; idx < W * W; idx += kTcThreads) wmin = fminf(wmin, tl.win_at(idx / W, idx % W));
    const float shift = block_min(wmin, red);
    const uint32_t idesc = instr_desc(g.M, g.N);
    const uint32_t crev_addr = saddr(crev);
    const uint32_t x_addr = saddr(xst);
    const int NR = kRowsPerStage;
    const int nsi = (W + NR - 1) / NR;  // stages per pass
    for (int jc = 0; jc < g.nchunks; ++jc) {
        // the previous pass must have finished reading the reversed chip before it is rebuilt
        if (jc > 0) mbar_wait(crev_free, (uint32_t)((jc - 1) & 1), err);
        // reversed, zero-padded chip columns [jc JC, jc JC + JC) as bf16 hi / lo
        for (int idx = tid; idx < KH * Q; idx += kTcThreads) {
            const int kc = idx / Q, q = idx - kc * Q;
            const int i = W - 1 - q;
            float x[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int j = jc * g.JC + 8 * kc + c;
                x[c] = (i >= 0 && i < R && j < R) ? (float)((double)tl.chip_at(i, j) - mean) : 0.0f;
            }
            uint4 hi, lo;
            split8(x, hi, lo);
            reinterpret_cast<uint4*>(crev)[(0 * KH + kc) * Q + q] = hi;
            reinterpret_cast<uint4*>(crev)[(1 * KH + kc) * Q + q] = lo;
        }
        fence_async_smem();
        __syncthreads();

        if (warp >= 1) {
            // producers (warps 1-7): kRowsPerStage window rows per stage -> overlapping 16-byte
            // rows of this pass's columns.  Raw rows are fetched kPrefetch rows ahead (cp.async).
            const int pt = tid - 32;
            using Raw = typename Tiles::Raw;
            Raw* raw = reinterpret_cast<Raw*>(tsm + g.off_raw);
            const int ncols = min(g.RB, W - jc * g.JC);  // columns of this pass inside the window
            auto fetch_row = [&](int w) {
                if (w < W) {
                    Raw* dst = raw + (w % kPrefetch) * g.RB;
                    for (int x = pt; x < ncols; x += kProducers) tl.fetch(dst + x, w, jc * g.JC + x);
                }
                cp_async_commit();
            };
            for (int k = 0; k < kPrefetch; ++k) fetch_row(k);
            for (int si = 0; si < nsi; ++si) {
                const int it = jc * nsi + si;  // stage sequence number over all passes
                const int s = it % g.nst;
                // one producer waits for the stage; the named barrier hands the verdict to every
                // producer (all leave the loop together, so the barrier never strands one)
                if (pt == 0)
                    *stop = (it >= g.nst && !mbar_wait(&empty[s], (uint32_t)(((it / g.nst) & 1) ^ 1), err)) ? 1 : 0;
                cp_async_wait<kPrefetch - kRowsPerStage>();
                asm volatile("bar.sync 1, %0;" ::"n"(kProducers) : "memory");
                if (*stop) break;
                float* rb = rowbuf + s * NR * g.RB;
                for (int idx = pt; idx < NR * g.RB; idx += kProducers) {
                    const int k = idx / g.RB, x = idx - k * g.RB;
                    const int w = si * NR + k;
                    rb[idx] = (w < W && x < ncols) ? Tiles::amp(raw[(w % kPrefetch) * g.RB + x]) - shift : 0.0f;
                }
                asm volatile("bar.sync 1, %0;" ::"n"(kProducers) : "memory");
                for (int k = 0; k < NR; ++k) fetch_row((si + 1) * NR + kPrefetch - NR + k);
                uint4* xs = reinterpret_cast<uint4*>(xst + s * xstage_bytes);
                for (int idx = pt; idx < NR * XR; idx += kProducers) {
                    const int k = idx / XR, p = idx - k * XR;
                    const float* rr = rb + k * g.RB + p;
                    float x[8];
#pragma unroll
                    for (int c = 0; c < 8; ++c) x[c] = rr[c];
                    uint4 hi, lo;
                    split8(x, hi, lo);
                    xs[(2 * k) * XR + p] = hi;
                    xs[(2 * k + 1) * XR + p] = lo;
                }
                fence_async_smem();
                mbar_arrive(&full[s]);
            }
            cp_async_wait<0>();
        } else if (lane == 0) {
            // warp 0, lane 0: the MMA issuer.  Descriptors advance by plain additions: the start
            // address sits in the low 14 bits in 16-byte units and never carries out of them.
            const uint64_t a0 = kmajor_desc(x_addr, 128u, 128u);
            const uint64_t b0 = kmajor_desc(crev_addr + (uint32_t)(W - 1) * 16u, (uint32_t)Q * 16u, 128u);
            const uint64_t b_lo_off = (uint64_t)(KH * Q);        // hi -> lo plane of the chip
            const uint64_t b_ks_off = (uint64_t)(2 * Q);         // next 16 chip columns
            const uint64_t a_lo_off = (uint64_t)XR;              // hi -> lo rows of a window row
            int acc_slot = (jc * W) % g.nacc;
            int row = jc * W;
            for (int si = 0; si < nsi; ++si) {
                const int it = jc * nsi + si;
                const int s = it % g.nst;
                if (!mbar_wait(&full[s], (uint32_t)((it / g.nst) & 1), err)) break;
                tc_fence_after();
                uint64_t as = a0 + (uint64_t)(s * (xstage_bytes >> 4));
                for (int k = 0; k < NR; ++k, ++row, as += 2 * a_lo_off) {
                    const int w = si * NR + k;
                    if (w >= W) break;
                    const uint32_t dacc = tmem + (uint32_t)(acc_slot * g.N);
                    const uint32_t keep = row < g.nacc ? 0u : 1u;
                    if (++acc_slot == g.nacc) acc_slot = 0;
                    uint64_t a = as;
                    uint64_t b = b0 - (uint64_t)w;  // reversed chip from row W-1-w
#pragma unroll 4
                    for (int ks = 0; ks < g.JC / 16; ++ks, a += 16, b += b_ks_off) {
                        mma_bf16(dacc, a, b, idesc, ks ? 1u : keep);
                        mma_bf16(dacc, a, b + b_lo_off, idesc, 1u);
                        mma_bf16(dacc, a + a_lo_off, b, idesc, 1u);
                    }
                }
                mma_commit(&empty[s]);
            }
            mma_commit(crev_free);
        }
        __syncwarp();
    }
    if (warp == 0 && lane == 0) mma_commit(done);
    __syncwarp();

    // epilogue: accumulator lanes of warps 0-3 -> normalised surface -> first maximum
    float bv = -INFINITY;
    int bi = INT_MAX;
    if (warp < 4) {
        const bool ok = mbar_wait(done, 0u, err) && !*err;
        tc_fence_after();
        // M = 128: accumulator row v sits in lane v; M = 64: rows 16q .. 16q+15 sit in lanes
        // 32q .. 32q+15 of lane quarter q
        const int v = g.M == 128 ? warp * 32 + lane : (lane < 16 ? warp * 16 + lane : g.M);
        for (int u0 = 0; u0 < g.N; u0 += 16) {
            float d[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)u0, d);
            for (int a = 1; a < g.nacc; ++a) {
                float e[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(a * g.N + u0), e);
#pragma unroll
                for (int k = 0; k < 16; ++k) d[k] += e[k];
            }
            if (!ok || v >= C) continue;
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const int u = u0 + k;
                if (u < C) {
                    const int idx = u * C + v;
                    const float gv = d[k] * __ldg(inv + idx) * inv_sigma;
                    better(bv, bi, gv, idx);
                    if (gam) gam[idx] = gv;
                    if (surf) surf[idx] = gv;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, (uint32_t)g.tmem_cols);
    }
    if (tid == 0 && *err) atomicAdd(err_out, 1u);
    block_argmax(bv, bi, reinterpret_cast<float*>(red), reinterpret_cast<int*>(red) + kTcWarps);
    if (exact_peak && bi >= 0 && bi < C * C) {
        const int u = bi / C, v = bi - u * C;
        bv = placement_gamma(tl, g, u, v, mean, __ldg(inv + bi), inv_sigma, red);
    }
    return SurfaceMax{bv, bi, inv_sigma, mean};
}

}  // namespace

__global__ void __launch_bounds__(kTcThreads, 2)
tc_coarse_kernel(PairSource src, long long pair0, long long pairs, TcGeom g, const float* inv, int m,
                 CoarseOut* out, float* coarse_peak, float* surfaces, unsigned int* err)
{
    if (blockIdx.x >= pairs) return;
    const long long p = pair0 + blockIdx.x;
    const long long roff = src.ref_off[p], toff = src.tgt_off[p];
    if (roff < 0 || toff < 0) {
        if (threadIdx.x == 0) {
            out[p] = CoarseOut{-1, -1, -1, -1};
            coarse_peak[p] = NAN;
        }
        return;
    }
    CplxTiles tl{src.ref_base + roff, src.ref_stride, src.tgt_base + toff, src.tgt_stride};
    // the coarse maximum only places the refinement window: its value keeps the accumulation
    // error (a few 1e-7 relative), below the reported peak's tolerance
    const SurfaceMax sm = tc_surface(tl, g, inv + (long long)blockIdx.x * g.C * g.C, false, nullptr,
                                     surfaces ? surfaces + (size_t)p * g.C * g.C : nullptr, err);
    if (threadIdx.x == 0) {
        // nudge.cu:107-140
        const int u = sm.i / g.C, v = sm.i - u * g.C;
        const int E = g.R + 2 * m;
        int left = v - m;
        if (left < 0) left = 0;
        if (left + E > g.W) left = g.W - E;
        int top = u - m;
        if (top < 0) top = 0;
        if (top + E > g.W) top = g.W - E;
        out[p] = CoarseOut{u, v, top, left};
        coarse_peak[p] = sm.v;
    }
}

__global__ void __launch_bounds__(kTcThreads, 2)
tc_fine_kernel(RealTiles t, long long pair0, long long pairs, TcGeom g, const float* inv,
               const long long* ref_off, FineOut* fout, float* gam, float* surfaces, unsigned int* err)
{
    if (blockIdx.x >= pairs) return;
    const long long p = pair0 + blockIdx.x;
    if (ref_off[p] < 0) return;
    const float* base = t.base + (long long)blockIdx.x * t.stride;
    DenseTiles tl{base + t.chip_off, base + t.win_off, g.R, g.W};
    const SurfaceMax sm = tc_surface(tl, g, inv + (long long)blockIdx.x * g.C * g.C, true,
                                     gam + (long long)blockIdx.x * g.C * g.C,
                                     surfaces ? surfaces + (size_t)p * g.C * g.C : nullptr, err);
    if (threadIdx.x == 0) fout[p] = FineOut{sm.i / g.C, sm.i % g.C, sm.v, 0.0f};
}

}  // namespace ampcor_b200
