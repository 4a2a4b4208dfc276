// Tensor-core zoom of the refined correlation surfaces (sm_100a tcgen05, 3xTF32, FP32
// accumulation in tensor memory).
//
// The reference zooms each Cf x Cf refined surface G by a factor z with a zero-padded FFT and
// takes the first maximum of the Z x Z result (Z = z Cf; correlators/kernels.h zoomcor, maxcor).
// That band-limited interpolation is the matrix product Zm = U G U^T with U the Z x Cf Dirichlet
// interpolation matrix, so here it runs as two products per pair, both on the tensor cores:
//   T^T = U G^T  (Z x Cf): A = U (constant, loaded once per CTA), B = G;
//   Zm  = U T    (Z x Z):  A = U, B = T^T (written from the first product's accumulators),
// with every operand split as x = hi + lo (hi rounded to tf32, lo = x - hi) and three products
// hi.hi + hi.lo + lo.hi per K step, a relative error near 2^-21 per product (FP32 class).
// The accumulators of Zm are reduced straight to their first maximum; the zoomed surface is
// never stored.
//
// Operands sit in shared memory as K-major core matrices (8 rows x 16 bytes, no swizzle): row r,
// element k of a plane at float offset ((r / 8) KC + k / 4) 32 + (r % 8) 4 + k % 4, KC = 16-byte
// chunks per row.  One CTA of kTcZoomThreads (512) threads per SM walks the pairs of a chunk;
// lane 0 of the last warp issues the MMAs, all sixteen warps read accumulators (warp w reads lane
// quarter w % 4; the four warps of a quarter take turns over its columns).
// Every wait on an mbarrier is bounded; on expiry the kernel records an error, drains its MMAs
// and frees its tensor memory.
#include "kernels.cuh"
#include "tcgen05.cuh"
#include "tile_common.cuh"

namespace ampcor_b200 {

namespace {

constexpr int kZThreads = kTcZoomThreads;
constexpr int kZGroups = kZThreads / 128;  // warps per lane quarter
constexpr int kZBatch = 3;                 // 16-column accumulator loads in flight per thread
// the thread that issues every MMA (and the drain after an expired wait): lane 0 of the last
// warp, whose group reads no more accumulator chunks per unit than the first one
constexpr int kIssuer = kZThreads - 32;

// accumulator row of this thread in a tile of M rows: M = 128 puts row r in lane r, M = 64 puts
// rows 16q .. 16q+15 in lanes 32q .. 32q+15; -1 for lanes that hold no row
__device__ __forceinline__ int tile_row(int M, int quarter, int lane)
{
    if (M == 128) return quarter * 32 + lane;
    return lane < 16 ? quarter * 16 + lane : -1;
}

__device__ __forceinline__ uint32_t lane_base(int quarter) { return (uint32_t)(quarter * 32) << 16; }

}  // namespace

__global__ void __launch_bounds__(kZThreads, 1)
tc_zoom_kernel(const float* gam, long long pair0, long long pairs, const long long* ref_off,
               ZoomTcGeom zt, const float* uhl, const CoarseOut* coarse, const float* coarse_peak,
               const FineOut* fout, int margin, int refine_factor, int refine_margin, int ref_compat,
               float2* offsets, PairDiag* diag, unsigned int* err_out, int stall)
{
    extern __shared__ __align__(1024) unsigned char zsm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int quarter = warp & 3, group = warp >> 2;
    const int Cf = zt.Cf, Z = zt.Z, KC = zt.KC;
    float* ahi = reinterpret_cast<float*>(zsm + zt.off_ahi);
    float* bhi = reinterpret_cast<float*>(zsm + zt.off_bhi);
    float* blo = reinterpret_cast<float*>(zsm + zt.off_blo);
    float* ghi = reinterpret_cast<float*>(zsm + zt.off_ghi);
    float* glo = reinterpret_cast<float*>(zsm + zt.off_glo);
    uint64_t* bar = reinterpret_cast<uint64_t*>(zsm + zt.off_bar);  // the first product
    uint64_t* drain = bar + 1;
    uint64_t* ubar = bar + 2;  // the two accumulator buffers of Zm
    uint64_t* never = bar + 4;  // completed by nothing: the wait of a failure-detection test
    unsigned char* misc = zsm + zt.off_misc;
    uint32_t* tmem_s = reinterpret_cast<uint32_t*>(misc);
    volatile int* err = reinterpret_cast<volatile int*>(misc + 8);
    float* red = reinterpret_cast<float*>(misc + 16);

    // U (hi and lo planes, contiguous in global and shared memory) once per CTA; the B planes
    // start out zero (their rows past Z stay so)
    for (int i = tid; i < (zt.off_bhi - zt.off_ahi) / 16; i += kZThreads)
        reinterpret_cast<float4*>(ahi)[i] = __ldg(reinterpret_cast<const float4*>(uhl) + i);
    for (int i = tid; i < (zt.off_ghi - zt.off_bhi) / 16; i += kZThreads)
        reinterpret_cast<float4*>(bhi)[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (tid == 0) {
        *err = 0;
        mbar_init(bar, 1);
        mbar_init(drain, 1);
        mbar_init(ubar, 1);
        mbar_init(ubar + 1, 1);
        mbar_init(never, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        tmem_alloc(tmem_s, (uint32_t)zt.tmem_cols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_s;
    const uint32_t ahi_a = saddr(ahi), alo_a = saddr(zsm + zt.off_alo);
    const uint32_t bhi_a = saddr(bhi), blo_a = saddr(blo), ghi_a = saddr(ghi), glo_a = saddr(glo);
    const uint32_t rg_bytes = (uint32_t)KC * 128u;  // one 8-row group of a plane
    const int units = zt.mtiles * zt.nparts;        // (row tile, column part) units of Zm
    const int pch = zt.npart / 16;                  // 16-column accumulator chunks of a unit
    uint32_t phase = 0, uph0 = 0, uph1 = 0;
    bool issued = false;

    // A x B -> tensor memory at column d: K steps of 8 (two 16-byte chunks), three products each
    auto issue = [&](uint32_t d, uint32_t a_hi, uint32_t a_lo, uint32_t b_hi, uint32_t b_lo,
                     uint32_t idesc) {
        for (int s = 0; s < KC / 2; ++s) {
            const uint64_t ah = kmajor_desc(a_hi + s * 256u, 128u, rg_bytes);
            const uint64_t al = kmajor_desc(a_lo + s * 256u, 128u, rg_bytes);
            const uint64_t bh = kmajor_desc(b_hi + s * 256u, 128u, rg_bytes);
            const uint64_t bl = kmajor_desc(b_lo + s * 256u, 128u, rg_bytes);
            mma_tf32(d, ah, bh, idesc, s > 0 ? 1u : 0u);
            mma_tf32(d, ah, bl, idesc, 1u);
            mma_tf32(d, al, bh, idesc, 1u);
        }
    };
    auto wait_mma = [&]() {
        const bool ok = mbar_wait(bar, phase, err);
        phase ^= 1u;
        tc_fence_after();
        return ok;
    };

    // a failure-detection test: before any tensor-core work is issued, every thread waits on a
    // barrier that nothing completes; the bounded wait runs out, sets the error flag, and the CTA
    // skips its pairs and reports the time-out like any other expired wait
    if (stall) {
        mbar_wait(never, 0u, err, kStallCycles);
        __syncthreads();
    }

    for (long long b = blockIdx.x; b < pairs && !*err; b += gridDim.x) {
        const long long p = pair0 + b;
        if (ref_off[p] < 0) {
            if (tid == 0) {
                offsets[p] = make_float2(NAN, NAN);
                if (diag) diag[p] = PairDiag{-1, -1, -1, -1, -1, -1, -1, -1, NAN, NAN, NAN, 0.0f};
            }
            continue;
        }
        // G -> its tf32 planes (rows a, K = c), zero past Cf
        const float* src = gam + b * Cf * Cf;
        for (int t = tid; t < zt.NG * KC; t += kZThreads) {
            const int a = t % zt.NG, c4 = t / zt.NG;
            float h[4], l[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int c = 4 * c4 + k;
                const float x = (a < Cf && c < Cf) ? __ldg(src + a * Cf + c) : 0.0f;
                split_tf32(x, h[k], l[k]);
            }
            const int off = (a >> 3) * KC * 32 + c4 * 32 + (a & 7) * 4;
            *reinterpret_cast<float4*>(ghi + off) = make_float4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<float4*>(glo + off) = make_float4(l[0], l[1], l[2], l[3]);
        }
        fence_async_smem();
        __syncthreads();

        // T^T = U G^T: every row tile at once, tile mt at accumulator column 64 mt
        if (tid == kIssuer) {
            tc_fence_after();
            for (int mt = 0; mt < zt.mtiles; ++mt) {
                const int M = (mt == zt.mtiles - 1) ? zt.last_m : 128;
                const uint32_t arow = (uint32_t)(mt * 16) * rg_bytes;
                issue(tmem + (uint32_t)(64 * mt), ahi_a + arow, alo_a + arow, ghi_a, glo_a,
                      instr_desc_tf32(M, zt.NG));
            }
            mma_commit(bar);
            issued = true;
        }
        __syncwarp();
        {
            const bool ok = wait_mma();
            // row tiles go round the warp groups; each thread writes its row of T^T into the B
            // planes, split hi / lo
            for (int mt = group; mt < zt.mtiles; mt += kZGroups) {
                const int M = (mt == zt.mtiles - 1) ? zt.last_m : 128;
                const int row = tile_row(M, quarter, lane);
                const int q = mt * 128 + row;
                const bool keep = ok && row >= 0 && q < Z;
                const int rowbase = (q >> 3) * KC * 32 + (q & 7) * 4;
                // one 16-column chunk (four 16-byte K chunks) at a time
                for (int j = 0; 16 * j < zt.NG; ++j) {
                    uint32_t r[16];
                    tmem_ld16_async(tmem + lane_base(quarter) + (uint32_t)(64 * mt + 16 * j), r);
                    tmem_wait_ld(r);
                    if (!keep) continue;
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        const int c4 = 4 * j + cc;
                        if (c4 >= KC) break;
                        float h[4], l[4];
#pragma unroll
                        for (int k = 0; k < 4; ++k) split_tf32(__uint_as_float(r[4 * cc + k]), h[k], l[k]);
                        *reinterpret_cast<float4*>(bhi + rowbase + c4 * 32) = make_float4(h[0], h[1], h[2], h[3]);
                        *reinterpret_cast<float4*>(blo + rowbase + c4 * 32) = make_float4(l[0], l[1], l[2], l[3]);
                    }
                }
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();

        // Zm = U T, one (row tile, column part) unit at a time, double-buffered in tensor memory
        // (columns 0 and 256): the MMAs of the next unit run while the warps read this one
        auto issue_unit = [&](int un) {
            const int mt = un / zt.nparts, np = un - mt * zt.nparts;
            const int M = (mt == zt.mtiles - 1) ? zt.last_m : 128;
            const uint32_t arow = (uint32_t)(mt * 16) * rg_bytes;
            const uint32_t brow = (uint32_t)(np * zt.npart / 8) * rg_bytes;
            issue(tmem + (uint32_t)((un & 1) * 256), ahi_a + arow, alo_a + arow, bhi_a + brow,
                  blo_a + brow, instr_desc_tf32(M, zt.npart));
            mma_commit(ubar + (un & 1));
        };
        float bv = -INFINITY;
        int bi = INT_MAX;
        if (tid == kIssuer && units > 0 && !*err) issue_unit(0);
        for (int un = 0; un < units; ++un) {
            if (*err) break;
            if (tid == kIssuer && un + 1 < units) issue_unit(un + 1);
            __syncwarp();
            const bool odd = (un & 1) != 0;
            const bool ok = mbar_wait(ubar + (un & 1), odd ? uph1 : uph0, err);
            if (odd)
                uph1 ^= 1u;
            else
                uph0 ^= 1u;
            tc_fence_after();
            const int mt = un / zt.nparts, np = un - mt * zt.nparts;
            const int M = (mt == zt.mtiles - 1) ? zt.last_m : 128;
            const int row = tile_row(M, quarter, lane);
            const int pz = mt * 128 + row;
            const bool live = ok && row >= 0 && pz < Z;
            const uint32_t dbase = tmem + lane_base(quarter) + (uint32_t)((un & 1) * 256);
            // 16-column chunks go round the warp groups, kZBatch loads in flight; a thread
            // visits its columns in increasing order (parts in order, chunks in order), so a
            // strict comparison keeps the first maximum
            for (int c = group; c < pch; c += kZGroups * kZBatch) {
                uint32_t r[kZBatch][16];
#pragma unroll
                for (int j = 0; j < kZBatch; ++j)
                    if (c + kZGroups * j < pch) tmem_ld16_async(dbase + (uint32_t)(16 * (c + kZGroups * j)), r[j]);
#pragma unroll
                for (int j = 0; j < kZBatch; ++j)
                    if (c + kZGroups * j < pch) tmem_wait_ld(r[j]);
                if (!live) continue;
#pragma unroll
                for (int j = 0; j < kZBatch; ++j) {
                    const int ci = c + kZGroups * j;
                    if (ci >= pch) break;
                    const int q0 = np * zt.npart + 16 * ci;
                    float v[16];
#pragma unroll
                    for (int k = 0; k < 16; ++k) v[k] = q0 + k < Z ? __uint_as_float(r[j][k]) : -INFINITY;
                    float m = v[0];
#pragma unroll
                    for (int k = 1; k < 16; ++k) m = fmaxf(m, v[k]);
                    if (m > bv) {
                        int first = 15;
#pragma unroll
                        for (int k = 15; k >= 0; --k)
                            if (v[k] == m) first = k;
                        bv = m;
                        bi = pz * Z + q0 + first;
                    }
                }
            }
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
        }
        block_argmax_n<kZThreads>(bv, bi, red, reinterpret_cast<int*>(red + kZThreads / 32));
        if (tid == 0 && !*err) {
            const CoarseOut co = coarse[p];
            const FineOut fo = fout[p];
            const int fp = bi / Z, fq = bi - fp * Z;
            const float zoom = (float)(refine_factor * zt.z);
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
                diag[p] = PairDiag{co.u, co.v, co.top, co.left, fo.u, fo.v, fp, fq, coarse_peak[p],
                                   fo.peak, bv, 0.0f};
            }
        }
        if (*err) break;
    }

    // teardown: after an expired wait, let the issued MMAs finish before freeing their memory
    __syncthreads();
    if (*err && issued && tid == kIssuer) {
        mma_commit(drain);
        volatile int spare = 0;
        mbar_wait(drain, 0u, &spare);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, (uint32_t)zt.tmem_cols);
    }
    if (tid == 0 && *err) atomicAdd(err_out, 1u);
}

}  // namespace ampcor_b200
