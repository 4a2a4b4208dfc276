// Device-side declarations of the sm_100a batched tile correlator.
//
// The pipeline per tile pair (reference: lib/libampcor_cuda/correlators/Sequential.icc:47-141):
//   coarse_kernel  - gather the chip and search window from the complex64 sources, detect
//                    (detect.cu:78-115), chip mean/sigma (refStats.cu:118-302), FP64 window box
//                    statistics (sat.cu:81-149, tgtStats.cu:88-168), NCC over every placement
//                    (correlate.cu:160-318), first strict maximum (maxcor.cu:79-133) and nudge
//                    (nudge.cu:81-143), all in one CTA with the tiles resident in shared memory.
//   refine_kernel  - band-limited upsampling of the complex chip and of the (R+2m)^2
//                    neighbourhood of the coarse peak (the intent of Sequential.icc:703-1087 and
//                    migrate.cu:101-154), written out as refined amplitudes.
//   fine_kernel    - refined NCC, band-limited zoom of the refined surface (intent of
//                    Sequential.icc:1101-1286), first strict maximum and offset assembly
//                    (offsets.cu:86-129).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ampcor_b200 {

constexpr int kThreads = 512;            // threads per CTA, one CTA per tile pair
constexpr int kWarps = kThreads / 32;
// threads of the spectral correlation kernels (one FFT tile per CTA, the tile fills the shared
// memory): 16 warps at up to 128 registers.  32 warps at 64 registers ran slower on B200 (coarse
// 2.42 against 2.27 ms, fine 3.90 against 3.73 ms per production job).
constexpr int kSpecThreads = 512;
constexpr int kSpecWarps = kSpecThreads / 32;
constexpr int kMaxVB = 8;                // column blocks of a correlation surface
constexpr int kSlot = 33;                // row stride of a partial-sum slot (floats)
constexpr int kStatRows = 8;             // placement rows per window-statistics chunk
constexpr int kQB = 8;                   // outputs per thread in the interpolation kernels

// how one correlation surface (R x R chip over a W x W window, C = W-R+1 placements per axis)
// is split over the warps of a CTA, and where each region lives in shared memory
struct NccGeom {
    int R, W, C;
    int S;          // window row stride in shared memory (odd: conflict-free column walks)
    int CS;         // chip row stride in shared memory (odd)
    int n_ub;       // full 32-row placement blocks handled lane-per-row ("main" tasks)
    int n_vb;       // placement column blocks
    int n_kc;       // chip-row chunks per main task
    int n_main;     // n_ub * n_vb * n_kc <= kWarps
    int n_tkc;      // chip-row chunks (32 rows, one per lane) per leftover row
    int n_trans;    // leftover-row tasks: (C - 32 n_ub) * n_vb * n_tkc
    int vb_v0[kMaxVB];     // first placement column of the block
    int vb_w[kMaxVB];      // placement columns in the block
    int vb_nv[kMaxVB];     // register block width (>= vb_w, one of the compiled widths)
    int vb_steps[kMaxVB];  // ceil(R / nv): chip columns are zero-padded to steps * nv
    int stat_rows;  // placement rows per window-statistics chunk (<= kStatRows)
    // shared-memory regions, in floats from the start of the dynamic buffer
    int off_win, off_part, off_chip, off_inv, off_gam, off_trans, off_red, off_aux;
    int smem_bytes;
};

// band-limited interpolation of an N x N complex tile by f (f*N x f*N output)
struct InterpGeom {
    int N, f, F;     // F = f N
    int NS, YS;      // row strides (float2) of the input tile and the row-interpolated tile
    int taps_len;    // per phase s in [1, f): taps_len entries
    int off_x, off_y, off_taps;   // shared-memory regions (floats)
    int smem_bytes;
};

struct ZoomGeom {
    int Cf, z, Z;    // refined surface Cf x Cf zoomed to Z x Z, Z = z Cf
    int cb;          // output rows per thread (Cf % cb == 0)
    int taps_len;    // per phase s in [0, z)
};

// per-pair source of the complex64 tiles: a raster (or the arena of the reference worker),
// the chip of pair p at ref_base + ref_off[p] with row stride ref_stride pixels, the search
// window at tgt_base + tgt_off[p] with row stride tgt_stride
struct PairSource {
    const float2* ref_base;
    const long long* ref_off;
    long long ref_stride;
    const float2* tgt_base;
    const long long* tgt_off;
    long long tgt_stride;
    long long ref_count;  // samples behind ref_base (the raster or the arena)
    long long tgt_count;
    long long tgt_lines;  // lines of the secondary raster (tgt_count / tgt_stride); 0 for the arena
};

// coarse result of one pair
struct CoarseOut {
    int u, v;          // argmax placement
    int top, left;     // nudged corner of the refinement neighbourhood inside the window
};

// optional per-pair diagnostics (matches ampcor_pair_diag in the public header)
struct PairDiag {
    int coarse_u, coarse_v;
    int top, left;
    int refined_u, refined_v;
    int fine_p, fine_q;
    float coarse_peak;
    float refined_peak;
    float zoom_peak;
    float pad;
};

// dense fp32 amplitude tiles of a chunk of pairs (the refined tiles): the tile set of chunk-local
// pair q starts at base + q * stride; the chip (R x R, row stride R) at chip_off and the window
// (W x W, row stride W) at win_off within it
struct RealTiles {
    const float* base;
    long long stride;
    long long chip_off;
    long long win_off;
};

// the tensor-core form of one correlation surface: D[v][u] = sum_w sum_j A_w[v][j] B_w[j][u]
// accumulated in tensor memory, A_w[v][j] = t(w, v + j) (window row w, read through overlapping
// 16-byte rows X[p] = t(w, p .. p+7)), B_w[j][u] = r'(w - u, j) (the zero-mean chip, rows
// reversed, so that B_w is a window of one fixed buffer that slides by one row per window row)
struct TcGeom {
    int R, W, C;
    int M;          // accumulator lanes used (placement columns v): 64 when C <= 64, else 128
    int N;          // accumulator columns (placement rows u), multiple of 16, >= C
    int JC;         // chip columns per pass over the window rows (multiple of 16)
    int nchunks;    // passes: ceil(R / JC)
    int Q;          // rows of the reversed-chip buffer: W + N - 1
    int XR;         // 16-byte rows of one window-row operand: M + JC - 8
    int RB;         // floats of one window-row buffer: XR + 8
    int nst;        // operand stages in flight
    int nacc;       // accumulators: window row it goes to accumulator it % nacc
    int tmem_cols;  // tensor-memory columns allocated (power of two >= nacc N)
    int off_crev, off_x, off_row, off_raw, off_bar, off_misc;   // shared-memory regions, bytes
    int smem_bytes;
};

// refined-surface maximum of one pair
struct FineOut {
    int u, v;
    float peak;
    float pad;
};

__global__ void pair_offsets_kernel(const int* ulhc, long long pairs, long long ref_lines,
                                    long long ref_samples, long long tgt_lines,
                                    long long tgt_samples, int R, int W, long long* ref_off,
                                    long long* tgt_off, unsigned int* bad);

__global__ void arena_offsets_kernel(long long pairs, long long ref_cells, long long tgt_cells,
                                     long long* ref_off, long long* tgt_off);

__global__ void coarse_kernel(PairSource src, long long pair0, long long pairs, NccGeom g, int m,
                              CoarseOut* out, float* coarse_peak, float* surfaces);

__global__ void refine_kernel(PairSource src, long long pair0, long long pairs,
                              const CoarseOut* coarse, InterpGeom chip_g, InterpGeom win_g,
                              const float* chip_taps, const float* win_taps, float* refined,
                              long long refined_stride, int deramp);

__global__ void fine_kernel(const float* refined, long long refined_stride, long long pair0,
                            long long pairs, const long long* ref_off, NccGeom g, ZoomGeom zg,
                            const float* zoom_taps, const CoarseOut* coarse,
                            const float* coarse_peak, int margin, int refine_factor,
                            int refine_margin, int ref_compat, float2* offsets, PairDiag* diag,
                            float* surfaces);

// FP64 window statistics of every placement, 1/sqrt(sum (t - mu)^2) (0 for a flat box), for the
// tensor-core form: C^2 floats per chunk-local pair
__global__ void window_stats_cplx_kernel(PairSource src, long long pair0, long long pairs, NccGeom g,
                                         float* inv);
__global__ void window_stats_real_kernel(RealTiles t, long long pairs, NccGeom g, float* inv);

// tensor-core correlation (bf16x3 split products, FP32 accumulation in tensor memory)
__global__ void tc_coarse_kernel(PairSource src, long long pair0, long long pairs, TcGeom g,
                                 const float* inv, int m, CoarseOut* out, float* coarse_peak,
                                 float* surfaces, unsigned int* err);
__global__ void tc_fine_kernel(RealTiles t, long long pair0, long long pairs, TcGeom g,
                               const float* inv, const long long* ref_off, FineOut* fout,
                               float* gam, float* surfaces, unsigned int* err);

// zoom of the refined surfaces of a chunk (C^2 floats per chunk-local pair), offsets
__global__ void zoom_kernel(const float* gam, long long pair0, long long pairs,
                            const long long* ref_off, ZoomGeom zg, const float* zoom_ut,
                            const CoarseOut* coarse, const float* coarse_peak, const FineOut* fout,
                            int margin, int refine_factor, int refine_margin, int ref_compat,
                            float2* offsets, PairDiag* diag);

// tensor-core zoom (3xTF32): Zm = U G U^T with U the Z x Cf interpolation matrix, as
// T^T = U G^T then Zm = U T; planes of K-major core matrices (8 rows x 16 bytes), K = Cf padded
// to KC 16-byte chunks (KC even)
struct ZoomTcGeom {
    int Cf, z, Z;
    int KC;        // 4-float chunks per operand row
    int NG;        // rows of the G planes (Cf rounded to 16): N of the first product
    int mtiles;    // tiles of rows (of T^T and of Zm): 128 each, the last one last_m (64 or 128)
    int last_m;
    int nparts;    // accumulator parts of Zm columns (1 or 2), npart columns each, 256 apart
    int npart;
    int tmem_cols;
    int off_ahi, off_alo, off_bhi, off_blo, off_ghi, off_glo, off_bar, off_misc;  // smem bytes
    int smem_bytes;
};

// threads of tc_zoom_kernel: four warps per tensor-memory lane quarter
constexpr int kTcZoomThreads = 512;

// zoom of the refined surfaces of a chunk on the tensor cores; same outputs as zoom_kernel.
// uhl: the hi and lo planes of U, contiguous.  One CTA per SM walks the pairs.  stall != 0 (a
// failure-detection test) makes every CTA's first wait on a barrier nothing completes: the
// bounded wait runs out before any work is issued and the chunk reports a time-out in err_out.
__global__ void tc_zoom_kernel(const float* gam, long long pair0, long long pairs,
                               const long long* ref_off, ZoomTcGeom zt, const float* uhl,
                               const CoarseOut* coarse, const float* coarse_peak,
                               const FineOut* fout, int margin, int refine_factor,
                               int refine_margin, int ref_compat, float2* offsets, PairDiag* diag,
                               unsigned int* err_out, int stall);

// spectral form: FFT correlation of one tile pair per CTA (512 threads, one CTA per SM).  The
// N x N tile (N = N1 N2 >= W, row stride RS = N + 1 complex samples) holds the window in its real
// parts and the zero-mean chip in its imaginary parts.
struct SpecGeom {
    int R, W, C;      // chip, window, placements per axis
    int N, N1, N2;    // transform length and its two register radices
    int RS;           // tile row stride (complex samples)
    int off_z, off_tw, off_neg, off_half, off_red, off_inv, off_gam;  // shared-memory byte offsets
    // placement statistics computed in the kernel (no InvSource given): nseg threads per window
    // column, their FP64 partial sums (4 nseg W doubles) at off_gam (the surface buffer, idle
    // until the last transform step), the column sums in the tile's imaginary parts and, past the
    // tile, right after the partial sums
    int nseg;
    int smem_bytes;
    // staged form (spec_staged_kernel, windows copied in while the previous pair finishes): the
    // window's W rows of stage_rs floats at off_stage (over the tile's last rows), the copy's
    // mbarrier at off_bar (and the CTA's wait-failure flag right after it);
    // tile rows below stage_y0 are written straight from the staged copy, the rows from stage_y0 on
    // in groups of stage_pj x 16 rows read whole before they are written
    int off_stage, off_bar, stage_y0, stage_pj, stage_rs;
    int off_inv_raw, inv_rs;  // raster statistics as copied: C rows of inv_rs floats
    int smem_staged;  // 0: no staged form for this stage
};

// float amplitude tiles of chunk-local pair b (global pair pair0 + b): at base + off[pair0 + b]
// when off is given, else at base + b * step; rows stride apart
struct SpecSource {
    const float* chip;
    long long chip_stride;
    const long long* chip_off;
    long long chip_step;
    const float* win;
    long long win_stride;
    const long long* win_off;
    long long win_step;
};

// what a spectral correlation writes: stage 0 the coarse maximum (nudged corners, peak and
// optionally the surface), stage 1 the refined maximum and the refined surface for the zoom
struct SpecOut {
    int stage;
    int m;  // refinement margin (the nudge)
    CoarseOut* coarse;
    float* coarse_peak;
    FineOut* fine;
    float* gam;       // chunk-local refined surfaces (stage 1)
    float* surfaces;  // optional, indexed by global pair
};

// |z| of every sample of a complex array (n samples)
__global__ void detect_kernel(const float2* src, long long n, float* dst);
// FP64 box statistics of an amplitude raster, for windows that overlap (the coarse stage of a
// raster job): column sums over R rows (v1: sum a, v2: sum a^2) for box rows [row_lo, row_hi)
// (box row y covers raster rows y .. y + R - 1; row_lo a multiple of kVBlock, so that a band
// computes its rows exactly as the whole raster would), then per box row prefix sums and
// 1/sqrt(var) of the R x R box at every (y, x), x <= samples - R
constexpr int kVBlock = 64;  // rows slid per thread of the column sums
__global__ void box_vsum_kernel(const float* a, long long samples, int R, long long row_lo,
                                long long row_hi, double* v1, double* v2);
__global__ void box_inv_kernel(const double* v1, const double* v2, long long row_lo, long long row_hi,
                               long long samples, int R, float* inv);

// where a spectral correlation finds 1/sigma_box of placement (u, v) of chunk-local pair b:
// base + off[pair0 + b] + u stride + v when off is given, else base + b C^2 + u C + v
struct InvSource {
    const float* base;
    const long long* off;
    long long stride;
};

// per-pair chip statistics of a blocked spectral stage: the chip's FP64 mean and 1/|r - mean|
struct ChipStat {
    double mean;
    double inv_sigma;
};

// the transform lengths that are compiled, with their radices
bool spec_radices(int n, int& n1, int& n2);
int spec_next_length(int w);
// allow every instantiation its shared memory; call once per device
cudaError_t spec_set_smem_limits();
// refinement by zero-padded FFT for an N x N tile and factor f, when compiled (smem: its bytes)
bool spec_refine_supported(int n, int f, int& smem);
// refinement in strips through a per-pair buffer of N x 2N complex samples in global memory
// (ybuf, blocks of them): tiles too large for one CTA's shared memory (N in 96 .. 160, f = 2), and
// with `strips` the shorter compiled lengths too (less shared memory, more CTAs per SM)
bool spec_refine_big_supported(int n, int f, int& smem);
// refinement of raster windows by the staged kernel (one resident CTA per SM, the next tile copied
// in by the copy engine): whether compiled for N x N tiles and factor f, its shared memory and the
// width (floats) of the tensor map's box; tmap maps the secondary raster as floats (2 per sample)
// with boxes of box_x x N floats
bool spec_refine_staged_supported(int n, int f, int& smem, int& box_x);
cudaError_t launch_spec_refine_staged(int n, unsigned sms, cudaStream_t st, const CUtensorMap* tmap,
                                      const long long* off, long long stride, const CoarseOut* coarse,
                                      long long pair0, long long pairs, const long long* valid,
                                      const float2* twn, const float2* twf, float* refined,
                                      long long refined_stride, long long out_off, unsigned int* errs);
cudaError_t launch_spec_refine(int n, unsigned blocks, cudaStream_t st, const float2* base,
                               const long long* off, long long stride, const CoarseOut* coarse,
                               long long pair0, long long pairs, const long long* valid,
                               const float2* twn, const float2* twf, float* refined,
                               long long refined_stride, long long out_off, int deramp,
                               float2* ybuf, bool strips);

// blocked spectral correlation (windows too large for one tile; see spectral.cu): per chunk of
// pairs the chip statistics, the placement statistics when no raster gives them, the partial
// numerators of every (pair, chip block) and their per-pair reduction to the stage's outputs
cudaError_t launch_spec_chip_stats(unsigned blocks, cudaStream_t st, SpecSource src, long long pair0,
                                   long long pairs, const long long* valid, int R, ChipStat* out);
int spec_tile_stats_rows(int W, int C, int& smem);
cudaError_t launch_spec_tile_stats(unsigned blocks, cudaStream_t st, SpecSource src, long long pair0,
                                   long long pairs, const long long* valid, int R, int W, float* inv);
cudaError_t launch_spec_block(const SpecGeom& tile, int nb, unsigned blocks, cudaStream_t st,
                              SpecSource src, long long pair0, long long pairs,
                              const long long* valid, const ChipStat* cstat, const float2* tw,
                              float* part, double* scal);
int spec_reduce_smem(int C);
cudaError_t launch_spec_reduce(const SpecGeom& full, int K, unsigned blocks, cudaStream_t st,
                               SpecSource src, long long pair0, long long pairs,
                               const long long* valid, const ChipStat* cstat, InvSource inv,
                               const float* part, const double* scal, SpecOut out);
cudaError_t launch_spec(const SpecGeom& g, unsigned blocks, cudaStream_t st, SpecSource src,
                        long long pair0, long long pairs, const long long* valid, InvSource inv,
                        const float2* tw, SpecOut out);
// the staged form: min(pairs, sms) resident CTAs walk the chunk; a bounded wait that runs out is
// counted in errs.  Refined tiles: wmap and cmap null, no statistics given.  Raster windows:
// wmap, cmap and imap 2-D maps of the secondary and reference amplitude rasters and of the
// secondary's box statistics (inv) with boxes of stage_rs x W, (R + 6 & ~3) x R and inv_rs x C
// floats.  stall: the failure-detection test's wait on a barrier that nothing completes.
cudaError_t launch_spec_staged(const SpecGeom& g, unsigned sms, cudaStream_t st, SpecSource src,
                               long long pair0, long long pairs, const long long* valid, InvSource inv,
                               const float2* tw, SpecOut out, unsigned int* errs, const CUtensorMap* wmap,
                               const CUtensorMap* cmap, const CUtensorMap* imap, int stall);

}  // namespace ampcor_b200
