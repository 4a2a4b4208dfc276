// C ABI and host orchestration of the batched tile correlator.
//
// The worker (ampcor_handle) plays the role of ampcor::cuda::correlators::Sequential
// (lib/libampcor_cuda/correlators/Sequential.h, Sequential.icc): it derives the tile layouts from
// the constructor arguments, owns the host arena of the pair-by-pair API and runs the pipeline.
// Unlike the reference it allocates its device memory once and reuses it, runs the stages on its
// own stream with no synchronisation between them, and returns status codes instead of
// throwing.
#include "../../include/ampcor_b200.h"
#include "kernels.cuh"

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

using namespace ampcor_b200;

namespace {

const char* kVersion = "ampcor_b200 0.1.0 (sm_100a)";
const char* kCopyright =
    "ampcor_b200: B200-native batched tile correlator with the worker interface of "
    "isce-framework/ampcor";

std::mutex g_create_mutex;
std::string g_create_error;

constexpr int kCompiledNV[] = {9, 16, 17, 32, 33};

// correlation forms (the values ampcor_form returns and ampcor_configure takes)
constexpr int kFormPlain = 0;
constexpr int kFormTensor = 1;
constexpr int kFormSpectral = 2;

int round_nv(int w)
{
    for (int nv : kCompiledNV)
        if (nv >= w) return nv;
    return -1;
}

int odd_at_least(int x) { return (x % 2) ? x : x + 1; }

int ncc_block_width()
{
    const char* env = std::getenv("AMPCOR_NCC_BLOCK");
    if (env && std::atoi(env) == 16) return 16;
    return 32;
}
int round4(int x) { return (x + 3) & ~3; }

// split of one correlation surface over the warps of a CTA and its shared-memory layout;
// extra_win / extra_chip reserve room for the zoom stage of the fine kernel
bool plan_ncc(int R, int W, int extra_win, int extra_chip, NccGeom& g, std::string& err)
{
    std::memset(&g, 0, sizeof(g));
    const int C = W - R + 1;
    if (R < 2 || C < 1) {
        err = "chip must be at least 2x2 and no larger than the search window";
        return false;
    }
    g.R = R;
    g.W = W;
    g.C = C;
    // column blocks: a first block of up to bw + 1 placements, then blocks of bw (bw = 32, or 16
    // with AMPCOR_NCC_BLOCK=16 for a smaller unrolled loop; on B200 both run at the same speed)
    const int bw = ncc_block_width();
    const int blocks = (C <= bw + 1) ? 1 : 1 + (C - (bw + 1) + bw - 1) / bw;
    if (blocks > kMaxVB) {
        err = "search margin too large for this build (at most 8 column blocks)";
        return false;
    }
    g.n_vb = blocks;
    int v0 = 0;
    int need_s = W, need_cs = R;
    for (int b = 0; b < blocks; ++b) {
        const int w = (b == 0) ? C - bw * (blocks - 1) : bw;
        const int nv = round_nv(w);
        if (nv < 0) {
            err = "internal: no register block for width " + std::to_string(w);
            return false;
        }
        const int steps = (R + nv - 1) / nv;
        g.vb_v0[b] = v0;
        g.vb_w[b] = w;
        g.vb_nv[b] = nv;
        g.vb_steps[b] = steps;
        need_s = std::max(need_s, v0 + steps * nv + nv);
        need_cs = std::max(need_cs, steps * nv);
        v0 += w;
    }
    g.S = odd_at_least(need_s);
    g.CS = odd_at_least(need_cs);
    g.n_ub = C / 32;
    if (g.n_ub * g.n_vb > kWarps) {
        err = "search margin too large for this build (placement blocks exceed the warps)";
        return false;
    }
    g.n_kc = g.n_ub ? std::min(R, std::max(1, kWarps / (g.n_ub * g.n_vb))) : 0;
    g.n_main = g.n_ub * g.n_vb * g.n_kc;
    g.n_tkc = (R + 31) / 32;
    g.stat_rows = kStatRows;
    g.n_trans = (C - 32 * g.n_ub) * g.n_vb * g.n_tkc;

    const int win_f = std::max({W * g.S, g.n_main * 32 * kSlot, extra_win});
    const int chip_f = std::max({R * g.CS, 4 * kStatRows * (W + 1), extra_chip});
    int off = 0;
    g.off_win = off;
    off += round4(win_f);
    g.off_chip = off;
    off += round4(chip_f);
    g.off_inv = off;
    off += round4(C * C);
    g.off_gam = off;
    off += round4(C * C);
    g.off_trans = off;
    off += round4(std::max(1, g.n_trans) * kSlot);
    g.off_red = off;
    off += 128;
    g.off_aux = off;
    g.smem_bytes = off * 4;
    if (g.smem_bytes > 227 * 1024) {
        err = "tile geometry needs " + std::to_string(g.smem_bytes) +
              " bytes of shared memory; this build supports at most 232448";
        return false;
    }
    return true;
}

bool plan_interp(int N, int f, InterpGeom& ig, std::string& err)
{
    std::memset(&ig, 0, sizeof(ig));
    if (N % kQB) {
        err = "refinement tiles must be a multiple of 8 pixels (chip and chip + 2 * refine margin)";
        return false;
    }
    ig.N = N;
    ig.f = f;
    ig.F = f * N;
    ig.NS = odd_at_least(N);
    ig.YS = odd_at_least(ig.F);
    ig.taps_len = 2 * N + 2 * kQB;
    int off = 0;
    ig.off_x = off;
    off += round4(2 * N * ig.NS);
    ig.off_y = off;
    off += round4(2 * N * ig.YS);
    ig.off_taps = off;
    off += round4(std::max(1, f - 1) * ig.taps_len);
    ig.smem_bytes = off * 4;
    if (ig.smem_bytes > 227 * 1024) {
        err = "refinement tile too large for shared memory in this build";
        return false;
    }
    return true;
}

// the tensor-core form of one surface: needs C <= 128 (the accumulator's 128 lanes hold the
// placement columns) and C <= 256 accumulator columns
bool plan_tc(int R, int W, int raw_bytes, TcGeom& g, std::string& err)
{
    std::memset(&g, 0, sizeof(g));
    const int C = W - R + 1;
    if (C < 1 || C > 128) {
        err = "the tensor-core form needs at most 128 placements per axis";
        return false;
    }
    g.R = R;
    g.W = W;
    g.C = C;
    g.M = C <= 64 ? 64 : 128;
    g.N = (C + 15) / 16 * 16;
    g.JC = std::min(64, (R + 15) / 16 * 16);
    g.nchunks = (R + g.JC - 1) / g.JC;
    g.Q = W + g.N - 1;
    g.XR = g.M + g.JC - 8;
    g.RB = g.XR + 8;
    g.nst = 3;  // stages of 2 window rows each
    // the tensor cores truncate when they add into an FP32 accumulator, which shrinks long sums
    // by a relative amount that grows with the number of additions; spreading the window rows over
    // several accumulators (summed with round-to-nearest at the end) divides that bias by their
    // count.  256 columns per CTA keeps two CTAs per SM within the 512 columns of an SM.
    g.nacc = std::max(1, std::min(8, 256 / g.N));
    g.tmem_cols = 32;
    while (g.tmem_cols < g.nacc * g.N) g.tmem_cols *= 2;
    auto up = [](int x, int a) { return (x + a - 1) / a * a; };
    int off = 0;
    g.off_crev = off;
    off = up(off + 2 * (g.JC / 8) * g.Q * 16, 1024);
    const int rows_per_stage = 2, prefetch = 2 * rows_per_stage;
    g.off_x = off;
    off = up(off + g.nst * rows_per_stage * 2 * g.XR * 16, 1024);
    g.off_row = off;
    off = up(off + g.nst * rows_per_stage * g.RB * 4, 128);
    g.off_raw = off;  // raw window rows in flight, RB elements each (complex64 or fp32)
    off = up(off + prefetch * g.RB * raw_bytes, 128);
    g.off_bar = off;
    off = up(off + (2 * g.nst + 2) * 8, 128);
    g.off_misc = off;
    off += 256;
    g.smem_bytes = off;
    if (g.Q > 16383 || g.smem_bytes > 227 * 1024) {
        err = "tile geometry too large for the tensor-core form";
        return false;
    }
    return true;
}

// the spectral form of one surface: transform length N >= W from the compiled lengths; shared
// memory: the N x (N + 1) complex tile, twiddles, the partner table of the spectrum product and
// a reduction scratch
bool plan_spec(int R, int W, SpecGeom& g, std::string& err)
{
    std::memset(&g, 0, sizeof(g));
    g.R = R;
    g.W = W;
    g.C = W - R + 1;
    g.N = spec_next_length(W);
    if (g.N == 0 || !spec_radices(g.N, g.N1, g.N2)) {
        err = "the spectral form needs a window of at most 160 samples";
        return false;
    }
    auto up = [](long x, long a) { return (x + a - 1) / a * a; };
    g.RS = g.N + 1;
    long off = up((long)g.N * g.RS * 8, 16);
    g.off_z = 0;
    g.off_tw = (int)off;
    off = up(off + (long)g.N * 8, 16);
    g.off_neg = (int)off;
    off = up(off + (long)g.N * 4, 16);
    g.off_half = (int)off;  // one position of every Hermitian pair of the spectrum
    off = up(off + (long)(g.N / 2 + 1) * 4, 16);
    g.off_red = (int)off;
    off += 2L * kSpecWarps * 8;
    g.off_inv = (int)off;  // the placement statistics, prefetched with the tiles
    off = up(off + (long)g.C * g.C * 4, 16);
    g.off_gam = (int)off;  // the normalised surface; before the last step, the statistics' scratch
    const long limit = 227L * 1024;
    // column sums (two floats a placement row and window column) past the tile's imaginary parts
    const long over = std::max<long>(0, 2L * g.C * g.W - (long)g.N * g.RS) * 4;
    g.nseg = std::max(1, kSpecThreads / g.W);
    while (g.nseg > 1 && off + 32L * g.nseg * g.W + over > limit) --g.nseg;
    off = up(off + std::max<long>((long)g.C * g.C * 4, 32L * g.nseg * g.W + over), 16);
    if (off > limit) {
        err = "tile geometry too large for the spectral form";
        return false;
    }
    g.smem_bytes = (int)off;
    return true;
}

// The staged form of a stage (spec_staged_kernel), a layout of its own: the tile, then the
// window's W rows of stage_rs floats at off_stage, which the correlation leaves alone from its
// inverse column pass on (it keeps its first rows_out + (rows_out + 1) / 2 rows): at the tile's
// end where the tile has room, else right after the kept rows and on past the tile; the
// statistics' column sums fit below them.  Tile rows below the staged bytes are written as they
// are read, the others in pieces of kStagePieces row groups, none of which may reach the staged
// rows of a later piece.  Rows whose samples may sit off 16-byte boundaries (`dense` false, or W
// not a multiple of 4) get 3 + W floats rounded up to 16 bytes.
constexpr int kStagePieces = 5;  // spec_staged_kernel's PJ

bool plan_spec_staged(int R, int W, bool dense, SpecGeom& g)
{
    std::string e;
    if (!plan_spec(R, W, g, e)) return false;
    auto up = [](long x, long a) { return (x + a - 1) / a * a; };
    const int N = g.N, C = g.C;
    const long row = (long)g.RS * 8, tile = (long)N * row;
    g.stage_rs = dense && W % 4 == 0 ? W : (W + 6) & ~3;
    const long stage = (long)W * g.stage_rs * 4;
    const int np = (C + 1) / 2;
    const long kept = (long)(C + np <= N ? C + np : C) * row;
    const long S = up(std::max(kept, tile - stage), 128);
    if (2L * C * W * 4 > S) return false;
    const int y0 = (int)std::min<long>(N, S / row) / kSpecWarps * kSpecWarps;
    const int JN = (N + kSpecWarps - 1) / kSpecWarps;
    for (int j0 = 0; j0 < JN; j0 += kStagePieces) {
        const long y1 = (long)std::min(j0 + kStagePieces, JN) * kSpecWarps;
        if (y1 <= y0 || y1 >= W) continue;
        if (y1 * row > S + y1 * g.stage_rs * 4) return false;
    }
    g.off_stage = (int)S;
    g.stage_y0 = y0;
    g.stage_pj = kStagePieces;
    long off = up(std::max(tile, S + stage), 16);
    g.off_tw = (int)off;
    off = up(off + (long)N * 8, 16);
    g.off_neg = (int)off;
    off = up(off + (long)N * 4, 16);
    g.off_half = (int)off;
    off = up(off + (long)(N / 2 + 1) * 4, 16);
    g.off_red = (int)off;
    off += 4L * kSpecWarps * 8;
    g.off_inv = (int)off;
    off = up(off + (long)C * C * 4, 16);
    g.off_gam = (int)off;  // the surface; before the last step, the statistics' partial sums
    const long limit = 227L * 1024 - 32;
    g.nseg = std::max(1, kSpecThreads / W);
    while (g.nseg > 1 && off + 32L * g.nseg * W > limit) --g.nseg;
    off = up(off + std::max<long>((long)C * C * 4, 32L * g.nseg * W), 128);
    // raster statistics as the copy engine brings them (rows from the window's 16-byte boundary)
    g.inv_rs = (C + 6) & ~3;
    g.off_inv_raw = dense ? 0 : (int)off;
    if (!dense) off = up(off + (long)C * g.inv_rs * 4, 16);
    g.off_bar = (int)off;
    off += 32;  // the copy's mbarrier, the wait-failure flag, the failure-detection test's mbarrier
    g.smem_staged = off <= 227L * 1024 ? (int)off : 0;
    return g.smem_staged > 0;
}

// A stage of the spectral form whose window is too large for one tile: the chip splits into nb x nb
// square blocks of side B (B divides R), each block's sub-window (B + C - 1 samples a side) one
// tile; the largest B whose tile fits is taken.  `full` describes the whole stage for the
// reduction.
struct SpecBlocks {
    bool on = false;
    int B = 0, nb = 0, K = 0;
    SpecGeom tile{};
    SpecGeom full{};
};

bool plan_spec_tile(int B, int S, int C, SpecGeom& g)
{
    std::memset(&g, 0, sizeof(g));
    g.R = B;
    g.W = S;
    g.C = C;
    g.N = spec_next_length(S);
    if (g.N == 0 || !spec_radices(g.N, g.N1, g.N2)) return false;
    auto up = [](long x, long a) { return (x + a - 1) / a * a; };
    g.RS = g.N + 1;
    long off = up((long)g.N * g.RS * 8, 16);
    g.off_z = 0;
    g.off_tw = (int)off;
    off = up(off + (long)g.N * 8, 16);
    g.off_neg = (int)off;
    off = up(off + (long)g.N * 4, 16);
    g.off_half = (int)off;
    off = up(off + (long)(g.N / 2 + 1) * 4, 16);
    g.off_red = (int)off;
    off += 2L * kSpecWarps * 8;
    g.smem_bytes = (int)off;
    return off <= 227L * 1024;
}

bool plan_spec_blocked(int R, int W, SpecBlocks& b, std::string& err)
{
    b = SpecBlocks{};
    const int C = W - R + 1;
    int tile_smem = 0;
    if (R < 1 || C < 1 || spec_tile_stats_rows(W, C, tile_smem) == 0 || spec_reduce_smem(C) > 227 * 1024) {
        err = "the blocked spectral form needs a window of at most 512 samples and at most 165 "
              "placements per axis";
        return false;
    }
    for (int B = R; B >= 1; --B) {
        if (R % B) continue;
        const int nb = R / B;
        if (nb * nb > 64) break;
        if (!plan_spec_tile(B, B + C - 1, C, b.tile)) continue;
        b.on = true;
        b.B = B;
        b.nb = nb;
        b.K = nb * nb;
        b.full.R = R;
        b.full.W = W;
        b.full.C = C;
        return true;
    }
    err = "no block of the chip fits the spectral form (the search margin is too large)";
    return false;
}

// the tensor-core zoom: operand planes, accumulator parts and row tiles; false when Zm does not fit
// (more than 512 accumulator columns or more shared memory than a CTA has)
bool plan_zoom_tc(int Cf, int z, ZoomTcGeom& g)
{
    std::memset(&g, 0, sizeof(g));
    g.Cf = Cf;
    g.z = z;
    g.Z = Cf * z;
    const int KP = (Cf + 7) / 8 * 8;
    g.KC = KP / 4;
    g.NG = (Cf + 15) / 16 * 16;
    if (g.NG > 64) return false;
    const int zq = (g.Z + 15) / 16 * 16;
    g.nparts = zq > 256 ? 2 : 1;
    g.npart = ((zq + g.nparts - 1) / g.nparts + 15) / 16 * 16;
    if (g.npart > 256) return false;
    const int full = g.Z / 128, rem = g.Z - 128 * full;
    g.mtiles = full + (rem ? 1 : 0);
    g.last_m = (rem == 0 || rem > 64) ? 128 : 64;
    // accumulators: two buffers of one Zm unit (npart columns) at columns 0 and 256; the row
    // tiles of T^T at columns 64 mt
    g.tmem_cols = 512;
    if (64 * g.mtiles > 512) return false;
    const long rg = (long)g.KC * 128;
    const long plane_a = (long)((g.Z + 7) / 8) * rg;
    const long plane_b = (long)(g.nparts * g.npart / 8) * rg;
    const long plane_g = (long)(g.NG / 8) * rg;
    // the last row tile may read row groups past U; they must land in the next plane (U's lo
    // plane, then the B planes)
    const long over = (long)(128 * (g.mtiles - 1) + g.last_m - (g.Z + 7) / 8 * 8) / 8 * rg;
    if (over > plane_b) return false;
    long off = 0;
    g.off_ahi = 0;
    g.off_alo = (int)(off += plane_a);
    g.off_bhi = (int)(off += plane_a);
    g.off_blo = (int)(off += plane_b);
    g.off_ghi = (int)(off += plane_b);
    g.off_glo = (int)(off += plane_g);
    off += plane_g;
    g.off_bar = (int)off;
    off += 48;  // five mbarriers (the fifth is waited on only by failure-detection tests)
    g.off_misc = (int)off;
    off += 256;  // tensor-memory address, error flag, and the block maximum's per-warp slots
    g.smem_bytes = (int)off;
    return off <= 227L * 1024;
}

double dirichlet(int N, double d);

// hi and lo tf32 planes of U (U[p][a] = D_Cf(p / z - a), an identity row for p % z == 0), rows of
// K-major core matrices; K past Cf is zero
std::vector<float> zoom_u_planes(const ZoomTcGeom& g)
{
    const int rows = (g.Z + 7) / 8 * 8;
    const size_t plane = (size_t)rows * g.KC * 4;
    std::vector<float> out(2 * plane, 0.0f);
    for (int p = 0; p < g.Z; ++p)
        for (int a = 0; a < g.Cf; ++a) {
            const int s = p % g.z, b = p / g.z;
            const float u = s == 0 ? (b == a ? 1.0f : 0.0f) : (float)dirichlet(g.Cf, (double)p / g.z - a);
            // round to tf32: nearest, ties away from zero
            uint32_t bits;
            std::memcpy(&bits, &u, 4);
            bits = (bits + 0x1000u) & 0xFFFFE000u;
            float hi;
            std::memcpy(&hi, &bits, 4);
            const float lo = u - hi;
            const size_t off = (size_t)((p / 8) * g.KC + a / 4) * 32 + (p % 8) * 4 + a % 4;
            out[off] = hi;
            out[plane + off] = lo;
        }
    return out;
}

// exp(-2 pi i m / N), m < N, rounded from FP64
std::vector<float> spec_twiddle_table(int N)
{
    std::vector<float> t(2 * (size_t)N);
    for (int m = 0; m < N; ++m) {
        t[2 * m] = (float)std::cos(2.0 * M_PI * m / N);
        t[2 * m + 1] = (float)-std::sin(2.0 * M_PI * m / N);
    }
    return t;
}

// shared memory of the statistics kernels: the staged window and the FP64 column-sum chunk
// (unpadded window rows: the statistics walk columns, one thread per column; the chunk of
// column sums shrinks until two CTAs fit on an SM)
NccGeom stats_layout(const NccGeom& g)
{
    NccGeom s = g;
    s.S = g.W;
    s.off_win = 0;
    s.off_chip = round4(g.W * g.W);
    s.stat_rows = kStatRows;
    while (s.stat_rows > 1 && (s.off_chip + 4 * s.stat_rows * (g.W + 1)) * 4 > 110 * 1024) s.stat_rows /= 2;
    s.smem_bytes = (s.off_chip + 4 * s.stat_rows * (g.W + 1)) * 4;
    return s;
}

// band-limited interpolation kernel of an N-periodic sequence (Nyquist pair halved for even N):
// the zero-padded inverse FFT with a 1/N scale, written as a sum of cosines
double dirichlet(int N, double d)
{
    double s = 1.0;
    if (N % 2) {
        for (int n = 1; n <= (N - 1) / 2; ++n) s += 2.0 * std::cos(2.0 * M_PI * n * d / N);
    } else {
        for (int n = 1; n < N / 2; ++n) s += 2.0 * std::cos(2.0 * M_PI * n * d / N);
        s += std::cos(M_PI * d);
    }
    return s / N;
}

// taps[s][d] = D_N(d - (N-1) + s/f) for phases s in [s0, f)
std::vector<float> taps_table(int N, int f, int s0, int len)
{
    std::vector<float> t((size_t)(f - s0) * len);
    for (int s = s0; s < f; ++s)
        for (int d = 0; d < len; ++d)
            t[(size_t)(s - s0) * len + d] = (float)dirichlet(N, d - (N - 1) + (double)s / f);
    return t;
}

}  // namespace

// bands of a host-buffer job of the spectral form: the rasters go up band by band while the pairs
// whose tiles lie in the bands already up are correlated
constexpr int kHostBands = 12;

struct ampcor_handle {
    ampcor_params prm{};
    int R = 0, W = 0, C = 0, M = 0, E = 0, f = 0, m = 0, z = 0, Rf = 0, Wf = 0, Cf = 0, Z = 0;
    NccGeom gc{}, gf{};
    InterpGeom ic{}, iw{};
    ZoomGeom zg{};
    int refine_smem = 0;
    cudaStream_t stream = nullptr;
    // host-buffer jobs: raster bands uploaded on their own stream, one event per band
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t band_ev[kHostBands + 1] = {};
    float* d_chip_taps = nullptr;
    float* d_win_taps = nullptr;
    float* d_zoom_taps = nullptr;
    float* d_zoom_ut = nullptr;
    // arena API
    float2* h_arena = nullptr;
    float2* d_arena = nullptr;
    float* h_offsets = nullptr;
    // per-pair buffers
    size_t cap = 0;
    long long* d_ref_off = nullptr;
    long long* d_tgt_off = nullptr;
    CoarseOut* d_coarse = nullptr;
    float* d_coarse_peak = nullptr;
    float2* d_offsets = nullptr;
    PairDiag* d_diag = nullptr;
    unsigned int* d_bad = nullptr;
    // refined amplitudes of one chunk of pairs
    float* d_refined = nullptr;
    size_t chunk = 0;
    size_t chunk_override = 0;
    long long refined_stride = 0;
    // host-path staging
    void* d_ref_raster = nullptr;
    void* d_tgt_raster = nullptr;
    size_t raster_bytes_ref = 0, raster_bytes_tgt = 0;
    int32_t* d_ulhc = nullptr;
    size_t ulhc_cap = 0;
    float* d_job_offsets = nullptr;
    size_t job_offsets_cap = 0;
    ampcor_pair_diag* d_job_diag = nullptr;
    size_t job_diag_cap = 0;
    // correlation form (kFormPlain, kFormTensor, kFormSpectral)
    int form = 0;
    SpecGeom spc{}, spf{};
    // the staged forms of both stages (spec_staged_kernel: one resident CTA per SM, windows
    // copied in while the previous pair finishes), where planned; sms: the device's
    // multiprocessors
    SpecGeom spc_st{}, spf_st{};
    bool coarse_staged = false, fine_staged = false;
    bool staged_on = false;  // the staged forms are allowed (AMPCOR_STAGED is not 0)
    int sms = 0;
    // tensor-core zoom (both the tensor-core and the spectral forms), when Zm fits
    bool zoom_tc = false;
    ZoomTcGeom ztc{};
    float* d_zoom_uhl = nullptr;
    float* d_tw_c = nullptr;
    float* d_tw_f = nullptr;
    // refinement by zero-padded FFT (spectral form): twiddles of R, f R, E and f E, in that order;
    // tiles too large to stage whole go through a per-pair buffer (d_upy, chunk x upy_len)
    bool refine_fft = false;
    float* d_tw_refine = nullptr;
    bool refine_big = false;
    bool refine_strips = false;  // every refinement through the strip kernel (AMPCOR_REFINE_STRIPS)
    float2* d_upy = nullptr;
    long long upy_len = 0;
    // blocked spectral stages (coarse, fine): chip statistics, placement statistics, partial
    // numerators and their scalars, all per chunk
    SpecBlocks bc{}, bf{};
    ChipStat* d_cstat = nullptr;
    float* d_inv_blk = nullptr;
    float* d_part = nullptr;
    double* d_scal = nullptr;
    // forms the geometry allows
    bool plain_ok = false, tensor_ok = false, spectral_ok = false;
    // amplitude rasters of the spectral form (reference and secondary, one allocation), and the
    // box statistics of the secondary raster (FP64 column sums, 1/sigma of every box)
    float* d_amp = nullptr;
    size_t amp_cap = 0;
    double* d_vsum = nullptr;
    size_t vsum_cap = 0;
    float* d_inv_raster = nullptr;
    size_t inv_raster_cap = 0;
    // tensor-core form
    TcGeom tcc{}, tcf{};
    NccGeom gsc{}, gsf{};
    int zoom_smem = 0;
    float* d_inv_c = nullptr;
    float* d_inv_f = nullptr;
    float* d_gam = nullptr;
    FineOut* d_fine_out = nullptr;
    size_t fine_cap = 0;
    unsigned int* d_tc_err = nullptr;
    // batches whose tensor-core zoom is made to time out (ampcor_inject_timeout)
    int inject_timeouts = 0;
    // per-kernel timing: (start, stop) event pairs of each launch, per kernel kind
    // (0 coarse correlation, 1 refinement, 2 fine correlation, 3 coarse statistics,
    //  4 fine statistics, 5 zoom)
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> marks[6];
    uint64_t mark_kernels[6] = {0, 0, 0, 0, 0, 0};
    std::string err;
};

namespace {

int fail(ampcor_handle* h, int code, const std::string& msg)
{
    if (h) h->err = msg;
    return code;
}

int cuda_fail(ampcor_handle* h, cudaError_t e, const char* what)
{
    return fail(h, AMPCOR_E_CUDA, std::string(what) + ": " + cudaGetErrorName(e) + " (" +
                                      cudaGetErrorString(e) + ")");
}

#define CK(h, call, what)                                  \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, what); \
    } while (0)

template <typename T>
int grow(ampcor_handle* h, T*& ptr, size_t& cap, size_t n, const char* what)
{
    if (cap >= n && ptr) return AMPCOR_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void**)&ptr, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) {
        ptr = nullptr;
        return fail(h, AMPCOR_E_NOMEM, std::string("allocating ") + what + ": " + cudaGetErrorName(e));
    }
    cap = n;
    return AMPCOR_OK;
}

int ensure_pairs(ampcor_handle* h, size_t pairs)
{
    if (h->cap >= pairs && h->d_ref_off) return AMPCOR_OK;
    cudaFree(h->d_ref_off);
    cudaFree(h->d_tgt_off);
    cudaFree(h->d_coarse);
    cudaFree(h->d_coarse_peak);
    cudaFree(h->d_offsets);
    cudaFree(h->d_diag);
    h->d_ref_off = h->d_tgt_off = nullptr;
    h->d_coarse = nullptr;
    h->d_coarse_peak = nullptr;
    h->d_offsets = nullptr;
    h->d_diag = nullptr;
    h->cap = 0;
    const size_t n = std::max<size_t>(pairs, 1);
    if (cudaMalloc(&h->d_ref_off, n * sizeof(long long)) != cudaSuccess ||
        cudaMalloc(&h->d_tgt_off, n * sizeof(long long)) != cudaSuccess ||
        cudaMalloc(&h->d_coarse, n * sizeof(CoarseOut)) != cudaSuccess ||
        cudaMalloc(&h->d_coarse_peak, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&h->d_offsets, n * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&h->d_diag, n * sizeof(PairDiag)) != cudaSuccess)
        return fail(h, AMPCOR_E_NOMEM, "allocating per-pair device buffers");
    h->cap = n;
    return AMPCOR_OK;
}

// the chunk of pairs whose refined amplitudes are resident at once: a few waves of CTAs,
// small enough that the refined tiles mostly stay in L2 between the refine and fine kernels
size_t default_chunk()
{
    const char* env = std::getenv("AMPCOR_CHUNK");
    if (env) {
        long v = std::strtol(env, nullptr, 10);
        if (v > 0) return (size_t)v;
    }
    return 148 * 4;
}

void free_chunk_scratch(ampcor_handle* h)
{
    cudaFree(h->d_refined);
    cudaFree(h->d_inv_c);
    cudaFree(h->d_inv_f);
    cudaFree(h->d_gam);
    cudaFree(h->d_cstat);
    cudaFree(h->d_inv_blk);
    cudaFree(h->d_part);
    cudaFree(h->d_scal);
    cudaFree(h->d_upy);
    h->d_refined = nullptr;
    h->d_inv_c = h->d_inv_f = h->d_gam = nullptr;
    h->d_cstat = nullptr;
    h->d_inv_blk = nullptr;
    h->d_part = nullptr;
    h->d_scal = nullptr;
    h->d_upy = nullptr;
}

// a failed chunk-scratch allocation releases what was allocated, so that the next call starts
// over, and clears the runtime's record of the failure (it is reported here, not by a later launch)
int scratch_fail(ampcor_handle* h, const std::string& what)
{
    free_chunk_scratch(h);
    cudaGetLastError();
    return fail(h, AMPCOR_E_NOMEM, what);
}

int ensure_refined(ampcor_handle* h)
{
    if (h->d_refined) return AMPCOR_OK;
    h->chunk = h->chunk_override ? h->chunk_override : default_chunk();
    h->refined_stride = (long long)h->Rf * h->Rf + (long long)h->Wf * h->Wf;
    // 16 floats of slack: staged copies round rows out to 16-byte boundaries
    cudaError_t e = cudaMalloc(&h->d_refined, (h->chunk * h->refined_stride + 16) * sizeof(float));
    if (e != cudaSuccess) {
        h->d_refined = nullptr;
        return scratch_fail(h, std::string("allocating refinement scratch: ") + cudaGetErrorName(e));
    }
    const size_t n = h->chunk;
    // per-pair placement statistics: only the tensor-core form stages them in memory (the
    // spectral form takes them from the raster or computes them in the correlation kernel)
    if (h->form == kFormTensor &&
        (cudaMalloc(&h->d_inv_c, n * h->C * h->C * sizeof(float)) != cudaSuccess ||
         cudaMalloc(&h->d_inv_f, n * h->Cf * h->Cf * sizeof(float)) != cudaSuccess))
        return scratch_fail(h, "allocating placement statistics scratch");
    if (h->form != kFormPlain && cudaMalloc(&h->d_gam, n * h->Cf * h->Cf * sizeof(float)) != cudaSuccess)
        return scratch_fail(h, "allocating refined-surface scratch");
    if (h->form == kFormSpectral && (h->bc.on || h->bf.on)) {
        const size_t K = (size_t)std::max(h->bc.on ? h->bc.K : 0, h->bf.on ? h->bf.K : 0);
        const size_t parts = std::max(h->bc.on ? (size_t)h->bc.K * h->C * h->C : 0,
                                      h->bf.on ? (size_t)h->bf.K * h->Cf * h->Cf : 0);
        const size_t cells = std::max(h->bc.on ? (size_t)h->C * h->C : 0, h->bf.on ? (size_t)h->Cf * h->Cf : 0);
        if (cudaMalloc(&h->d_cstat, n * sizeof(ChipStat)) != cudaSuccess ||
            cudaMalloc(&h->d_inv_blk, n * cells * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&h->d_part, n * parts * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&h->d_scal, n * K * 2 * sizeof(double)) != cudaSuccess)
            return scratch_fail(h, "allocating blocked-correlation scratch");
    }
    if (h->form == kFormSpectral && h->refine_big &&
        cudaMalloc(&h->d_upy, n * (size_t)h->upy_len * sizeof(float2)) != cudaSuccess)
        return scratch_fail(h, "allocating refinement scratch");
    return AMPCOR_OK;
}


int ensure_fine_out(ampcor_handle* h, size_t pairs)
{
    if (h->fine_cap >= pairs && h->d_fine_out) return AMPCOR_OK;
    cudaFree(h->d_fine_out);
    h->d_fine_out = nullptr;
    h->fine_cap = 0;
    if (cudaMalloc(&h->d_fine_out, std::max<size_t>(pairs, 1) * sizeof(FineOut)) != cudaSuccess)
        return fail(h, AMPCOR_E_NOMEM, "allocating refined maxima");
    h->fine_cap = std::max<size_t>(pairs, 1);
    return AMPCOR_OK;
}

// record an event (profiling only); returns nullptr when profiling is off
cudaEvent_t mark(ampcor_handle* h, cudaStream_t st)
{
    if (!h->profiling) return nullptr;
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    cudaEventRecord(e, st);
    return e;
}

// a timed stage region holding `kernels` kernel launches
void keep(ampcor_handle* h, int stage, cudaEvent_t a, cudaEvent_t b, int kernels = 1)
{
    if (a && b) {
        h->marks[stage].emplace_back(a, b);
        h->mark_kernels[stage] += (uint64_t)kernels;
    }
}

// plain FP32 form: coarse over all pairs, then (refine -> fine) per chunk on stream st
int run_plain(ampcor_handle* h, const PairSource& src, long long pairs, float2* offsets,
              PairDiag* diag, float* coarse_surfaces, float* refined_surfaces, cudaStream_t st)
{
    if (pairs == 0) return AMPCOR_OK;
    int rc = ensure_refined(h);
    if (rc) return rc;
    cudaEvent_t a = mark(h, st);
    coarse_kernel<<<(unsigned)pairs, kThreads, h->gc.smem_bytes, st>>>(
        src, 0, pairs, h->gc, h->m, h->d_coarse, h->d_coarse_peak, coarse_surfaces);
    CK(h, cudaGetLastError(), "launching the coarse correlation kernel");
    keep(h, 0, a, mark(h, st));
    for (long long c0 = 0; c0 < pairs; c0 += (long long)h->chunk) {
        const long long n = std::min<long long>((long long)h->chunk, pairs - c0);
        a = mark(h, st);
        refine_kernel<<<(unsigned)n, kThreads, h->refine_smem, st>>>(
            src, c0, n, h->d_coarse, h->ic, h->iw, h->d_chip_taps, h->d_win_taps, h->d_refined,
            h->refined_stride, (h->prm.flags & AMPCOR_FLAG_DERAMP) ? 1 : 0);
        CK(h, cudaGetLastError(), "launching the refinement kernel");
        cudaEvent_t b = mark(h, st);
        keep(h, 1, a, b);
        fine_kernel<<<(unsigned)n, kThreads, h->gf.smem_bytes, st>>>(
            h->d_refined, h->refined_stride, c0, n, src.ref_off, h->gf, h->zg, h->d_zoom_taps,
            h->d_coarse, h->d_coarse_peak, h->M, h->f, h->m,
            (h->prm.flags & AMPCOR_FLAG_REF_COMPAT) ? 1 : 0, offsets, diag, refined_surfaces);
        CK(h, cudaGetLastError(), "launching the fine correlation kernel");
        // the fine stage starts at the event that ends the refine stage
        keep(h, 2, b, mark(h, st));
    }
    return AMPCOR_OK;
}

void drop_marks(ampcor_handle* h)
{
    for (auto& k : h->mark_kernels) k = 0;
    std::vector<cudaEvent_t> seen;
    for (auto& v : h->marks) {
        for (auto& pr : v) {
            for (cudaEvent_t e : {pr.first, pr.second})
                if (std::find(seen.begin(), seen.end(), e) == seen.end()) seen.push_back(e);
        }
        v.clear();
    }
    for (cudaEvent_t e : seen) cudaEventDestroy(e);
}

// the zoom of a chunk: tensor cores where Zm fits, else the FP32 kernel
int launch_zoom(ampcor_handle* h, long long c0, unsigned n, const PairSource& src, float2* offsets,
                PairDiag* diag, cudaStream_t st)
{
    const int compat = (h->prm.flags & AMPCOR_FLAG_REF_COMPAT) ? 1 : 0;
    if (h->zoom_tc) {
        const unsigned blocks = std::min<unsigned>(n, 148u);
        tc_zoom_kernel<<<blocks, kTcZoomThreads, h->ztc.smem_bytes, st>>>(
            h->d_gam, c0, n, src.ref_off, h->ztc, h->d_zoom_uhl, h->d_coarse, h->d_coarse_peak,
            h->d_fine_out, h->M, h->f, h->m, compat, offsets, diag, h->d_tc_err, h->inject_timeouts > 0 ? 1 : 0);
    } else {
        zoom_kernel<<<n, 256, h->zoom_smem, st>>>(h->d_gam, c0, n, src.ref_off, h->zg, h->d_zoom_ut,
                                                  h->d_coarse, h->d_coarse_peak, h->d_fine_out, h->M,
                                                  h->f, h->m, compat, offsets, diag);
    }
    CK(h, cudaGetLastError(), "launching the zoom kernel");
    return AMPCOR_OK;
}

// tensor-core form, per chunk: coarse statistics -> coarse correlation -> refinement -> fine
// statistics -> fine correlation -> zoom
int run_tensor(ampcor_handle* h, const PairSource& src, long long pairs, float2* offsets,
               PairDiag* diag, float* coarse_surfaces, float* refined_surfaces, cudaStream_t st)
{
    if (pairs == 0) return AMPCOR_OK;
    int rc = ensure_refined(h);
    if (rc) return rc;
    if ((rc = ensure_fine_out(h, (size_t)pairs))) return rc;
    const RealTiles rt{h->d_refined, h->refined_stride, 0, (long long)h->Rf * h->Rf};
    for (long long c0 = 0; c0 < pairs; c0 += (long long)h->chunk) {
        const unsigned n = (unsigned)std::min<long long>((long long)h->chunk, pairs - c0);
        cudaEvent_t a = mark(h, st);
        window_stats_cplx_kernel<<<n, kThreads, h->gsc.smem_bytes, st>>>(src, c0, n, h->gsc, h->d_inv_c);
        cudaEvent_t b = mark(h, st);
        keep(h, 3, a, b);
        tc_coarse_kernel<<<n, 256, h->tcc.smem_bytes, st>>>(src, c0, n, h->tcc, h->d_inv_c, h->m,
                                                            h->d_coarse, h->d_coarse_peak,
                                                            coarse_surfaces, h->d_tc_err);
        cudaEvent_t c = mark(h, st);
        keep(h, 0, b, c);
        refine_kernel<<<n, kThreads, h->refine_smem, st>>>(src, c0, n, h->d_coarse, h->ic, h->iw,
                                                           h->d_chip_taps, h->d_win_taps,
                                                           h->d_refined, h->refined_stride, (h->prm.flags & AMPCOR_FLAG_DERAMP) ? 1 : 0);
        cudaEvent_t d = mark(h, st);
        keep(h, 1, c, d);
        window_stats_real_kernel<<<n, kThreads, h->gsf.smem_bytes, st>>>(rt, n, h->gsf, h->d_inv_f);
        cudaEvent_t e = mark(h, st);
        keep(h, 4, d, e);
        tc_fine_kernel<<<n, 256, h->tcf.smem_bytes, st>>>(rt, c0, n, h->tcf, h->d_inv_f, src.ref_off,
                                                          h->d_fine_out, h->d_gam, refined_surfaces,
                                                          h->d_tc_err);
        cudaEvent_t f = mark(h, st);
        keep(h, 2, e, f);
        CK(h, cudaGetLastError(), "launching the tensor-core pipeline");
        if ((rc = launch_zoom(h, c0, n, src, offsets, diag, st))) return rc;
        keep(h, 5, f, mark(h, st));
    }
    return AMPCOR_OK;
}

// spectral form: amplitudes of both rasters once, then per chunk: coarse statistics -> coarse
// correlation (FFT) -> refinement -> fine statistics -> fine correlation (FFT) -> zoom
// the amplitude rasters of a spectral job and, where the windows tile a raster, its box statistics
struct SpecRasters {
    float* amp_ref = nullptr;
    float* amp_tgt = nullptr;
    bool shared = false;        // one raster holds chips and windows
    bool raster_stats = false;  // coarse box statistics once per raster, else inside the kernel
    long long rows = 0;         // box rows of the secondary raster (tgt_lines - R + 1)
    size_t cells = 0;           // rows * stride
    InvSource inv_c{nullptr, nullptr, 0};
};

// buffers of a spectral job of `pairs` pairs; no launches
// cuTensorMapEncodeTiled from the driver (the runtime is linked statically; the driver's entry
// point is looked up once)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled()
{
    static const EncodeTiledFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return static_cast<EncodeTiledFn>(nullptr);
        return reinterpret_cast<EncodeTiledFn>(f);
    }();
    return fn;
}

// a 2-D map of a float raster (lines x samples) whose boxes are bx x by floats (bx a multiple of
// 4); false where the driver has no tensor maps or the raster breaks the copy engine's alignment
// rules (a 16-byte aligned base, lines a multiple of 16 bytes)
bool raster_map(CUtensorMap& m, const float* base, long long lines, long long samples, int bx, int by)
{
    const EncodeTiledFn fn = encode_tiled();
    if (!fn || (reinterpret_cast<uintptr_t>(base) & 15) || (samples & 3) || lines < 1 || bx % 4 || bx < 4 ||
        bx > 256 || by < 1 || by > 256)
        return false;
    const cuuint64_t dim[2] = {(cuuint64_t)samples, (cuuint64_t)lines};
    const cuuint64_t stride[1] = {(cuuint64_t)samples * 4};
    const cuuint32_t box[2] = {(cuuint32_t)bx, (cuuint32_t)by};
    const cuuint32_t es[2] = {1, 1};
    return fn(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dim, stride, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int spec_rasters(ampcor_handle* h, const PairSource& src, long long pairs, SpecRasters& r)
{
    int rc = ensure_refined(h);
    if (rc) return rc;
    if ((rc = ensure_fine_out(h, (size_t)pairs))) return rc;
    r.shared = src.ref_base == src.tgt_base;
    const size_t need = (size_t)src.ref_count + (r.shared ? 0 : (size_t)src.tgt_count);
    // 16 floats of slack here and below: staged copies round rows out to 16-byte boundaries
    // the secondary's amplitudes start on a 16-byte boundary (tensor copies of its windows)
    const size_t ref_span = ((size_t)src.ref_count + 3) & ~(size_t)3;
    const size_t need_al = r.shared ? need : ref_span + (size_t)src.tgt_count;
    if ((rc = grow(h, h->d_amp, h->amp_cap, need_al + 16, "amplitude rasters"))) return rc;
    r.amp_ref = h->d_amp;
    r.amp_tgt = r.shared ? h->d_amp : h->d_amp + ref_span;
    // coarse box statistics once per raster where the windows tile a raster (they overlap), else
    // inside the correlation kernel from the window it holds (as for every fine window)
    r.rows = src.tgt_lines - h->R + 1;
    r.raster_stats = src.tgt_lines > 0 && r.rows > 0 && src.tgt_stride <= 12288;
    r.inv_c = InvSource{nullptr, nullptr, 0};
    if (r.raster_stats) {
        r.cells = (size_t)r.rows * (size_t)src.tgt_stride;
        if ((rc = grow(h, h->d_vsum, h->vsum_cap, 2 * r.cells, "box statistics")) ||
            (rc = grow(h, h->d_inv_raster, h->inv_raster_cap, r.cells + 16, "box statistics")))
            return rc;
        r.inv_c = InvSource{h->d_inv_raster, src.tgt_off, src.tgt_stride};
    }
    return AMPCOR_OK;
}

// amplitudes of samples [ref_lo, ref_hi) of the reference source and [tgt_lo, tgt_hi) of the
// secondary, box statistics of box rows [box_lo, box_hi); a band gives the same values as the
// whole raster
int spec_band(ampcor_handle* h, const PairSource& src, const SpecRasters& r, long long ref_lo,
              long long ref_hi, long long tgt_lo, long long tgt_hi, long long box_lo, long long box_hi,
              cudaStream_t st)
{
    auto detect = [&](const float2* x, long long n, float* y) {
        const long long blocks = std::min<long long>((n + 1023) / 1024, 148 * 16);
        if (n > 0) detect_kernel<<<(unsigned)std::max<long long>(blocks, 1), 256, 0, st>>>(x, n, y);
        return n > 0 ? 1 : 0;
    };
    cudaEvent_t a0 = mark(h, st);
    int kernels = 0;
    if (r.shared) {
        const long long lo = std::min(ref_lo, tgt_lo), hi = std::max(ref_hi, tgt_hi);
        kernels += detect(src.ref_base + lo, hi - lo, r.amp_ref + lo);
    } else {
        kernels += detect(src.ref_base + ref_lo, ref_hi - ref_lo, r.amp_ref + ref_lo);
        kernels += detect(src.tgt_base + tgt_lo, tgt_hi - tgt_lo, r.amp_tgt + tgt_lo);
    }
    CK(h, cudaGetLastError(), "launching the detection kernel");
    if (r.raster_stats && box_hi > box_lo) {
        const long long vlo = box_lo / kVBlock * kVBlock;
        const dim3 vg((unsigned)((src.tgt_stride + 255) / 256), (unsigned)((box_hi - vlo + kVBlock - 1) / kVBlock));
        box_vsum_kernel<<<vg, 256, 0, st>>>(r.amp_tgt, src.tgt_stride, h->R, vlo, box_hi, h->d_vsum,
                                            h->d_vsum + r.cells);
        const int psmem = (int)((2 * (src.tgt_stride + 1) + 2 * kWarps) * sizeof(double));
        box_inv_kernel<<<(unsigned)(box_hi - box_lo), kThreads, psmem, st>>>(
            h->d_vsum, h->d_vsum + r.cells, box_lo, box_hi, src.tgt_stride, h->R, h->d_inv_raster);
        CK(h, cudaGetLastError(), "launching the box statistics kernels");
        kernels += 2;
    }
    keep(h, 3, a0, mark(h, st), kernels);
    return AMPCOR_OK;
}

// the correlation pipeline of pairs [p0, p1), chunk by chunk
int spec_pairs(ampcor_handle* h, const PairSource& src, const SpecRasters& r, long long p0, long long p1,
               float2* offsets, PairDiag* diag, float* coarse_surfaces, float* refined_surfaces,
               cudaStream_t st)
{
    int rc = AMPCOR_OK;
    const SpecSource cs{r.amp_ref, src.ref_stride, src.ref_off, 0, r.amp_tgt, src.tgt_stride, src.tgt_off, 0};
    const SpecSource fs{h->d_refined, h->Rf, nullptr, h->refined_stride,
                        h->d_refined + (long long)h->Rf * h->Rf, h->Wf, nullptr, h->refined_stride};
    // the staged coarse stage takes its windows from the secondary's amplitude raster through a
    // tensor map and its statistics from the raster
    CUtensorMap wmap{}, cmap{}, imap{};
    const bool coarse_st =
        h->coarse_staged && r.inv_c.base && src.tgt_stride > 0 && src.ref_stride > 0 &&
        raster_map(wmap, r.amp_tgt, src.tgt_count / src.tgt_stride, src.tgt_stride, h->spc_st.stage_rs, h->W) &&
        raster_map(cmap, r.amp_ref, src.ref_count / src.ref_stride, src.ref_stride, (h->R + 6) & ~3, h->R) &&
        raster_map(imap, r.inv_c.base, r.rows, src.tgt_stride, h->spc_st.inv_rs, h->C);
    // the window refinement of a raster job in the staged form: its tiles come from the secondary
    // raster (as floats, two a sample) through a tensor map
    CUtensorMap rmap{};
    int rs_smem = 0, rs_box = 0;
    const bool refine_st =
        h->staged_on && h->refine_fft && !h->refine_strips && !(h->prm.flags & AMPCOR_FLAG_DERAMP) &&
        src.tgt_lines > 0 && src.tgt_stride > 0 && spec_refine_staged_supported(h->E, h->f, rs_smem, rs_box) &&
        raster_map(rmap, reinterpret_cast<const float*>(src.tgt_base), src.tgt_count / src.tgt_stride,
                   2 * src.tgt_stride, rs_box, h->E);
    for (long long c0 = p0; c0 < p1; c0 += (long long)h->chunk) {
        const unsigned n = (unsigned)std::min<long long>((long long)h->chunk, p1 - c0);
        cudaEvent_t b = mark(h, st);
        const SpecOut co{0, h->m, h->d_coarse, h->d_coarse_peak, nullptr, nullptr, coarse_surfaces};
        if (h->bc.on) {
            InvSource ic = r.inv_c;
            CK(h, launch_spec_chip_stats(n, st, cs, c0, n, src.ref_off, h->R, h->d_cstat),
               "launching the chip statistics");
            int kernels = 1;
            if (!ic.base) {
                CK(h, launch_spec_tile_stats(n, st, cs, c0, n, src.ref_off, h->R, h->W, h->d_inv_blk),
                   "launching the placement statistics");
                ic = InvSource{h->d_inv_blk, nullptr, 0};
                ++kernels;
            }
            cudaEvent_t b2 = mark(h, st);
            keep(h, 3, b, b2, kernels);
            b = b2;
            CK(h, launch_spec_block(h->bc.tile, h->bc.nb, n * (unsigned)h->bc.K, st, cs, c0, n, src.ref_off,
                                    h->d_cstat, reinterpret_cast<const float2*>(h->d_tw_c), h->d_part, h->d_scal),
               "launching the blocked coarse correlation");
            CK(h, launch_spec_reduce(h->bc.full, h->bc.K, n, st, cs, c0, n, src.ref_off, h->d_cstat, ic,
                                     h->d_part, h->d_scal, co),
               "launching the coarse reduction");
        } else {
            if (coarse_st)
                CK(h, launch_spec_staged(h->spc_st, (unsigned)h->sms, st, cs, c0, n, src.ref_off, r.inv_c,
                                         reinterpret_cast<const float2*>(h->d_tw_c), co, h->d_tc_err,
                                         &wmap, &cmap, &imap, h->inject_timeouts > 0 ? 1 : 0),
                   "launching the staged coarse correlation");
            else
                CK(h, launch_spec(h->spc, n, st, cs, c0, n, src.ref_off, r.inv_c,
                                  reinterpret_cast<const float2*>(h->d_tw_c), co),
                   "launching the spectral coarse correlation");
        }
        cudaEvent_t c = mark(h, st);
        keep(h, 0, b, c, h->bc.on ? 2 : 1);
        if (h->refine_fft) {
            const float2* tw = reinterpret_cast<const float2*>(h->d_tw_refine);
            CK(h, launch_spec_refine(h->R, n, st, src.ref_base, src.ref_off, src.ref_stride, nullptr, c0,
                                     n, src.ref_off, tw, tw + h->R, h->d_refined, h->refined_stride, 0,
                                     (h->prm.flags & AMPCOR_FLAG_DERAMP) ? 1 : 0, h->d_upy, h->refine_strips),
               "launching the chip refinement");
            if (refine_st)
                CK(h, launch_spec_refine_staged(h->E, (unsigned)h->sms, st, &rmap, src.tgt_off, src.tgt_stride,
                                                h->d_coarse, c0, n, src.ref_off, tw + h->R + h->Rf,
                                                tw + h->R + h->Rf + h->E, h->d_refined, h->refined_stride,
                                                (long long)h->Rf * h->Rf, h->d_tc_err),
                   "launching the staged window refinement");
            else
                CK(h, launch_spec_refine(h->E, n, st, src.tgt_base, src.tgt_off, src.tgt_stride, h->d_coarse,
                                         c0, n, src.ref_off, tw + h->R + h->Rf, tw + h->R + h->Rf + h->E,
                                         h->d_refined, h->refined_stride, (long long)h->Rf * h->Rf,
                                         (h->prm.flags & AMPCOR_FLAG_DERAMP) ? 1 : 0, h->d_upy, h->refine_strips),
                   "launching the window refinement");
        } else {
            refine_kernel<<<n, kThreads, h->refine_smem, st>>>(src, c0, n, h->d_coarse, h->ic, h->iw,
                                                               h->d_chip_taps, h->d_win_taps,
                                                               h->d_refined, h->refined_stride, (h->prm.flags & AMPCOR_FLAG_DERAMP) ? 1 : 0);
            CK(h, cudaGetLastError(), "launching the refinement kernel");
        }
        cudaEvent_t e = mark(h, st);
        keep(h, 1, c, e, h->refine_fft ? 2 : 1);
        const SpecOut fo{1, 0, nullptr, nullptr, h->d_fine_out, h->d_gam, refined_surfaces};
        if (h->bf.on) {
            CK(h, launch_spec_chip_stats(n, st, fs, c0, n, src.ref_off, h->Rf, h->d_cstat),
               "launching the refined chip statistics");
            CK(h, launch_spec_tile_stats(n, st, fs, c0, n, src.ref_off, h->Rf, h->Wf, h->d_inv_blk),
               "launching the refined placement statistics");
            cudaEvent_t e2 = mark(h, st);
            keep(h, 4, e, e2, 2);
            e = e2;
            CK(h, launch_spec_block(h->bf.tile, h->bf.nb, n * (unsigned)h->bf.K, st, fs, c0, n, src.ref_off,
                                    h->d_cstat, reinterpret_cast<const float2*>(h->d_tw_f), h->d_part, h->d_scal),
               "launching the blocked fine correlation");
            CK(h, launch_spec_reduce(h->bf.full, h->bf.K, n, st, fs, c0, n, src.ref_off, h->d_cstat,
                                     InvSource{h->d_inv_blk, nullptr, 0}, h->d_part, h->d_scal, fo),
               "launching the fine reduction");
        } else {
            if (h->fine_staged)
                CK(h, launch_spec_staged(h->spf_st, (unsigned)h->sms, st, fs, c0, n, src.ref_off,
                                         InvSource{nullptr, nullptr, 0},
                                         reinterpret_cast<const float2*>(h->d_tw_f), fo, h->d_tc_err,
                                         nullptr, nullptr, nullptr, h->inject_timeouts > 0 ? 1 : 0),
                   "launching the staged fine correlation");
            else
                CK(h, launch_spec(h->spf, n, st, fs, c0, n, src.ref_off, InvSource{nullptr, nullptr, 0},
                                  reinterpret_cast<const float2*>(h->d_tw_f), fo),
                   "launching the spectral fine correlation");
        }
        cudaEvent_t f = mark(h, st);
        keep(h, 2, e, f, h->bf.on ? 2 : 1);
        if ((rc = launch_zoom(h, c0, n, src, offsets, diag, st))) return rc;
        keep(h, 5, f, mark(h, st));
    }
    return AMPCOR_OK;
}

int run_spectral(ampcor_handle* h, const PairSource& src, long long pairs, float2* offsets,
                 PairDiag* diag, float* coarse_surfaces, float* refined_surfaces, cudaStream_t st)
{
    if (pairs == 0) return AMPCOR_OK;
    SpecRasters r;
    int rc = spec_rasters(h, src, pairs, r);
    if (rc) return rc;
    if ((rc = spec_band(h, src, r, 0, src.ref_count, 0, src.tgt_count, 0, r.raster_stats ? r.rows : 0, st)))
        return rc;
    return spec_pairs(h, src, r, 0, pairs, offsets, diag, coarse_surfaces, refined_surfaces, st);
}

int run_pipeline(ampcor_handle* h, const PairSource& src, long long pairs, float2* offsets,
                 PairDiag* diag, float* coarse_surfaces, float* refined_surfaces, cudaStream_t st)
{
    int rc;
    switch (h->form) {
        case kFormSpectral:
            rc = run_spectral(h, src, pairs, offsets, diag, coarse_surfaces, refined_surfaces, st);
            break;
        case kFormTensor:
            rc = run_tensor(h, src, pairs, offsets, diag, coarse_surfaces, refined_surfaces, st);
            break;
        default:
            rc = run_plain(h, src, pairs, offsets, diag, coarse_surfaces, refined_surfaces, st);
    }
    if (h->inject_timeouts > 0) --h->inject_timeouts;
    return rc;
}

cudaStream_t pick(ampcor_handle* h, void* stream)
{
    return stream ? (cudaStream_t)stream : h->stream;
}

}  // namespace

extern "C" {

int ampcor_create(const ampcor_params* p, ampcor_handle** out)
{
    auto create_fail = [&](int code, const std::string& msg) {
        std::lock_guard<std::mutex> lk(g_create_mutex);
        g_create_error = msg;
        return code;
    };
    if (!p || !out) return create_fail(AMPCOR_E_ARG, "null argument");
    *out = nullptr;
    if (p->ref_lines != p->ref_samples || p->tgt_lines != p->tgt_samples)
        return create_fail(AMPCOR_E_SHAPE, "chips and search windows must be square");
    if (p->tgt_lines < p->ref_lines || (p->tgt_lines - p->ref_lines) % 2)
        return create_fail(AMPCOR_E_SHAPE, "window must exceed the chip by an even margin");
    if (p->refine_factor < 1 || p->zoom_factor < 1)
        return create_fail(AMPCOR_E_ARG, "refine and zoom factors must be positive");
    if (p->ref_lines > 4096 || p->refine_factor > 16 || p->zoom_factor > 64 ||
        p->refine_margin > 1024)
        return create_fail(AMPCOR_E_SHAPE, "geometry out of range");

    ampcor_handle* h = new (std::nothrow) ampcor_handle();
    if (!h) return create_fail(AMPCOR_E_NOMEM, "allocating the worker");
    h->prm = *p;
    h->R = (int)p->ref_lines;
    h->W = (int)p->tgt_lines;
    h->C = h->W - h->R + 1;
    h->M = (h->W - h->R) / 2;
    h->f = (int)p->refine_factor;
    h->m = (int)p->refine_margin;
    h->z = (int)p->zoom_factor;
    h->E = h->R + 2 * h->m;
    h->Rf = h->f * h->R;
    h->Wf = h->f * h->E;
    h->Cf = 2 * h->f * h->m + 1;
    h->Z = h->z * h->Cf;
    std::string err;
    if (h->E > h->W) {
        delete h;
        return create_fail(AMPCOR_E_SHAPE, "refinement neighbourhood (chip + 2 * refine margin) exceeds the window");
    }
    // zoom stage sizes (taps of z phases, the row-interpolated surface Cf x Z)
    h->zg.Cf = h->Cf;
    h->zg.z = h->z;
    h->zg.Z = h->Z;
    h->zg.cb = 1;
    for (int cb : {17, 13, 11, 5, 3})
        if (h->Cf % cb == 0) {
            h->zg.cb = cb;
            break;
        }
    h->zg.taps_len = 2 * h->Cf + 32;
    // the forms this geometry allows: the plain form (direct FP32 sums, whole tiles in shared
    // memory, refinement by interpolation taps), the tensor-core form (the same refinement) and
    // the spectral form (each correlation stage in one tile, or in chip blocks where the window
    // is too large; refinement by zero-padded FFT, or by taps where no FFT length is compiled)
    {
        std::string perr, terr, serr;
        const bool interp_ok = plan_interp(h->R, h->f, h->ic, perr) && plan_interp(h->E, h->f, h->iw, perr);
        h->plain_ok = plan_ncc(h->R, h->W, 0, 0, h->gc, perr) &&
                      plan_ncc(h->Rf, h->Wf, h->Cf * h->Z, h->z * h->zg.taps_len, h->gf, perr) && interp_ok;
        h->tensor_ok = h->plain_ok && plan_tc(h->R, h->W, 8, h->tcc, terr) && plan_tc(h->Rf, h->Wf, 4, h->tcf, terr);
        int sm_c = 0, sm_w = 0;
        const bool small_c = spec_refine_supported(h->R, h->f, sm_c), small_w = spec_refine_supported(h->E, h->f, sm_w);
        const bool big_c = !small_c && spec_refine_big_supported(h->R, h->f, sm_c);
        const bool big_w = !small_w && spec_refine_big_supported(h->E, h->f, sm_w);
        h->refine_fft = (small_c || big_c) && (small_w || big_w) &&
                        !(std::getenv("AMPCOR_REFINE_TAPS") && interp_ok);
        int sm_sc = 0, sm_sw = 0;
        h->refine_strips = h->refine_fft && std::getenv("AMPCOR_REFINE_STRIPS") &&
                           std::atoi(std::getenv("AMPCOR_REFINE_STRIPS")) == 1 &&
                           spec_refine_big_supported(h->R, h->f, sm_sc) && spec_refine_big_supported(h->E, h->f, sm_sw);
        h->refine_big = h->refine_fft && (big_c || big_w || h->refine_strips);
        h->upy_len = std::max((long long)h->R * h->Rf, (long long)h->E * h->Wf);
        const bool direct_c = plan_spec(h->R, h->W, h->spc, serr);
        const bool coarse_ok = direct_c || plan_spec_blocked(h->R, h->W, h->bc, serr);
        const bool direct_f = coarse_ok && plan_spec(h->Rf, h->Wf, h->spf, serr);
        // staged forms where they fit (AMPCOR_STAGED=0 keeps spec_kernel); the refined tiles of a
        // pair are dense rows of one buffer, staged whole when its rows are 16-byte multiples
        const char* stg = std::getenv("AMPCOR_STAGED");
        const bool staged_on = !(stg && std::strcmp(stg, "0") == 0);
        h->staged_on = staged_on;
        h->coarse_staged = staged_on && direct_c && plan_spec_staged(h->R, h->W, false, h->spc_st);
        h->fine_staged = staged_on && direct_f &&
                         plan_spec_staged(h->Rf, h->Wf, h->Rf % 2 == 0 && h->Wf % 2 == 0, h->spf_st) &&
                         h->spf_st.stage_rs == h->Wf;
        const bool fine_ok = coarse_ok && (direct_f || plan_spec_blocked(h->Rf, h->Wf, h->bf, serr));
        h->spectral_ok = fine_ok && (h->refine_fft || interp_ok);
        if (direct_c || !h->spectral_ok) h->bc = SpecBlocks{};
        if (direct_f || !h->spectral_ok) h->bf = SpecBlocks{};
        if (!h->spectral_ok && serr.empty()) serr = "no refinement of these tiles is compiled";
        if (!h->plain_ok && !h->spectral_ok) {
            delete h;
            return create_fail(AMPCOR_E_SHAPE, perr + "; " + serr);
        }
        h->refine_smem = std::max(h->ic.smem_bytes, h->iw.smem_bytes);
        // the spectral form where the geometry allows it, else the tensor-core form, else the plain
        // form; AMPCOR_FLAG_PLAIN_FP32 (or AMPCOR_FORM=plain|tensor|spectral) chooses among those
        // allowed
        const char* env = std::getenv("AMPCOR_FORM");
        h->form = h->spectral_ok ? kFormSpectral : h->tensor_ok ? kFormTensor : kFormPlain;
        if ((p->flags & AMPCOR_FLAG_PLAIN_FP32) && !h->plain_ok) {
            delete h;
            return create_fail(AMPCOR_E_SHAPE, "this geometry has no plain FP32 form: " + perr);
        }
        if (p->flags & AMPCOR_FLAG_PLAIN_FP32) h->form = kFormPlain;
        if (env && std::strcmp(env, "plain") == 0 && h->plain_ok) h->form = kFormPlain;
        if (env && std::strcmp(env, "tensor") == 0 && h->tensor_ok) h->form = kFormTensor;
        if (env && std::strcmp(env, "spectral") == 0 && h->spectral_ok) h->form = kFormSpectral;
        h->gsc = stats_layout(h->gc);
        h->gsf = stats_layout(h->gf);
        const int Zp = (h->Z + 7) & ~7;
        h->zoom_smem = (round4(h->Cf * h->Cf) + 2 * h->Cf * Zp + 64) * 4;
        h->zoom_tc = plan_zoom_tc(h->Cf, h->z, h->ztc) && !std::getenv("AMPCOR_ZOOM_FP32");
        if (!h->zoom_tc && h->zoom_smem > 227 * 1024) {
            delete h;
            return create_fail(AMPCOR_E_SHAPE, "the zoomed surface is too large for this build");
        }
    }

    cudaError_t e = cudaSetDevice(p->device);
    if (e != cudaSuccess) {
        delete h;
        return create_fail(AMPCOR_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorName(e));
    }
    auto cuda_create_fail = [&](cudaError_t ce, const char* what) {
        ampcor_destroy(h);
        return create_fail(AMPCOR_E_CUDA, std::string(what) + ": " + cudaGetErrorName(ce));
    };
    if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return cuda_create_fail(e, "creating the worker stream");
    if ((e = cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, p->device)) != cudaSuccess)
        return cuda_create_fail(e, "reading the multiprocessor count");
    // the opt-in limit is per kernel and process-wide: raise it to the device maximum once so
    // that workers of different geometries can coexist
    const int kMaxSmem = 227 * 1024;
    if ((e = cudaFuncSetAttribute(coarse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kMaxSmem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(fine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kMaxSmem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(refine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kMaxSmem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(window_stats_cplx_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kMaxSmem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(window_stats_real_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kMaxSmem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(tc_coarse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kMaxSmem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(tc_fine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kMaxSmem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(zoom_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kMaxSmem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(tc_zoom_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kMaxSmem)) != cudaSuccess ||
        (e = spec_set_smem_limits()) != cudaSuccess)
        return cuda_create_fail(e, "configuring kernel shared memory");

    const std::vector<float> ct = taps_table(h->R, h->f, 1, h->ic.taps_len);
    const std::vector<float> wt = taps_table(h->E, h->f, 1, h->iw.taps_len);
    const std::vector<float> zt = taps_table(h->Cf, h->z, 0, h->zg.taps_len);
    // transposed zoom interpolation matrix, Ut[l][q] = D_Cf(q / z - l), rows padded to 8
    std::vector<float> zut;
    {
        const int Zp = (h->Z + 7) & ~7;
        zut.assign((size_t)h->Cf * Zp, 0.0f);
        for (int l = 0; l < h->Cf; ++l)
            for (int q = 0; q < h->Z; ++q) {
                const int s = q % h->z, b = q / h->z;
                zut[(size_t)l * Zp + q] = s == 0 ? (b == l ? 1.0f : 0.0f)
                                                 : (float)dirichlet(h->Cf, (double)q / h->z - l);
            }
    }
    auto upload = [&](float*& d, const std::vector<float>& v) {
        cudaError_t ue = cudaMalloc(&d, std::max<size_t>(v.size(), 1) * sizeof(float));
        if (ue != cudaSuccess) return ue;
        if (!v.empty()) ue = cudaMemcpy(d, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice);
        return ue;
    };
    if ((e = upload(h->d_chip_taps, ct)) != cudaSuccess || (e = upload(h->d_win_taps, wt)) != cudaSuccess ||
        (e = upload(h->d_zoom_taps, zt)) != cudaSuccess || (e = upload(h->d_zoom_ut, zut)) != cudaSuccess ||
        (e = upload(h->d_tw_c, spec_twiddle_table(std::max(h->bc.on ? h->bc.tile.N : h->spc.N, 1)))) != cudaSuccess ||
        (e = upload(h->d_tw_f, spec_twiddle_table(std::max(h->bf.on ? h->bf.tile.N : h->spf.N, 1)))) != cudaSuccess ||
        (h->zoom_tc && (e = upload(h->d_zoom_uhl, zoom_u_planes(h->ztc))) != cudaSuccess))
        return cuda_create_fail(e, "uploading interpolation taps");
    if (h->refine_fft) {
        std::vector<float> tw;
        for (int n : {h->R, h->Rf, h->E, h->Wf}) {
            const std::vector<float> t = spec_twiddle_table(n);
            tw.insert(tw.end(), t.begin(), t.end());
        }
        if ((e = upload(h->d_tw_refine, tw)) != cudaSuccess)
            return cuda_create_fail(e, "uploading refinement twiddles");
    }
    if ((e = cudaMalloc(&h->d_bad, sizeof(unsigned int))) != cudaSuccess ||
        (e = cudaMemset(h->d_bad, 0, sizeof(unsigned int))) != cudaSuccess ||
        (e = cudaMalloc(&h->d_tc_err, sizeof(unsigned int))) != cudaSuccess ||
        (e = cudaMemset(h->d_tc_err, 0, sizeof(unsigned int))) != cudaSuccess)
        return cuda_create_fail(e, "allocating the error counters");
    *out = h;
    return AMPCOR_OK;
}

int ampcor_destroy(ampcor_handle* h)
{
    if (!h) return AMPCOR_E_ARG;
    cudaSetDevice(h->prm.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->d_chip_taps);
    cudaFree(h->d_win_taps);
    cudaFree(h->d_zoom_taps);
    cudaFree(h->d_zoom_ut);
    cudaFree(h->d_arena);
    cudaFree(h->d_ref_off);
    cudaFree(h->d_tgt_off);
    cudaFree(h->d_coarse);
    cudaFree(h->d_coarse_peak);
    cudaFree(h->d_offsets);
    cudaFree(h->d_diag);
    cudaFree(h->d_bad);
    cudaFree(h->d_refined);
    cudaFree(h->d_ref_raster);
    cudaFree(h->d_tgt_raster);
    cudaFree(h->d_ulhc);
    cudaFree(h->d_job_offsets);
    cudaFree(h->d_job_diag);
    cudaFree(h->d_inv_c);
    cudaFree(h->d_inv_f);
    cudaFree(h->d_gam);
    cudaFree(h->d_fine_out);
    cudaFree(h->d_tw_c);
    cudaFree(h->d_tw_f);
    cudaFree(h->d_zoom_uhl);
    cudaFree(h->d_tw_refine);
    cudaFree(h->d_amp);
    cudaFree(h->d_vsum);
    cudaFree(h->d_inv_raster);
    cudaFree(h->d_tc_err);
    cudaFree(h->d_cstat);
    cudaFree(h->d_inv_blk);
    cudaFree(h->d_part);
    cudaFree(h->d_scal);
    cudaFree(h->d_upy);
    drop_marks(h);
    if (h->h_arena) cudaFreeHost(h->h_arena);
    if (h->h_offsets) cudaFreeHost(h->h_offsets);
    for (cudaEvent_t e : h->band_ev)
        if (e) cudaEventDestroy(e);
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return AMPCOR_OK;
}

static int ensure_arena(ampcor_handle* h)
{
    if (h->h_arena) return AMPCOR_OK;
    const size_t pixels = h->prm.pairs * ((size_t)h->R * h->R + (size_t)h->W * h->W);
    cudaError_t e = cudaMallocHost(&h->h_arena, std::max<size_t>(pixels, 1) * sizeof(float2));
    if (e != cudaSuccess) {
        h->h_arena = nullptr;
        return fail(h, AMPCOR_E_NOMEM, "allocating the host tile arena");
    }
    std::memset(h->h_arena, 0, pixels * sizeof(float2));
    return AMPCOR_OK;
}

static int add_tile(ampcor_handle* h, uint64_t pid, const void* tile, uint64_t row_stride, bool ref)
{
    if (!h) return AMPCOR_E_ARG;
    if (!tile) return fail(h, AMPCOR_E_ARG, "null tile");
    if (pid >= h->prm.pairs) return fail(h, AMPCOR_E_ARG, "pair id out of range");
    const int dim = ref ? h->R : h->W;
    if (row_stride < (uint64_t)dim) return fail(h, AMPCOR_E_ARG, "row stride smaller than the tile");
    int rc = ensure_arena(h);
    if (rc) return rc;
    const size_t cells = (size_t)h->R * h->R + (size_t)h->W * h->W;
    float2* dst = h->h_arena + pid * cells + (ref ? 0 : (size_t)h->R * h->R);
    const float2* src = static_cast<const float2*>(tile);
    for (int r = 0; r < dim; ++r) std::memcpy(dst + (size_t)r * dim, src + r * row_stride, dim * sizeof(float2));
    return AMPCOR_OK;
}

int ampcor_add_reference(ampcor_handle* h, uint64_t pid, const void* tile, uint64_t row_stride)
{
    return add_tile(h, pid, tile, row_stride, true);
}

int ampcor_add_target(ampcor_handle* h, uint64_t pid, const void* tile, uint64_t row_stride)
{
    return add_tile(h, pid, tile, row_stride, false);
}

int ampcor_adjust(ampcor_handle* h, const float** offsets)
{
    if (!h || !offsets) return fail(h, AMPCOR_E_ARG, "null argument");
    *offsets = nullptr;
    const size_t P = h->prm.pairs;
    int rc = ensure_arena(h);
    if (rc) return rc;
    CK(h, cudaSetDevice(h->prm.device), "cudaSetDevice");
    const size_t cells = (size_t)h->R * h->R + (size_t)h->W * h->W;
    if (!h->d_arena) CK(h, cudaMalloc(&h->d_arena, std::max<size_t>(P * cells, 1) * sizeof(float2)), "allocating the device arena");
    if (!h->h_offsets) CK(h, cudaMallocHost(&h->h_offsets, std::max<size_t>(2 * P, 1) * sizeof(float)), "allocating the offset field");
    if ((rc = ensure_pairs(h, P))) return rc;
    cudaStream_t st = h->stream;
    if (P) {
        CK(h, cudaMemcpyAsync(h->d_arena, h->h_arena, P * cells * sizeof(float2), cudaMemcpyHostToDevice, st),
           "pushing the tile arena");
        arena_offsets_kernel<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(
            (long long)P, (long long)h->R * h->R, (long long)h->W * h->W, h->d_ref_off, h->d_tgt_off);
        CK(h, cudaGetLastError(), "launching the arena offsets kernel");
        const long long cells = (long long)P * ((long long)h->R * h->R + (long long)h->W * h->W);
        PairSource src{h->d_arena, h->d_ref_off, h->R, h->d_arena, h->d_tgt_off, h->W, cells, cells, 0};
        if ((rc = run_pipeline(h, src, (long long)P, h->d_offsets, h->d_diag, nullptr, nullptr, st))) return rc;
        CK(h, cudaMemcpyAsync(h->h_offsets, h->d_offsets, 2 * P * sizeof(float), cudaMemcpyDeviceToHost, st),
           "harvesting the offset field");
    }
    CK(h, cudaStreamSynchronize(st), "running the correlation pipeline");
    *offsets = h->h_offsets;
    return AMPCOR_OK;
}

int ampcor_diagnostics(ampcor_handle* h, ampcor_pair_diag* diag)
{
    if (!h || !diag) return fail(h, AMPCOR_E_ARG, "null argument");
    if (!h->d_diag) return fail(h, AMPCOR_E_STATE, "no adjust has run");
    CK(h, cudaSetDevice(h->prm.device), "cudaSetDevice");
    static_assert(sizeof(ampcor_pair_diag) == sizeof(PairDiag), "diagnostic layout");
    CK(h, cudaMemcpy(diag, h->d_diag, h->prm.pairs * sizeof(PairDiag), cudaMemcpyDeviceToHost),
       "copying diagnostics");
    return AMPCOR_OK;
}

static int check_job(ampcor_handle* h, const ampcor_job* j)
{
    if (!h) return AMPCOR_E_ARG;
    if (!j) return fail(h, AMPCOR_E_ARG, "null job");
    if (j->pairs && (!j->ref || !j->tgt || !j->ulhc || !j->offsets))
        return fail(h, AMPCOR_E_ARG, "null raster, corner or offset pointer");
    if (j->ref_lines <= 0 || j->ref_samples <= 0 || j->tgt_lines <= 0 || j->tgt_samples <= 0)
        return fail(h, AMPCOR_E_ARG, "empty raster");
    if (j->pairs > 0x7fffffffull) return fail(h, AMPCOR_E_ARG, "too many pairs in one batch");
    return AMPCOR_OK;
}

int ampcor_correlate(ampcor_handle* h, const ampcor_job* j, void* stream)
{
    int rc = check_job(h, j);
    if (rc) return rc;
    CK(h, cudaSetDevice(h->prm.device), "cudaSetDevice");
    if ((rc = ensure_pairs(h, j->pairs))) return rc;
    cudaStream_t st = pick(h, stream);
    if (j->pairs == 0) return AMPCOR_OK;
    pair_offsets_kernel<<<(unsigned)((j->pairs + 255) / 256), 256, 0, st>>>(
        j->ulhc, (long long)j->pairs, j->ref_lines, j->ref_samples, j->tgt_lines, j->tgt_samples,
        h->R, h->W, h->d_ref_off, h->d_tgt_off, h->d_bad);
    CK(h, cudaGetLastError(), "launching the pair offsets kernel");
    PairSource src{static_cast<const float2*>(j->ref), h->d_ref_off, j->ref_samples,
                   static_cast<const float2*>(j->tgt), h->d_tgt_off, j->tgt_samples,
                   j->ref_lines * j->ref_samples, j->tgt_lines * j->tgt_samples, j->tgt_lines};
    return run_pipeline(h, src, (long long)j->pairs, reinterpret_cast<float2*>(j->offsets),
                        reinterpret_cast<PairDiag*>(j->diag), j->coarse_surfaces,
                        j->refined_surfaces, st);
}

int ampcor_synchronize(ampcor_handle* h, void* stream)
{
    if (!h) return AMPCOR_E_ARG;
    CK(h, cudaSetDevice(h->prm.device), "cudaSetDevice");
    cudaStream_t st = pick(h, stream);
    unsigned int bad = 0, tcerr = 0;
    CK(h, cudaMemcpyAsync(&bad, h->d_bad, sizeof(bad), cudaMemcpyDeviceToHost, st), "reading the bounds counter");
    CK(h, cudaMemcpyAsync(&tcerr, h->d_tc_err, sizeof(tcerr), cudaMemcpyDeviceToHost, st), "reading the error counter");
    CK(h, cudaStreamSynchronize(st), "running the correlation pipeline");
    if (tcerr) {
        CK(h, cudaMemsetAsync(h->d_tc_err, 0, sizeof(unsigned int), st), "resetting the error counter");
        CK(h, cudaStreamSynchronize(st), "resetting the error counter");
        return fail(h, AMPCOR_E_CUDA, std::to_string(tcerr) +
                           " tile pair(s) or resident blocks timed out in a bounded device wait");
    }
    if (bad) {
        CK(h, cudaMemsetAsync(h->d_bad, 0, sizeof(unsigned int), st), "resetting the bounds counter");
        CK(h, cudaStreamSynchronize(st), "resetting the bounds counter");
        return fail(h, AMPCOR_E_BOUNDS, std::to_string(bad) + " tile pair(s) leave their raster; their offsets are NaN");
    }
    return AMPCOR_OK;
}

// A host-buffer job of the spectral form in at most kHostBands groups of consecutive pairs,
// growing from one wave: group g needs the raster rows up to the deepest chip and window of
// pairs 0 .. end of g (so pairs in raster order need about a band each); those rows go up on
// the copy stream while the compute stream
// correlates group g - 1, then the compute stream detects the new rows, extends the box
// statistics to the box rows they complete and correlates group g.  Same kernels and the same
// values as one upload followed by the whole job; the upload hides behind all but the first band.
int correlate_host_banded(ampcor_handle* h, const ampcor_job* j)
{
    int rc = AMPCOR_OK;
    cudaStream_t st = h->stream;
    if (!h->copy_stream)
        CK(h, cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking), "creating the upload stream");
    for (cudaEvent_t& e : h->band_ev)
        if (!e) CK(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "creating the band events");
    if ((rc = ensure_pairs(h, j->pairs))) return rc;
    const long long P = (long long)j->pairs;
    const long long rs = j->ref_samples, ts = j->tgt_samples;
    const long long rlines = j->ref_lines, tlines = j->tgt_lines;
    // the raster buffers may still be read by the previous job's kernels
    CK(h, cudaEventRecord(h->band_ev[kHostBands], st), "ordering the upload");
    CK(h, cudaStreamWaitEvent(h->copy_stream, h->band_ev[kHostBands], 0), "ordering the upload");
    CK(h, cudaMemcpyAsync(h->d_ulhc, j->ulhc, 4 * P * sizeof(int32_t), cudaMemcpyHostToDevice, st),
       "uploading the pair corners");
    pair_offsets_kernel<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(h->d_ulhc, P, rlines, rs, tlines, ts, h->R,
                                                                      h->W, h->d_ref_off, h->d_tgt_off, h->d_bad);
    CK(h, cudaGetLastError(), "launching the pair offsets kernel");
    const float2* dref = reinterpret_cast<const float2*>(h->d_ref_raster);
    const float2* dtgt = reinterpret_cast<const float2*>(h->d_tgt_raster);
    PairSource src{dref, h->d_ref_off, rs, dtgt, h->d_tgt_off, ts, rlines * rs, tlines * ts, tlines};
    SpecRasters r;
    if ((rc = spec_rasters(h, src, P, r))) return rc;
    const float2* href = static_cast<const float2*>(j->ref);
    const float2* htgt = static_cast<const float2*>(j->tgt);
    // group ends on whole waves of the correlation kernels (two CTAs per SM at most) once a job
    // has a few waves per group
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long granule = std::min<long long>(2LL * std::max(sms, 1), std::max<long long>(1, P / (4 * kHostBands)));
    long long up_r = 0, up_t = 0, boxes = 0, need_r = 0, need_t = 0, p0 = 0;
    // the first group is one granule (its upload is the one nothing hides); each next group is
    // twice the one before (its rows go up while the one before is correlated, and uploading a
    // pair's rows takes about half as long as correlating it), the last takes the rest
    long long size = std::min(P, granule);
    for (int g = 0; g < kHostBands && p0 < P; ++g) {
        long long p1 = p0 + (size + granule / 2) / granule * granule;
        if (g + 1 == kHostBands || p1 > P) p1 = P;
        size = size * 2;
        if (p1 <= p0) continue;
        for (long long p = p0; p < p1; ++p) {
            need_r = std::max<long long>(need_r, std::min<long long>((long long)j->ulhc[4 * p] + h->R, rlines));
            need_t = std::max<long long>(need_t, std::min<long long>((long long)j->ulhc[4 * p + 2] + h->W, tlines));
        }
        const long long nr = p1 == P ? rlines : std::max(need_r, up_r);
        const long long nt = p1 == P ? tlines : std::max(need_t, up_t);
        if (nr > up_r)
            CK(h, cudaMemcpyAsync(static_cast<float2*>(h->d_ref_raster) + up_r * rs, href + up_r * rs, (nr - up_r) * rs * sizeof(float2),
                                  cudaMemcpyHostToDevice, h->copy_stream),
               "uploading the reference raster");
        if (nt > up_t)
            CK(h, cudaMemcpyAsync(static_cast<float2*>(h->d_tgt_raster) + up_t * ts, htgt + up_t * ts, (nt - up_t) * ts * sizeof(float2),
                                  cudaMemcpyHostToDevice, h->copy_stream),
               "uploading the secondary raster");
        CK(h, cudaEventRecord(h->band_ev[g], h->copy_stream), "recording a band");
        CK(h, cudaStreamWaitEvent(st, h->band_ev[g], 0), "waiting for a band");
        const long long nb = r.raster_stats ? std::max<long long>(0, std::min(r.rows, nt - h->R + 1)) : 0;
        if ((rc = spec_band(h, src, r, up_r * rs, nr * rs, up_t * ts, nt * ts, boxes, std::max(boxes, nb), st)))
            return rc;
        boxes = std::max(boxes, nb);
        up_r = nr;
        up_t = nt;
        if ((rc = spec_pairs(h, src, r, p0, p1, reinterpret_cast<float2*>(h->d_job_offsets),
                             j->diag ? reinterpret_cast<PairDiag*>(h->d_job_diag) : nullptr, nullptr, nullptr, st)))
            return rc;
        p0 = p1;
    }
    CK(h, cudaMemcpyAsync(j->offsets, h->d_job_offsets, 2 * P * sizeof(float), cudaMemcpyDeviceToHost, st),
       "downloading the offsets");
    if (j->diag)
        CK(h, cudaMemcpyAsync(j->diag, h->d_job_diag, P * sizeof(ampcor_pair_diag), cudaMemcpyDeviceToHost, st),
           "downloading the diagnostics");
    return AMPCOR_OK;
}

int ampcor_correlate_host(ampcor_handle* h, const ampcor_job* j)
{
    int rc = check_job(h, j);
    if (rc) return rc;
    CK(h, cudaSetDevice(h->prm.device), "cudaSetDevice");
    if (j->pairs == 0) return AMPCOR_OK;
    const size_t rb = (size_t)j->ref_lines * j->ref_samples * sizeof(float2);
    const size_t tb = (size_t)j->tgt_lines * j->tgt_samples * sizeof(float2);
    if (h->raster_bytes_ref < rb) {
        cudaFree(h->d_ref_raster);
        h->d_ref_raster = nullptr;
        h->raster_bytes_ref = 0;
        CK(h, cudaMalloc(&h->d_ref_raster, rb), "allocating the reference raster");
        h->raster_bytes_ref = rb;
    }
    if (h->raster_bytes_tgt < tb) {
        cudaFree(h->d_tgt_raster);
        h->d_tgt_raster = nullptr;
        h->raster_bytes_tgt = 0;
        CK(h, cudaMalloc(&h->d_tgt_raster, tb), "allocating the secondary raster");
        h->raster_bytes_tgt = tb;
    }
    if ((rc = grow(h, h->d_ulhc, h->ulhc_cap, 4 * j->pairs, "pair corners"))) return rc;
    if ((rc = grow(h, h->d_job_offsets, h->job_offsets_cap, 2 * j->pairs, "offsets"))) return rc;
    if (j->diag && (rc = grow(h, h->d_job_diag, h->job_diag_cap, j->pairs, "diagnostics"))) return rc;
    cudaStream_t st = h->stream;
    if (h->form == kFormSpectral && j->pairs >= 2 * kHostBands && !j->coarse_surfaces && !j->refined_surfaces &&
        j->ref != j->tgt) {
        if ((rc = correlate_host_banded(h, j))) return rc;
        return ampcor_synchronize(h, st);
    }
    CK(h, cudaMemcpyAsync(h->d_ref_raster, j->ref, rb, cudaMemcpyHostToDevice, st), "uploading the reference raster");
    CK(h, cudaMemcpyAsync(h->d_tgt_raster, j->tgt, tb, cudaMemcpyHostToDevice, st), "uploading the secondary raster");
    CK(h, cudaMemcpyAsync(h->d_ulhc, j->ulhc, 4 * j->pairs * sizeof(int32_t), cudaMemcpyHostToDevice, st),
       "uploading the pair corners");
    ampcor_job dj = *j;
    dj.ref = h->d_ref_raster;
    dj.tgt = h->d_tgt_raster;
    dj.ulhc = h->d_ulhc;
    dj.offsets = h->d_job_offsets;
    dj.diag = j->diag ? h->d_job_diag : nullptr;
    dj.coarse_surfaces = nullptr;
    dj.refined_surfaces = nullptr;
    if ((rc = ampcor_correlate(h, &dj, st))) return rc;
    CK(h, cudaMemcpyAsync(j->offsets, h->d_job_offsets, 2 * j->pairs * sizeof(float), cudaMemcpyDeviceToHost, st),
       "downloading the offsets");
    if (j->diag)
        CK(h, cudaMemcpyAsync(j->diag, h->d_job_diag, j->pairs * sizeof(ampcor_pair_diag), cudaMemcpyDeviceToHost, st),
           "downloading the diagnostics");
    return ampcor_synchronize(h, st);
}

int ampcor_profile(ampcor_handle* h, int enable)
{
    if (!h) return AMPCOR_E_ARG;
    CK(h, cudaSetDevice(h->prm.device), "cudaSetDevice");
    drop_marks(h);
    h->profiling = enable != 0;
    return AMPCOR_OK;
}

int ampcor_stage_times(ampcor_handle* h, double* coarse_ms, double* refine_ms, double* fine_ms,
                       uint64_t* launches)
{
    if (!h) return AMPCOR_E_ARG;
    CK(h, cudaSetDevice(h->prm.device), "cudaSetDevice");
    double t[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    uint64_t n = 0;
    for (int s = 0; s < 6; ++s)
        for (auto& pr : h->marks[s]) {
            CK(h, cudaEventSynchronize(pr.second), "waiting for a stage event");
            float ms = 0.0f;
            CK(h, cudaEventElapsedTime(&ms, pr.first, pr.second), "reading a stage event");
            t[s] += ms;
            ++n;
        }
    drop_marks(h);
    if (coarse_ms) *coarse_ms = t[0] + t[3];
    if (refine_ms) *refine_ms = t[1];
    if (fine_ms) *fine_ms = t[2] + t[4] + t[5];
    if (launches) *launches = n;
    return AMPCOR_OK;
}

int ampcor_kernel_times(ampcor_handle* h, double* ms, uint64_t* launches)
{
    if (!h || !ms || !launches) return fail(h, AMPCOR_E_ARG, "null argument");
    CK(h, cudaSetDevice(h->prm.device), "cudaSetDevice");
    for (int s = 0; s < 6; ++s) {
        ms[s] = 0.0;
        launches[s] = 0;
        for (auto& pr : h->marks[s]) {
            CK(h, cudaEventSynchronize(pr.second), "waiting for a kernel event");
            float x = 0.0f;
            CK(h, cudaEventElapsedTime(&x, pr.first, pr.second), "reading a kernel event");
            ms[s] += x;
        }
        launches[s] = h->mark_kernels[s];
    }
    drop_marks(h);
    return AMPCOR_OK;
}

int ampcor_configure(ampcor_handle* h, int form, uint64_t chunk)
{
    if (!h) return AMPCOR_E_ARG;
    CK(h, cudaSetDevice(h->prm.device), "cudaSetDevice");
    CK(h, cudaStreamSynchronize(h->stream), "waiting for the worker");
    if (form == kFormTensor) {
        if (!h->tensor_ok) return fail(h, AMPCOR_E_SHAPE, "this geometry has no tensor-core form");
    } else if (form == kFormSpectral) {
        if (!h->spectral_ok) return fail(h, AMPCOR_E_SHAPE, "this geometry has no spectral form");
    } else if (form == kFormPlain) {
        if (!h->plain_ok) return fail(h, AMPCOR_E_SHAPE, "this geometry has no plain FP32 form");
    } else if (form != -1) {
        return fail(h, AMPCOR_E_ARG, "form must be -1, 0, 1 or 2");
    }
    const bool switching = form != -1 && form != h->form;
    if (form != -1) h->form = form;
    if (chunk && chunk != h->chunk) {
        // the chunk scratch is sized on first use
        free_chunk_scratch(h);
        h->chunk_override = (size_t)chunk;
    } else if (switching && h->d_refined) {
        // a form switch needs the chunk scratch of the new form
        free_chunk_scratch(h);
    }
    return AMPCOR_OK;
}

int ampcor_inject_timeout(ampcor_handle* h, int batches)
{
    if (!h) return AMPCOR_E_ARG;
    if (batches < 0) return fail(h, AMPCOR_E_ARG, "batches must not be negative");
    if (!h->zoom_tc || h->form == kFormPlain)
        return fail(h, AMPCOR_E_STATE, "the worker's form has no bounded tensor-core waits");
    h->inject_timeouts = batches;
    return AMPCOR_OK;
}

int ampcor_chunk(const ampcor_handle* h, uint64_t* chunk)
{
    if (!h || !chunk) return AMPCOR_E_ARG;
    *chunk = h->chunk_override ? h->chunk_override : default_chunk();
    return AMPCOR_OK;
}

int ampcor_form(const ampcor_handle* h)
{
    if (!h) return -1;
    return h->form;
}

int ampcor_surface_dims(const ampcor_handle* h, int32_t* coarse, int32_t* refined, int32_t* zoomed)
{
    if (!h) return AMPCOR_E_ARG;
    if (coarse) *coarse = h->C;
    if (refined) *refined = h->Cf;
    if (zoomed) *zoomed = h->Z;
    return AMPCOR_OK;
}

const char* ampcor_last_error(const ampcor_handle* h)
{
    if (h) return h->err.c_str();
    std::lock_guard<std::mutex> lk(g_create_mutex);
    return g_create_error.c_str();
}

const char* ampcor_version(void) { return kVersion; }
const char* ampcor_copyright(void) { return kCopyright; }

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Allocation-free entry point.
//
// Some callers cannot allocate device memory while they run: applications that reserve the whole
// GPU up front for their own memory pool (a caching allocator that owns every byte, so a stray
// cudaMalloc fails or fragments it), and real-time or on-board processing chains that forbid any
// allocation after start-up.  ampcor_correlate_noalloc() serves them: every intermediate of the
// pipeline lives in the fixed device array below, which the CUDA runtime creates when it loads
// this library's device code on a device (with lazy module loading, at the first call that needs
// it: a call with no pairs at start-up does that and launches nothing) and keeps until the process
// exits (kNoAllocBytes per device).  The array is shared by all calls; calls that overlap on the
// GPU race.  Every call waits for its stream, so none runs on a capturing stream.
// ------------------------------------------------------------------------------------------

namespace {

constexpr long long kNoAllocMaxPairs = 16384;                // pairs per call
constexpr long long kNoAllocTapFloats = 16384;               // interpolation tap tables
constexpr long long kNoAllocRefinedBytes = 40ll << 20;       // refined amplitudes of a chunk
constexpr long long kNoAllocTapsOff = 0;
constexpr long long kNoAllocRefOff = kNoAllocTapsOff + kNoAllocTapFloats * 4;
constexpr long long kNoAllocTgtOff = kNoAllocRefOff + kNoAllocMaxPairs * 8;
constexpr long long kNoAllocCoarseOff = kNoAllocTgtOff + kNoAllocMaxPairs * 8;
constexpr long long kNoAllocPeakOff = kNoAllocCoarseOff + kNoAllocMaxPairs * 16;
constexpr long long kNoAllocBadOff = kNoAllocPeakOff + kNoAllocMaxPairs * 4;
constexpr long long kNoAllocRefinedOff = kNoAllocBadOff + 256;
constexpr long long kNoAllocBytes = kNoAllocRefinedOff + kNoAllocRefinedBytes;
constexpr int kNoAllocMaxDevices = 64;

static_assert(kNoAllocRefinedOff % 256 == 0, "scratch regions stay 256-byte aligned");

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

std::mutex g_noalloc_mutex;
void* g_noalloc_base[kNoAllocMaxDevices] = {};
float g_noalloc_taps[kNoAllocTapFloats];

int noalloc_fail(char* errbuf, size_t errlen, int code, const char* what, cudaError_t e = cudaSuccess)
{
    if (errbuf && errlen) {
        if (e != cudaSuccess)
            std::snprintf(errbuf, errlen, "%s: %s", what, cudaGetErrorName(e));
        else
            std::snprintf(errbuf, errlen, "%s", what);
    }
    return code;
}

void taps_fill(int N, int f, int s0, int len, float* out)
{
    for (int s = s0; s < f; ++s)
        for (int d = 0; d < len; ++d)
            out[(size_t)(s - s0) * len + d] = (float)dirichlet(N, d - (N - 1) + (double)s / f);
}

}  // namespace

extern "C" int ampcor_correlate_noalloc(const ampcor_params* p, const ampcor_job* j, void* stream,
                                        char* errbuf, size_t errlen)
{
    if (errbuf && errlen) errbuf[0] = '\0';
    if (!p || !j) return noalloc_fail(errbuf, errlen, AMPCOR_E_ARG, "null argument");
    if (p->ref_lines != p->ref_samples || p->tgt_lines != p->tgt_samples)
        return noalloc_fail(errbuf, errlen, AMPCOR_E_SHAPE, "chips and search windows must be square");
    if (p->tgt_lines < p->ref_lines || (p->tgt_lines - p->ref_lines) % 2)
        return noalloc_fail(errbuf, errlen, AMPCOR_E_SHAPE, "window must exceed the chip by an even margin");
    if (p->refine_factor < 1 || p->zoom_factor < 1 || p->ref_lines > 4096 || p->refine_factor > 16 ||
        p->zoom_factor > 64 || p->refine_margin > 1024)
        return noalloc_fail(errbuf, errlen, AMPCOR_E_SHAPE, "geometry out of range");
    if (j->pairs > (uint64_t)kNoAllocMaxPairs)
        return noalloc_fail(errbuf, errlen, AMPCOR_E_ARG,
                            "ampcor_correlate_noalloc takes at most 16384 pairs per call");
    if (j->pairs && (!j->ref || !j->tgt || !j->ulhc || !j->offsets))
        return noalloc_fail(errbuf, errlen, AMPCOR_E_ARG, "null raster, corner or offset pointer");
    if (j->pairs && (j->ref_lines <= 0 || j->ref_samples <= 0 || j->tgt_lines <= 0 || j->tgt_samples <= 0))
        return noalloc_fail(errbuf, errlen, AMPCOR_E_ARG, "empty raster");
    if (p->device < 0 || p->device >= kNoAllocMaxDevices)
        return noalloc_fail(errbuf, errlen, AMPCOR_E_ARG, "device ordinal out of range");

    const int R = (int)p->ref_lines, W = (int)p->tgt_lines, f = (int)p->refine_factor;
    const int m = (int)p->refine_margin, z = (int)p->zoom_factor;
    const int E = R + 2 * m, Rf = f * R, Wf = f * E, Cf = 2 * f * m + 1, Z = z * Cf, M = (W - R) / 2;
    if (E > W)
        return noalloc_fail(errbuf, errlen, AMPCOR_E_SHAPE,
                            "refinement neighbourhood (chip + 2 * refine margin) exceeds the window");
    ZoomGeom zg{};
    zg.Cf = Cf;
    zg.z = z;
    zg.Z = Z;
    zg.cb = 1;
    for (int cb : {17, 13, 11, 5, 3})
        if (Cf % cb == 0) {
            zg.cb = cb;
            break;
        }
    zg.taps_len = 2 * Cf + 32;
    NccGeom gc{}, gf{};
    InterpGeom ic{}, iw{};
    std::string err;
    if (!plan_ncc(R, W, 0, 0, gc, err) || !plan_ncc(Rf, Wf, Cf * Z, z * zg.taps_len, gf, err) ||
        !plan_interp(R, f, ic, err) || !plan_interp(E, f, iw, err))
        return noalloc_fail(errbuf, errlen, AMPCOR_E_SHAPE, "tile geometry not supported by this build");
    const long long chip_taps = (long long)(f - 1) * ic.taps_len;
    const long long win_taps = (long long)(f - 1) * iw.taps_len;
    const long long zoom_taps = (long long)z * zg.taps_len;
    if (chip_taps + win_taps + zoom_taps > kNoAllocTapFloats)
        return noalloc_fail(errbuf, errlen, AMPCOR_E_SHAPE, "interpolation tables exceed the fixed scratch");
    const long long refined_stride = (long long)Rf * Rf + (long long)Wf * Wf;
    const long long chunk = kNoAllocRefinedBytes / (refined_stride * 4);
    if (chunk < 1)
        return noalloc_fail(errbuf, errlen, AMPCOR_E_SHAPE, "refined tiles exceed the fixed scratch");

    cudaError_t e = cudaSetDevice(p->device);
    if (e != cudaSuccess) return noalloc_fail(errbuf, errlen, AMPCOR_E_CUDA, "cudaSetDevice", e);
    cudaStream_t st = (cudaStream_t)stream;
    // every call waits for its stream before it returns, which a capturing stream does not allow
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    if ((e = cudaStreamIsCapturing(st, &capture)) != cudaSuccess)
        return noalloc_fail(errbuf, errlen, AMPCOR_E_CUDA, "querying the stream", e);
    if (capture != cudaStreamCaptureStatusNone)
        return noalloc_fail(errbuf, errlen, AMPCOR_E_ARG,
                            "ampcor_correlate_noalloc waits for its stream and cannot run on a capturing stream");

    std::lock_guard<std::mutex> lk(g_noalloc_mutex);
    // a failure once work is queued still waits for the stream, so that the shared array is idle
    // whenever the lock is released
    auto queued_fail = [&](int code, const char* what, cudaError_t qe) {
        cudaStreamSynchronize(st);
        return noalloc_fail(errbuf, errlen, code, what, qe);
    };
    // the device address of the fixed array, looked up once per device with that device current
    if (!g_noalloc_base[p->device]) {
        void* base = nullptr;
        e = cudaGetSymbolAddress(&base, g_noalloc_scratch);
        if (e != cudaSuccess) return noalloc_fail(errbuf, errlen, AMPCOR_E_CUDA, "cudaGetSymbolAddress", e);
        g_noalloc_base[p->device] = base;
    }
    unsigned char* base = static_cast<unsigned char*>(g_noalloc_base[p->device]);
    float* taps = reinterpret_cast<float*>(base + kNoAllocTapsOff);
    long long* ref_off = reinterpret_cast<long long*>(base + kNoAllocRefOff);
    long long* tgt_off = reinterpret_cast<long long*>(base + kNoAllocTgtOff);
    CoarseOut* coarse = reinterpret_cast<CoarseOut*>(base + kNoAllocCoarseOff);
    float* peak = reinterpret_cast<float*>(base + kNoAllocPeakOff);
    unsigned int* bad = reinterpret_cast<unsigned int*>(base + kNoAllocBadOff);
    float* refined = reinterpret_cast<float*>(base + kNoAllocRefinedOff);

    const int kMaxSmem = 227 * 1024;
    if ((e = cudaFuncSetAttribute(coarse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(fine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(refine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem)) != cudaSuccess)
        return noalloc_fail(errbuf, errlen, AMPCOR_E_CUDA, "configuring kernel shared memory", e);
    // an empty batch only loads the device code and looks up the array (a start-up call)
    if (j->pairs == 0) return AMPCOR_OK;

    // tap tables: computed on the host into a fixed buffer; a copy from pageable memory has left
    // the buffer when cudaMemcpyAsync returns, so the buffer is free again under the lock
    taps_fill(R, f, 1, ic.taps_len, g_noalloc_taps);
    taps_fill(E, f, 1, iw.taps_len, g_noalloc_taps + chip_taps);
    taps_fill(Cf, z, 0, zg.taps_len, g_noalloc_taps + chip_taps + win_taps);
    if ((e = cudaMemcpyAsync(taps, g_noalloc_taps, (chip_taps + win_taps + zoom_taps) * sizeof(float),
                             cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return queued_fail(AMPCOR_E_CUDA, "uploading interpolation taps", e);
    // the bounds counter keeps the previous call's value: clear it
    if ((e = cudaMemsetAsync(bad, 0, sizeof(unsigned int), st)) != cudaSuccess)
        return queued_fail(AMPCOR_E_CUDA, "clearing the bounds counter", e);

    const long long P = (long long)j->pairs;
    pair_offsets_kernel<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(
        j->ulhc, P, j->ref_lines, j->ref_samples, j->tgt_lines, j->tgt_samples, R, W, ref_off, tgt_off, bad);
    PairSource src{static_cast<const float2*>(j->ref), ref_off, j->ref_samples,
                   static_cast<const float2*>(j->tgt), tgt_off, j->tgt_samples,
                   j->ref_lines * j->ref_samples, j->tgt_lines * j->tgt_samples, j->tgt_lines};
    coarse_kernel<<<(unsigned)P, kThreads, gc.smem_bytes, st>>>(src, 0, P, gc, m, coarse, peak,
                                                                j->coarse_surfaces);
    const int refine_smem = std::max(ic.smem_bytes, iw.smem_bytes);
    for (long long c0 = 0; c0 < P; c0 += chunk) {
        const long long n = std::min(chunk, P - c0);
        refine_kernel<<<(unsigned)n, kThreads, refine_smem, st>>>(src, c0, n, coarse, ic, iw, taps,
                                                                  taps + chip_taps, refined, refined_stride,
                                                                  (p->flags & AMPCOR_FLAG_DERAMP) ? 1 : 0);
        fine_kernel<<<(unsigned)n, kThreads, gf.smem_bytes, st>>>(
            refined, refined_stride, c0, n, ref_off, gf, zg, taps + chip_taps + win_taps, coarse, peak, M, f,
            m, (p->flags & AMPCOR_FLAG_REF_COMPAT) ? 1 : 0, reinterpret_cast<float2*>(j->offsets),
            reinterpret_cast<PairDiag*>(j->diag), j->refined_surfaces);
    }
    if ((e = cudaGetLastError()) != cudaSuccess)
        return queued_fail(AMPCOR_E_CUDA, "launching the correlation kernels", e);
    unsigned int nbad = 0;
    if ((e = cudaMemcpyAsync(&nbad, bad, sizeof(nbad), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return queued_fail(AMPCOR_E_CUDA, "running the correlation pipeline", e);
    if (nbad)
        return noalloc_fail(errbuf, errlen, AMPCOR_E_BOUNDS,
                            "tile pair(s) leave their raster; their offsets are NaN");
    return AMPCOR_OK;
}
