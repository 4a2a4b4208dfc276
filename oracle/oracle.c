/*
 * FP64 CPU oracle for the ampcor batched tile correlator.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the ampcor_b200 package, its CUDA
 * kernels or its C ABI) links, loads or calls this file; only the tests, the smoke check
 * and the CPU-baseline leg of the benchmark do, and only as the checker.
 *
 * Two restatements live here:
 *
 *  1. oracle_coarse_cpu(): the reference CPU coarse correlator, formula for formula
 *     (lib/libampcor/correlators/Sequential.cc:17-97 with the amplitude/accumulate steps of
 *     lib/libampcor/correlators/Sequential.icc:16-182 and the summed-area table of
 *     lib/libampcor/correlators/SumArea.icc:66-180).  Its quirks are kept on purpose: the
 *     chip is NOT mean-subtracted (the std::for_each at Sequential.icc:86 mutates nothing) so
 *     the chip "variance" is the raw sum of squares (Sequential.cc:55); amplitudes are the
 *     float std::abs of complex<float> stored as double (Sequential.icc:38-50).  Its argmax is
 *     the one the integer offsets are compared with, bit for bit.
 *
 *  2. oracle_adjust(): the full pipeline in FP64, written to the intended math of the CUDA
 *     worker (lib/libampcor_cuda/correlators/Sequential.icc:47-141):
 *       detect (detect.cu:78-115) -> chip mean/sigma (refStats.cu:118-302)
 *       -> window box means (sat.cu:81-149, tgtStats.cu:88-168)
 *       -> NCC (correlate.cu:160-318) -> first strict maximum (maxcor.cu:79-133)
 *       -> nudge (nudge.cu:81-143) -> band-limited FFT upsampling of the complex chip and of
 *          the (R+2m)^2 neighbourhood (intent of Sequential.icc:703-1087, migrate.cu:101-154)
 *       -> refined NCC -> band-limited zoom of the refined surface (intent of
 *          Sequential.icc:1101-1286) -> first strict maximum -> offsets (offsets.cu:86-129).
 *     The reference CUDA refine/zoom/offset stages are defective (forward transform used as
 *     the inverse, no spectrum split, no 1/N, only 32 columns copied, refine margin subtracted
 *     twice); this oracle implements what they intend.  With ORACLE_REF_COMPAT the offset is
 *     assembled with the reference's formula (offsets.cu:124-125) and the zoomed surface is
 *     taken as a magnitude (c2r.cu:130).
 *
 * The band-limited upsampling is computed as the separable Dirichlet-kernel matrix that the
 * zero-padded FFT is equal to (the spectrum of an N-sample row zero-padded to f*N samples,
 * with the Nyquist bin split in half for even N, then inverse transformed and scaled by 1/N).
 * tests/test_oracle.py checks this against numpy.fft in FP64.
 *
 * Zero-variance placements (a flat window) and flat chips give correlation 0 here and on the
 * GPU; the reference divides by zero there.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef long long i64;

/* where the tiles of pair p live: complex64 pixels (interleaved float re, im) */
typedef struct {
    const float *ref_base;   /* complex64 raster (or arena) holding the chips */
    const i64 *ref_off;      /* per pair: offset of the chip's upper-left pixel, in pixels */
    i64 ref_stride;          /* row stride of the chip source, in pixels */
    const float *tgt_base;   /* complex64 raster (or arena) holding the search windows */
    const i64 *tgt_off;      /* per pair: offset of the window's upper-left pixel */
    i64 tgt_stride;          /* row stride of the window source, in pixels */
} oracle_src;

typedef struct {
    int R;          /* chip dimension */
    int W;          /* search window dimension, R + 2*margin */
    int f;          /* refine factor */
    int m;          /* refine margin */
    int z;          /* zoom factor */
    int flags;      /* ORACLE_REF_COMPAT */
} oracle_geom;

#define ORACLE_REF_COMPAT 1
#define ORACLE_DERAMP 2     /* remove the linear phase ramp of each complex tile before refining */

/* per-pair diagnostics */
typedef struct {
    int coarse_u, coarse_v;     /* coarse argmax (placement row, col) */
    int top, left;              /* nudged neighbourhood corner inside the window */
    int fine_p, fine_q;         /* argmax on the zoomed surface */
    int refined_u, refined_v;   /* argmax on the refined surface */
    double coarse_peak;         /* coarse NCC maximum */
    double coarse_gap;          /* coarse: maximum minus second largest value */
    double refined_peak;        /* refined NCC maximum (the reported peak correlation) */
    double zoom_peak;           /* zoomed surface maximum */
    double zoom_gap;            /* zoomed: maximum minus second largest value */
} oracle_diag;

/* ------------------------------------------------------------------------------------- */
/* small helpers                                                                          */
/* ------------------------------------------------------------------------------------- */

/* first (row-major) strict maximum, maxcor.cu:114-126: start at cell 0, replace on '>' */
int oracle_argmax_first(const double *a, i64 n)
{
    i64 best = 0;
    double high = a[0];
    for (i64 k = 1; k < n; ++k) {
        if (a[k] > high) { high = a[k]; best = k; }
    }
    return (int)best;
}

static double second_largest_excluding(const double *a, i64 n, i64 skip)
{
    double s = -HUGE_VAL;
    for (i64 k = 0; k < n; ++k) if (k != skip && a[k] > s) s = a[k];
    return s;
}

/* amplitude as the reference CPU path computes it: float |z| (hypotf) widened to double */
static inline double amp_cpu(const float *px) { return (double)hypotf(px[0], px[1]); }

/* amplitude in FP64 */
static inline double amp64(const float *px)
{
    double re = px[0], im = px[1];
    return sqrt(re * re + im * im);
}

/* ------------------------------------------------------------------------------------- */
/* stage functions (exported for the known-answer tests)                                  */
/* ------------------------------------------------------------------------------------- */

/* inclusive summed-area table, SumArea.icc:143-180 (top row, left column, then interior) */
void oracle_sat(const double *x, int rows, int cols, double *sat)
{
    sat[0] = x[0];
    for (int j = 1; j < cols; ++j) sat[j] = x[j] + sat[j - 1];
    for (int i = 1; i < rows; ++i) sat[(i64)i * cols] = x[(i64)i * cols] + sat[(i64)(i - 1) * cols];
    for (int i = 1; i < rows; ++i)
        for (int j = 1; j < cols; ++j) {
            i64 k = (i64)i * cols + j;
            sat[k] = x[k] + sat[k - 1] + sat[k - cols] - sat[k - cols - 1];
        }
}

/* box sum over rows [r0, r1) and columns [c0, c1) from an inclusive SAT, SumArea.icc:66-140 */
double oracle_box(const double *sat, int cols, int r0, int c0, int r1, int c1)
{
    double s = sat[(i64)(r1 - 1) * cols + (c1 - 1)];
    if (r0 > 0) s -= sat[(i64)(r0 - 1) * cols + (c1 - 1)];
    if (c0 > 0) s -= sat[(i64)(r1 - 1) * cols + (c0 - 1)];
    if (r0 > 0 && c0 > 0) s += sat[(i64)(r0 - 1) * cols + (c0 - 1)];
    return s;
}

/*
 * Normalized cross-correlation surface of an R x R chip over every placement inside a
 * W x W window (C = W - R + 1 per axis): the chip is made zero-mean, each placement's window
 * mean comes from the summed-area table, and
 *     gamma(u,v) = sum r'(t - mu) / (|r'| * sqrt(sum (t - mu)^2)),
 * correlate.cu:213-313.  Returns sigma_r = |r'|.
 */
double oracle_ncc(const double *chip, int R, const double *win, int W, double *gamma,
                  double *scratch /* W*W doubles + R*R doubles */)
{
    const int C = W - R + 1;
    const double cells = (double)R * (double)R;
    double *sat = scratch;
    double *rp = scratch + (i64)W * W;

    double mean = 0.0;
    for (i64 k = 0; k < (i64)R * R; ++k) mean += chip[k];
    mean /= cells;
    double ss = 0.0;
    for (i64 k = 0; k < (i64)R * R; ++k) { rp[k] = chip[k] - mean; ss += rp[k] * rp[k]; }
    const double sigma = sqrt(ss);

    oracle_sat(win, W, W, sat);
    for (int u = 0; u < C; ++u) {
        for (int v = 0; v < C; ++v) {
            const double mu = oracle_box(sat, W, u, v, u + R, v + R) / cells;
            double num = 0.0, var = 0.0;
            for (int i = 0; i < R; ++i) {
                const double *trow = win + (i64)(u + i) * W + v;
                const double *rrow = rp + (i64)i * R;
#pragma omp simd reduction(+ : num, var)
                for (int j = 0; j < R; ++j) {
                    const double t = trow[j] - mu;
                    num += rrow[j] * t;
                    var += t * t;
                }
            }
            const double den = sigma * sqrt(var);
            gamma[(i64)u * C + v] = (var > 0.0 && sigma > 0.0) ? num / den : 0.0;
        }
    }
    return sigma;
}

/* nudge.cu:107-140: move the (R+2m)^2 neighbourhood so that it fits inside the W x W window */
void oracle_nudge(int u, int v, int R, int W, int m, int *top, int *left)
{
    const int E = R + 2 * m;
    int l = v - m;
    if (l < 0) l = 0;
    if (l + E > W) l = W - E;
    int t = u - m;
    if (t < 0) t = 0;
    if (t + E > W) t = W - E;
    *top = t;
    *left = l;
}

/*
 * Band-limited interpolation kernel of an N-periodic sequence, evaluated at offset d:
 *   D_N(d) = (1/N) sum_n c_n cos(2 pi n d / N)
 * n over [-(N-1)/2, (N-1)/2] for odd N, over [-N/2, N/2] for even N with c = 1/2 at the
 * Nyquist pair.  Zero-padding the N-point spectrum to f*N points (negative frequencies kept
 * at the top, Nyquist bin split) and inverse transforming with a 1/N scale is the same as
 *   out[p] = sum_k D_N(p/f - k) in[k].
 */
double oracle_dirichlet(int N, double d)
{
    double s = 0.0;
    if (N % 2) {
        const int h = (N - 1) / 2;
        s = 1.0;
        for (int n = 1; n <= h; ++n) s += 2.0 * cos(2.0 * M_PI * n * d / N);
    } else {
        const int h = N / 2;
        s = 1.0;
        for (int n = 1; n < h; ++n) s += 2.0 * cos(2.0 * M_PI * n * d / N);
        s += cos(M_PI * d); /* two half-weight Nyquist terms */
    }
    return s / N;
}

/* interpolation matrix U (fN x N), row-major: U[p][k] = D_N(p/f - k) */
void oracle_interp_matrix(int N, int f, double *U)
{
    for (int p = 0; p < f * N; ++p)
        for (int k = 0; k < N; ++k) {
            if (p % f == 0) { U[(i64)p * N + k] = (p / f == k) ? 1.0 : 0.0; continue; }
            U[(i64)p * N + k] = oracle_dirichlet(N, (double)p / f - k);
        }
}

/*
 * Band-limited upsampling of a complex N x N tile (interleaved re/im doubles, row stride N)
 * to fN x fN: out = U in U^T.
 */
void oracle_upsample(const double *in, int N, int f, const double *U, double *out,
                     double *tmp /* N * fN complex */)
{
    const int F = f * N;
    /* rows: tmp[e][p] = sum_k in[e][k] U[p][k] */
    for (int e = 0; e < N; ++e)
        for (int p = 0; p < F; ++p) {
            double re = 0.0, im = 0.0;
            const double *u = U + (i64)p * N;
            const double *x = in + 2 * (i64)e * N;
            for (int k = 0; k < N; ++k) { re += u[k] * x[2 * k]; im += u[k] * x[2 * k + 1]; }
            tmp[2 * ((i64)e * F + p)] = re;
            tmp[2 * ((i64)e * F + p) + 1] = im;
        }
    /* columns: out[q][p] = sum_e U[q][e] tmp[e][p] */
    for (int q = 0; q < F; ++q) {
        const double *u = U + (i64)q * N;
        for (int p = 0; p < F; ++p) {
            double re = 0.0, im = 0.0;
            for (int e = 0; e < N; ++e) {
                re += u[e] * tmp[2 * ((i64)e * F + p)];
                im += u[e] * tmp[2 * ((i64)e * F + p) + 1];
            }
            out[2 * ((i64)q * F + p)] = re;
            out[2 * ((i64)q * F + p) + 1] = im;
        }
    }
}

/*
 * Band-limited zoom of a real Cf x Cf surface by z (Cf odd: no Nyquist bin), real part
 * (or magnitude when use_abs, as c2r.cu:130 does): Z = U G U^T with U = interp(Cf, z).
 */
void oracle_zoom(const double *G, int Cf, int z, const double *U, int use_abs, double *Zm,
                 double *tmp /* Cf * z*Cf */)
{
    const int Z = z * Cf;
    for (int a = 0; a < Cf; ++a)
        for (int q = 0; q < Z; ++q) {
            double s = 0.0;
            const double *u = U + (i64)q * Cf;
            for (int l = 0; l < Cf; ++l) s += G[(i64)a * Cf + l] * u[l];
            tmp[(i64)a * Z + q] = s;
        }
    for (int p = 0; p < Z; ++p) {
        const double *u = U + (i64)p * Cf;
        for (int q = 0; q < Z; ++q) {
            double s = 0.0;
            for (int a = 0; a < Cf; ++a) s += u[a] * tmp[(i64)a * Z + q];
            Zm[(i64)p * Z + q] = use_abs ? fabs(s) : s;
        }
    }
}

/* ------------------------------------------------------------------------------------- */
/* the reference CPU coarse correlator                                                    */
/* ------------------------------------------------------------------------------------- */

/*
 * Sequential.cc:17-97 for every pair: amplitudes (float |z| as double), rVar = sum a_r^2 of
 * the raw chip, per anchor tAvg = SAT box / R^2, num = sum a_r (t - tAvg),
 * tVar = sum (t - tAvg)^2, cor = num / sqrt(rVar * tVar).
 * cor (P x C^2, may be NULL), argmax (2P: row, col), gap (P, may be NULL): top-2 gap.
 *
 * as_built selects where tAvg comes from.  0: the window's own box mean (the summed-area table
 * of the window amplitudes, the intent, and what the reference's CUDA worker computes:
 * sat.cu:81-149, tgtStats.cu:88-168).  1: the arithmetic of the reference's CPU code as it is
 * written: Sequential.cc:48 builds its table as `sat_type sat(tgt.layout())`, i.e. over a new
 * grid of the window's layout rather than over the window, so with that storage zero every box
 * sum and tAvg are 0 and cor is the uncentred sum a_r t / sqrt(sum a_r^2 sum t^2); the sums then
 * run in the reference's order, one term at a time (no vectorised reduction), so that the values
 * match the compiled reference (oracle/_ref) to the last bit.
 */
void oracle_coarse_cpu(const oracle_src *src, i64 pairs, int R, int W,
                       double *cor, int *argmax, double *gap, int threads, int as_built)
{
    const int C = W - R + 1;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel
    {
        double *ref = (double *)malloc(sizeof(double) * (size_t)R * R);
        double *tgt = (double *)malloc(sizeof(double) * (size_t)W * W);
        double *sat = (double *)malloc(sizeof(double) * (size_t)W * W);
        double *g = (double *)malloc(sizeof(double) * (size_t)C * C);
#pragma omp for schedule(dynamic, 1)
        for (i64 p = 0; p < pairs; ++p) {
            const float *rb = src->ref_base + 2 * src->ref_off[p];
            const float *tb = src->tgt_base + 2 * src->tgt_off[p];
            for (int i = 0; i < R; ++i)
                for (int j = 0; j < R; ++j)
                    ref[(i64)i * R + j] = amp_cpu(rb + 2 * ((i64)i * src->ref_stride + j));
            for (int i = 0; i < W; ++i)
                for (int j = 0; j < W; ++j)
                    tgt[(i64)i * W + j] = amp_cpu(tb + 2 * ((i64)i * src->tgt_stride + j));
            double rVar = 0.0;
            for (i64 k = 0; k < (i64)R * R; ++k) rVar += ref[k] * ref[k];
            oracle_sat(tgt, W, W, sat);
            const double cells = (double)R * R;
            for (int u = 0; u < C; ++u)
                for (int v = 0; v < C; ++v) {
                    double num = 0.0, tVar = 0.0;
                    if (as_built) {
                        for (int i = 0; i < R; ++i)
                            for (int j = 0; j < R; ++j) {
                                const double rv = ref[(i64)i * R + j];
                                const double tv = tgt[(i64)(u + i) * W + v + j];
                                num += rv * tv;
                                tVar += tv * tv;
                            }
                    } else {
                        const double tAvg = oracle_box(sat, W, u, v, u + R, v + R) / cells;
                        for (int i = 0; i < R; ++i)
#pragma omp simd reduction(+ : num, tVar)
                            for (int j = 0; j < R; ++j) {
                                const double rv = ref[(i64)i * R + j];
                                const double tv = tgt[(i64)(u + i) * W + v + j] - tAvg;
                                num += rv * tv;
                                tVar += tv * tv;
                            }
                    }
                    g[(i64)u * C + v] = num / sqrt(rVar * tVar);
                }
            const int k = oracle_argmax_first(g, (i64)C * C);
            argmax[2 * p] = k / C;
            argmax[2 * p + 1] = k % C;
            if (gap) gap[p] = g[k] - second_largest_excluding(g, (i64)C * C, k);
            if (cor) memcpy(cor + p * (i64)C * C, g, sizeof(double) * (size_t)C * C);
        }
        free(ref); free(tgt); free(sat); free(g);
    }
}

/* ------------------------------------------------------------------------------------- */
/* the full pipeline                                                                       */
/* ------------------------------------------------------------------------------------- */

/* The opt-in deramp before refinement, in FP64: phi_s = arg sum z(y, x+1) conj z(y, x),
 * phi_l = arg sum z(y+1, x) conj z(y, x) over the N x N tile (interleaved complex), then
 * z(y, x) *= exp(-i (phi_s x + phi_l y)).  The reference's _deramp (Sequential.icc:1094-1098) is an
 * empty stub that runs after refinement, where a phase ramp cannot change the amplitudes. */
void oracle_deramp(double *t, int N)
{
    double sr = 0.0, si = 0.0, lr = 0.0, li = 0.0;
    for (int y = 0; y < N; ++y)
        for (int x = 0; x < N; ++x) {
            const double zr = t[2 * ((i64)y * N + x)], zi = t[2 * ((i64)y * N + x) + 1];
            if (x + 1 < N) {
                const double wr = t[2 * ((i64)y * N + x + 1)], wi = t[2 * ((i64)y * N + x + 1) + 1];
                sr += wr * zr + wi * zi;
                si += wi * zr - wr * zi;
            }
            if (y + 1 < N) {
                const double wr = t[2 * ((i64)(y + 1) * N + x)], wi = t[2 * ((i64)(y + 1) * N + x) + 1];
                lr += wr * zr + wi * zi;
                li += wi * zr - wr * zi;
            }
        }
    const double ps = atan2(si, sr), pl = atan2(li, lr);
    for (int y = 0; y < N; ++y)
        for (int x = 0; x < N; ++x) {
            const double ph = ps * x + pl * y, c = cos(ph), sn = sin(ph);
            double *z = t + 2 * ((i64)y * N + x);
            const double zr = z[0], zi = z[1];
            z[0] = zr * c + zi * sn;
            z[1] = zi * c - zr * sn;
        }
}

void oracle_adjust(const oracle_src *src, i64 pairs, const oracle_geom *g,
                   float *offsets, oracle_diag *diag, double *coarse_surfaces,
                   double *refined_surfaces, int threads)
{
    const int R = g->R, W = g->W, f = g->f, m = g->m, z = g->z;
    const int M = (W - R) / 2;
    const int C = W - R + 1;
    const int E = R + 2 * m;
    const int Rf = f * R, Wf = f * E, Cf = 2 * f * m + 1, Z = z * Cf;
    const int compat = (g->flags & ORACLE_REF_COMPAT) != 0;
    const int deramp = (g->flags & ORACLE_DERAMP) != 0;

    double *Ur = (double *)malloc(sizeof(double) * (size_t)Rf * R);
    double *Ue = (double *)malloc(sizeof(double) * (size_t)Wf * E);
    double *Uz = (double *)malloc(sizeof(double) * (size_t)Z * Cf);
    oracle_interp_matrix(R, f, Ur);
    oracle_interp_matrix(E, f, Ue);
    oracle_interp_matrix(Cf, z, Uz);

#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel
    {
        const size_t big = (size_t)(Wf > W ? Wf : W);
        double *chip = (double *)malloc(sizeof(double) * (size_t)Rf * Rf);
        double *win = (double *)malloc(sizeof(double) * big * big);
        double *scratch = (double *)malloc(sizeof(double) * (big * big + (size_t)Rf * Rf));
        double *gam = (double *)malloc(sizeof(double) * (size_t)C * C);
        double *gf = (double *)malloc(sizeof(double) * (size_t)Cf * Cf);
        double *cin = (double *)malloc(sizeof(double) * 2 * (size_t)E * E);
        double *cout = (double *)malloc(sizeof(double) * 2 * (size_t)Wf * Wf);
        double *ctmp = (double *)malloc(sizeof(double) * 2 * (size_t)E * Wf);
        double *zm = (double *)malloc(sizeof(double) * (size_t)Z * Z);
        double *ztmp = (double *)malloc(sizeof(double) * (size_t)Cf * Z);
#pragma omp for schedule(dynamic, 1)
        for (i64 p = 0; p < pairs; ++p) {
            const float *rb = src->ref_base + 2 * src->ref_off[p];
            const float *tb = src->tgt_base + 2 * src->tgt_off[p];
            /* coarse */
            for (int i = 0; i < R; ++i)
                for (int j = 0; j < R; ++j)
                    chip[(i64)i * R + j] = amp64(rb + 2 * ((i64)i * src->ref_stride + j));
            for (int i = 0; i < W; ++i)
                for (int j = 0; j < W; ++j)
                    win[(i64)i * W + j] = amp64(tb + 2 * ((i64)i * src->tgt_stride + j));
            oracle_ncc(chip, R, win, W, gam, scratch);
            const int kc = oracle_argmax_first(gam, (i64)C * C);
            const int cu = kc / C, cv = kc % C;
            int top, left;
            oracle_nudge(cu, cv, R, W, m, &top, &left);
            if (coarse_surfaces) memcpy(coarse_surfaces + p * (i64)C * C, gam, sizeof(double) * (size_t)C * C);

            /* refine the complex chip */
            for (int i = 0; i < R; ++i)
                for (int j = 0; j < R; ++j) {
                    const float *px = rb + 2 * ((i64)i * src->ref_stride + j);
                    cin[2 * ((i64)i * R + j)] = px[0];
                    cin[2 * ((i64)i * R + j) + 1] = px[1];
                }
            if (deramp) oracle_deramp(cin, R);
            oracle_upsample(cin, R, f, Ur, cout, ctmp);
            for (i64 k = 0; k < (i64)Rf * Rf; ++k)
                chip[k] = sqrt(cout[2 * k] * cout[2 * k] + cout[2 * k + 1] * cout[2 * k + 1]);
            /* refine the neighbourhood of the coarse peak */
            for (int i = 0; i < E; ++i)
                for (int j = 0; j < E; ++j) {
                    const float *px = tb + 2 * ((i64)(top + i) * src->tgt_stride + left + j);
                    cin[2 * ((i64)i * E + j)] = px[0];
                    cin[2 * ((i64)i * E + j) + 1] = px[1];
                }
            if (deramp) oracle_deramp(cin, E);
            oracle_upsample(cin, E, f, Ue, cout, ctmp);
            for (i64 k = 0; k < (i64)Wf * Wf; ++k)
                win[k] = sqrt(cout[2 * k] * cout[2 * k] + cout[2 * k + 1] * cout[2 * k + 1]);
            oracle_ncc(chip, Rf, win, Wf, gf, scratch);
            const int kr = oracle_argmax_first(gf, (i64)Cf * Cf);
            if (refined_surfaces) memcpy(refined_surfaces + p * (i64)Cf * Cf, gf, sizeof(double) * (size_t)Cf * Cf);

            /* zoom */
            oracle_zoom(gf, Cf, z, Uz, compat, zm, ztmp);
            const int kz = oracle_argmax_first(zm, (i64)Z * Z);
            const int fp = kz / Z, fq = kz % Z;

            /* offsets: (top - M) + p/(f z); the reference subtracts the refine margin again */
            const double zoom = (double)f * z;
            double dy = (double)(top - M) + fp / zoom;
            double dx = (double)(left - M) + fq / zoom;
            if (compat) { dy -= m; dx -= m; }
            offsets[2 * p] = (float)dy;
            offsets[2 * p + 1] = (float)dx;

            if (diag) {
                oracle_diag *d = diag + p;
                d->coarse_u = cu; d->coarse_v = cv;
                d->top = top; d->left = left;
                d->fine_p = fp; d->fine_q = fq;
                d->refined_u = kr / Cf; d->refined_v = kr % Cf;
                d->coarse_peak = gam[kc];
                d->coarse_gap = gam[kc] - second_largest_excluding(gam, (i64)C * C, kc);
                d->refined_peak = gf[kr];
                d->zoom_peak = zm[kz];
                d->zoom_gap = zm[kz] - second_largest_excluding(zm, (i64)Z * Z, kz);
            }
        }
        free(chip); free(win); free(scratch); free(gam); free(gf);
        free(cin); free(cout); free(ctmp); free(zm); free(ztmp);
    }
    free(Ur); free(Ue); free(Uz);
}

/* raw cross-correlation sum_ij chip(i,j) win(u+i, v+j) over every placement (the numerator of
   the stand-alone prototype tests/cuda/tile-correlate.cu:409-486, no mean removal) */
void oracle_xcorr(const double *chip, int R, const double *win, int W, double *out)
{
    const int C = W - R + 1;
    for (int u = 0; u < C; ++u)
        for (int v = 0; v < C; ++v) {
            double s = 0.0;
            for (int i = 0; i < R; ++i)
                for (int j = 0; j < R; ++j) s += chip[(i64)i * R + j] * win[(i64)(u + i) * W + v + j];
            out[(i64)u * C + v] = s;
        }
}
