/*
 * Host-side generator of warped secondary rasters for the synthetic benchmark workloads:
 *   out(y, x) = in(y - dy(y, x), x - dx(y, x))
 * with (dy, dx) a bivariate quadratic in the normalised coordinates Y = (y - H/2)/(H/2),
 * X = (x - W/2)/(W/2), evaluated by a separable Kaiser-windowed sinc of half-width 8 in FP64.
 * Samples outside the raster read as zero.  This is input generation, not part of the
 * correlator.
 */
#include <math.h>
#include <stddef.h>

static double bessel_i0(double x)
{
    double s = 1.0, t = 1.0;
    for (int k = 1; k < 40; ++k) {
        t *= (x / (2.0 * k)) * (x / (2.0 * k));
        s += t;
        if (t < 1e-17 * s) break;
    }
    return s;
}

#define HALF 8
#define BETA 8.0

static void weights(double frac, double *w, double i0b)
{
    /* taps at integer offsets k - HALF + 1 .. k + HALF relative to floor */
    for (int k = 0; k < 2 * HALF; ++k) {
        const double t = (double)(k - HALF + 1) - frac;
        const double a = t / HALF;
        double win = 0.0;
        if (fabs(a) < 1.0) win = bessel_i0(BETA * sqrt(1.0 - a * a)) / i0b;
        const double sinc = (t == 0.0) ? 1.0 : sin(M_PI * t) / (M_PI * t);
        w[k] = sinc * win;
    }
}

void synth_warp(const float *in, float *out, long long H, long long W, const double *cy,
                const double *cx)
{
    const double i0b = bessel_i0(BETA);
#pragma omp parallel for schedule(dynamic, 16)
    for (long long y = 0; y < H; ++y) {
        double wy[2 * HALF], wx[2 * HALF];
        const double Y = (y - H / 2.0) / (H / 2.0);
        for (long long x = 0; x < W; ++x) {
            const double X = (x - W / 2.0) / (W / 2.0);
            const double dy = cy[0] + cy[1] * Y + cy[2] * X + cy[3] * Y * Y + cy[4] * X * Y + cy[5] * X * X;
            const double dx = cx[0] + cx[1] * Y + cx[2] * X + cx[3] * Y * Y + cx[4] * X * Y + cx[5] * X * X;
            const double sy = y - dy, sx = x - dx;
            const double fy = floor(sy), fx = floor(sx);
            weights(sy - fy, wy, i0b);
            weights(sx - fx, wx, i0b);
            double re = 0.0, im = 0.0;
            for (int a = 0; a < 2 * HALF; ++a) {
                const long long r = (long long)fy + a - HALF + 1;
                if (r < 0 || r >= H) continue;
                double rr = 0.0, ri = 0.0;
                const float *row = in + 2 * r * W;
                for (int b = 0; b < 2 * HALF; ++b) {
                    const long long c = (long long)fx + b - HALF + 1;
                    if (c < 0 || c >= W) continue;
                    rr += wx[b] * row[2 * c];
                    ri += wx[b] * row[2 * c + 1];
                }
                re += wy[a] * rr;
                im += wy[a] * ri;
            }
            out[2 * (y * W + x)] = (float)re;
            out[2 * (y * W + x) + 1] = (float)im;
        }
    }
}
