// Host run of the spectral form's FFT templates (ampcor_b200/csrc/fft.cuh): every compiled
// transform length against a direct FP64 DFT, the inverse round trip, and the in-place 2-D tile
// correlation against FP64 direct sums.  Exit status 0 when all errors are within bounds.
#include "fft.cuh"
#include <cstdio>
#include <cmath>
#include <vector>
#include <random>
using namespace ampcor_b200::fft;
struct NoSync { __host__ __device__ void operator()() const {} };

template <int N1, int N2>
double check1d(std::mt19937& g)
{
    constexpr int N = N1 * N2;
    std::normal_distribution<double> nd;
    std::vector<float2> x(N), tw(N);
    for (int m = 0; m < N; ++m) tw[m] = make_float2((float)cos(2 * M_PI * m / N), (float)-sin(2 * M_PI * m / N));
    for (auto& v : x) v = make_float2((float)nd(g), (float)nd(g));
    std::vector<float2> y = x;
    for (int n2 = 0; n2 < N2; ++n2) fwd_a<N1, N2>(y.data(), 1, n2, tw.data());
    for (int k1 = 0; k1 < N1; ++k1) step_b<N1, N2, -1>(y.data(), 1, k1);
    double err = 0, mag = 0;
    for (int k = 0; k < N; ++k) {
        double re = 0, im = 0;
        for (int n = 0; n < N; ++n) {
            const double a = -2 * M_PI * (double)n * k / N;
            re += x[n].x * cos(a) - x[n].y * sin(a);
            im += x[n].x * sin(a) + x[n].y * cos(a);
        }
        const float2 v = y[pos_of<N1, N2>(k)];
        err = fmax(err, hypot(v.x - re, v.y - im));
        mag = fmax(mag, hypot(re, im));
    }
    for (int k1 = 0; k1 < N1; ++k1) step_b<N1, N2, 1>(y.data(), 1, k1);
    for (int n2 = 0; n2 < N2; ++n2) inv_a<N1, N2>(y.data(), 1, n2, tw.data());
    double rerr = 0;
    for (int n = 0; n < N; ++n) rerr = fmax(rerr, hypot(y[n].x / N - x[n].x, y[n].y / N - x[n].y));
    printf("N=%3d (%2dx%2d): fwd err/mag %.2e, roundtrip err %.2e\n", N, N1, N2, err / mag, rerr);
    return fmax(err / mag, rerr);
}

template <int N1, int N2>
double check2d(int W, int R, std::mt19937& g, bool centre_in_pass = false)
{
    constexpr int N = N1 * N2;
    const int C = W - R + 1, RS = N + 1;
    std::uniform_real_distribution<double> ud(0.0, 2.0);
    std::vector<float> t(W * W), r(R * R), raw(R * R);
    for (auto& v : t) v = (float)ud(g);
    double mr = 0;
    for (auto& v : raw) { v = (float)ud(g); mr += v; }
    mr /= R * R;
    for (int k = 0; k < R * R; ++k) r[k] = (float)(raw[k] - mr);
    std::vector<float2> Z(N * RS, make_float2(0, 0)), tw(N);
    for (int m = 0; m < N; ++m) tw[m] = make_float2((float)cos(2 * M_PI * m / N), (float)-sin(2 * M_PI * m / N));
    // with centre_in_pass the tile takes the raw chip and the window, and the first transform pass
    // takes both means off
    double mw = 0;
    for (auto v : t) mw += v;
    mw /= (double)W * W;
    for (int y = 0; y < W; ++y) for (int x = 0; x < W; ++x) Z[y * RS + x].x = t[y * W + x];
    // the chip centred as the kernel does it (two float subtractions carrying the FP64 mean)
    const float mhi = (float)mr, mlo = (float)(mr - (double)mhi);
    for (int y = 0; y < R; ++y)
        for (int x = 0; x < R; ++x) Z[y * RS + x].y = centre_in_pass ? (raw[y * R + x] - mhi) - mlo : r[y * R + x];
    Centre ctr{0.0f, 0};
    if (centre_in_pass) ctr = Centre{(float)mw, W};
    std::vector<int> neg(N), half(half_count<N1, N2>());
    for (int q = 0; q < N; ++q) neg[q] = neg_pos<N1, N2>(q);
    half_positions<N1, N2>(half.data());
    std::vector<float> num(C * N);
    correlate_tile<N1, N2>(Z.data(), RS, W, C, tw.data(), neg.data(), half.data(), ctr, 0, 1, NoSync{},
                           [&](int u, int v, float2 val) { num[u * N + v] = val.x; });
    double err = 0, mag = 0;
    for (int u = 0; u < C; ++u) for (int v = 0; v < C; ++v) {
        double s = 0;
        for (int i = 0; i < R; ++i)
            for (int j = 0; j < R; ++j)
                s += (centre_in_pass ? (double)raw[i * R + j] - mr : (double)r[i * R + j]) * t[(u + i) * W + v + j];
        const double f = num[u * N + v] / (4.0 * N * N);
        err = fmax(err, fabs(f - s));
        mag = fmax(mag, fabs(s));
    }
    printf("2-D N=%d W=%d R=%d C=%d%s: max err %.3e, max |num| %.3e\n", N, W, R, C,
           centre_in_pass ? " (centred in the first pass)" : "", err, mag);
    return err / mag;
}

// the refinement sequence of the spectral form (rows: N-point FFT, pad, F-point inverse; then the
// columns), against the direct FP64 Dirichlet interpolation of the same tile
static double dirichlet(int N, double d)
{
    double s = 1.0;
    if (N % 2) {
        for (int n = 1; n <= (N - 1) / 2; ++n) s += 2.0 * cos(2.0 * M_PI * n * d / N);
    } else {
        for (int n = 1; n < N / 2; ++n) s += 2.0 * cos(2.0 * M_PI * n * d / N);
        s += cos(M_PI * d);
    }
    return s / N;
}

template <int N1, int N2, int F1, int F2>
double check_upsample(std::mt19937& g)
{
    constexpr int N = N1 * N2, F = F1 * F2, f = F / N;
    std::normal_distribution<double> nd;
    std::vector<float2> X(N * N), Y(F * N), B(F), Out(F * F), twn(N), twf(F);
    for (int m = 0; m < N; ++m) twn[m] = make_float2((float)cos(2 * M_PI * m / N), (float)-sin(2 * M_PI * m / N));
    for (int m = 0; m < F; ++m) twf[m] = make_float2((float)cos(2 * M_PI * m / F), (float)-sin(2 * M_PI * m / F));
    for (auto& v : X) v = make_float2((float)nd(g), (float)nd(g));
    std::vector<float2> X0 = X;
    // the refinement's order: the 2-D forward transform (rows, then columns), the padded inverse
    // down the N columns (F x N), then the padded inverse along each of the F rows
    for (int y = 0; y < N; ++y) {
        for (int n2 = 0; n2 < N2; ++n2) fwd_a<N1, N2>(X.data() + y * N, 1, n2, twn.data());
        for (int k1 = 0; k1 < N1; ++k1) step_b<N1, N2, -1>(X.data() + y * N, 1, k1);
    }
    for (int x = 0; x < N; ++x) {
        for (int n2 = 0; n2 < N2; ++n2) fwd_a<N1, N2>(X.data() + x, N, n2, twn.data());
        for (int k1 = 0; k1 < N1; ++k1) step_b<N1, N2, -1>(X.data() + x, N, k1);
        for (int k1 = 0; k1 < F1; ++k1) step_b_pad<N1, N2, F1, F2>(X.data() + x, N, Y.data() + x, N, k1);
        for (int n2 = 0; n2 < F2; ++n2) inv_a<F1, F2>(Y.data() + x, N, n2, twf.data());
    }
    for (int y = 0; y < F; ++y) {
        for (int k1 = 0; k1 < F1; ++k1) step_b_pad<N1, N2, F1, F2>(Y.data() + y * N, 1, B.data(), 1, k1);
        for (int n2 = 0; n2 < F2; ++n2)
            inv_a_store<F1, F2>(B.data(), 1, n2, twf.data(), [&](int n, float2 v) { Out[y * F + n] = v; });
    }
    // direct: out = |A X A^T|, A[i][n] = D_N(i / f - n)
    std::vector<double> A(F * N);
    for (int i = 0; i < F; ++i)
        for (int n = 0; n < N; ++n) A[i * N + n] = (i % f == 0) ? (i / f == n ? 1.0 : 0.0) : dirichlet(N, (double)i / f - n);
    double err = 0, mag = 0;
    std::vector<double> Tr(F * N), Ti(F * N);
    for (int i = 0; i < F; ++i)
        for (int n = 0; n < N; ++n) {
            double sr = 0, si = 0;
            for (int m = 0; m < N; ++m) { sr += A[i * N + m] * X0[m * N + n].x; si += A[i * N + m] * X0[m * N + n].y; }
            Tr[i * N + n] = sr; Ti[i * N + n] = si;
        }
    for (int i = 0; i < F; ++i)
        for (int j = 0; j < F; ++j) {
            double sr = 0, si = 0;
            for (int n = 0; n < N; ++n) { sr += Tr[i * N + n] * A[j * N + n]; si += Ti[i * N + n] * A[j * N + n]; }
            const double ref = hypot(sr, si);
            const float2 v = Out[i * F + j];
            const double got = hypot((double)v.x, (double)v.y) / ((double)N * N);
            err = fmax(err, fabs(got - ref));
            mag = fmax(mag, ref);
        }
    printf("upsample %d -> %d: max |amplitude error| %.3e (max amplitude %.3f)\n", N, F, err, mag);
    return err / mag;
}

int main()
{
    std::mt19937 g(1);
    double e = 0;
    e = fmax(e, check1d<4, 4>(g));
    e = fmax(e, check1d<4, 6>(g));
    e = fmax(e, check1d<4, 8>(g));
    e = fmax(e, check1d<5, 8>(g));
    e = fmax(e, check1d<6, 8>(g));
    e = fmax(e, check1d<8, 8>(g));
    e = fmax(e, check1d<8, 10>(g));
    e = fmax(e, check1d<8, 12>(g));
    e = fmax(e, check1d<8, 16>(g));
    e = fmax(e, check1d<10, 16>(g));
    e = fmax(e, check1d<12, 12>(g));
    e = fmax(e, check1d<3, 5>(g));
    e = fmax(e, check1d<16, 15>(g));
    double e2 = 0;
    e2 = fmax(e2, check2d<8, 16>(128, 64, g));
    e2 = fmax(e2, check2d<10, 16>(160, 128, g));
    e2 = fmax(e2, check2d<8, 12>(90, 60, g));
    e2 = fmax(e2, check2d<6, 8>(48, 32, g));
    e2 = fmax(e2, check2d<12, 12>(144, 128, g));
    e2 = fmax(e2, check2d<8, 16>(128, 64, g, true));
    e2 = fmax(e2, check2d<10, 16>(160, 128, g, true));
    e2 = fmax(e2, check2d<8, 12>(90, 60, g, true));
    // odd first and second radices and short lengths
    e2 = fmax(e2, check2d<5, 8>(40, 32, g, true));
    e2 = fmax(e2, check2d<8, 15>(120, 96, g, true));
    e2 = fmax(e2, check2d<4, 6>(24, 16, g, true));
    e2 = fmax(e2, check2d<8, 10>(80, 64, g, true));
    e2 = fmax(e2, check2d<4, 4>(16, 8, g, true));
    e2 = fmax(e2, check2d<4, 8>(32, 20, g, true));
    // an even number of placement rows, and windows whose placement rows leave no room for the
    // packed rows (each row then transformed alone)
    e2 = fmax(e2, check2d<8, 16>(128, 63, g, true));
    e2 = fmax(e2, check2d<10, 16>(160, 32, g, true));
    e2 = fmax(e2, check2d<12, 12>(144, 16, g, true));
    double e3 = 0;
    e3 = fmax(e3, check_upsample<8, 8, 8, 16>(g));
    e3 = fmax(e3, check_upsample<8, 10, 10, 16>(g));
    e3 = fmax(e3, check_upsample<4, 8, 8, 8>(g));
    e3 = fmax(e3, check_upsample<5, 8, 8, 10>(g));
    // lengths of the strip-buffered refinement (chip 128, neighbourhood 144)
    e3 = fmax(e3, check_upsample<8, 16, 16, 16>(g));
    e3 = fmax(e3, check_upsample<12, 12, 12, 24>(g));
    printf("worst 1-D %.2e, worst 2-D (relative to the largest numerator) %.2e, worst upsampling %.2e\n",
           e, e2, e3);
    return (e < 2e-6 && e2 < 5e-6 && e3 < 2e-6) ? 0 : 1;
}
