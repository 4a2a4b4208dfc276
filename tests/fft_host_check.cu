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
double check2d(int W, int R, std::mt19937& g)
{
    constexpr int N = N1 * N2;
    const int C = W - R + 1, RS = N + 1;
    std::uniform_real_distribution<double> ud(0.0, 2.0);
    std::vector<float> t(W * W), r(R * R);
    for (auto& v : t) v = (float)ud(g);
    double mr = 0;
    for (auto& v : r) { v = (float)ud(g); mr += v; }
    mr /= R * R;
    for (auto& v : r) v = (float)(v - mr);
    std::vector<float2> Z(N * RS, make_float2(0, 0)), tw(N);
    for (int m = 0; m < N; ++m) tw[m] = make_float2((float)cos(2 * M_PI * m / N), (float)-sin(2 * M_PI * m / N));
    for (int y = 0; y < W; ++y) for (int x = 0; x < W; ++x) Z[y * RS + x].x = t[y * W + x];
    for (int y = 0; y < R; ++y) for (int x = 0; x < R; ++x) Z[y * RS + x].y = r[y * R + x];
    std::vector<int> neg(N);
    for (int q = 0; q < N; ++q) neg[q] = neg_pos<N1, N2>(q);
    correlate_tile<N1, N2>(Z.data(), RS, W, C, tw.data(), neg.data(), 0, 1, NoSync{});
    double err = 0, mag = 0;
    for (int u = 0; u < C; ++u) for (int v = 0; v < C; ++v) {
        double s = 0;
        for (int i = 0; i < R; ++i) for (int j = 0; j < R; ++j) s += (double)r[i * R + j] * t[(u + i) * W + v + j];
        const double f = Z[u * RS + v].x / (4.0 * N * N);
        err = fmax(err, fabs(f - s));
        mag = fmax(mag, fabs(s));
    }
    printf("2-D N=%d W=%d R=%d C=%d: max err %.3e, max |num| %.3e\n", N, W, R, C, err, mag);
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
    printf("worst 1-D %.2e, worst 2-D (relative to the largest numerator) %.2e\n", e, e2);
    return (e < 2e-6 && e2 < 5e-6) ? 0 : 1;
}
