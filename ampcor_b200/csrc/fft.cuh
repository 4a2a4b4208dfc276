// Shared-memory FFTs of the spectral correlation form (host + device templates).
//
// A length-N transform (N = N1 * N2, both at most 16 and built from the radices 2, 3, 4, 5) runs
// as two in-place steps over a row or column of a 2-D tile:
//
//   n = N2 n1 + n2,  k = k1 + N1 k2
//   step A (one task per n2): y[k1] = DFT_N1(x[N2 n1 + n2])[k1] * W_N^(n2 k1), stored where
//                             x[N2 k1 + n2] was
//   step B (one task per k1): X[k1 + N1 k2] = DFT_N2(y[N2 k1 + n2])[k2], stored at N2 k1 + k2
//
// so the spectrum sits in a fixed permutation of the frequencies (position N2 k1 + k2 holds
// frequency k1 + N1 k2) and the inverse runs the two steps backwards from that permutation to
// natural order.  Neither step needs a scratch buffer: a task reads and writes the same positions.
// The short DFTs run in registers (mixed-radix Cooley-Tukey over compile-time indices); their
// twiddles come from a compile-time table of cos / sin (2 pi m / 240), evaluated from Taylor
// series after an exact reduction of m to the first octant.
#pragma once

#include <cuda_runtime.h>

#ifndef HD
#define HD __host__ __device__ __forceinline__
#endif

namespace ampcor_b200 {
namespace fft {

// ---- compile-time cos / sin of 2 pi m / 240 -------------------------------------------------

constexpr double kPi = 3.14159265358979323846264338327950288;

constexpr double taylor_cos(double x)
{
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 14; ++k) {
        term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
        sum += term;
    }
    return sum;
}

constexpr double taylor_sin(double x)
{
    double term = x, sum = x;
    for (int k = 1; k < 14; ++k) {
        term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
        sum += term;
    }
    return sum;
}

struct Tw240 {
    float c[240];
    float s[240];
};

// angle 2 pi q / 240: quadrant q / 60, remainder r; r <= 30 is within pi/4 of the quadrant start,
// larger r is within pi/4 of its end
constexpr Tw240 make_tw240()
{
    Tw240 t{};
    for (int q = 0; q < 240; ++q) {
        const int quad = q / 60, r = q % 60;
        double c = 0.0, s = 0.0;
        if (r <= 30) {
            const double phi = kPi * r / 120.0;
            c = taylor_cos(phi);
            s = taylor_sin(phi);
        } else {
            const double phi = kPi * (60 - r) / 120.0;
            c = taylor_sin(phi);
            s = taylor_cos(phi);
        }
        double cc = c, ss = s;
        if (quad == 1) {
            cc = -s;
            ss = c;
        } else if (quad == 2) {
            cc = -c;
            ss = -s;
        } else if (quad == 3) {
            cc = s;
            ss = -c;
        }
        t.c[q] = (float)cc;
        t.s[q] = (float)ss;
    }
    return t;
}

__constant__ Tw240 kTw240Dev = make_tw240();
constexpr Tw240 kTw240Host = make_tw240();

HD float tw_cos(int i)
{
#ifdef __CUDA_ARCH__
    return kTw240Dev.c[i];
#else
    return kTw240Host.c[i];
#endif
}

HD float tw_sin(int i)
{
#ifdef __CUDA_ARCH__
    return kTw240Dev.s[i];
#else
    return kTw240Host.s[i];
#endif
}

// ---- complex helpers ----------------------------------------------------------------------

HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
HD float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// a * conj(b)
HD float2 cmulc(float2 a, float2 b) { return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }
// a * (s i), s = +-1
template <int S>
HD float2 mul_si(float2 a) { return S > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x); }

// v * exp(S 2 pi i m / N) for a compile-time N (240 % N == 0) and a constant-after-unrolling m
template <int N, int S>
HD float2 twiddle(float2 v, int m)
{
    static_assert(240 % N == 0, "register DFT length must divide 240");
    m %= N;
    if (m == 0) return v;
    if ((4 * m) % N == 0) {
        const int j = (4 * m) / N;
        if (j == 1) return mul_si<S>(v);
        if (j == 2) return make_float2(-v.x, -v.y);
        return mul_si<-S>(v);
    }
    const int i = m * (240 / N);
    const float c = tw_cos(i), s = S > 0 ? tw_sin(i) : -tw_sin(i);
    return make_float2(v.x * c - v.y * s, v.x * s + v.y * c);
}

// ---- register DFTs (natural order in and out; S = -1 forward, +1 inverse, unnormalised) --------

template <int N, int S>
struct Dft;

template <int S>
struct Dft<1, S> {
    HD static void run(float2 (&)[1]) {}
};

template <int S>
struct Dft<2, S> {
    HD static void run(float2 (&a)[2])
    {
        const float2 t = a[0];
        a[0] = cadd(t, a[1]);
        a[1] = csub(t, a[1]);
    }
};

template <int S>
struct Dft<3, S> {
    HD static void run(float2 (&a)[3])
    {
        // X1,2 = a0 - (a1 + a2) / 2 +- S i sin(2 pi / 3) (a1 - a2)
        const float h = 0.866025403784438646763723170752936183f;
        const float2 t = cadd(a[1], a[2]);
        const float2 d = csub(a[1], a[2]);
        const float2 m = make_float2(a[0].x - 0.5f * t.x, a[0].y - 0.5f * t.y);
        const float2 r = mul_si<S>(make_float2(h * d.x, h * d.y));
        a[0] = cadd(a[0], t);
        a[1] = cadd(m, r);
        a[2] = csub(m, r);
    }
};

template <int S>
struct Dft<4, S> {
    HD static void run(float2 (&a)[4])
    {
        const float2 s02 = cadd(a[0], a[2]), d02 = csub(a[0], a[2]);
        const float2 s13 = cadd(a[1], a[3]), d13 = mul_si<S>(csub(a[1], a[3]));
        a[0] = cadd(s02, s13);
        a[2] = csub(s02, s13);
        a[1] = cadd(d02, d13);
        a[3] = csub(d02, d13);
    }
};

template <int S>
struct Dft<5, S> {
    HD static void run(float2 (&a)[5])
    {
        // X_k = a0 + sum_{n=1,2} [cos(2 pi n k / 5) (a_n + a_{5-n}) + S i sin(2 pi n k / 5) (a_n - a_{5-n})]
        const float c1 = 0.309016994374947424102293417182819059f;   // cos(2 pi / 5)
        const float c2 = -0.809016994374947424102293417182819059f;  // cos(4 pi / 5)
        const float s1 = 0.951056516295153572116439333379382143f;   // sin(2 pi / 5)
        const float s2 = 0.587785252292473129168705954639072769f;   // sin(4 pi / 5)
        const float2 p1 = cadd(a[1], a[4]), m1 = csub(a[1], a[4]);
        const float2 p2 = cadd(a[2], a[3]), m2 = csub(a[2], a[3]);
        const float2 a0 = a[0];
        const float2 r1 = make_float2(a0.x + c1 * p1.x + c2 * p2.x, a0.y + c1 * p1.y + c2 * p2.y);
        const float2 r2 = make_float2(a0.x + c2 * p1.x + c1 * p2.x, a0.y + c2 * p1.y + c1 * p2.y);
        // sin(2 pi 2 k / 5) for k = 2 is sin(8 pi / 5) = -sin(2 pi / 5)
        const float2 i1 = mul_si<S>(make_float2(s1 * m1.x + s2 * m2.x, s1 * m1.y + s2 * m2.y));
        const float2 i2 = mul_si<S>(make_float2(s2 * m1.x - s1 * m2.x, s2 * m1.y - s1 * m2.y));
        a[0] = cadd(a0, cadd(p1, p2));
        a[1] = cadd(r1, i1);
        a[4] = csub(r1, i1);
        a[2] = cadd(r2, i2);
        a[3] = csub(r2, i2);
    }
};

// composite N = P Q: n = n1 + P n2, k = Q k1 + k2
template <int N, int S>
struct Dft {
    static constexpr int P = (N % 4 == 0) ? 4 : (N % 2 == 0) ? 2 : (N % 3 == 0) ? 3 : 5;
    static constexpr int Q = N / P;
    static_assert(P * Q == N && Q > 1, "unsupported register DFT length");
    HD static void run(float2 (&a)[N])
    {
        float2 y[P][Q];
#pragma unroll
        for (int n1 = 0; n1 < P; ++n1)
#pragma unroll
            for (int n2 = 0; n2 < Q; ++n2) y[n1][n2] = a[n1 + P * n2];
#pragma unroll
        for (int n1 = 0; n1 < P; ++n1) Dft<Q, S>::run(y[n1]);
#pragma unroll
        for (int n1 = 1; n1 < P; ++n1)
#pragma unroll
            for (int k2 = 1; k2 < Q; ++k2) y[n1][k2] = twiddle<N, S>(y[n1][k2], n1 * k2);
#pragma unroll
        for (int k2 = 0; k2 < Q; ++k2) {
            float2 t[P];
#pragma unroll
            for (int n1 = 0; n1 < P; ++n1) t[n1] = y[n1][k2];
            Dft<P, S>::run(t);
#pragma unroll
            for (int k1 = 0; k1 < P; ++k1) a[Q * k1 + k2] = t[k1];
        }
    }
};

// ---- the two in-place steps of a length N1 N2 transform ----------------------------------
// base: element 0 of the row or column; es: element stride (1 along a row, the row stride down a
// column); tw[m] = exp(-2 pi i m / N) for m < N.

template <int N1, int N2>
HD void fwd_a(float2* base, int es, int n2, const float2* tw)
{
    float2 a[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) a[n1] = base[(N2 * n1 + n2) * es];
    Dft<N1, -1>::run(a);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) a[k1] = cmul(a[k1], tw[n2 * k1]);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) base[(N2 * k1 + n2) * es] = a[k1];
}

// fwd_a with a constant m taken off every input on the way in
template <int N1, int N2>
HD void fwd_a_minus(float2* base, int es, int n2, const float2* tw, float2 m)
{
    float2 a[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
        const float2 v = base[(N2 * n1 + n2) * es];
        a[n1] = make_float2(v.x - m.x, v.y - m.y);
    }
    Dft<N1, -1>::run(a);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) a[k1] = cmul(a[k1], tw[n2 * k1]);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) base[(N2 * k1 + n2) * es] = a[k1];
}

// Centring applied on the way in (the first pass over the rows): element n of row y gets sx
// taken off its real part when y < wx and n < wx, and (ci_hi, then ci_lo) off its imaginary part
// when y < ci and n < ci.  A zero shift leaves the tile as it is.
struct Centre {
    float sx;
    int wx;
    float ci_hi = 0.0f, ci_lo = 0.0f;
    int ci = 0;
};

template <int N1, int N2>
HD void fwd_a_centred(float2* row, int y, int n2, const float2* tw, const Centre& c)
{
    const int lim = y < c.wx ? c.wx : 0;
    const int ilim = y < c.ci ? c.ci : 0;
    float2 a[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
        const int n = N2 * n1 + n2;
        float2 v = row[n];
        if (n < lim) v.x -= c.sx;
        if (n < ilim) v.y = (v.y - c.ci_hi) - c.ci_lo;
        a[n1] = v;
    }
    Dft<N1, -1>::run(a);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) a[k1] = cmul(a[k1], tw[n2 * k1]);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) row[N2 * k1 + n2] = a[k1];
}

template <int N1, int N2, int S>
HD void step_b(float2* base, int es, int k1)
{
    float2 a[N2];
#pragma unroll
    for (int j = 0; j < N2; ++j) a[j] = base[(N2 * k1 + j) * es];
    Dft<N2, S>::run(a);
#pragma unroll
    for (int j = 0; j < N2; ++j) base[(N2 * k1 + j) * es] = a[j];
}

template <int N1, int N2>
HD void inv_a(float2* base, int es, int n2, const float2* tw)
{
    float2 a[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) a[k1] = base[(N2 * k1 + n2) * es];
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) a[k1] = cmulc(a[k1], tw[n2 * k1]);
    Dft<N1, 1>::run(a);
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) base[(N2 * n1 + n2) * es] = a[n1];
}

// inv_a that writes back only the outputs n < lim (the rows a later step reads)
template <int N1, int N2>
HD void inv_a_lim(float2* base, int es, int n2, const float2* tw, int lim)
{
    float2 a[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) a[k1] = base[(N2 * k1 + n2) * es];
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) a[k1] = cmulc(a[k1], tw[n2 * k1]);
    Dft<N1, 1>::run(a);
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1)
        if (N2 * n1 + n2 < lim) base[(N2 * n1 + n2) * es] = a[n1];
}

// inv_a whose natural-order outputs go to store(n, value) instead of back into the tile
template <int N1, int N2, class Store>
HD void inv_a_store(const float2* base, int es, int n2, const float2* tw, Store store)
{
    float2 a[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) a[k1] = base[(N2 * k1 + n2) * es];
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) a[k1] = cmulc(a[k1], tw[n2 * k1]);
    Dft<N1, 1>::run(a);
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) store(N2 * n1 + n2, a[n1]);
}

// Two tasks of one step at a time, their loads issued before either's arithmetic and their
// stores after it (the tasks of a step touch disjoint elements): twice the independent work per
// thread between two shared-memory round trips.
template <int N1, int N2>
HD void fwd_a_centred2(float2* ra, int ya, int n2a, float2* rb, int yb, int n2b, const float2* tw,
                       const Centre& c)
{
    const int la = ya < c.wx ? c.wx : 0, lb = yb < c.wx ? c.wx : 0;
    const int ia = ya < c.ci ? c.ci : 0, ib = yb < c.ci ? c.ci : 0;
    float2 a[N1], b[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
        a[n1] = ra[N2 * n1 + n2a];
        b[n1] = rb[N2 * n1 + n2b];
    }
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
        const int na = N2 * n1 + n2a, nb = N2 * n1 + n2b;
        if (na < la) a[n1].x -= c.sx;
        if (na < ia) a[n1].y = (a[n1].y - c.ci_hi) - c.ci_lo;
        if (nb < lb) b[n1].x -= c.sx;
        if (nb < ib) b[n1].y = (b[n1].y - c.ci_hi) - c.ci_lo;
    }
    Dft<N1, -1>::run(a);
    Dft<N1, -1>::run(b);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) {
        a[k1] = cmul(a[k1], tw[n2a * k1]);
        b[k1] = cmul(b[k1], tw[n2b * k1]);
    }
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
        ra[N2 * k1 + n2a] = a[k1];
        rb[N2 * k1 + n2b] = b[k1];
    }
}

template <int N1, int N2>
HD void fwd_a2(float2* ba, int n2a, float2* bb, int n2b, int es, const float2* tw)
{
    float2 a[N1], b[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
        a[n1] = ba[(N2 * n1 + n2a) * es];
        b[n1] = bb[(N2 * n1 + n2b) * es];
    }
    Dft<N1, -1>::run(a);
    Dft<N1, -1>::run(b);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) {
        a[k1] = cmul(a[k1], tw[n2a * k1]);
        b[k1] = cmul(b[k1], tw[n2b * k1]);
    }
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
        ba[(N2 * k1 + n2a) * es] = a[k1];
        bb[(N2 * k1 + n2b) * es] = b[k1];
    }
}

template <int N1, int N2, int S>
HD void step_b2(float2* ba, int k1a, float2* bb, int k1b, int es)
{
    float2 a[N2], b[N2];
#pragma unroll
    for (int j = 0; j < N2; ++j) {
        a[j] = ba[(N2 * k1a + j) * es];
        b[j] = bb[(N2 * k1b + j) * es];
    }
    Dft<N2, S>::run(a);
    Dft<N2, S>::run(b);
#pragma unroll
    for (int j = 0; j < N2; ++j) {
        ba[(N2 * k1a + j) * es] = a[j];
        bb[(N2 * k1b + j) * es] = b[j];
    }
}

template <int N1, int N2>
HD void inv_a_lim2(float2* ba, int n2a, float2* bb, int n2b, int es, const float2* tw, int lim)
{
    float2 a[N1], b[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
        a[k1] = ba[(N2 * k1 + n2a) * es];
        b[k1] = bb[(N2 * k1 + n2b) * es];
    }
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) {
        a[k1] = cmulc(a[k1], tw[n2a * k1]);
        b[k1] = cmulc(b[k1], tw[n2b * k1]);
    }
    Dft<N1, 1>::run(a);
    Dft<N1, 1>::run(b);
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
        if (N2 * n1 + n2a < lim) ba[(N2 * n1 + n2a) * es] = a[n1];
        if (N2 * n1 + n2b < lim) bb[(N2 * n1 + n2b) * es] = b[n1];
    }
}

// row_tasks two at a time: f2(ya, ja, yb, jb) for the tasks t and t + nt, f(y, j) for an odd
// last one
template <class F, class F2>
HD void row_tasks2(int rows, int J, int tid, int nt, F f, F2 f2)
{
    const int dj = nt / rows, dy = nt - dj * rows;
    auto step = [&](int& y, int& j) {
        y += dy;
        j += dj;
        if (y >= rows) {
            y -= rows;
            ++j;
        }
    };
    int j = tid / rows, y = tid - j * rows;
    while (j < J) {
        int yb = y, jb = j;
        step(yb, jb);
        if (jb >= J) {
            f(y, j);
            break;
        }
        f2(y, j, yb, jb);
        y = yb;
        j = jb;
        step(y, j);
    }
}

// tasks t = tid, tid + nt, ... below n, two at a time: f2(ta, tb), and f(t) for an odd last one
template <class F, class F2>
HD void tasks2(int n, int tid, int nt, F f, F2 f2)
{
    int t = tid;
    for (; t + nt < n; t += 2 * nt) f2(t, t + nt);
    if (t < n) f(t);
}

// position of frequency k in the permuted spectrum, and the frequency at position p
template <int N1, int N2>
HD int pos_of(int k) { return N2 * (k % N1) + k / N1; }
template <int N1, int N2>
HD int freq_at(int p) { return p / N2 + N1 * (p % N2); }

// One cell pair of the correlation spectrum.  The tile holds Z = FFT2(t + i r) for two real
// tiles t (window) and r (chip); with T = (Z(k) + conj Z(-k)) / 2 and R = (Z(k) - conj Z(-k)) / 2i
// the correlation spectrum is T conj R, Hermitian because the correlation is real.  a = Z(k),
// b = Z(-k); returns 4 T conj R (the factor 4 is folded into the final scale).
HD float2 corr_cell(float2 a, float2 b)
{
    const float2 t = make_float2(a.x + b.x, a.y - b.y);
    const float2 r = make_float2(a.y + b.y, b.x - a.x);
    return cmulc(t, r);
}

// position of -k for the frequency k held at position p (the partner of a cell in the
// correlation spectrum)
template <int N1, int N2>
HD int neg_pos(int p)
{
    constexpr int N = N1 * N2;
    return pos_of<N1, N2>((N - freq_at<N1, N2>(p)) % N);
}

// Zero padding of an N-point spectrum to F points (band-limited upsampling by F / N): the source
// frequency of padded frequency kp and its weight.  The low half keeps its place, the high half
// moves to the top, an even N's Nyquist bin is split in two halves (the Dirichlet kernel's
// cos(pi d) term); w = 0 in the zero gap.
template <int N, int F>
HD int pad_source(int kp, float& w)
{
    w = 1.0f;
    if (kp < (N + 1) / 2) return kp;
    if (kp > F - (N + 1) / 2) return kp - (F - N);
    if ((N & 1) == 0 && (kp == N / 2 || kp == F - N / 2)) {
        w = 0.5f;
        return N / 2;
    }
    w = 0.0f;
    return 0;
}

// The first inverse step (step B) of an F-point transform whose input is an N-point spectrum
// padded to F points (pad_source): the task of k1 gathers its F2 inputs straight from the
// N-point spectrum at src (element stride src_es, in the N-point permutation), weighted, and
// writes the step's outputs to dst (element stride dst_es).  src and dst must not overlap.
template <int N1, int N2, int F1, int F2>
HD void step_b_pad(const float2* src, int src_es, float2* dst, int dst_es, int k1)
{
    constexpr int N = N1 * N2, F = F1 * F2;
    float2 a[F2];
#pragma unroll
    for (int j = 0; j < F2; ++j) {
        float w;
        const int k = pad_source<N, F>(k1 + F1 * j, w);
        const float2 v = src[pos_of<N1, N2>(k) * src_es];
        a[j] = make_float2(w * v.x, w * v.y);
    }
    Dft<F2, 1>::run(a);
#pragma unroll
    for (int j = 0; j < F2; ++j) dst[(F2 * k1 + j) * dst_es] = a[j];
}

// f(y, j) for every y < rows and j < J, spread over nt threads (thread tid first) in the order
// t = j rows + y, so that lanes take consecutive y; the runtime division happens once per pass,
// not once per task
template <class F>
HD void row_tasks(int rows, int J, int tid, int nt, F f)
{
    const int dj = nt / rows, dy = nt - dj * rows;
    int j = tid / rows, y = tid - j * rows;
    while (j < J) {
        f(y, j);
        y += dy;
        j += dj;
        if (y >= rows) {
            y -= rows;
            ++j;
        }
    }
}

// The correlation spectrum is Hermitian (the correlation is real), so the inverse transform needs
// one position of every pair (p, neg_pos(p)).  The half taken is {p : p <= neg_pos(p)}: in the
// permuted order it is the block of positions N2 k1 + k2 with k1 below N1 / 2 (give or take the
// ends), nearly contiguous, so lanes walking it hit distinct banks.  half_positions writes its N/2 + 1
// positions in increasing order (one thread; the device builds the list with a warp ballot).
template <int N1, int N2>
HD constexpr int half_count() { return N1 * N2 / 2 + 1; }

template <int N1, int N2>
HD bool in_half(int p) { return p <= neg_pos<N1, N2>(p); }

template <int N1, int N2>
HD void half_positions(int* out)
{
    int c = 0;
    for (int p = 0; p < N1 * N2; ++p)
        if (in_half<N1, N2>(p)) out[c++] = p;
}

// One task of the pass that joins the columns' forward step B, the correlation spectrum and the
// inverse's step B on the Hermitian half.  The group of column x at positions N2 k1 + k2 holds
// the frequencies whose negatives sit in column xn = neg_pos(x) at positions N2 k1n + k2n, with
// k1n = -k1 mod N1 and k2n = -k2 mod N2 when k1 = 0, N2 - 1 - k2 otherwise (pos_of, freq_at).  The
// task takes both groups through the forward step B, forms the cell pairs in registers, and writes
// the inverse step B of column x back into the group (of both groups when x is its own partner:
// the columns of frequencies 0 and N/2).  Every (column, group) belongs to one task, so the pass
// runs in place without a barrier between its steps.
template <int N1, int N2, bool K0>
HD void spectrum_groups(float2* Z, int RS, int x, int xn, int k1)
{
    const int k1n = K0 ? 0 : N1 - k1;
    const bool self_col = x == xn, self = self_col && k1 == k1n;
    float2 a[N2], b[N2];
#pragma unroll
    for (int j = 0; j < N2; ++j) a[j] = Z[(N2 * k1 + j) * RS + x];
    Dft<N2, -1>::run(a);
    if (self) {
#pragma unroll
        for (int j = 0; j < N2; ++j) b[j] = a[j];
    } else {
#pragma unroll
        for (int j = 0; j < N2; ++j) b[j] = Z[(N2 * k1n + j) * RS + xn];
        Dft<N2, -1>::run(b);
    }
    // s: the spectrum of column x, group k1; b becomes that of the partner group (x's own group
    // k1n when the column is its own partner)
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
        const int k2n = K0 ? (N2 - k2) % N2 : N2 - 1 - k2;
        const float2 c = corr_cell(a[k2], b[k2n]);
        a[k2] = c;
    }
    if (self_col && !self) {
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
            const int k2n = K0 ? (N2 - k2) % N2 : N2 - 1 - k2;
            b[k2n] = make_float2(a[k2].x, -a[k2].y);
        }
        Dft<N2, 1>::run(b);
#pragma unroll
        for (int j = 0; j < N2; ++j) Z[(N2 * k1n + j) * RS + x] = b[j];
    }
    Dft<N2, 1>::run(a);
#pragma unroll
    for (int j = 0; j < N2; ++j) Z[(N2 * k1 + j) * RS + x] = a[j];
}

// ---- the 2-D correlation of one tile pair -------------------------------------------------
//
// Z: an N x N tile (row stride RS, odd, so that lanes walking rows or columns hit distinct banks)
// holding t + i r: the window t in the real parts, the chip r in the imaginary parts, zero
// outside them, centred on the way in as `centre` says.  Rows at and past rows_in are all zero.
// neg[p] = neg_pos(p) for p < N; half: the half_positions list.
// The correlation goes to store(u, v, value) for u < rows_out and v < N: value.x is
// 4 N^2 sum_ij r(i, j) t(u + i, v + j)
// (circular indices, which never wrap for the placements of a window of at most N samples); the
// stores of a row go to rows of the tile no later step reads, so store may write into the tile's
// rows below rows_out.  The tasks of each phase are spread over the nt threads; sync() separates
// the phases (__syncthreads on the device).  cols_done() runs in every thread after the inverse
// column pass, from which point the correlation touches only the tile's first rows_out +
// (rows_out + 1) / 2 rows (rows_out where those do not fit in the tile).
//
// The inverse runs on the Hermitian half: the columns of the half only (N/2 + 1 of N), after which
// every placement row is Hermitian along its row; two such rows A, B go through one transform as
// A + i B (real and imaginary parts of the result), packed into the free rows past rows_out where
// the tile has them, else each row is completed from its partners and transformed alone.
struct NoHook {
    HD void operator()() const {}
};

// PAIR: 2 runs every pass two tasks at a time, 1 only the passes of N1-point steps (fewer
// registers), 0 none
template <int N1, int N2, int PAIR = 0, class Sync, class Store, class Hook = NoHook>
HD void correlate_tile(float2* Z, int RS, int rows_in, int rows_out, const float2* tw,
                       const int* neg, const int* half, const Centre& centre, int tid, int nt,
                       Sync sync, Store store, Hook cols_done = Hook{})
{
    constexpr int N = N1 * N2;
    // forward along rows (centring the tile on the way in): lanes take consecutive rows
    if constexpr (PAIR >= 1)
        row_tasks2(
            rows_in, N2, tid, nt, [&](int y, int n2) { fwd_a_centred<N1, N2>(Z + y * RS, y, n2, tw, centre); },
            [&](int ya, int na, int yb, int nb) {
                fwd_a_centred2<N1, N2>(Z + ya * RS, ya, na, Z + yb * RS, yb, nb, tw, centre);
            });
    else
        row_tasks(rows_in, N2, tid, nt, [&](int y, int n2) { fwd_a_centred<N1, N2>(Z + y * RS, y, n2, tw, centre); });
    sync();
    if constexpr (PAIR >= 2)
        row_tasks2(
            rows_in, N1, tid, nt, [&](int y, int k1) { step_b<N1, N2, -1>(Z + y * RS, 1, k1); },
            [&](int ya, int ka, int yb, int kb) { step_b2<N1, N2, -1>(Z + ya * RS, ka, Z + yb * RS, kb, 1); });
    else
        row_tasks(rows_in, N1, tid, nt, [&](int y, int k1) { step_b<N1, N2, -1>(Z + y * RS, 1, k1); });
    sync();
    // forward along columns: lanes take consecutive columns
    if constexpr (PAIR >= 1)
        tasks2(
            N * N2, tid, nt, [&](int t) { fwd_a<N1, N2>(Z + t % N, RS, t / N, tw); },
            [&](int ta, int tb) { fwd_a2<N1, N2>(Z + ta % N, ta / N, Z + tb % N, tb / N, RS, tw); });
    else
        for (int t = tid; t < N * N2; t += nt) fwd_a<N1, N2>(Z + t % N, RS, t / N, tw);
    sync();
    // the columns' forward step B, the correlation spectrum and the inverse's step B on the
    // columns of the Hermitian half, one task per pair of column groups
    constexpr int NH = half_count<N1, N2>();
    for (int t = tid; t < NH * N1; t += nt) {
        const int c = t % NH, k1 = t / NH;
        const int x = half[c], xn = neg[x];
        if (x == xn && k1 > (N1 - k1) % N1) continue;  // done by the task of the partner group
        if (k1 == 0)
            spectrum_groups<N1, N2, true>(Z, RS, x, xn, k1);
        else
            spectrum_groups<N1, N2, false>(Z, RS, x, xn, k1);
    }
    sync();
    // (only the placement rows are read from here on)
    if constexpr (PAIR >= 1)
        tasks2(
            NH * N2, tid, nt, [&](int t) { inv_a_lim<N1, N2>(Z + half[t % NH], RS, t / NH, tw, rows_out); },
            [&](int ta, int tb) {
                inv_a_lim2<N1, N2>(Z + half[ta % NH], ta / NH, Z + half[tb % NH], tb / NH, RS, tw, rows_out);
            });
    else
        for (int t = tid; t < NH * N2; t += nt) inv_a_lim<N1, N2>(Z + half[t % NH], RS, t / NH, tw, rows_out);
    sync();
    cols_done();
    const int np = (rows_out + 1) / 2;
    if (rows_out + np <= N) {
        // placement rows 2q and 2q + 1 as one row A + i B at tile row rows_out + q; positions off
        // the half take the conjugates of their partners
        for (int t = tid; t < np * N; t += nt) {
            const int q = t / N, x = t - q * N;
            const int sx = in_half<N1, N2>(x) ? x : neg[x];
            const float cj = sx == x ? 1.0f : -1.0f;
            const float2 a = Z[2 * q * RS + sx];
            const float2 b = 2 * q + 1 < rows_out ? Z[(2 * q + 1) * RS + sx] : make_float2(0.0f, 0.0f);
            Z[(rows_out + q) * RS + x] = make_float2(a.x - cj * b.y, cj * a.y + b.x);
        }
        sync();
        float2* P = Z + rows_out * RS;
        row_tasks(np, N1, tid, nt, [&](int y, int k1) { step_b<N1, N2, 1>(P + y * RS, 1, k1); });
        sync();
        // the last step hands its outputs to store(u, v, value) instead of writing them back
        row_tasks(np, N2, tid, nt, [&](int y, int n2) {
            inv_a_store<N1, N2>(P + y * RS, 1, n2, tw, [&](int n, float2 v) {
                store(2 * y, n, make_float2(v.x, 0.0f));
                if (2 * y + 1 < rows_out) store(2 * y + 1, n, make_float2(v.y, 0.0f));
            });
        });
        sync();
    } else {
        // every placement row completed from its partners, then transformed alone
        for (int t = tid; t < rows_out * N; t += nt) {
            const int y = t / N, x = t - y * N;
            if (!in_half<N1, N2>(x)) {
                const float2 v = Z[y * RS + neg[x]];
                Z[y * RS + x] = make_float2(v.x, -v.y);
            }
        }
        sync();
        row_tasks(rows_out, N1, tid, nt, [&](int y, int k1) { step_b<N1, N2, 1>(Z + y * RS, 1, k1); });
        sync();
        row_tasks(rows_out, N2, tid, nt, [&](int y, int n2) {
            inv_a_store<N1, N2>(Z + y * RS, 1, n2, tw, [&](int n, float2 v) { store(y, n, v); });
        });
        sync();
    }
}

}  // namespace fft
}  // namespace ampcor_b200
