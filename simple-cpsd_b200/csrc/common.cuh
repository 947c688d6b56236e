// common.cuh -- complex arithmetic, compile-time twiddles, register DFTs and
// the two-level line FFT used by every transform kernel (sm_100a).
//
// A line of length N = P*Q (P | Q) is transformed by a group of P adjacent
// lanes of one warp.  Lane t starts with x[t + P*m] (m < Q) in registers,
// does a Q-point DFT in registers, multiplies by W_N^{t q}, exchanges through
// a group-private shared buffer and finishes with Q/P P-point DFTs; it ends
// holding X[(t*U + u) + Q*s] (U = Q/P, u < U, s < P) in v[u*P + s].  Sign
// +1 is FFTPACK's backward transform (e^{+i}), -1 its forward (e^{-i});
// both are unnormalised, as in fftpack/dcfftb.f and dcfftf.f.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

#define CPSD_HD __host__ __device__ __forceinline__
#define CPSD_D __device__ __forceinline__

template <typename T>
struct cx {
    T x, y;
};

template <typename T> CPSD_HD cx<T> mk(T a, T b) { return cx<T>{a, b}; }
template <typename T> CPSD_HD cx<T> operator+(cx<T> a, cx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T> CPSD_HD cx<T> operator-(cx<T> a, cx<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T> CPSD_HD cx<T> operator*(T s, cx<T> a) { return {s * a.x, s * a.y}; }
template <typename T> CPSD_HD cx<T> cmul(cx<T> a, cx<T> b)
{
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T> CPSD_HD cx<T> conj(cx<T> a) { return {a.x, -a.y}; }
// multiply by i*S (S = +1 or -1)
template <int S, typename T> CPSD_HD cx<T> mul_is(cx<T> a)
{
    return S > 0 ? cx<T>{-a.y, a.x} : cx<T>{a.y, -a.x};
}

// ---------------------------------------------------------------------------
// compile-time cos/sin of 2*pi*k/n: exact integer reduction to the nearest
// quarter turn, then Taylor series on |d| <= pi/4.
namespace ctw {
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double taylor_cos(double d)
{
    double term = 1.0, sum = 1.0, d2 = d * d;
    for (int k = 1; k < 14; ++k) {
        term *= -d2 / ((2.0 * k - 1.0) * (2.0 * k));
        sum += term;
    }
    return sum;
}
constexpr double taylor_sin(double d)
{
    double term = d, sum = d, d2 = d * d;
    for (int k = 1; k < 14; ++k) {
        term *= -d2 / ((2.0 * k) * (2.0 * k + 1.0));
        sum += term;
    }
    return sum;
}
// cos(2 pi k / n) and sin(2 pi k / n)
constexpr double cos_turn(long k, long n)
{
    long m = ((k % n) + n) % n;
    long q = (4 * m + n / 2) / n;           // nearest quarter turn
    long num = 4 * m - q * n;               // d = 2 pi num / (4 n)
    double d = 2.0 * kPi * (double)num / (4.0 * (double)n);
    double c = taylor_cos(d), s = taylor_sin(d);
    switch (q & 3) {
    case 0: return c;
    case 1: return -s;
    case 2: return -c;
    default: return s;
    }
}
constexpr double sin_turn(long k, long n)
{
    long m = ((k % n) + n) % n;
    long q = (4 * m + n / 2) / n;
    long num = 4 * m - q * n;
    double d = 2.0 * kPi * (double)num / (4.0 * (double)n);
    double c = taylor_cos(d), s = taylor_sin(d);
    switch (q & 3) {
    case 0: return s;
    case 1: return c;
    case 2: return -s;
    default: return -c;
    }
}
}  // namespace ctw

// W_N^{K} with the transform's sign: exp(SIGN * 2 pi i K / N), as constants.
template <int N, int SIGN, int K>
struct Tw {
    static constexpr double c = ctw::cos_turn(K, N);
    static constexpr double s = SIGN * ctw::sin_turn(K, N);
};

template <int N, int SIGN, int K, typename T>
CPSD_D cx<T> twmul(cx<T> a)
{
    if constexpr (K % N == 0) {
        return a;
    } else if constexpr ((4 * K) % N == 0) {
        // multiples of a quarter turn: exact
        constexpr int q = ((4 * K) / N) & 3;
        if constexpr (q == 1) return mul_is<SIGN>(a);
        else if constexpr (q == 2) return cx<T>{-a.x, -a.y};
        else return mul_is<-SIGN>(a);
    } else {
        const T c = (T)Tw<N, SIGN, K>::c, s = (T)Tw<N, SIGN, K>::s;
        return cx<T>{a.x * c - a.y * s, a.x * s + a.y * c};
    }
}

// static_for<B, E>(f): f(std::integral_constant<int, i>) for i in [B, E)
template <int B, int E>
struct SFor {
    template <typename F>
    CPSD_D static void run(F &&f)
    {
        if constexpr (B < E) {
            f(std::integral_constant<int, B>{});
            SFor<B + 1, E>::run(f);
        }
    }
};

// ---------------------------------------------------------------------------
// In-register DFT of size N on v[0..N): v[k] <- sum_j v[j] W_N^{jk} (sign SIGN)
template <int N, int SIGN, typename T>
struct DFT;

template <int SIGN, typename T>
struct DFT<1, SIGN, T> {
    CPSD_D static void run(cx<T> *) {}
};
template <int SIGN, typename T>
struct DFT<2, SIGN, T> {
    CPSD_D static void run(cx<T> *v)
    {
        cx<T> a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    }
};
template <int SIGN, typename T>
struct DFT<3, SIGN, T> {
    CPSD_D static void run(cx<T> *v)
    {
        // W_3 = -1/2 + i SIGN sqrt(3)/2
        const T h = (T)0.5, r3 = (T)0.86602540378443864676;
        cx<T> a = v[0], b = v[1], c = v[2];
        cx<T> t1 = b + c;
        cx<T> t2 = a - h * t1;
        cx<T> d = b - c;
        cx<T> t3 = mul_is<SIGN>(r3 * d);
        v[0] = a + t1;
        v[1] = t2 + t3;
        v[2] = t2 - t3;
    }
};
template <int SIGN, typename T>
struct DFT<4, SIGN, T> {
    CPSD_D static void run(cx<T> *v)
    {
        cx<T> a = v[0], b = v[1], c = v[2], d = v[3];
        cx<T> s0 = a + c, s1 = a - c, s2 = b + d, s3 = mul_is<SIGN>(b - d);
        v[0] = s0 + s2;
        v[1] = s1 + s3;
        v[2] = s0 - s2;
        v[3] = s1 - s3;
    }
};
// composite: decimation in time with radix R (4 if possible, else 2, else 3)
template <int N, int SIGN, typename T>
struct DFT {
    static constexpr int R = (N % 4 == 0) ? 4 : ((N % 2 == 0) ? 2 : 3);
    static constexpr int M = N / R;
    static_assert(M * R == N && M > 1, "unsupported DFT size");
    CPSD_D static void run(cx<T> *v)
    {
        cx<T> sub[R][M];
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int m = 0; m < M; ++m) sub[r][m] = v[r + R * m];
#pragma unroll
        for (int r = 0; r < R; ++r) DFT<M, SIGN, T>::run(sub[r]);
        SFor<0, M>::run([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            cx<T> t[R];
            SFor<0, R>::run([&](auto rc) {
                constexpr int r = decltype(rc)::value;
                t[r] = twmul<N, SIGN, r * k>(sub[r][k]);
            });
            DFT<R, SIGN, T>::run(t);
#pragma unroll
            for (int q = 0; q < R; ++q) v[k + M * q] = t[q];
        });
    }
};

// ---------------------------------------------------------------------------
// line shapes: N = P*Q with P | Q, P lanes per line
template <int N>
struct LineShape;
template <> struct LineShape<8> { static constexpr int P = 2; };
template <> struct LineShape<12> { static constexpr int P = 2; };
template <> struct LineShape<16> { static constexpr int P = 4; };
template <> struct LineShape<24> { static constexpr int P = 2; };
template <> struct LineShape<32> { static constexpr int P = 4; };
template <> struct LineShape<48> { static constexpr int P = 4; };
template <> struct LineShape<64> { static constexpr int P = 8; };
template <> struct LineShape<128> { static constexpr int P = 8; };

template <int N>
struct Line {
    static constexpr int P = LineShape<N>::P;
    static constexpr int Q = N / P;
    static constexpr int U = Q / P;
    static_assert(P * Q == N && U * P == Q, "line shape");
    // exchange buffer: N complex plus one pad slot per U consecutive q
    static constexpr int XB = N + P;
    CPSD_HD static int xb_index(int q, int s) { return q * P + s + q / U; }
    // index held by lane t in output register u*P + s
    CPSD_HD static int out_index(int t, int u, int s) { return (t * U + u) + Q * s; }
    // index lane t must load into input register m
    CPSD_HD static int in_index(int t, int m) { return t + P * m; }
};

// Two-level transform of one line by P lanes (see file header).
// tw: the twiddles in the order the lanes read them, tw[q*P + t] = W_N^{t q}
// (q < Q, t < P) for this SIGN, so the P lanes of a group read P consecutive
// entries for every q (no shared-memory bank conflicts).  xb: the group's
// exchange buffer (Line<N>::XB entries).  All lanes of the warp must call it
// together.
template <int N, int SIGN, typename T>
CPSD_D void line_fft(cx<T> *v, int t, cx<T> *xb, const cx<T> *__restrict__ tw)
{
    using L = Line<N>;
    constexpr int P = L::P, Q = L::Q, U = L::U;
    DFT<Q, SIGN, T>::run(v);
#pragma unroll
    for (int q = 1; q < Q; ++q) v[q] = cmul(v[q], tw[q * P + t]);
#pragma unroll
    for (int q = 0; q < Q; ++q) xb[L::xb_index(q, t)] = v[q];
    __syncwarp();
#pragma unroll
    for (int u = 0; u < U; ++u) {
        cx<T> w[P];
        const int q = t * U + u;
#pragma unroll
        for (int s = 0; s < P; ++s) w[s] = xb[L::xb_index(q, s)];
        DFT<P, SIGN, T>::run(w);
#pragma unroll
        for (int s = 0; s < P; ++s) v[u * P + s] = w[s];
    }
    __syncwarp();
}

// The transposed algorithm (decimation in frequency): lane t starts with
// x[(t*U + u) + Q*s] in v[u*P + s] -- the output distribution of line_fft --
// and ends with X[t + P*m] in v[m], its input distribution.  P-point DFTs,
// twiddle W_N^{q t'}, one exchange, then the Q-point DFT in registers.
// tw: tw[t'*Q + q] = W_N^{q t'} (t' < P, q < Q) for this SIGN.
template <int N, int SIGN, typename T>
CPSD_D void line_fft_dif(cx<T> *v, int t, cx<T> *xb, const cx<T> *__restrict__ tw)
{
    using L = Line<N>;
    constexpr int P = L::P, Q = L::Q, U = L::U;
#pragma unroll
    for (int u = 0; u < U; ++u) {
        cx<T> w[P];
#pragma unroll
        for (int s = 0; s < P; ++s) w[s] = v[u * P + s];
        DFT<P, SIGN, T>::run(w);
        const int q = t * U + u;
#pragma unroll
        for (int tp = 0; tp < P; ++tp) xb[L::xb_index(q, tp)] = (tp == 0) ? w[0] : cmul(w[tp], tw[tp * Q + q]);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < Q; ++q) v[q] = xb[L::xb_index(q, t)];
    __syncwarp();
    DFT<Q, SIGN, T>::run(v);
}

// ---------------------------------------------------------------------------
// shared-memory padding: a 128-byte wavefront holds kSlots<T> complex values;
// lanes of one access phase must hit distinct slots.
template <typename T>
constexpr int kSlots = 128 / (int)sizeof(cx<T>);

// smallest v >= base with v = want (mod m)
constexpr int pad_to(int base, int m, int want)
{
    return base + (((want - base) % m) + m) % m;
}

// stride between the exchange buffers of consecutive line groups of P lanes:
// the groups sharing an access phase then start on different slots
template <typename T, int N>
constexpr int group_stride()
{
    return (Line<N>::P >= kSlots<T>) ? Line<N>::XB : pad_to(Line<N>::XB, kSlots<T>, Line<N>::P);
}

// ---------------------------------------------------------------------------
// error flags written by kernels (host reads them after a step)
enum : int {
    CPSD_DEVFLAG_BAD_INDEX = 1,
};
