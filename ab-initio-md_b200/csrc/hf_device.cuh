// Device building blocks of the McMurchie-Davidson integrals (sm_100a).
//
// Boys function F_n(x): positive power series (small x) or erf + upward
// recursion (x >= n + 1.5), without tables (Helgaker, Jorgensen & Olsen
// 2000, sec. 9.8; the reference tabulates, aimd/qc/boys.py:88-114). Hermite expansion coefficients E^{ij}_t by the
// Obara-Saika-type recursion of McMurchie & Davidson (aimd/qc/hermite.py:110),
// Hermite Coulomb integrals R_tuv by the level recursion, evaluated in place
// (aimd/qc/hermite.py:145).
//
// Everything is templated on the angular momenta of a quartet class, so the
// work arrays have compile-time sizes and small classes live in registers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hf {

constexpr int LMAX = 2;            // s, p, d: every built-in basis set
constexpr int PPW = 16;            // doubles per primitive-pair record
constexpr double PI = 3.14159265358979323846;
constexpr double TWO_PI_2_5 = 34.98683665524972;   // 2 pi^(5/2)

__host__ __device__ constexpr int nherm(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }
__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
// Contraction cap per block angular momentum: s blocks may carry 2
// contractions (cc-pVDZ first-row atoms), others one. Larger general
// contractions are split into blocks of at most this size on the host.
__host__ __device__ constexpr int ncon_cap(int l) { return l == 0 ? 2 : 1; }
// Linear Hermite index of (t, u, v): by total degree, then t descending,
// then u descending (the reference's ordering, aimd/qc/hermite.py:73-80).
__host__ __device__ constexpr int hidx(int t, int u, int v) {
    return nherm(t + u + v - 1) + (u + v) * (u + v + 1) / 2 + v;
}
// Cartesian component i of angular momentum l in PySCF order.
__host__ __device__ constexpr int cart_x(int l, int i) {
    int n = 0;
    for (int lx = l; lx >= 0; --lx)
        for (int ly = l - lx; ly >= 0; --ly) { if (n == i) return lx; ++n; }
    return 0;
}
__host__ __device__ constexpr int cart_y(int l, int i) {
    int n = 0;
    for (int lx = l; lx >= 0; --lx)
        for (int ly = l - lx; ly >= 0; --ly) { if (n == i) return ly; ++n; }
    return 0;
}
__host__ __device__ constexpr int cart_z(int l, int i) { return l - cart_x(l, i) - cart_y(l, i); }

// pair class index <-> (la, lb), la >= lb
__host__ __device__ constexpr int pcls(int la, int lb) { return la * (la + 1) / 2 + lb; }
__host__ __device__ constexpr int cls_la(int c) { return c == 0 ? 0 : (c < 3 ? 1 : 2); }
__host__ __device__ constexpr int cls_lb(int c) { return c - pcls(cls_la(c), 0); }
constexpr int NCLS = 6;
// Sub-classes: within an angular class, pairs are grouped by their number of
// surviving primitive pairs (buckets 1, 2-3, 4-7, 8-15, 16-31, 32+) and by
// their contraction-combination count (1, 2, 4), so that the lanes of a warp
// walk loops of similar length. Segment id = class * NSUB + sub.
constexpr int NPPB = 6, NCONB = 3, NSUB = NPPB * NCONB, NSEG = NCLS * NSUB;
__host__ __device__ inline int npp_bucket(int npp) {
    int b = 0;
    while (b < NPPB - 1 && npp >= (2 << b)) ++b;
    return b;
}

// Normalisation of Cartesian component (lx, ly, lz) relative to x^l:
// sqrt((2l-1)!! / ((2lx-1)!! (2ly-1)!! (2lz-1)!!)).
__host__ __device__ constexpr double dfact_odd(int n) { double r = 1.0; for (int k = n; k > 1; k -= 2) r *= k; return r; }
__host__ __device__ inline double cart_norm(int lx, int ly, int lz) {
    return sqrt(dfact_odd(2 * (lx + ly + lz) - 1) / (dfact_odd(2 * lx - 1) * dfact_odd(2 * ly - 1) * dfact_odd(2 * lz - 1)));
}

// ---------------------------------------------------------------- accumulation

// Order-independent sums: J, K and the nuclear gradients are accumulated as
// 64-bit fixed-point integers (value * scale, rounded to nearest), so the
// total is the same bits whatever order threads and CTAs add in (integer
// addition is associative, and wraps modulo 2^64, so only each addend and
// the final total need to fit in 63 bits). The float value is restored once
// at the end. Gradients: scale 2^44 (resolution 5.7e-14 Eh/bohr, range
// +-5.2e5). J and K: scale jk_fix_for(max |D|), 2^44 for densities of
// magnitude 1, so that the builds of small difference densities keep the
// relative resolution of a full build.
typedef unsigned long long facc;
constexpr double FIX_G = 17592186044416.0;        // 2^44
__device__ __forceinline__ facc to_fixed(double v, double scale) {
    return static_cast<facc>(__double2ll_rn(v * scale));
}
__device__ __forceinline__ void fadd(facc* p, double v, double scale) { atomicAdd(p, to_fixed(v, scale)); }
__host__ __device__ __forceinline__ double from_fixed(facc u, double scale) {
    return static_cast<double>(static_cast<long long>(u)) / scale;
}
// J/K scale for a density of largest element m in [2^(e-1), 2^e): 2^(45-e)
// (2^44 at m = 1), e clamped to [-60, 30]. J and K are linear in D, so their
// elements stay below 2^18 m (far above any molecular Coulomb or exchange
// element per unit density) and every sum fits; m = 0 or NaN gives e = 0.
__device__ __forceinline__ double jk_fix_for(double m) {
    int e = 0;
    if (m > 0.0 && m <= 1.0e300) frexp(m, &e);
    e = e < -60 ? -60 : (e > 30 ? 30 : e);
    return ldexp(1.0, 45 - e);
}

// ---------------------------------------------------------------- Boys

// Coefficient a_k of the positive series F_N(x) = e^{-x} sum_k a_k (2x)^k,
// a_k = 1 / ((2N+1)(2N+3)...(2N+2k+1)).
__host__ __device__ constexpr double boys_series_coef(int N, int k) {
    double a = 1.0;
    for (int j = 0; j <= k; ++j) a /= (2 * N + 2 * j + 1);
    return a;
}

// F_N(x) without tables (no memory traffic in the integral loops):
//   x <  N + 1.5: the positive series above in Horner form, 22 + 2N terms
//                 (relative truncation < 1e-15 on the whole interval);
//   x >= N + 1.5: F_0 = sqrt(pi/x) erf(sqrt(x)) / 2 and the upward recursion
//                 F_{m+1} = ((2m+1) F_m - e^{-x}) / (2x), stable there
//                 (measured relative error < 1.5e-15 for N <= 10).
// Both are standard evaluations of F_N (Helgaker, Jorgensen & Olsen 2000,
// sec. 9.8); the reference tabulates instead (aimd/qc/boys.py:88-114).
// ex = e^{-x} is passed in by the caller, which needs it anyway.
template <int N>
__device__ __forceinline__ double boys_top(double x, double ex) {
    if (x < N + 1.5) {
        constexpr int NT = 22 + 2 * N;
        const double y = 2.0 * x;
        double s = boys_series_coef(N, NT - 1);
#pragma unroll
        for (int k = NT - 2; k >= 0; --k) s = fma(s, y, boys_series_coef(N, k));
        return ex * s;
    }
    const double sx = sqrt(x);
    // sqrt(pi)/2 erf(sqrt x)/sqrt x; from x = 36 on erf(sqrt x) is 1 in double
    // precision (erfc(6) = 2.2e-17, below half an ulp of 1)
    double f = 0.88622692545275801365 * (x < 36.0 ? erf(sx) : 1.0) / sx;
    if (N > 0) {
        const double inv2x = 0.5 / x;
#pragma unroll
        for (int m = 0; m < N; ++m) f = ((2 * m + 1) * f - ex) * inv2x;
    }
    return f;
}

// FP32 F_N(x) for x < 40 (the mixed-precision quartets): the same series
// with 16 + N terms (relative truncation < 2e-8 at x = N + 1.5), or erf and
// the upward recursion above N + 1.5.
template <int N>
__device__ __forceinline__ float boys_top_f(float x, float ex) {
    if (x < N + 1.5f) {
        constexpr int NT = 16 + N;
        const float y = 2.0f * x;
        float s = static_cast<float>(boys_series_coef(N, NT - 1));
#pragma unroll
        for (int k = NT - 2; k >= 0; --k) s = fmaf(s, y, static_cast<float>(boys_series_coef(N, k)));
        return ex * s;
    }
    const float sx = sqrtf(x);
    float f = 0.886226925f * erff(sx) / sx;
    if (N > 0) {
        const float inv2x = 0.5f / x;
#pragma unroll
        for (int m = 0; m < N; ++m) f = ((2 * m + 1) * f - ex) * inv2x;
    }
    return f;
}

// g[n] = (-2 alpha)^n F_n(T), n = 0..L: the level seeds of hermite_r.
template <int L>
__device__ __forceinline__ void boys_scaled(double alpha, double T, double (&g)[L + 1]) {
    const double ex = exp(-T);
    double f = boys_top<L>(T, ex);
    const double m2a = -2.0 * alpha;
    double pw[L + 1];
    pw[0] = 1.0;
#pragma unroll
    for (int n = 1; n <= L; ++n) pw[n] = pw[n - 1] * m2a;
    g[L] = pw[L] * f;
#pragma unroll
    for (int n = L - 1; n >= 0; --n) {
        f = (2.0 * T * f + ex) * (1.0 / (2 * n + 1));
        g[n] = pw[n] * f;
    }
}
// FP32 quartets: below T = 40 in FP32; from T = 40 on (where F_n(T) alone
// can leave the FP32 range) in FP64, in the asymptotic form
// (-2a)^n F_n = (-a/T)^n (2n-1)!! F_0, F_0 = sqrt(pi/T)/2, e^-T < 5e-18.
template <int L>
__device__ __forceinline__ void boys_scaled(float alpha, float T, float (&g)[L + 1]) {
    if (T >= 40.0f) {
        const double td = T;
        double gn = 0.88622692545275801365 / sqrt(td);
        const double s = -static_cast<double>(alpha) / td;
        g[0] = static_cast<float>(gn);
#pragma unroll
        for (int n = 1; n <= L; ++n) {
            gn *= (2 * n - 1) * s;
            g[n] = static_cast<float>(gn);
        }
        return;
    }
    const float ex = expf(-T);
    float f = boys_top_f<L>(T, ex);
    const float m2a = -2.0f * alpha;
    float pw[L + 1];
    pw[0] = 1.0f;
#pragma unroll
    for (int n = 1; n <= L; ++n) pw[n] = pw[n - 1] * m2a;
    g[L] = pw[L] * f;
#pragma unroll
    for (int n = L - 1; n >= 0; --n) {
        f = (2.0f * T * f + ex) * (1.0f / (2 * n + 1));
        g[n] = pw[n] * f;
    }
}

// scale * R_tuv(alpha, PQ) for all t+u+v <= L, in place: levels n = L..0,
// each level overwriting the previous one in decreasing Hermite index
// (entries h only read lower indices of the level above). R[0] of level n
// is scale (-2a)^n F_n; the recursion is linear in these seeds. R is a
// register array or a pointer (shared memory) with NH(L) entries.
// RT = double (plain path) or float (mixed-precision quartets).
template <int L, typename RT, typename Arr>
__device__ __forceinline__ void hermite_r_scaled(RT alpha, RT X, RT Y, RT Z, RT scale, Arr&& R) {
    const RT T = alpha * (X * X + Y * Y + Z * Z);
    RT g[L + 1];
    boys_scaled<L>(alpha, T, g);
#pragma unroll
    for (int n = 0; n <= L; ++n) g[n] *= scale;
    R[0] = g[L];
#pragma unroll
    for (int n = L - 1; n >= 0; --n) {
        // level n from level n+1; degrees d = L-n .. 1, decreasing index
#pragma unroll
        for (int d = L - n; d >= 1; --d) {
#pragma unroll
            for (int t = 0; t <= d; ++t) {
#pragma unroll
                for (int u = 0; u <= d - t; ++u) {
                    const int v = d - t - u;
                    RT r;
                    if (t > 0) {
                        r = X * R[hidx(t - 1, u, v)];
                        if (t > 1) r += (t - 1) * R[hidx(t - 2, u, v)];
                    } else if (u > 0) {
                        r = Y * R[hidx(t, u - 1, v)];
                        if (u > 1) r += (u - 1) * R[hidx(t, u - 2, v)];
                    } else {
                        r = Z * R[hidx(t, u, v - 1)];
                        if (v > 1) r += (v - 1) * R[hidx(t, u, v - 2)];
                    }
                    R[hidx(t, u, v)] = r;
                }
            }
        }
        R[0] = g[n];
    }
}

template <int L, typename RT>
__device__ __forceinline__ void hermite_r(RT alpha, RT X, RT Y, RT Z, RT (&R)[nherm(L)]) {
    hermite_r_scaled<L>(alpha, X, Y, Z, RT(1), R);
}

// E^{ij}_t for i <= IM, j <= JM, t <= i + j, one direction: e[i][j][t].
// pa = P - A, pb = P - B, oo2p = 1/(2p), e00 = E^{00}_0.
template <int IM, int JM, typename RT>
__device__ __forceinline__ void hermite_e(RT pa, RT pb, RT oo2p, RT e00, RT (&e)[IM + 1][JM + 1][IM + JM + 1]) {
#pragma unroll
    for (int i = 0; i <= IM; ++i)
#pragma unroll
        for (int j = 0; j <= JM; ++j)
#pragma unroll
            for (int t = 0; t <= IM + JM; ++t) e[i][j][t] = RT(0);
    e[0][0][0] = e00;
#pragma unroll
    for (int j = 1; j <= JM; ++j)
#pragma unroll
        for (int t = 0; t <= j; ++t) {
            RT v = pb * e[0][j - 1][t];
            if (t + 1 <= j - 1) v += (t + 1) * e[0][j - 1][t + 1];
            if (t > 0) v += oo2p * e[0][j - 1][t - 1];
            e[0][j][t] = v;
        }
#pragma unroll
    for (int i = 1; i <= IM; ++i)
#pragma unroll
        for (int j = 0; j <= JM; ++j)
#pragma unroll
            for (int t = 0; t <= i + j; ++t) {
                RT v = pa * e[i - 1][j][t];
                if (t + 1 <= i - 1 + j) v += (t + 1) * e[i - 1][j][t + 1];
                if (t > 0) v += oo2p * e[i - 1][j][t - 1];
                e[i][j][t] = v;
            }
}

// ---------------------------------------------------------------- data

// Primitive-pair record (PPW doubles), pair oriented so that l_A >= l_B:
//   0 a, 1 b, 2 K = exp(-mu |A-B|^2), 3..5 P, 6..8 P - A, 9..11 P - B,
//   12..15 contraction products c_A[ca] c_B[cb] at the compact index
//          ca * nB + cb (nA, nB: the blocks' actual contraction counts),
//          zeros after nA * nB; the bra rows and ket contraction groups of
//          the quartet kernels use the same compact index
struct PairView {
    const int* pa_blk;      // [npair] block A (l_A >= l_B)
    const int* pb_blk;      // [npair] block B
    const int64_t* slot;    // [npair] first record of the pair
    const int* npp;         // [npair] surviving primitive pairs
    const double* rec;      // records
};

struct BlockView {
    const int* atom;
    const int* l;
    const int* ncon;
    const int* ao;          // AO of (contraction 0, component 0)
};

}  // namespace hf
