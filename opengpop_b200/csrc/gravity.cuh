// gravity.cuh -- fused normalised spherical-harmonic gravity (Gottlieb's derived-Legendre method,
// as in lib/force_model/src/acceleration/gravity_source_device.cu:63-239) for K objects per thread.
//
// The reference builds the whole P-bar triangle, four N x T term arrays and two Thrust segment
// reductions in HBM per evaluation (about 25 launches). Here each thread walks the triangle column
// by column with a two-term recursion held in registers, reading the pre-scaled coefficient table
// from shared memory by broadcast (every lane of a warp reads the same entry). Per (n, m) term and
// object: 3 FP64 ops for the recursion and 6 FMAs into per-column sums; per column the sums are
// combined with the cos/sin(m lambda) recursion of eq. 3-18. The (R/r)^n factor of eq. 4-12 rides
// in the recursion variable, so no per-degree sums are needed. With K objects per thread every
// table entry loaded from shared memory feeds K independent chains; with two objects the columns
// are also walked two at a time, so each thread carries two independent recursions.
//
// Mixed precision: terms of degree n <= 8 (and all per-column combining, the central term, frame
// rotations and the final assembly) stay FP64; the n > 8 recursion and sums run in FP32 with
// packed f32x2 FMAs (for K = 2 the recursion of the two objects shares one packed instruction),
// per column, and each column's FP32 sums are added into the FP64 totals (two-level summation: at
// most 62 FP32 terms per partial sum).
#pragma once
#include "common.cuh"
#include "model.h"

namespace gpop {

constexpr int kMixedSplit = 8; // highest degree kept in FP64 in the mixed mode

// Unroll factors of the column walks (measured on B200, 65,536 objects at 70x70: the two-object
// FP32 walk runs 6 % faster at 8 than at 4, and 10 % slower at 32).
#ifndef GPOP_COL32X2_UNROLL
#define GPOP_COL32X2_UNROLL 8
#endif
#ifndef GPOP_COL64_UNROLL
#define GPOP_COL64_UNROLL 4
#endif
// Two objects per thread walk the columns two at a time (two independent recursions per thread
// hide each other's latency). Measured on B200, 65,536 objects at 70x70, with the corrector state
// in shared memory: mixed 123.9 -> 139.4 M object-steps/s (pair unroll 4: 137.6, 8: 139.4, 12:
// 139.0; three columns at a time 130.5, four 121.3), FP64 72.3 -> 73.8 M (pair unroll 2).
#ifndef GPOP_COLPAIR_UNROLL
#define GPOP_COLPAIR_UNROLL 8
#endif
#ifndef GPOP_COLGROUP_UNROLL
#define GPOP_COLGROUP_UNROLL 4
#endif
#ifndef GPOP_PAIR_COLUMNS
#define GPOP_PAIR_COLUMNS 1
#endif
#ifndef GPOP_PAIR_COLUMNS64
#define GPOP_PAIR_COLUMNS64 1
#endif
#ifndef GPOP_COL64PAIR_UNROLL
#define GPOP_COL64PAIR_UNROLL 2
#endif
constexpr int kCol32x2Unroll = GPOP_COL32X2_UNROLL;
constexpr int kCol64Unroll = GPOP_COL64_UNROLL;
constexpr int kColPairUnroll = GPOP_COLPAIR_UNROLL;
constexpr int kColGroupUnroll = GPOP_COLGROUP_UNROLL;
constexpr bool kPairColumns = GPOP_PAIR_COLUMNS != 0;
constexpr bool kPairColumns64 = GPOP_PAIR_COLUMNS64 != 0;
constexpr int kCol64PairUnroll = GPOP_COL64PAIR_UNROLL;
// FP64 with one object per thread also walks two columns at a time (20,000 objects at 70x70:
// 36.6 -> 40.0 M object-steps/s)
#ifndef GPOP_PAIR_COLUMNS64_ONE
#define GPOP_PAIR_COLUMNS64_ONE 1
#endif
constexpr bool kPairColumns64One = GPOP_PAIR_COLUMNS64_ONE != 0;
// the FP32 group walk runs its last N mod U terms in blocks of two (mixed 139.4 -> 140.5 M)
#ifndef GPOP_BLOCK_REMAINDER
#define GPOP_BLOCK_REMAINDER 1
#endif
constexpr bool kBlockRemainder = GPOP_BLOCK_REMAINDER != 0;

struct GravSmem {
    const GravEntry64* t64; // FP64 mode: full table; mixed mode: head table (n <= 8)
    const GravEntry32* t32; // mixed mode: full FP32 table (recursion constant stored negated, twice)
    int L; // degree summed (<= Lt)
    int Lt; // degree of the table layout (columns of Lt - m + 1 entries)
    double radius, gm;
    const int* cb64 = nullptr; // lane layout: first 16-byte unit of each FP64 (or head) column
    const int* cb32 = nullptr; // lane layout: the same for the FP32 table
};

// Columns of the lane-layout tables (build_lane_blob): column m starts at 16-byte unit cb[m].
__device__ __forceinline__ const GravEntry64* lane_col64(const GravSmem& g, int m)
{
    return reinterpret_cast<const GravEntry64*>(reinterpret_cast<const uint4*>(g.t64) + g.cb64[m]);
}
__device__ __forceinline__ const GravEntry32* lane_col32(const GravSmem& g, int m)
{
    return reinterpret_cast<const GravEntry32*>(reinterpret_cast<const uint4*>(g.t32) + g.cb32[m]);
}
// Column m of the FP64 table (degree Lt64: the full table, or the n <= 8 head in mixed mode) and of
// the FP32 table, in the plain (LANE = false) or the lane layout.
template <bool LANE>
__device__ __forceinline__ const GravEntry64* col64(const GravSmem& g, int m, int Lt64)
{
    if constexpr (LANE)
        return lane_col64(g, m);
    else
        return g.t64 + grav_col_offset(m, Lt64);
}
template <bool LANE> __device__ __forceinline__ const GravEntry32* col32(const GravSmem& g, int m)
{
    if constexpr (LANE)
        return lane_col32(g, m);
    else
        return g.t32 + grav_col_offset(m, g.Lt);
}

template <int K> struct ColSums64 {
    double g1[K], g2[K], j1[K], j2[K], h1[K], h2[K];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int k = 0; k < K; ++k)
            g1[k] = g2[k] = j1[k] = j2[k] = h1[k] = h2[k] = 0.0;
    }
    __device__ __forceinline__ void add(const GravEntry64* __restrict__ e, const double (&Q)[K])
    {
        const double2* p = reinterpret_cast<const double2*>(e);
        const double2 g = p[1], j = p[2], h = p[3];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            g1[k] = fma(g.x, Q[k], g1[k]);
            g2[k] = fma(g.y, Q[k], g2[k]);
            j1[k] = fma(j.x, Q[k], j1[k]);
            j2[k] = fma(j.y, Q[k], j2[k]);
            h1[k] = fma(h.x, Q[k], h1[k]);
            h2[k] = fma(h.y, Q[k], h2[k]);
        }
    }
};

// One FP64 term at entry e: t2 holds c(n) w Q(n-2) on entry and c(n+1) w Q(n-1) on exit.
template <int K>
__device__ __forceinline__ void term64(const GravEntry64* __restrict__ e, const double (&u)[K],
    const double (&w)[K], double (&Q1)[K], double (&Q2)[K], double (&t2)[K], ColSums64<K>& s)
{
    const double cn = reinterpret_cast<const double2*>(e + 1)[0].x;
    double Q[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        Q[k] = fma(u[k], Q1[k], -t2[k]);
        t2[k] = (cn * w[k]) * Q1[k];
        Q2[k] = Q1[k];
        Q1[k] = Q[k];
    }
    s.add(e, Q);
}

// Walks column entries e[first..last] in FP64, continuing the recursion from Q1 = Q(n-1),
// Q2 = Q(n-2) of each object. The product c(n+1) w Q(n-1) of the next term is formed while the
// current term accumulates, so one FMA separates consecutive Q values on the dependency chain.
// (The entry after the last one of column m < L is the first entry of column m+1, in bounds.)
template <int K>
__device__ __forceinline__ void column64(const GravEntry64* __restrict__ e, int first, int last,
    const double (&u)[K], const double (&w)[K], double (&Q1)[K], double (&Q2)[K], ColSums64<K>& s)
{
    if (first > last)
        return;
    double t2[K];
    {
        const double c = reinterpret_cast<const double2*>(e + first)[0].x;
#pragma unroll
        for (int k = 0; k < K; ++k)
            t2[k] = (c * w[k]) * Q2[k];
    }
#pragma unroll(kCol64Unroll)
    for (int i = first; i <= last; ++i)
        term64<K>(e + i, u, w, Q1, Q2, t2, s);
}

// Two FP64 columns walked side by side: N terms at entries ea[0..N-1] and eb[0..N-1], each with
// the operations of column64 in its order (bit-identical sums).
template <int K>
__device__ __forceinline__ void column64_pair(const GravEntry64* __restrict__ ea,
    const GravEntry64* __restrict__ eb, int N, const double (&u)[K], const double (&w)[K],
    double (&Qa1)[K], double (&Qa2)[K], ColSums64<K>& sa, double (&Qb1)[K], double (&Qb2)[K],
    ColSums64<K>& sb)
{
    if (N <= 0)
        return;
    double ta[K], tb[K];
    {
        const double ca = reinterpret_cast<const double2*>(ea)[0].x;
        const double cb = reinterpret_cast<const double2*>(eb)[0].x;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            ta[k] = (ca * w[k]) * Qa2[k];
            tb[k] = (cb * w[k]) * Qb2[k];
        }
    }
#pragma unroll(kCol64PairUnroll)
    for (int t = 0; t < N; ++t) {
        term64<K>(ea + t, u, w, Qa1, Qa2, ta, sa);
        term64<K>(eb + t, u, w, Qb1, Qb2, tb, sb);
    }
}

// FP32 column walk; the table holds (-c, -c, g1, g2 | j1, j2, h1, h2).
template <int K> struct ColSums32 {
    float2 g[K], j[K], h[K];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int k = 0; k < K; ++k)
            g[k] = j[k] = h[k] = make_float2(0.f, 0.f);
    }
};

__device__ __forceinline__ void column32(const GravEntry32* __restrict__ e, int first, int last,
    float u, float w, float& Q1, float& Q2, ColSums32<1>& s)
{
    if (first > last)
        return;
    float t2 = (reinterpret_cast<const float4*>(e + first)[0].x * w) * Q2;
#pragma unroll 4
    for (int i = first; i <= last; ++i) {
        const float4* p = reinterpret_cast<const float4*>(e + i);
        const float4 a = p[0], b = p[1];
        const float cn = reinterpret_cast<const float4*>(e + i + 1)[0].x;
        const float Q = fmaf(u, Q1, t2);
        t2 = (cn * w) * Q1;
        const float2 QQ = make_float2(Q, Q);
        s.g[0] = __ffma2_rn(QQ, make_float2(a.z, a.w), s.g[0]);
        s.j[0] = __ffma2_rn(QQ, make_float2(b.x, b.y), s.j[0]);
        s.h[0] = __ffma2_rn(QQ, make_float2(b.z, b.w), s.h[0]);
        Q2 = Q1;
        Q1 = Q;
    }
}

// Two objects: the recursion of both objects is one packed chain (Q = (Q_A, Q_B)).
// One term at entry e: t2 holds -c(n) w Q(n-2) on entry and -c(n+1) w Q(n-1) on exit.
__device__ __forceinline__ void term32x2(const GravEntry32* __restrict__ e, float2 u, float2 w,
    float2& Q1, float2& Q2, float2& t2, ColSums32<2>& s)
{
    const float4* p = reinterpret_cast<const float4*>(e);
    const float4 a = p[0], b = p[1];
    const float4 an = reinterpret_cast<const float4*>(e + 1)[0];
    const float2 Q = __ffma2_rn(u, Q1, t2);
    t2 = __fmul2_rn(__fmul2_rn(make_float2(an.x, an.y), w), Q1);
    const float2 QA = make_float2(Q.x, Q.x), QB = make_float2(Q.y, Q.y);
    const float2 cg = make_float2(a.z, a.w), cj = make_float2(b.x, b.y), ch = make_float2(b.z, b.w);
    s.g[0] = __ffma2_rn(QA, cg, s.g[0]);
    s.j[0] = __ffma2_rn(QA, cj, s.j[0]);
    s.h[0] = __ffma2_rn(QA, ch, s.h[0]);
    s.g[1] = __ffma2_rn(QB, cg, s.g[1]);
    s.j[1] = __ffma2_rn(QB, cj, s.j[1]);
    s.h[1] = __ffma2_rn(QB, ch, s.h[1]);
    Q2 = Q1;
    Q1 = Q;
}

__device__ __forceinline__ float2 first_t2(const GravEntry32* __restrict__ e, float2 w, float2 Q2)
{
    const float4 a0 = reinterpret_cast<const float4*>(e)[0];
    return __fmul2_rn(__fmul2_rn(make_float2(a0.x, a0.y), w), Q2);
}

// The single term at entry e of a column whose walk ends there (t2 formed from Q2 first).
__device__ __forceinline__ void last_term32x2(const GravEntry32* __restrict__ e, float2 u, float2 w,
    float2& Q1, float2& Q2, ColSums32<2>& s)
{
    const float4* p = reinterpret_cast<const float4*>(e);
    const float4 a = p[0], b = p[1];
    const float2 t2 = __fmul2_rn(__fmul2_rn(make_float2(a.x, a.y), w), Q2);
    const float2 Q = __ffma2_rn(u, Q1, t2);
    const float2 QA = make_float2(Q.x, Q.x), QB = make_float2(Q.y, Q.y);
    const float2 cg = make_float2(a.z, a.w), cj = make_float2(b.x, b.y), ch = make_float2(b.z, b.w);
    s.g[0] = __ffma2_rn(QA, cg, s.g[0]);
    s.j[0] = __ffma2_rn(QA, cj, s.j[0]);
    s.h[0] = __ffma2_rn(QA, ch, s.h[0]);
    s.g[1] = __ffma2_rn(QB, cg, s.g[1]);
    s.j[1] = __ffma2_rn(QB, cj, s.j[1]);
    s.h[1] = __ffma2_rn(QB, ch, s.h[1]);
    Q2 = Q1;
    Q1 = Q;
}

__device__ __forceinline__ void column32x2(const GravEntry32* __restrict__ e, int first, int last,
    float2 u, float2 w, float2& Q1, float2& Q2, ColSums32<2>& s)
{
    if (first > last)
        return;
    float2 t2 = first_t2(e + first, w, Q2);
#pragma unroll(kCol32x2Unroll)
    for (int i = first; i <= last; ++i)
        term32x2(e + i, u, w, Q1, Q2, t2, s);
}

template <int K>
__device__ __forceinline__ void column32k(const GravEntry32* __restrict__ e, int first, int last,
    const float (&u)[K], const float (&w)[K], float (&Q1)[K], float (&Q2)[K], ColSums32<K>& s)
{
    if constexpr (K == 1) {
        column32(e, first, last, u[0], w[0], Q1[0], Q2[0], s);
    } else {
        static_assert(K == 2, "FP32 path packs one or two objects");
        float2 U = make_float2(u[0], u[1]), W = make_float2(w[0], w[1]);
        float2 A = make_float2(Q1[0], Q1[1]), B = make_float2(Q2[0], Q2[1]);
        column32x2(e, first, last, U, W, A, B, s);
        Q1[0] = A.x;
        Q1[1] = A.y;
        Q2[0] = B.x;
        Q2[1] = B.y;
    }
}

// C FP32 columns of two objects walked side by side: N terms at entries e[c][0..N-1], each column
// with the operations of column32x2 in its order (bit-identical sums).
template <int C, int PU = kColPairUnroll>
__device__ __forceinline__ void column32x2_group(const GravEntry32* const (&e)[C], int N, float2 u,
    float2 w, float2 (&Q1)[C], float2 (&Q2)[C], ColSums32<2> (&s)[C])
{
    if (N <= 0)
        return;
    float2 t[C];
#pragma unroll
    for (int c = 0; c < C; ++c)
        t[c] = first_t2(e[c], w, Q2[c]);
    if constexpr (kBlockRemainder) {
        // blocks of U terms, then blocks of 2, then at most one term: every block is straight-line
        // code whose loads can all be issued before its first term
        constexpr int U = C == 2 ? PU : kColGroupUnroll;
        int i = 0;
#pragma unroll 1
        for (; i + U <= N; i += U)
#pragma unroll
            for (int j = 0; j < U; ++j)
#pragma unroll
                for (int c = 0; c < C; ++c)
                    term32x2(e[c] + i + j, u, w, Q1[c], Q2[c], t[c], s[c]);
#pragma unroll 1
        for (; i + 2 <= N; i += 2)
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int c = 0; c < C; ++c)
                    term32x2(e[c] + i + j, u, w, Q1[c], Q2[c], t[c], s[c]);
        if (i < N)
#pragma unroll
            for (int c = 0; c < C; ++c)
                term32x2(e[c] + i, u, w, Q1[c], Q2[c], t[c], s[c]);
    } else {
#pragma unroll(C == 2 ? PU : kColGroupUnroll)
        for (int i = 0; i < N; ++i)
#pragma unroll
            for (int c = 0; c < C; ++c)
                term32x2(e[c] + i, u, w, Q1[c], Q2[c], t[c], s[c]);
    }
}

// Mixed precision, two objects, degree L > 8: the walk of gravity_itrs<true, 2> with the FP32
// parts of the columns taken kHeadGroup (columns m <= 8) or kTailGroup (m > 8) columns at a time.
// Every column's sums, their combination and the order of the combinations are those of the
// one-column walk, so the accelerations are bit-identical to it.
// Start values of a two-object walk at Earth-fixed (x, y, z): q = R/r, u = q eps, w = q^2 and the
// eq. 3-18 seeds x/r, y/r (the arithmetic of the walks' own constructors).
struct WalkStart {
    double q[2], u[2], w[2], C1[2], S1[2];
};
__device__ __forceinline__ void walk_start(double radius, const double (&x)[2], const double (&y)[2],
    const double (&z)[2], WalkStart& s)
{
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const double r = sqrt(x[k] * x[k] + y[k] * y[k] + z[k] * z[k]);
        const double eps = z[k] / r;
        s.q[k] = radius / r;
        s.u[k] = s.q[k] * eps;
        s.w[k] = s.q[k] * s.q[k];
        s.C1[k] = x[k] / r;
        s.S1[k] = y[k] / r;
    }
}

// PU: the unroll of the two-column FP32 walk (the split block runs faster at 4, the plain block
// at 8).
template <bool LANE, int PU = kColPairUnroll> struct MixedWalk2 {
    static constexpr int K = 2;
    const GravSmem& gs;
    int L;
    double q[K], u[K], w[K], C1[K], S1[K], Cm[K], Sm[K], Cp[K], Sp[K], qm[K];
    double G[K], H[K], J[K], KK[K];
    float2 uf, wf;
    float cf[K], sf[K], cpf[K], spf[K], qmf[K], c1f[K], s1f[K], qf[K];
    float Gf[K], Hf[K], Jf[K], Kf[K];

    __device__ __forceinline__ MixedWalk2(const GravSmem& g, const double (&r)[K], const double (&x)[K],
        const double (&y)[K], const double (&z)[K])
        : gs(g)
        , L(g.L)
    {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double eps = z[k] / r[k];
            q[k] = gs.radius / r[k];
            u[k] = q[k] * eps;
            w[k] = q[k] * q[k];
            C1[k] = x[k] / r[k];
            S1[k] = y[k] / r[k];
            Cm[k] = 1.0;
            Sm[k] = 0.0;
            Cp[k] = 0.0;
            Sp[k] = 0.0;
            qm[k] = 1.0;
            G[k] = H[k] = J[k] = KK[k] = 0.0;
        }
        uf = make_float2((float)u[0], (float)u[1]);
        wf = make_float2((float)w[0], (float)w[1]);
    }
    __device__ __forceinline__ MixedWalk2(const GravSmem& g, const WalkStart& s)
        : gs(g)
        , L(g.L)
    {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            q[k] = s.q[k];
            u[k] = s.u[k];
            w[k] = s.w[k];
            C1[k] = s.C1[k];
            S1[k] = s.S1[k];
            Cm[k] = 1.0;
            Sm[k] = 0.0;
            Cp[k] = 0.0;
            Sp[k] = 0.0;
            qm[k] = 1.0;
            G[k] = H[k] = J[k] = KK[k] = 0.0;
        }
        uf = make_float2((float)u[0], (float)u[1]);
        wf = make_float2((float)w[0], (float)w[1]);
    }
    // eq. 4-11 for column m in FP64, then the cos/sin(m lambda) and q^m recursions step on
    __device__ __forceinline__ void combine64(int m, const ColSums64<K>& s)
    {
        const double dm = (double)m;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            G[k] += Cm[k] * s.g1[k] + Sm[k] * s.g2[k];
            J[k] += dm * (Cp[k] * s.j1[k] + Sp[k] * s.j2[k]);
            KK[k] -= dm * (Sp[k] * s.j1[k] - Cp[k] * s.j2[k]);
            H[k] += Cp[k] * s.h1[k] + Sp[k] * s.h2[k];
            Cp[k] = Cm[k];
            Sp[k] = Sm[k];
            const double Cn = C1[k] * Cm[k] - S1[k] * Sm[k];
            const double Sn = S1[k] * Cm[k] + C1[k] * Sm[k];
            Cm[k] = Cn;
            Sm[k] = Sn;
            qm[k] *= q[k];
        }
    }
    // columns m .. m + C - 1 (<= 8): FP64 terms n <= 8 of each, then the FP32 terms 9..L of all
    // of them side by side (L - 8 terms each), then the combinations in order
    template <int C> __device__ __forceinline__ void head_group(int m)
    {
        ColSums64<K> s[C];
        ColSums32<K> f[C];
        float2 Q1f[C], Q2f[C];
        const GravEntry32* e[C];
        double qs[K];
#pragma unroll
        for (int k = 0; k < K; ++k)
            qs[k] = qm[k];
        double Q1[C][K], Q2[C][K];
        const GravEntry64* e64[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            if (c > 0) {
#pragma unroll
                for (int k = 0; k < K; ++k)
                    qs[k] = qs[k] * q[k]; // the value combine64 gives qm at column m + c
            }
            s[c].zero();
            f[c].zero();
#pragma unroll
            for (int k = 0; k < K; ++k) {
                Q1[c][k] = qs[k];
                Q2[c][k] = 0.0;
            }
            e64[c] = col64<LANE>(gs, m + c, kMixedSplit);
            s[c].add(e64[c], Q1[c]);
            e[c] = col32<LANE>(gs, m + c) + (kMixedSplit + 1 - m - c);
        }
        if constexpr (C == 2) { // FP64 terms of both columns side by side; column m has one more
            column64_pair<K>(e64[0] + 1, e64[1] + 1, kMixedSplit - m - 1, u, w, Q1[0], Q2[0], s[0],
                Q1[1], Q2[1], s[1]);
            column64<K>(e64[0], kMixedSplit - m, kMixedSplit - m, u, w, Q1[0], Q2[0], s[0]);
        } else {
#pragma unroll
            for (int c = 0; c < C; ++c)
                column64<K>(e64[c], 1, kMixedSplit - m - c, u, w, Q1[c], Q2[c], s[c]);
        }
#pragma unroll
        for (int c = 0; c < C; ++c) {
            Q1f[c] = make_float2((float)Q1[c][0], (float)Q1[c][1]);
            Q2f[c] = make_float2((float)Q2[c][0], (float)Q2[c][1]);
        }
        if constexpr (C == 1)
            column32x2(e[0], 0, L - kMixedSplit - 1, uf, wf, Q1f[0], Q2f[0], f[0]);
        else
            column32x2_group<C, PU>(e, L - kMixedSplit, uf, wf, Q1f, Q2f, f);
#pragma unroll
        for (int c = 0; c < C; ++c) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                s[c].g1[k] += (double)f[c].g[k].x;
                s[c].g2[k] += (double)f[c].g[k].y;
                s[c].j1[k] += (double)f[c].j[k].x;
                s[c].j2[k] += (double)f[c].j[k].y;
                s[c].h1[k] += (double)f[c].h[k].x;
                s[c].h2[k] += (double)f[c].h[k].y;
            }
            combine64(m + c, s[c]);
        }
    }
    // the recursions of combine64 over one column, without its sums (for a walk that starts past it)
    __device__ __forceinline__ void skip64()
    {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            Cp[k] = Cm[k];
            Sp[k] = Sm[k];
            const double Cn = C1[k] * Cm[k] - S1[k] * Sm[k];
            const double Sn = S1[k] * Cm[k] + C1[k] * Sm[k];
            Cm[k] = Cn;
            Sm[k] = Sn;
            qm[k] *= q[k];
        }
    }
    // FP32 state of the columns m > 8 from the FP64 recursions after column 8
    __device__ __forceinline__ void to_tail()
    {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            cf[k] = (float)Cm[k];
            sf[k] = (float)Sm[k];
            cpf[k] = (float)Cp[k];
            spf[k] = (float)Sp[k];
            qmf[k] = (float)qm[k];
            c1f[k] = (float)C1[k];
            s1f[k] = (float)S1[k];
            qf[k] = (float)q[k];
            Gf[k] = Hf[k] = Jf[k] = Kf[k] = 0.f;
        }
    }
    __device__ __forceinline__ void combine32(int m, const ColSums32<K>& f)
    {
        const float dm = (float)m;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            Gf[k] += cf[k] * f.g[k].x + sf[k] * f.g[k].y;
            Jf[k] += dm * (cpf[k] * f.j[k].x + spf[k] * f.j[k].y);
            Kf[k] -= dm * (spf[k] * f.j[k].x - cpf[k] * f.j[k].y);
            Hf[k] += cpf[k] * f.h[k].x + spf[k] * f.h[k].y;
            cpf[k] = cf[k];
            spf[k] = sf[k];
            const float cn = c1f[k] * cf[k] - s1f[k] * sf[k];
            const float sn = s1f[k] * cf[k] + c1f[k] * sf[k];
            cf[k] = cn;
            sf[k] = sn;
            qmf[k] *= qf[k];
        }
    }
    // columns m .. m + C - 1 (> 8, m + C - 1 <= L) in FP32: the n = m term (Q = q^m) of each, the
    // L - m - C + 1 terms all of them have left side by side, the remaining terms of the longer
    // columns one column at a time, then the combinations in order
    template <int C> __device__ __forceinline__ void tail_group(int m)
    {
        ColSums32<K> f[C];
        float2 Q1f[C], Q2f[C];
        const GravEntry32* e[C];
        float qs[K];
#pragma unroll
        for (int k = 0; k < K; ++k)
            qs[k] = qmf[k];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            if (c > 0) {
#pragma unroll
                for (int k = 0; k < K; ++k)
                    qs[k] = qs[k] * qf[k]; // the value combine32 gives qmf at column m + c
            }
            const GravEntry32* base = col32<LANE>(gs, m + c);
            const float4* p = reinterpret_cast<const float4*>(base);
            const float4 a = p[0], b = p[1];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const float2 QQ = make_float2(qs[k], qs[k]);
                f[c].g[k] = __fmul2_rn(QQ, make_float2(a.z, a.w));
                f[c].j[k] = __fmul2_rn(QQ, make_float2(b.x, b.y));
                f[c].h[k] = __fmul2_rn(QQ, make_float2(b.z, b.w));
            }
            Q1f[c] = make_float2(qs[0], qs[1]);
            Q2f[c] = make_float2(0.f, 0.f);
            e[c] = base + 1;
        }
        const int N = L - m - (C - 1);
        if constexpr (C > 1) {
            column32x2_group<C, PU>(e, N, uf, wf, Q1f, Q2f, f);
            if constexpr (C == 2) {
                last_term32x2(e[0] + N, uf, wf, Q1f[0], Q2f[0], f[0]); // column m: one term more
            } else {
#pragma unroll
                for (int c = 0; c + 1 < C; ++c) // column m + c has C - 1 - c terms more
                    column32x2(e[c] - 1, N + 1, L - m - c, uf, wf, Q1f[c], Q2f[c], f[c]);
            }
        } else {
            column32x2(e[0] - 1, 1, L - m, uf, wf, Q1f[0], Q2f[0], f[0]);
        }
#pragma unroll
        for (int c = 0; c < C; ++c)
            combine32(m + c, f[c]);
    }
};

#ifndef GPOP_HEAD_GROUP
#define GPOP_HEAD_GROUP 2
#endif
#ifndef GPOP_TAIL_GROUP
#define GPOP_TAIL_GROUP 2
#endif
constexpr int kHeadGroup = GPOP_HEAD_GROUP;

constexpr int kTailGroup = GPOP_TAIL_GROUP;


// Eq. 4-13: Earth-fixed acceleration from the totals G, H, J, K of eq. 4-11.
__device__ __forceinline__ void assemble_itrs(double gm, double x, double y, double z, double r,
    double G, double H, double J, double KK, double& ax, double& ay, double& az)
{
    const double Gk = G + 1.0;
    const double Lambda = Gk + z * H / r;
    const double c = -gm / (r * r);
    ax = c * (Lambda * x / r - J);
    ay = c * (Lambda * y / r - KK);
    az = c * (Lambda * z / r - H);
}

// The mixed two-object walk from column m0 (a multiple of kHeadGroup, <= 8; the recursions
// already stepped to it) to L: head groups, then the FP32 tail, whose totals are added into the
// FP64 ones.
template <bool LANE, int PU>
__device__ __forceinline__ void walk_groups_from(MixedWalk2<LANE, PU>& W, int m0)
{
    constexpr int K = 2;
    const int L = W.L;
    int m = m0;
#pragma unroll 1
    for (; m + kHeadGroup - 1 <= kMixedSplit; m += kHeadGroup)
        W.template head_group<kHeadGroup>(m);
    if constexpr (kHeadGroup > 1) { // 9 head columns: what the groups left
        constexpr int rest = (kMixedSplit + 1) % kHeadGroup;
        if constexpr (rest > 0)
            W.template head_group<rest>(m);
    }
    W.to_tail();
    m = kMixedSplit + 1;
#pragma unroll 1
    for (; m + kTailGroup - 1 <= L; m += kTailGroup)
        W.template tail_group<kTailGroup>(m);
    if constexpr (kTailGroup > 2) {
        if (m + 1 <= L) {
            W.template tail_group<2>(m);
            m += 2;
        }
    }
    if constexpr (kTailGroup > 1) {
        if (m <= L)
            W.template tail_group<1>(m);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
        W.G[k] += (double)W.Gf[k];
        W.H[k] += (double)W.Hf[k];
        W.J[k] += (double)W.Jf[k];
        W.KK[k] += (double)W.Kf[k];
    }
}

template <bool LANE>
__device__ __forceinline__ void gravity_itrs_groups(const GravSmem& gs, const double (&x)[2],
    const double (&y)[2], const double (&z)[2], double (&ax)[2], double (&ay)[2], double (&az)[2])
{
    constexpr int K = 2;
    double r[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
        r[k] = sqrt(x[k] * x[k] + y[k] * y[k] + z[k] * z[k]);
    MixedWalk2<LANE> W(gs, r, x, y, z);
    walk_groups_from(W, 0);
#pragma unroll
    for (int k = 0; k < K; ++k)
        assemble_itrs(gs.gm, x[k], y[k], z[k], r[k], W.G[k], W.H[k], W.J[k], W.KK[k], ax[k], ay[k],
            az[k]);
}

// FP64, K objects: columns (0, 1), (2, 3), ... walked side by side, each combined in order as the
// one-column walk does (bit-identical accelerations).
template <bool LANE, int K> struct PairWalk64 {
    const GravSmem& gs;
    int L;
    double r[K], q[K], u[K], w[K], C1[K], S1[K], Cm[K], Sm[K], Cp[K], Sp[K], qm[K];
    double G[K], H[K], J[K], KK[K];

    __device__ __forceinline__ PairWalk64(const GravSmem& g, const double (&x)[K], const double (&y)[K],
        const double (&z)[K])
        : gs(g)
        , L(g.L)
    {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            r[k] = sqrt(x[k] * x[k] + y[k] * y[k] + z[k] * z[k]);
            const double eps = z[k] / r[k];
            q[k] = gs.radius / r[k];
            u[k] = q[k] * eps;
            w[k] = q[k] * q[k];
            C1[k] = x[k] / r[k];
            S1[k] = y[k] / r[k];
            Cm[k] = 1.0;
            Sm[k] = 0.0;
            Cp[k] = 0.0;
            Sp[k] = 0.0;
            qm[k] = 1.0;
            G[k] = H[k] = J[k] = KK[k] = 0.0;
        }
    }
    __device__ __forceinline__ PairWalk64(const GravSmem& g, const WalkStart& s)
        : gs(g)
        , L(g.L)
    {
        static_assert(K == 2, "a walk start carries two objects");
#pragma unroll
        for (int k = 0; k < K; ++k) {
            r[k] = 0.0; // not needed: the caller assembles
            q[k] = s.q[k];
            u[k] = s.u[k];
            w[k] = s.w[k];
            C1[k] = s.C1[k];
            S1[k] = s.S1[k];
            Cm[k] = 1.0;
            Sm[k] = 0.0;
            Cp[k] = 0.0;
            Sp[k] = 0.0;
            qm[k] = 1.0;
            G[k] = H[k] = J[k] = KK[k] = 0.0;
        }
    }
    // the cos/sin(m lambda) and q^m recursions over one column
    __device__ __forceinline__ void step()
    {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            Cp[k] = Cm[k];
            Sp[k] = Sm[k];
            const double Cn = C1[k] * Cm[k] - S1[k] * Sm[k];
            const double Sn = S1[k] * Cm[k] + C1[k] * Sm[k];
            Cm[k] = Cn;
            Sm[k] = Sn;
            qm[k] *= q[k];
        }
    }
    __device__ __forceinline__ void combine(int m, const ColSums64<K>& s)
    {
        const double dm = (double)m;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            G[k] += Cm[k] * s.g1[k] + Sm[k] * s.g2[k];
            J[k] += dm * (Cp[k] * s.j1[k] + Sp[k] * s.j2[k]);
            KK[k] -= dm * (Sp[k] * s.j1[k] - Cp[k] * s.j2[k]);
            H[k] += Cp[k] * s.h1[k] + Sp[k] * s.h2[k];
        }
        step();
    }
    // columns [m0, m1) (m1 <= L + 1), two at a time from m0
    __device__ __forceinline__ void walk(int m0, int m1)
    {
#pragma unroll 1
        for (int m = m0; m < m1; m += 2) {
            ColSums64<K> sa, sb;
            double Qa1[K], Qa2[K], Qb1[K], Qb2[K];
            sa.zero();
#pragma unroll
            for (int k = 0; k < K; ++k) {
                Qa1[k] = qm[k];
                Qa2[k] = 0.0;
            }
            const GravEntry64* ea = col64<LANE>(gs, m, gs.Lt);
            sa.add(ea, Qa1);
            if (m + 1 < m1) {
                sb.zero();
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    Qb1[k] = qm[k] * q[k];
                    Qb2[k] = 0.0;
                }
                const GravEntry64* eb = col64<LANE>(gs, m + 1, gs.Lt);
                sb.add(eb, Qb1);
                column64_pair<K>(ea + 1, eb + 1, L - m - 1, u, w, Qa1, Qa2, sa, Qb1, Qb2, sb);
                column64<K>(ea, L - m, L - m, u, w, Qa1, Qa2, sa);
                combine(m, sa);
                combine(m + 1, sb);
            } else {
                column64<K>(ea, 1, L - m, u, w, Qa1, Qa2, sa);
                combine(m, sa);
            }
        }
    }
};

template <bool LANE, int K>
__device__ __forceinline__ void gravity_itrs_pairs64(const GravSmem& gs, const double (&x)[K],
    const double (&y)[K], const double (&z)[K], double (&ax)[K], double (&ay)[K], double (&az)[K])
{
    PairWalk64<LANE, K> W(gs, x, y, z);
    W.walk(0, gs.L + 1);
#pragma unroll
    for (int k = 0; k < K; ++k)
        assemble_itrs(gs.gm, x[k], y[k], z[k], W.r[k], W.G[k], W.H[k], W.J[k], W.KK[k], ax[k], ay[k],
            az[k]);
}

// ---- column-split walk of two objects (gj8_split_kernel) ----
// Each object's columns are walked as two pieces, each summed from zero into its own totals (G, H,
// J, K of eq. 4-11): the low columns m < kSplitColumn and the columns from kSplitColumn on. The
// object's totals are low + high, in that order, whichever threads walked the pieces, so every
// object of a launch takes the same arithmetic. The high piece starts from the cos/sin(m lambda)
// and q^m recursions stepped over the low columns without their sums. Both need L > 8.
constexpr int kSplitColumn = 4;
// Unroll of the split walks' two-column FP32 walk (65,536 objects, mixed: 156.3 M object-steps/s
// at 4, 156.0 at 6, 154.2 at 8, 153.4 at 12).
#ifndef GPOP_SPLIT_PAIR_UNROLL
#define GPOP_SPLIT_PAIR_UNROLL 4
#endif
constexpr int kSplitPairUnroll = GPOP_SPLIT_PAIR_UNROLL;
static_assert(kSplitColumn % kHeadGroup == 0 && kSplitColumn <= kMixedSplit,
    "the split falls between head groups");

struct SplitTotals {
    double G[2], H[2], J[2], K[2];
};

template <bool MIXED>
__device__ __forceinline__ void split_low(const GravSmem& gs, const WalkStart& ws, SplitTotals& t)
{
    if constexpr (MIXED) {
        MixedWalk2<false, kSplitPairUnroll> W(gs, ws);
#pragma unroll 1
        for (int m = 0; m < kSplitColumn; m += kHeadGroup)
            W.template head_group<kHeadGroup>(m);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            t.G[k] = W.G[k];
            t.H[k] = W.H[k];
            t.J[k] = W.J[k];
            t.K[k] = W.KK[k];
        }
    } else {
        PairWalk64<false, 2> W(gs, ws);
        W.walk(0, kSplitColumn);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            t.G[k] = W.G[k];
            t.H[k] = W.H[k];
            t.J[k] = W.J[k];
            t.K[k] = W.KK[k];
        }
    }
}

template <bool MIXED>
__device__ __forceinline__ void split_high(const GravSmem& gs, const WalkStart& ws, SplitTotals& t)
{
    if constexpr (MIXED) {
        MixedWalk2<false, kSplitPairUnroll> W(gs, ws);
#pragma unroll
        for (int m = 0; m < kSplitColumn; ++m)
            W.skip64();
        walk_groups_from(W, kSplitColumn);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            t.G[k] = W.G[k];
            t.H[k] = W.H[k];
            t.J[k] = W.J[k];
            t.K[k] = W.KK[k];
        }
    } else {
        PairWalk64<false, 2> W(gs, ws);
#pragma unroll
        for (int m = 0; m < kSplitColumn; ++m)
            W.step();
        W.walk(kSplitColumn, gs.L + 1);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            t.G[k] = W.G[k];
            t.H[k] = W.H[k];
            t.J[k] = W.J[k];
            t.K[k] = W.KK[k];
        }
    }
}

// Accelerations of K objects in the Earth-fixed frame (eq. 4-13 of gravity_source_device.cu:212-239).
template <bool MIXED, int K>
__device__ __forceinline__ void gravity_itrs(const GravSmem& gs, const double (&x)[K],
    const double (&y)[K], const double (&z)[K], double (&ax)[K], double (&ay)[K], double (&az)[K])
{
    if constexpr (MIXED && K == 2 && kPairColumns) {
        if (gs.L > kMixedSplit) {
            gravity_itrs_groups<false>(gs, x, y, z, ax, ay, az);
            return;
        }
    }
    if constexpr (!MIXED && (K == 2 || kPairColumns64One) && kPairColumns64) {
        gravity_itrs_pairs64<false, K>(gs, x, y, z, ax, ay, az);
        return;
    }
    const int L = gs.L;
    double r[K], q[K], u[K], w[K], C1[K], S1[K], Cm[K], Sm[K], Cp[K], Sp[K], qm[K];
    double G[K], H[K], J[K], KK[K];
    float uf[K], wf[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        r[k] = sqrt(x[k] * x[k] + y[k] * y[k] + z[k] * z[k]);
        const double eps = z[k] / r[k]; // eq. 3-3
        q[k] = gs.radius / r[k];
        u[k] = q[k] * eps;
        w[k] = q[k] * q[k];
        C1[k] = x[k] / r[k]; // eq. 3-18 seeds
        S1[k] = y[k] / r[k];
        Cm[k] = 1.0;
        Sm[k] = 0.0;
        Cp[k] = 0.0;
        Sp[k] = 0.0;
        qm[k] = 1.0;
        G[k] = H[k] = J[k] = KK[k] = 0.0;
        uf[k] = (float)u[k];
        wf[k] = (float)w[k];
    }
    // Mixed mode: columns m <= 8 are combined in FP64 below; the columns m > 8 (every term of
    // degree > 8) are walked, combined and summed in FP32 after this loop.
    const int Lhead = (MIXED && L > kMixedSplit) ? kMixedSplit : L;
    for (int m = 0; m <= Lhead; ++m) {
        ColSums64<K> s;
        s.zero();
        double Q1[K], Q2[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            Q1[k] = qm[k];
            Q2[k] = 0.0;
        }
        if constexpr (!MIXED) {
            const GravEntry64* e = gs.t64 + grav_col_offset(m, gs.Lt);
            s.add(e, Q1); // n = m
            column64<K>(e, 1, L - m, u, w, Q1, Q2, s);
        } else {
            ColSums32<K> f;
            f.zero();
            const GravEntry32* e32 = gs.t32 + grav_col_offset(m, gs.Lt);
            float Q1f[K], Q2f[K];
            if (m <= kMixedSplit) {
                const int top = L < kMixedSplit ? L : kMixedSplit;
                const GravEntry64* e = gs.t64 + grav_col_offset(m, kMixedSplit);
                s.add(e, Q1);
                column64<K>(e, 1, top - m, u, w, Q1, Q2, s);
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    Q1f[k] = (float)Q1[k];
                    Q2f[k] = (float)Q2[k];
                }
                column32k<K>(e32, kMixedSplit + 1 - m, L - m, uf, wf, Q1f, Q2f, f);
            } else {
                // n = m term (Q = q^m), then the rest of the column with Q(m-1, m) = 0
                const float4* p = reinterpret_cast<const float4*>(e32);
                const float4 a = p[0], b = p[1];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const float Qm = (float)qm[k];
                    const float2 QQ = make_float2(Qm, Qm);
                    f.g[k] = __ffma2_rn(QQ, make_float2(a.z, a.w), f.g[k]);
                    f.j[k] = __ffma2_rn(QQ, make_float2(b.x, b.y), f.j[k]);
                    f.h[k] = __ffma2_rn(QQ, make_float2(b.z, b.w), f.h[k]);
                    Q1f[k] = Qm;
                    Q2f[k] = 0.f;
                }
                column32k<K>(e32, 1, L - m, uf, wf, Q1f, Q2f, f);
            }
#pragma unroll
            for (int k = 0; k < K; ++k) {
                s.g1[k] += (double)f.g[k].x;
                s.g2[k] += (double)f.g[k].y;
                s.j1[k] += (double)f.j[k].x;
                s.j2[k] += (double)f.j[k].y;
                s.h1[k] += (double)f.h[k].x;
                s.h2[k] += (double)f.h[k].y;
            }
        }
        // eq. 4-11 per column: G with (C_m, S_m); J, K, H with (C_{m-1}, S_{m-1})
        const double dm = (double)m;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            G[k] += Cm[k] * s.g1[k] + Sm[k] * s.g2[k];
            J[k] += dm * (Cp[k] * s.j1[k] + Sp[k] * s.j2[k]);
            KK[k] -= dm * (Sp[k] * s.j1[k] - Cp[k] * s.j2[k]);
            H[k] += Cp[k] * s.h1[k] + Sp[k] * s.h2[k];
            Cp[k] = Cm[k];
            Sp[k] = Sm[k];
            const double Cn = C1[k] * Cm[k] - S1[k] * Sm[k];
            const double Sn = S1[k] * Cm[k] + C1[k] * Sm[k];
            Cm[k] = Cn;
            Sm[k] = Sn;
            qm[k] *= q[k];
        }
    }
    if constexpr (MIXED) {
        if (L > kMixedSplit) {
            // the n = m term (Q = q^m) and the rest of each column in FP32; the column sums are
            // combined with FP32 cos/sin(m lambda) and (R/r)^m recursions into FP32 partial G, J,
            // K, H, added to the FP64 totals once
            float cf[K], sf[K], cpf[K], spf[K], qmf[K], c1f[K], s1f[K], qf[K];
            float Gf[K], Hf[K], Jf[K], Kf[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                cf[k] = (float)Cm[k];
                sf[k] = (float)Sm[k];
                cpf[k] = (float)Cp[k];
                spf[k] = (float)Sp[k];
                qmf[k] = (float)qm[k];
                c1f[k] = (float)C1[k];
                s1f[k] = (float)S1[k];
                qf[k] = (float)q[k];
                Gf[k] = Hf[k] = Jf[k] = Kf[k] = 0.f;
            }
            for (int m = kMixedSplit + 1; m <= L; ++m) {
                ColSums32<K> f;
                f.zero();
                const GravEntry32* e32 = gs.t32 + grav_col_offset(m, gs.Lt);
                const float4* p = reinterpret_cast<const float4*>(e32);
                const float4 a = p[0], b = p[1];
                float Q1f[K], Q2f[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const float2 QQ = make_float2(qmf[k], qmf[k]);
                    f.g[k] = __fmul2_rn(QQ, make_float2(a.z, a.w));
                    f.j[k] = __fmul2_rn(QQ, make_float2(b.x, b.y));
                    f.h[k] = __fmul2_rn(QQ, make_float2(b.z, b.w));
                    Q1f[k] = qmf[k];
                    Q2f[k] = 0.f;
                }
                column32k<K>(e32, 1, L - m, uf, wf, Q1f, Q2f, f);
                const float dm = (float)m;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    Gf[k] += cf[k] * f.g[k].x + sf[k] * f.g[k].y;
                    Jf[k] += dm * (cpf[k] * f.j[k].x + spf[k] * f.j[k].y);
                    Kf[k] -= dm * (spf[k] * f.j[k].x - cpf[k] * f.j[k].y);
                    Hf[k] += cpf[k] * f.h[k].x + spf[k] * f.h[k].y;
                    cpf[k] = cf[k];
                    spf[k] = sf[k];
                    const float cn = c1f[k] * cf[k] - s1f[k] * sf[k];
                    const float sn = s1f[k] * cf[k] + c1f[k] * sf[k];
                    cf[k] = cn;
                    sf[k] = sn;
                    qmf[k] *= qf[k];
                }
            }
#pragma unroll
            for (int k = 0; k < K; ++k) {
                G[k] += (double)Gf[k];
                H[k] += (double)Hf[k];
                J[k] += (double)Jf[k];
                KK[k] += (double)Kf[k];
            }
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) { // eq. 4-13
        const double Gk = G[k] + 1.0;
        const double Lambda = Gk + z[k] * H[k] / r[k];
        const double c = -gs.gm / (r[k] * r[k]);
        ax[k] = c * (Lambda * x[k] / r[k] - J[k]);
        ay[k] = c * (Lambda * y[k] / r[k] - KK[k]);
        az[k] = c * (Lambda * z[k] / r[k] - H[k]);
    }
}

// ---- mixed precision with compensated FP32 sums (GPOP_MIXED_COMPENSATED) ----
// The same split as the mixed walk (terms of degree <= 8 in FP64, every term of degree > 8 in
// FP32), with each FP32 column sum carried as a value and a compensation term: every product
// Q(n) x coefficient is added by Knuth's TwoSum, whose rounding error goes into the compensation
// (compensated summation). Each column's sum and compensation are then added to the FP64 column
// sums and combined in FP64. The walk is plain (one column at a time); it exists to measure the
// error and the cost of compensation against the two-level sums of the default mixed walk.

// s + c <- s + c + p, with the rounding error of s + p kept in c (TwoSum; no contraction).
__device__ __forceinline__ void two_sum_add(float& s, float& c, float p)
{
    const float t = __fadd_rn(s, p);
    const float z = __fsub_rn(t, s);
    const float e = __fadd_rn(__fsub_rn(s, __fsub_rn(t, z)), __fsub_rn(p, z));
    s = t;
    c = __fadd_rn(c, e);
}

// FP32 terms first..last of a column (entries e[first..last]) for K objects, continuing the
// recursion from Q1 = Q(n-1), Q2 = Q(n-2), compensated sums into sum/cmp [k][g1 g2 j1 j2 h1 h2].
template <int K>
__device__ __forceinline__ void column32_comp(const GravEntry32* __restrict__ e, int first, int last,
    const float (&u)[K], const float (&w)[K], float (&Q1)[K], float (&Q2)[K], float (&sum)[K][6],
    float (&cmp)[K][6])
{
    for (int i = first; i <= last; ++i) {
        const float4* p = reinterpret_cast<const float4*>(e + i);
        const float4 a = p[0], b = p[1]; // (-c, -c, g1, g2 | j1, j2, h1, h2)
        const float coef[6] = { a.z, a.w, b.x, b.y, b.z, b.w };
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const float t2 = (a.x * w[k]) * Q2[k];
            const float Q = fmaf(u[k], Q1[k], t2);
#pragma unroll
            for (int c = 0; c < 6; ++c)
                two_sum_add(sum[k][c], cmp[k][c], __fmul_rn(Q, coef[c]));
            Q2[k] = Q1[k];
            Q1[k] = Q;
        }
    }
}

template <int K>
__device__ __forceinline__ void gravity_itrs_comp(const GravSmem& gs, const double (&x)[K],
    const double (&y)[K], const double (&z)[K], double (&ax)[K], double (&ay)[K], double (&az)[K])
{
    const int L = gs.L;
    double r[K], q[K], u[K], w[K], C1[K], S1[K], Cm[K], Sm[K], Cp[K], Sp[K], qm[K];
    double G[K], H[K], J[K], KK[K];
    float uf[K], wf[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        r[k] = sqrt(x[k] * x[k] + y[k] * y[k] + z[k] * z[k]);
        const double eps = z[k] / r[k];
        q[k] = gs.radius / r[k];
        u[k] = q[k] * eps;
        w[k] = q[k] * q[k];
        C1[k] = x[k] / r[k];
        S1[k] = y[k] / r[k];
        Cm[k] = 1.0;
        Sm[k] = 0.0;
        Cp[k] = 0.0;
        Sp[k] = 0.0;
        qm[k] = 1.0;
        G[k] = H[k] = J[k] = KK[k] = 0.0;
        uf[k] = (float)u[k];
        wf[k] = (float)w[k];
    }
    for (int m = 0; m <= L; ++m) {
        ColSums64<K> s;
        s.zero();
        float sum[K][6], cmp[K][6], Q1f[K], Q2f[K];
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int c = 0; c < 6; ++c)
                sum[k][c] = cmp[k][c] = 0.f;
        const GravEntry32* e32 = gs.t32 + grav_col_offset(m, gs.Lt);
        if (m <= kMixedSplit) { // FP64 terms n = m..8, then FP32 terms 9..L
            double Q1[K], Q2[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                Q1[k] = qm[k];
                Q2[k] = 0.0;
            }
            const int top = L < kMixedSplit ? L : kMixedSplit;
            const GravEntry64* e = gs.t64 + grav_col_offset(m, kMixedSplit);
            s.add(e, Q1);
            column64<K>(e, 1, top - m, u, w, Q1, Q2, s);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                Q1f[k] = (float)Q1[k];
                Q2f[k] = (float)Q2[k];
            }
            column32_comp<K>(e32, kMixedSplit + 1 - m, L - m, uf, wf, Q1f, Q2f, sum, cmp);
        } else { // FP32 terms n = m..L: Q(m) = q^m, Q(m-1) = 0
            const float4* p = reinterpret_cast<const float4*>(e32);
            const float4 a = p[0], b = p[1];
            const float coef[6] = { a.z, a.w, b.x, b.y, b.z, b.w };
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const float Qm = (float)qm[k];
#pragma unroll
                for (int c = 0; c < 6; ++c)
                    sum[k][c] = __fmul_rn(Qm, coef[c]);
                Q1f[k] = Qm;
                Q2f[k] = 0.f;
            }
            column32_comp<K>(e32, 1, L - m, uf, wf, Q1f, Q2f, sum, cmp);
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            s.g1[k] += (double)sum[k][0] + (double)cmp[k][0];
            s.g2[k] += (double)sum[k][1] + (double)cmp[k][1];
            s.j1[k] += (double)sum[k][2] + (double)cmp[k][2];
            s.j2[k] += (double)sum[k][3] + (double)cmp[k][3];
            s.h1[k] += (double)sum[k][4] + (double)cmp[k][4];
            s.h2[k] += (double)sum[k][5] + (double)cmp[k][5];
        }
        const double dm = (double)m;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            G[k] += Cm[k] * s.g1[k] + Sm[k] * s.g2[k];
            J[k] += dm * (Cp[k] * s.j1[k] + Sp[k] * s.j2[k]);
            KK[k] -= dm * (Sp[k] * s.j1[k] - Cp[k] * s.j2[k]);
            H[k] += Cp[k] * s.h1[k] + Sp[k] * s.h2[k];
            Cp[k] = Cm[k];
            Sp[k] = Sm[k];
            const double Cn = C1[k] * Cm[k] - S1[k] * Sm[k];
            const double Sn = S1[k] * Cm[k] + C1[k] * Sm[k];
            Cm[k] = Cn;
            Sm[k] = Sn;
            qm[k] *= q[k];
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) { // eq. 4-13
        const double Gk = G[k] + 1.0;
        const double Lambda = Gk + z[k] * H[k] / r[k];
        const double c = -gs.gm / (r[k] * r[k]);
        ax[k] = c * (Lambda * x[k] / r[k] - J[k]);
        ay[k] = c * (Lambda * y[k] / r[k] - KK[k]);
        az[k] = c * (Lambda * z[k] / r[k] - H[k]);
    }
}

// GCRS accelerations of K objects at GCRS positions r[k] with the ITRS->GCRS matrix M
// (column-major): r_itrs = M^T r, a = M a_itrs (the two cublasDgemvStridedBatched of
// gravity_source.cu:176-210).
// LANE: the tables are in the lane layout, two objects (K = 2) and, in mixed mode, L > 8; the
// walk is then the two-column walk (the other cases have no plain-walk form in that layout).
template <bool MIXED, int K, bool LANE = false, bool COMP = false>
__device__ __forceinline__ void gravity_gcrs(const GravSmem& gs, const double* __restrict__ M,
    const double (&r)[K][3], double (&a)[K][3])
{
    double m[9];
#pragma unroll
    for (int i = 0; i < 9; ++i)
        m[i] = __ldg(M + i);
    double px[K], py[K], pz[K], ax[K], ay[K], az[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        px[k] = m[0] * r[k][0] + m[1] * r[k][1] + m[2] * r[k][2];
        py[k] = m[3] * r[k][0] + m[4] * r[k][1] + m[5] * r[k][2];
        pz[k] = m[6] * r[k][0] + m[7] * r[k][1] + m[8] * r[k][2];
    }
    if constexpr (COMP) {
        static_assert(MIXED && !LANE, "compensated sums belong to the plain mixed walk");
        gravity_itrs_comp<K>(gs, px, py, pz, ax, ay, az);
    } else if constexpr (LANE) {
        static_assert(K == 2, "the lane-layout two-column walk carries two objects");
        if constexpr (MIXED)
            gravity_itrs_groups<true>(gs, px, py, pz, ax, ay, az);
        else
            gravity_itrs_pairs64<true, 2>(gs, px, py, pz, ax, ay, az);
    } else {
        gravity_itrs<MIXED, K>(gs, px, py, pz, ax, ay, az);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
        a[k][0] = m[0] * ax[k] + m[3] * ay[k] + m[6] * az[k];
        a[k][1] = m[1] * ax[k] + m[4] * ay[k] + m[7] * az[k];
        a[k][2] = m[2] * ax[k] + m[5] * ay[k] + m[8] * az[k];
    }
}

// One object (startup, single-evaluation and unit kernels).
template <bool MIXED, bool COMP = false>
__device__ __forceinline__ void gravity_gcrs1(const GravSmem& gs, const double* __restrict__ M,
    const double* r, double* a)
{
    double rr[1][3] = { { r[0], r[1], r[2] } };
    double aa[1][3];
    gravity_gcrs<MIXED, 1, false, COMP>(gs, M, rr, aa);
    a[0] = aa[0][0];
    a[1] = aa[0][1];
    a[2] = aa[0][2];
}

template <bool MIXED>
__device__ __forceinline__ void gravity_itrs1(const GravSmem& gs, double x, double y, double z,
    double& ax, double& ay, double& az)
{
    double X[1] = { x }, Y[1] = { y }, Z[1] = { z }, AX[1], AY[1], AZ[1];
    gravity_itrs<MIXED, 1>(gs, X, Y, Z, AX, AY, AZ);
    ax = AX[0];
    ay = AY[0];
    az = AZ[0];
}

} // namespace gpop
