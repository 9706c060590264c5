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
// table entry loaded from shared memory feeds K independent chains.
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

struct GravSmem {
    const GravEntry64* t64; // FP64 mode: full table; mixed mode: head table (n <= 8)
    const GravEntry32* t32; // mixed mode: full FP32 table (recursion constant stored negated, twice)
    int L;
    double radius, gm;
};

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
#pragma unroll 4
    for (int i = first; i <= last; ++i) {
        const double cn = reinterpret_cast<const double2*>(e + i + 1)[0].x;
        double Q[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            Q[k] = fma(u[k], Q1[k], -t2[k]);
            t2[k] = (cn * w[k]) * Q1[k];
            Q2[k] = Q1[k];
            Q1[k] = Q[k];
        }
        s.add(e + i, Q);
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
__device__ __forceinline__ void column32x2(const GravEntry32* __restrict__ e, int first, int last,
    float2 u, float2 w, float2& Q1, float2& Q2, ColSums32<2>& s)
{
    if (first > last)
        return;
    const float4 a0 = reinterpret_cast<const float4*>(e + first)[0];
    float2 t2 = __fmul2_rn(__fmul2_rn(make_float2(a0.x, a0.y), w), Q2);
#pragma unroll 4
    for (int i = first; i <= last; ++i) {
        const float4* p = reinterpret_cast<const float4*>(e + i);
        const float4 a = p[0], b = p[1];
        const float4 an = reinterpret_cast<const float4*>(e + i + 1)[0];
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

// Accelerations of K objects in the Earth-fixed frame (eq. 4-13 of gravity_source_device.cu:212-239).
template <bool MIXED, int K>
__device__ __forceinline__ void gravity_itrs(const GravSmem& gs, const double (&x)[K],
    const double (&y)[K], const double (&z)[K], double (&ax)[K], double (&ay)[K], double (&az)[K])
{
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
    for (int m = 0; m <= L; ++m) {
        ColSums64<K> s;
        s.zero();
        double Q1[K], Q2[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            Q1[k] = qm[k];
            Q2[k] = 0.0;
        }
        if constexpr (!MIXED) {
            const GravEntry64* e = gs.t64 + grav_col_offset(m, L);
            s.add(e, Q1); // n = m
            column64<K>(e, 1, L - m, u, w, Q1, Q2, s);
        } else {
            ColSums32<K> f;
            f.zero();
            const GravEntry32* e32 = gs.t32 + grav_col_offset(m, L);
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

// ---- one object, two cursors ----
// The triangle is split at column kSplit(L) into two contiguous groups of columns with about the
// same number of terms; one thread walks both groups in lockstep (two independent recursion and
// accumulation chains), so the FP pipes see twice the independent work per warp without more
// threads per object. All lanes of a warp hold different objects but walk the same entries, so
// control flow stays uniform.
__host__ __device__ __forceinline__ int cursor_split(int L)
{
    const int E = (L + 1) * (L + 2) / 2;
    int m = 0;
    while (m < L && grav_col_offset(m + 1, L) <= E / 2)
        ++m;
    return m + 1; // first column of the second group
}

struct Col64 {
    double Q1, Q2, g1, g2, j1, j2, h1, h2;
    double Cm, Sm, Cp, Sp, qm;
    int m, i, last; // current column, next entry in it, last column of the group
};

__device__ __forceinline__ void col64_step(Col64& c, const GravEntry64* __restrict__ e, double u, double w)
{
    const double2* p = reinterpret_cast<const double2*>(e);
    const double cc = p[0].x;
    const double2 g = p[1], j = p[2], h = p[3];
    const double Q = fma(u, c.Q1, -(cc * w) * c.Q2);
    c.g1 = fma(g.x, Q, c.g1);
    c.g2 = fma(g.y, Q, c.g2);
    c.j1 = fma(j.x, Q, c.j1);
    c.j2 = fma(j.y, Q, c.j2);
    c.h1 = fma(h.x, Q, c.h1);
    c.h2 = fma(h.y, Q, c.h2);
    c.Q2 = c.Q1;
    c.Q1 = Q;
}

struct ObjTotals {
    double G, H, J, K;
};

// eq. 4-11 column combination, then the eq. 3-18 step to the next column.
__device__ __forceinline__ void col64_finish(Col64& c, ObjTotals& t, double C1, double S1, double q)
{
    const double dm = (double)c.m;
    t.G += c.Cm * c.g1 + c.Sm * c.g2;
    t.J += dm * (c.Cp * c.j1 + c.Sp * c.j2);
    t.K -= dm * (c.Sp * c.j1 - c.Cp * c.j2);
    t.H += c.Cp * c.h1 + c.Sp * c.h2;
    c.Cp = c.Cm;
    c.Sp = c.Sm;
    const double Cn = C1 * c.Cm - S1 * c.Sm;
    const double Sn = S1 * c.Cm + C1 * c.Sm;
    c.Cm = Cn;
    c.Sm = Sn;
    c.qm *= q;
    c.m += 1;
}

// Opens column c.m: n = m term with Q = q^m.
__device__ __forceinline__ void col64_open(Col64& c, const GravEntry64* __restrict__ tab, int L)
{
    const GravEntry64* e = tab + grav_col_offset(c.m, L);
    const double2* p = reinterpret_cast<const double2*>(e);
    const double2 g = p[1], j = p[2], h = p[3];
    c.Q1 = c.qm;
    c.Q2 = 0.0;
    c.g1 = g.x * c.Q1;
    c.g2 = g.y * c.Q1;
    c.j1 = j.x * c.Q1;
    c.j2 = j.y * c.Q1;
    c.h1 = h.x * c.Q1;
    c.h2 = h.y * c.Q1;
    c.i = 1;
}

__device__ __forceinline__ void cursor_seed(Col64& c, int m0, int last, double C1, double S1, double q)
{
    c.Cm = 1.0;
    c.Sm = 0.0;
    c.Cp = 0.0;
    c.Sp = 0.0;
    c.qm = 1.0;
    for (int m = 0; m < m0; ++m) { // the same recursion as walking the columns one by one
        c.Cp = c.Cm;
        c.Sp = c.Sm;
        const double Cn = C1 * c.Cm - S1 * c.Sm;
        const double Sn = S1 * c.Cm + C1 * c.Sm;
        c.Cm = Cn;
        c.Sm = Sn;
        c.qm *= q;
    }
    c.m = m0;
    c.last = last;
}

__device__ __forceinline__ void gravity_itrs_fp64_c2(const GravSmem& gs, double x, double y,
    double z, double& ax, double& ay, double& az)
{
    const int L = gs.L;
    const double r = sqrt(x * x + y * y + z * z);
    const double eps = z / r;
    const double q = gs.radius / r;
    const double u = q * eps, w = q * q;
    const double C1 = x / r, S1 = y / r;
    ObjTotals t { 0.0, 0.0, 0.0, 0.0 };
    const int split = cursor_split(L);
    Col64 A, B;
    cursor_seed(A, 0, split - 1, C1, S1, q);
    cursor_seed(B, split, L, C1, S1, q);
    col64_open(A, gs.t64, L);
    col64_open(B, gs.t64, L);
    bool a_on = true, b_on = split <= L;
    while (a_on || b_on) {
        if (a_on && b_on) {
            const int ra = (L - A.m) - A.i + 1, rb = (L - B.m) - B.i + 1;
            const int k = ra < rb ? ra : rb;
            const GravEntry64* ea = gs.t64 + grav_col_offset(A.m, L) + A.i;
            const GravEntry64* eb = gs.t64 + grav_col_offset(B.m, L) + B.i;
#pragma unroll 2
            for (int s = 0; s < k; ++s) {
                col64_step(A, ea + s, u, w);
                col64_step(B, eb + s, u, w);
            }
            A.i += k;
            B.i += k;
        } else if (a_on) {
            const GravEntry64* ea = gs.t64 + grav_col_offset(A.m, L);
#pragma unroll 2
            for (int s = A.i; s <= L - A.m; ++s)
                col64_step(A, ea + s, u, w);
            A.i = L - A.m + 1;
        } else {
            const GravEntry64* eb = gs.t64 + grav_col_offset(B.m, L);
#pragma unroll 2
            for (int s = B.i; s <= L - B.m; ++s)
                col64_step(B, eb + s, u, w);
            B.i = L - B.m + 1;
        }
        if (a_on && A.i > L - A.m) {
            const bool more = A.m < A.last;
            col64_finish(A, t, C1, S1, q);
            if (more)
                col64_open(A, gs.t64, L);
            else
                a_on = false;
        }
        if (b_on && B.i > L - B.m) {
            const bool more = B.m < B.last;
            col64_finish(B, t, C1, S1, q);
            if (more)
                col64_open(B, gs.t64, L);
            else
                b_on = false;
        }
    }
    const double G = t.G + 1.0; // eq. 4-13
    const double Lambda = G + z * t.H / r;
    const double c = -gs.gm / (r * r);
    ax = c * (Lambda * x / r - t.J);
    ay = c * (Lambda * y / r - t.K);
    az = c * (Lambda * z / r - t.H);
}

// Mixed precision with two cursors: FP32 lockstep walk over the n > 8 entries; the FP64 head
// (n <= 8) of a column m <= 8 runs when the cursor opens that column.
struct Col32 {
    float Q1, Q2;
    float2 g, j, h;
    double Cm, Sm, Cp, Sp, qm;
    int m, i, last;
};

__device__ __forceinline__ void col32_step(Col32& c, const GravEntry32* __restrict__ e, float u, float w)
{
    const float4* p = reinterpret_cast<const float4*>(e);
    const float4 a = p[0], b = p[1];
    const float Q = fmaf(u, c.Q1, (a.x * w) * c.Q2);
    const float2 QQ = make_float2(Q, Q);
    c.g = __ffma2_rn(QQ, make_float2(a.z, a.w), c.g);
    c.j = __ffma2_rn(QQ, make_float2(b.x, b.y), c.j);
    c.h = __ffma2_rn(QQ, make_float2(b.z, b.w), c.h);
    c.Q2 = c.Q1;
    c.Q1 = Q;
}

__device__ __forceinline__ void col32_finish(Col32& c, ObjTotals& t, double C1, double S1, double q)
{
    const double dm = (double)c.m;
    const double g1 = c.g.x, g2 = c.g.y, j1 = c.j.x, j2 = c.j.y, h1 = c.h.x, h2 = c.h.y;
    t.G += c.Cm * g1 + c.Sm * g2;
    t.J += dm * (c.Cp * j1 + c.Sp * j2);
    t.K -= dm * (c.Sp * j1 - c.Cp * j2);
    t.H += c.Cp * h1 + c.Sp * h2;
    c.Cp = c.Cm;
    c.Sp = c.Sm;
    const double Cn = C1 * c.Cm - S1 * c.Sm;
    const double Sn = S1 * c.Cm + C1 * c.Sm;
    c.Cm = Cn;
    c.Sm = Sn;
    c.qm *= q;
    c.m += 1;
}

// Opens column c.m in mixed mode; returns with c.i = first FP32 entry of the column.
__device__ __forceinline__ void col32_open(Col32& c, const GravSmem& gs, ObjTotals& t, double u,
    double w)
{
    const int L = gs.L;
    const GravEntry32* e32 = gs.t32 + grav_col_offset(c.m, L);
    c.g = c.j = c.h = make_float2(0.f, 0.f);
    if (c.m <= kMixedSplit) {
        // FP64 head n = m..min(8, L), combined into the totals right away
        const int top = L < kMixedSplit ? L : kMixedSplit;
        const GravEntry64* e = gs.t64 + grav_col_offset(c.m, kMixedSplit);
        double Q1[1] = { c.qm }, Q2[1] = { 0.0 };
        ColSums64<1> s;
        s.zero();
        s.add(e, Q1);
        const double uu[1] = { u }, ww[1] = { w };
        column64<1>(e, 1, top - c.m, uu, ww, Q1, Q2, s);
        const double dm = (double)c.m;
        t.G += c.Cm * s.g1[0] + c.Sm * s.g2[0];
        t.J += dm * (c.Cp * s.j1[0] + c.Sp * s.j2[0]);
        t.K -= dm * (c.Sp * s.j1[0] - c.Cp * s.j2[0]);
        t.H += c.Cp * s.h1[0] + c.Sp * s.h2[0];
        c.Q1 = (float)Q1[0];
        c.Q2 = (float)Q2[0];
        c.i = kMixedSplit + 1 - c.m;
    } else {
        const float4* p = reinterpret_cast<const float4*>(e32);
        const float4 a = p[0], b = p[1];
        const float Qm = (float)c.qm;
        const float2 QQ = make_float2(Qm, Qm);
        c.g = __fmul2_rn(QQ, make_float2(a.z, a.w));
        c.j = __fmul2_rn(QQ, make_float2(b.x, b.y));
        c.h = __fmul2_rn(QQ, make_float2(b.z, b.w));
        c.Q1 = Qm;
        c.Q2 = 0.f;
        c.i = 1;
    }
}

__device__ __forceinline__ void gravity_itrs_mixed_c2(const GravSmem& gs, double x, double y,
    double z, double& ax, double& ay, double& az)
{
    const int L = gs.L;
    const double r = sqrt(x * x + y * y + z * z);
    const double eps = z / r;
    const double q = gs.radius / r;
    const double u = q * eps, w = q * q;
    const float uf = (float)u, wf = (float)w;
    const double C1 = x / r, S1 = y / r;
    ObjTotals t { 0.0, 0.0, 0.0, 0.0 };
    const int split = cursor_split(L);
    Col32 A, B;
    {
        Col64 tmp;
        cursor_seed(tmp, 0, split - 1, C1, S1, q);
        A.Cm = tmp.Cm; A.Sm = tmp.Sm; A.Cp = tmp.Cp; A.Sp = tmp.Sp; A.qm = tmp.qm; A.m = tmp.m; A.last = tmp.last;
        cursor_seed(tmp, split, L, C1, S1, q);
        B.Cm = tmp.Cm; B.Sm = tmp.Sm; B.Cp = tmp.Cp; B.Sp = tmp.Sp; B.qm = tmp.qm; B.m = tmp.m; B.last = tmp.last;
    }
    col32_open(A, gs, t, u, w);
    bool a_on = true, b_on = split <= L;
    if (b_on)
        col32_open(B, gs, t, u, w);
    while (a_on || b_on) {
        if (a_on && b_on) {
            const int ra = (L - A.m) - A.i + 1, rb = (L - B.m) - B.i + 1;
            const int k = ra < rb ? ra : rb;
            const GravEntry32* ea = gs.t32 + grav_col_offset(A.m, L) + A.i;
            const GravEntry32* eb = gs.t32 + grav_col_offset(B.m, L) + B.i;
#pragma unroll 2
            for (int s = 0; s < k; ++s) {
                col32_step(A, ea + s, uf, wf);
                col32_step(B, eb + s, uf, wf);
            }
            A.i += k;
            B.i += k;
        } else if (a_on) {
            const GravEntry32* ea = gs.t32 + grav_col_offset(A.m, L);
#pragma unroll 2
            for (int s = A.i; s <= L - A.m; ++s)
                col32_step(A, ea + s, uf, wf);
            A.i = L - A.m + 1;
        } else {
            const GravEntry32* eb = gs.t32 + grav_col_offset(B.m, L);
#pragma unroll 2
            for (int s = B.i; s <= L - B.m; ++s)
                col32_step(B, eb + s, uf, wf);
            B.i = L - B.m + 1;
        }
        if (a_on && A.i > L - A.m) {
            const bool more = A.m < A.last;
            col32_finish(A, t, C1, S1, q);
            if (more)
                col32_open(A, gs, t, u, w);
            else
                a_on = false;
        }
        if (b_on && B.i > L - B.m) {
            const bool more = B.m < B.last;
            col32_finish(B, t, C1, S1, q);
            if (more)
                col32_open(B, gs, t, u, w);
            else
                b_on = false;
        }
    }
    const double G = t.G + 1.0; // eq. 4-13
    const double Lambda = G + z * t.H / r;
    const double c = -gs.gm / (r * r);
    ax = c * (Lambda * x / r - t.J);
    ay = c * (Lambda * y / r - t.K);
    az = c * (Lambda * z / r - t.H);
}

template <bool MIXED>
__device__ __forceinline__ void gravity_gcrs_c2(const GravSmem& gs, const double* __restrict__ M,
    const double (&r)[1][3], double (&a)[1][3])
{
    double m[9];
#pragma unroll
    for (int i = 0; i < 9; ++i)
        m[i] = __ldg(M + i);
    const double px = m[0] * r[0][0] + m[1] * r[0][1] + m[2] * r[0][2];
    const double py = m[3] * r[0][0] + m[4] * r[0][1] + m[5] * r[0][2];
    const double pz = m[6] * r[0][0] + m[7] * r[0][1] + m[8] * r[0][2];
    double ax, ay, az;
    if constexpr (MIXED)
        gravity_itrs_mixed_c2(gs, px, py, pz, ax, ay, az);
    else
        gravity_itrs_fp64_c2(gs, px, py, pz, ax, ay, az);
    a[0][0] = m[0] * ax + m[3] * ay + m[6] * az;
    a[0][1] = m[1] * ax + m[4] * ay + m[7] * az;
    a[0][2] = m[2] * ax + m[5] * ay + m[8] * az;
}

// GCRS accelerations of K objects at GCRS positions r[k] with the ITRS->GCRS matrix M
// (column-major): r_itrs = M^T r, a = M a_itrs (the two cublasDgemvStridedBatched of
// gravity_source.cu:176-210).
template <bool MIXED, int K>
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
    gravity_itrs<MIXED, K>(gs, px, py, pz, ax, ay, az);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        a[k][0] = m[0] * ax[k] + m[3] * ay[k] + m[6] * az[k];
        a[k][1] = m[1] * ax[k] + m[4] * ay[k] + m[7] * az[k];
        a[k][2] = m[2] * ax[k] + m[5] * ay[k] + m[8] * az[k];
    }
}

// One object (startup, single-evaluation and unit kernels).
template <bool MIXED>
__device__ __forceinline__ void gravity_gcrs1(const GravSmem& gs, const double* __restrict__ M,
    const double* r, double* a)
{
    double rr[1][3] = { { r[0], r[1], r[2] } };
    double aa[1][3];
    gravity_gcrs<MIXED, 1>(gs, M, rr, aa);
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
