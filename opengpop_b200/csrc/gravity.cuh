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

// Unroll factors of the column walks (measured on B200, 65,536 objects at 70x70: the two-object
// FP32 walk runs 6 % faster at 8 than at 4, and 10 % slower at 32).
#ifndef GPOP_COL32X2_UNROLL
#define GPOP_COL32X2_UNROLL 8
#endif
#ifndef GPOP_COL64_UNROLL
#define GPOP_COL64_UNROLL 4
#endif
constexpr int kCol32x2Unroll = GPOP_COL32X2_UNROLL;
constexpr int kCol64Unroll = GPOP_COL64_UNROLL;

struct GravSmem {
    const GravEntry64* t64; // FP64 mode: full table; mixed mode: head table (n <= 8)
    const GravEntry32* t32; // mixed mode: full FP32 table (recursion constant stored negated, twice)
    int L; // degree summed (<= Lt)
    int Lt; // degree of the table layout (columns of Lt - m + 1 entries)
    double radius, gm;
    const int* cb64 = nullptr; // lane layout: first 16-byte unit of each FP64 (or head) column
    const int* cb32 = nullptr; // lane layout: the same for the FP32 table
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
#pragma unroll(kCol64Unroll)
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
#pragma unroll(kCol32x2Unroll)
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
