// gravity.cuh -- fused normalised spherical-harmonic gravity (Gottlieb's derived-Legendre method,
// as in lib/force_model/src/acceleration/gravity_source_device.cu:63-239), one object per thread.
//
// The reference builds the whole P-bar triangle, four N x T term arrays and two Thrust segment
// reductions in HBM per evaluation (about 25 launches). Here each thread walks the triangle column
// by column with a two-term recursion held in registers, reading the pre-scaled coefficient table
// from shared memory by broadcast (every lane of a warp reads the same entry). Per (n, m) term:
// 3 FP64 ops for the recursion and 6 FMAs into per-column sums; per column the sums are combined
// with the cos/sin(m lambda) recursion of eq. 3-18. The (R/r)^n factor of eq. 4-12 rides in the
// recursion variable, so no per-degree sums are needed.
//
// Mixed precision: terms of degree n <= 8 (and all per-column combining, the central term, frame
// rotations and the final assembly) stay FP64; the n > 8 recursion and sums run in FP32 with
// packed f32x2 FMAs, per column, and each column's FP32 sums are added into the FP64 totals
// (two-level summation: at most 62 FP32 terms per partial sum).
#pragma once
#include "common.cuh"
#include "model.h"

namespace gpop {

constexpr int kMixedSplit = 8; // highest degree kept in FP64 in the mixed mode

struct GravSmem {
    const GravEntry64* t64; // FP64 mode: full table; mixed mode: head table (n <= 8)
    const GravEntry32* t32; // mixed mode: full FP32 table
    int L;
    double radius, gm;
};

__device__ __forceinline__ void col_accum64(const GravEntry64* __restrict__ e, double Q, double& g1,
    double& g2, double& j1, double& j2, double& h1, double& h2)
{
    const double2* p = reinterpret_cast<const double2*>(e);
    double2 g = p[1], j = p[2], h = p[3];
    g1 = fma(g.x, Q, g1);
    g2 = fma(g.y, Q, g2);
    j1 = fma(j.x, Q, j1);
    j2 = fma(j.y, Q, j2);
    h1 = fma(h.x, Q, h1);
    h2 = fma(h.y, Q, h2);
}

// Walks column entries e[first..last] (n = m + first .. m + last) in FP64, continuing the
// recursion from (Q1, Q2) = (Q(n-1), Q(n-2)).
__device__ __forceinline__ void column64(const GravEntry64* __restrict__ e, int first, int last,
    double u, double w, double& Q1, double& Q2, double& g1, double& g2, double& j1, double& j2,
    double& h1, double& h2)
{
#pragma unroll 2
    for (int k = first; k <= last; ++k) {
        double c = reinterpret_cast<const double2*>(e + k)[0].x;
        double Q = fma(u, Q1, -(c * w) * Q2);
        col_accum64(e + k, Q, g1, g2, j1, j2, h1, h2);
        Q2 = Q1;
        Q1 = Q;
    }
}

__device__ __forceinline__ void column32(const GravEntry32* __restrict__ e, int first, int last,
    float u, float w, float& Q1, float& Q2, float2& g, float2& j, float2& h)
{
#pragma unroll 2
    for (int k = first; k <= last; ++k) {
        const float4* p = reinterpret_cast<const float4*>(e + k);
        float4 a = p[0]; // c, pad, g1, g2
        float4 b = p[1]; // j1, j2, h1, h2
        float Q = fmaf(u, Q1, -(a.x * w) * Q2);
        float2 QQ = make_float2(Q, Q);
        g = __ffma2_rn(QQ, make_float2(a.z, a.w), g);
        j = __ffma2_rn(QQ, make_float2(b.x, b.y), j);
        h = __ffma2_rn(QQ, make_float2(b.z, b.w), h);
        Q2 = Q1;
        Q1 = Q;
    }
}

// Acceleration in the Earth-fixed frame (eq. 4-13 of gravity_source_device.cu:212-239).
template <bool MIXED>
__device__ __forceinline__ void gravity_itrs(const GravSmem& gs, double x, double y, double z,
    double& ax, double& ay, double& az)
{
    const int L = gs.L;
    const double r = sqrt(x * x + y * y + z * z);
    const double eps = z / r; // eq. 3-3
    const double q = gs.radius / r;
    const double u = q * eps;
    const double w = q * q;
    const double C1 = x / r, S1 = y / r; // eq. 3-18 seeds
    double Cm = 1.0, Sm = 0.0, Cp = 0.0, Sp = 0.0; // C_m, S_m and C_{m-1}, S_{m-1}
    double qm = 1.0; // q^m
    double G = 0.0, H = 0.0, J = 0.0, K = 0.0;
    const float uf = (float)u, wf = (float)w;
    for (int m = 0; m <= L; ++m) {
        double g1 = 0, g2 = 0, j1 = 0, j2 = 0, h1 = 0, h2 = 0;
        double Q1 = qm, Q2 = 0.0;
        if (!MIXED) {
            const GravEntry64* e = gs.t64 + grav_col_offset(m, L);
            col_accum64(e, Q1, g1, g2, j1, j2, h1, h2); // n = m
            column64(e, 1, L - m, u, w, Q1, Q2, g1, g2, j1, j2, h1, h2);
        } else {
            float2 fg = make_float2(0.f, 0.f), fj = fg, fh = fg;
            const GravEntry32* e32 = gs.t32 + grav_col_offset(m, L);
            if (m <= kMixedSplit) {
                const int top = L < kMixedSplit ? L : kMixedSplit;
                const GravEntry64* e = gs.t64 + grav_col_offset(m, kMixedSplit);
                col_accum64(e, Q1, g1, g2, j1, j2, h1, h2);
                column64(e, 1, top - m, u, w, Q1, Q2, g1, g2, j1, j2, h1, h2);
                float Q1f = (float)Q1, Q2f = (float)Q2;
                column32(e32, kMixedSplit + 1 - m, L - m, uf, wf, Q1f, Q2f, fg, fj, fh);
            } else {
                float Q1f = (float)qm, Q2f = 0.f;
                const float4* p = reinterpret_cast<const float4*>(e32);
                float4 a = p[0], b = p[1];
                float2 QQ = make_float2(Q1f, Q1f);
                fg = __ffma2_rn(QQ, make_float2(a.z, a.w), fg);
                fj = __ffma2_rn(QQ, make_float2(b.x, b.y), fj);
                fh = __ffma2_rn(QQ, make_float2(b.z, b.w), fh);
                column32(e32, 1, L - m, uf, wf, Q1f, Q2f, fg, fj, fh);
            }
            g1 += (double)fg.x;
            g2 += (double)fg.y;
            j1 += (double)fj.x;
            j2 += (double)fj.y;
            h1 += (double)fh.x;
            h2 += (double)fh.y;
        }
        // eq. 4-11 per column: G with (C_m, S_m); J, K, H with (C_{m-1}, S_{m-1})
        const double dm = (double)m;
        G += Cm * g1 + Sm * g2;
        J += dm * (Cp * j1 + Sp * j2);
        K -= dm * (Sp * j1 - Cp * j2);
        H += Cp * h1 + Sp * h2;
        Cp = Cm;
        Sp = Sm;
        const double Cn = C1 * Cm - S1 * Sm;
        const double Sn = S1 * Cm + C1 * Sm;
        Cm = Cn;
        Sm = Sn;
        qm *= q;
    }
    // eq. 4-13
    G = G + 1.0;
    const double Lambda = G + z * H / r;
    const double c = -gs.gm / (r * r);
    ax = c * (Lambda * x / r - J);
    ay = c * (Lambda * y / r - K);
    az = c * (Lambda * z / r - H);
}

// GCRS acceleration at GCRS position r with the ITRS->GCRS matrix M (column-major, 9 doubles):
// r_itrs = M^T r, a = M a_itrs (the two cublasDgemvStridedBatched of gravity_source.cu:176-210).
template <bool MIXED>
__device__ __forceinline__ void gravity_gcrs(const GravSmem& gs, const double* __restrict__ M,
    const double* r, double* a)
{
    double m[9];
#pragma unroll
    for (int i = 0; i < 9; ++i)
        m[i] = __ldg(M + i);
    const double px = m[0] * r[0] + m[1] * r[1] + m[2] * r[2];
    const double py = m[3] * r[0] + m[4] * r[1] + m[5] * r[2];
    const double pz = m[6] * r[0] + m[7] * r[1] + m[8] * r[2];
    double ax, ay, az;
    gravity_itrs<MIXED>(gs, px, py, pz, ax, ay, az);
    a[0] = m[0] * ax + m[3] * ay + m[6] * az;
    a[1] = m[1] * ax + m[4] * ay + m[7] * az;
    a[2] = m[2] * ax + m[5] * ay + m[8] * az;
}

__device__ __forceinline__ void gravity_identity_fp64(const GravSmem& gs, const double* r, double* a, bool mixed)
{
    if (mixed)
        gravity_itrs<true>(gs, r[0], r[1], r[2], a[0], a[1], a[2]);
    else
        gravity_itrs<false>(gs, r[0], r[1], r[2], a[0], a[1], a[2]);
}

} // namespace gpop
