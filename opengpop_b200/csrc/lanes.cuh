// lanes.cuh -- gravity with the columns of the triangle split over the P lanes of an object
// (lane l of P takes m = l, l + P, ...); the per-object sums are added with warp shuffles among
// the lanes named by `mask` (the whole warp, or the object's aligned group of P lanes), so every
// lane of the object ends with the same result. Used where one object per thread leaves
// the GPU idle: long single requests of a batch and the variational/adjoint kernels. The tables
// are in the lane layout (build_lane_blob), so the lanes' simultaneous reads of different columns
// fall in different shared-memory banks.
#pragma once
#include "gravity.cuh"
#include "kernels.h"

namespace gpop {

// Lane setup by prefix products over the object's lanes (log2 P shuffle steps) instead of each
// lane's own powers of (C1 + i S1) and q (tuned batch rates on B200, object-steps/s per SM:
// degree 8 with 32 lanes 3.5e5 -> 4.7e5, degree 70 with 32 lanes 1.49e5 -> 1.65e5).
#ifndef GPOP_LANE_SCAN
#define GPOP_LANE_SCAN 1
#endif
constexpr bool kLaneScan = GPOP_LANE_SCAN != 0;

// Stages a lane-layout blob into shared memory (after a 128-byte mbarrier slot) and binds it.
__device__ __forceinline__ bool bind_lane_table(uint8_t* smem, const TableSrc& ts, unsigned* err, GravSmem& g)
{
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem);
    uint8_t* tab = smem + 128;
    const bool ok = stage_to_smem(tab, ts.src, ts.bytes, mbar, err, ts.wait_spins);
    g.L = ts.L;
    g.Lt = ts.L;
    g.radius = ts.radius;
    g.gm = ts.gm;
    g.cb64 = reinterpret_cast<const int*>(tab);
    g.cb32 = reinterpret_cast<const int*>(tab + 512);
    g.t64 = reinterpret_cast<const GravEntry64*>(tab + kLaneOff64);
    g.t32 = reinterpret_cast<const GravEntry32*>(tab + ts.off32);
    return ok;
}

__device__ __forceinline__ void cmul(double ac, double as, double bc, double bs, double& rc, double& rs)
{
    const double c = ac * bc - as * bs;
    const double s = as * bc + ac * bs;
    rc = c;
    rs = s;
}

#ifndef GPOP_LANE_PAIR_COLUMNS
#define GPOP_LANE_PAIR_COLUMNS 1
#endif
constexpr bool kLanePairColumns = GPOP_LANE_PAIR_COLUMNS != 0;

// Eq. 4-11 for column m of a lane walk, then the lane's cos/sin(m lambda) and q^m recursions step
// P columns on (z^P; from column 0 the m - 1 values jump to z^(P-1)).
template <int K>
__device__ __forceinline__ void lane_combine(int m, const ColSums64<K>& s, const double (&CP)[K],
    const double (&SP)[K], const double (&CPm1)[K], const double (&SPm1)[K], const double (&qP)[K],
    double (&Cm)[K], double (&Sm)[K], double (&Cp)[K], double (&Sp)[K], double (&qm)[K],
    double (&G)[K], double (&H)[K], double (&J)[K], double (&KK)[K])
{
    const double dm = (double)m;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        G[k] += Cm[k] * s.g1[k] + Sm[k] * s.g2[k];
        J[k] += dm * (Cp[k] * s.j1[k] + Sp[k] * s.j2[k]);
        KK[k] -= dm * (Sp[k] * s.j1[k] - Cp[k] * s.j2[k]);
        H[k] += Cp[k] * s.h1[k] + Sp[k] * s.h2[k];
        if (m == 0) {
            Cp[k] = CPm1[k];
            Sp[k] = SPm1[k];
        } else {
            cmul(Cp[k], Sp[k], CP[k], SP[k], Cp[k], Sp[k]);
        }
        cmul(Cm[k], Sm[k], CP[k], SP[k], Cm[k], Sm[k]);
        qm[k] *= qP[k];
    }
}

// (C1 + i S1)^p by binary powering (p >= 0).
__device__ __forceinline__ void cpow(double c1, double s1, int p, double& rc, double& rs)
{
    double xc = 1.0, xs = 0.0, bc = c1, bs = s1;
    while (p > 0) {
        if (p & 1)
            cmul(xc, xs, bc, bs, xc, xs);
        p >>= 1;
        if (p)
            cmul(bc, bs, bc, bs, bc, bs);
    }
    rc = xc;
    rs = xs;
}

// Gravity in the Earth-fixed frame of K objects with the columns split over the P lanes of each
// object's group (lane l takes columns l, l + P, ...); the per-object totals are added across the
// P lanes. As gravity_itrs in mixed mode: the head columns m <= 8 are combined in FP64 (their
// terms of degree > 8 summed in FP32 per column), the columns m > 8 are walked, combined and
// summed in FP32 and added to the FP64 totals once. PAIRS: FP64 lanes walk two of their columns
// side by side (the one-object GJ8 lane kernel; kernels with fewer registers to spare keep one at a
// time).
template <bool MIXED, int K, bool PAIRS = false>
__device__ __forceinline__ void gravity_itrs_lk(const GravSmem& gs, int l, int P, const double (&x)[K],
    const double (&y)[K], const double (&z)[K], double (&ax)[K], double (&ay)[K], double (&az)[K],
    unsigned mask)
{
    const int L = gs.L;
    double r[K], q[K], u[K], w[K], C1[K], S1[K], CP[K], SP[K], Cm[K], Sm[K], Cp[K], Sp[K], CPm1[K], SPm1[K];
    double qm[K], qP[K], G[K], H[K], J[K], KK[K];
    float uf[K], wf[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        r[k] = sqrt(x[k] * x[k] + y[k] * y[k] + z[k] * z[k]);
        const double eps = z[k] / r[k];
        q[k] = gs.radius / r[k];
        u[k] = q[k] * eps;
        w[k] = q[k] * q[k];
        uf[k] = (float)u[k];
        wf[k] = (float)w[k];
        C1[k] = x[k] / r[k];
        S1[k] = y[k] / r[k];
        G[k] = H[k] = J[k] = KK[k] = 0.0;
        if (kLaneScan && P > 1) {
            // prefix products over the group's lanes (segments of width P): lane l ends with
            // z^(l+1) and q^(l+1), z = C1 + i S1; the lane's first column, the step between its
            // columns and the m - 1 values follow by shuffles
            double zc = C1[k], zs = S1[k], zq = q[k];
            for (int o = 1; o < P; o <<= 1) {
                const double pc = __shfl_up_sync(mask, zc, o, P), ps = __shfl_up_sync(mask, zs, o, P);
                const double pq = __shfl_up_sync(mask, zq, o, P);
                if (l >= o) {
                    cmul(pc, ps, zc, zs, zc, zs);
                    zq = pq * zq;
                }
            }
            const double c1 = __shfl_up_sync(mask, zc, 1, P), s1 = __shfl_up_sync(mask, zs, 1, P);
            const double q1 = __shfl_up_sync(mask, zq, 1, P);
            const double c2 = __shfl_up_sync(mask, zc, 2, P), s2 = __shfl_up_sync(mask, zs, 2, P);
            Cm[k] = l >= 1 ? c1 : 1.0; // z^l
            Sm[k] = l >= 1 ? s1 : 0.0;
            qm[k] = l >= 1 ? q1 : 1.0; // q^l
            Cp[k] = l >= 2 ? c2 : (l == 1 ? 1.0 : 0.0); // z^(l-1); column 0 has no J, K or H part
            Sp[k] = l >= 2 ? s2 : 0.0;
            CP[k] = __shfl_sync(mask, zc, P - 1, P); // z^P: step between this lane's columns
            SP[k] = __shfl_sync(mask, zs, P - 1, P);
            qP[k] = __shfl_sync(mask, zq, P - 1, P);
            CPm1[k] = __shfl_sync(mask, zc, P - 2, P); // z^(P-1): the m - 1 values of column P
            SPm1[k] = __shfl_sync(mask, zs, P - 2, P);
            continue;
        }
        cpow(C1[k], S1[k], P, CP[k], SP[k]); // step between this lane's columns
        cpow(C1[k], S1[k], l, Cm[k], Sm[k]);
        if (l > 0)
            cpow(C1[k], S1[k], l - 1, Cp[k], Sp[k]);
        else
            Cp[k] = Sp[k] = 0.0; // column 0 has no J, K or H part
        cpow(C1[k], S1[k], P - 1, CPm1[k], SPm1[k]); // the m - 1 values of column P
        qm[k] = 1.0;
        qP[k] = 1.0;
        for (int i = 0; i < l; ++i)
            qm[k] *= q[k];
        for (int i = 0; i < P; ++i)
            qP[k] *= q[k];
    }
    const int Lhead = (MIXED && L > kMixedSplit) ? kMixedSplit : L;
    // column bases of the lane's next column are read one column ahead (they are shared-memory
    // loads the walk's first table read depends on)
    int b64 = gs.cb64[l], b32 = gs.cb32[l];
    int m = l;
    if constexpr (!MIXED && PAIRS && kLanePairColumns) {
        // FP64: two of this lane's columns (m and m + P) side by side, so each object carries two
        // independent recursions; each column's sums, and their combination, in the order of the
        // one-column loop below (bit-identical accelerations)
        for (; m + P <= Lhead; m += 2 * P) {
            const int mb = m + P;
            const int mn = mb + P < 127 ? mb + P : 127;
            const int bb64 = gs.cb64[mb], nb64 = gs.cb64[mn];
            ColSums64<K> sa, sb;
            sa.zero();
            sb.zero();
            double Qa1[K], Qa2[K], Qb1[K], Qb2[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                Qa1[k] = qm[k];
                Qa2[k] = 0.0;
                Qb1[k] = qm[k] * qP[k]; // the q^m the one-column loop carries into column m + P
                Qb2[k] = 0.0;
            }
            const GravEntry64* ea = reinterpret_cast<const GravEntry64*>(reinterpret_cast<const uint4*>(gs.t64) + b64);
            const GravEntry64* eb = reinterpret_cast<const GravEntry64*>(reinterpret_cast<const uint4*>(gs.t64) + bb64);
            sa.add(ea, Qa1);
            sb.add(eb, Qb1);
            column64_pair<K>(ea + 1, eb + 1, Lhead - mb, u, w, Qa1, Qa2, sa, Qb1, Qb2, sb);
            column64<K>(ea, Lhead - mb + 1, Lhead - m, u, w, Qa1, Qa2, sa);
            lane_combine<K>(m, sa, CP, SP, CPm1, SPm1, qP, Cm, Sm, Cp, Sp, qm, G, H, J, KK);
            lane_combine<K>(mb, sb, CP, SP, CPm1, SPm1, qP, Cm, Sm, Cp, Sp, qm, G, H, J, KK);
            b64 = nb64;
        }
    }
    for (; m <= Lhead; m += P) {
        const int mn = m + P < 127 ? m + P : 127;
        const int nb64 = gs.cb64[mn], nb32 = gs.cb32[mn];
        ColSums64<K> s;
        s.zero();
        double Q1[K], Q2[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            Q1[k] = qm[k];
            Q2[k] = 0.0;
        }
        const GravEntry64* e = reinterpret_cast<const GravEntry64*>(reinterpret_cast<const uint4*>(gs.t64) + b64);
        s.add(e, Q1);
        column64<K>(e, 1, Lhead - m, u, w, Q1, Q2, s);
        if constexpr (MIXED) {
            if (L > kMixedSplit) {
                ColSums32<K> f;
                f.zero();
                float Q1f[K], Q2f[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    Q1f[k] = (float)Q1[k];
                    Q2f[k] = (float)Q2[k];
                }
                column32k<K>(reinterpret_cast<const GravEntry32*>(reinterpret_cast<const uint4*>(gs.t32) + b32),
                    kMixedSplit + 1 - m, L - m, uf, wf, Q1f, Q2f, f);
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
        }
        const double dm = (double)m; // eq. 4-11
#pragma unroll
        for (int k = 0; k < K; ++k) {
            G[k] += Cm[k] * s.g1[k] + Sm[k] * s.g2[k];
            J[k] += dm * (Cp[k] * s.j1[k] + Sp[k] * s.j2[k]);
            KK[k] -= dm * (Sp[k] * s.j1[k] - Cp[k] * s.j2[k]);
            H[k] += Cp[k] * s.h1[k] + Sp[k] * s.h2[k];
            if (m == 0) {
                Cp[k] = CPm1[k];
                Sp[k] = SPm1[k];
            } else {
                cmul(Cp[k], Sp[k], CP[k], SP[k], Cp[k], Sp[k]);
            }
            cmul(Cm[k], Sm[k], CP[k], SP[k], Cm[k], Sm[k]);
            qm[k] *= qP[k];
        }
        b64 = nb64;
        b32 = nb32;
    }
    if constexpr (MIXED) {
        if (m <= L) { // this lane's columns m > 8, in FP32
            float cf[K], sf[K], cpf[K], spf[K], CPf[K], SPf[K], qmf[K], qPf[K];
            float Gf[K], Hf[K], Jf[K], Kf[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                cf[k] = (float)Cm[k];
                sf[k] = (float)Sm[k];
                cpf[k] = (float)Cp[k];
                spf[k] = (float)Sp[k];
                CPf[k] = (float)CP[k];
                SPf[k] = (float)SP[k];
                qmf[k] = (float)qm[k];
                qPf[k] = (float)qP[k];
                Gf[k] = Hf[k] = Jf[k] = Kf[k] = 0.f;
            }
            for (; m <= L; m += P) {
                const int nb = gs.cb32[m + P < 127 ? m + P : 127];
                ColSums32<K> f;
                const GravEntry32* e32 = reinterpret_cast<const GravEntry32*>(reinterpret_cast<const uint4*>(gs.t32) + b32);
                const float4* p = reinterpret_cast<const float4*>(e32);
                const float4 a = p[0], b = p[1];
                float Q1f[K], Q2f[K];
#pragma unroll
                for (int k = 0; k < K; ++k) { // n = m term (Q = q^m)
                    const float2 QQ = make_float2(qmf[k], qmf[k]);
                    f.g[k] = __fmul2_rn(QQ, make_float2(a.z, a.w));
                    f.j[k] = __fmul2_rn(QQ, make_float2(b.x, b.y));
                    f.h[k] = __fmul2_rn(QQ, make_float2(b.z, b.w));
                    Q1f[k] = qmf[k];
                    Q2f[k] = 0.f;
                }
                column32k<K>(e32, 1, L - m, uf, wf, Q1f, Q2f, f);
                const float dmf = (float)m;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    Gf[k] += cf[k] * f.g[k].x + sf[k] * f.g[k].y;
                    Jf[k] += dmf * (cpf[k] * f.j[k].x + spf[k] * f.j[k].y);
                    Kf[k] -= dmf * (spf[k] * f.j[k].x - cpf[k] * f.j[k].y);
                    Hf[k] += cpf[k] * f.h[k].x + spf[k] * f.h[k].y;
                    const float c1 = cf[k] * CPf[k] - sf[k] * SPf[k], s1 = sf[k] * CPf[k] + cf[k] * SPf[k];
                    const float c2 = cpf[k] * CPf[k] - spf[k] * SPf[k], s2 = spf[k] * CPf[k] + cpf[k] * SPf[k];
                    cf[k] = c1;
                    sf[k] = s1;
                    cpf[k] = c2;
                    spf[k] = s2;
                    qmf[k] *= qPf[k];
                }
                b32 = nb;
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
    for (int k = 0; k < K; ++k) {
        for (int o = P >> 1; o > 0; o >>= 1) {
            G[k] += __shfl_xor_sync(mask, G[k], o);
            H[k] += __shfl_xor_sync(mask, H[k], o);
            J[k] += __shfl_xor_sync(mask, J[k], o);
            KK[k] += __shfl_xor_sync(mask, KK[k], o);
        }
        const double Gt = G[k] + 1.0; // eq. 4-13
        const double Lambda = Gt + z[k] * H[k] / r[k];
        const double c = -gs.gm / (r[k] * r[k]);
        ax[k] = c * (Lambda * x[k] / r[k] - J[k]);
        ay[k] = c * (Lambda * y[k] / r[k] - KK[k]);
        az[k] = c * (Lambda * z[k] / r[k] - H[k]);
    }
}

template <bool MIXED>
__device__ __forceinline__ void gravity_itrs_lanes(const GravSmem& gs, int l, int P, double x,
    double y, double z, double& ax, double& ay, double& az, unsigned mask = 0xffffffffu)
{
    const double X[1] = { x }, Y[1] = { y }, Z[1] = { z };
    double AX[1], AY[1], AZ[1];
    gravity_itrs_lk<MIXED, 1>(gs, l, P, X, Y, Z, AX, AY, AZ, mask);
    ax = AX[0];
    ay = AY[0];
    az = AZ[0];
}

// K objects: GCRS positions r[k] with the ITRS<-GCRS matrix M of gravity_gcrs.
template <bool MIXED, int K, bool PAIRS = false>
__device__ __forceinline__ void gravity_gcrs_lk(const GravSmem& gs, int l, int P, const double* __restrict__ M,
    const double (&r)[K][3], double (&a)[K][3], unsigned mask)
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
    gravity_itrs_lk<MIXED, K, PAIRS>(gs, l, P, px, py, pz, ax, ay, az, mask);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        a[k][0] = m[0] * ax[k] + m[3] * ay[k] + m[6] * az[k];
        a[k][1] = m[1] * ax[k] + m[4] * ay[k] + m[7] * az[k];
        a[k][2] = m[2] * ax[k] + m[5] * ay[k] + m[8] * az[k];
    }
}

template <bool MIXED>
__device__ __forceinline__ void gravity_gcrs_lanes(const GravSmem& gs, int l, int P,
    const double* __restrict__ M, const double* r, double* a, unsigned mask = 0xffffffffu)
{
    double m[9];
#pragma unroll
    for (int i = 0; i < 9; ++i)
        m[i] = __ldg(M + i);
    const double px = m[0] * r[0] + m[1] * r[1] + m[2] * r[2];
    const double py = m[3] * r[0] + m[4] * r[1] + m[5] * r[2];
    const double pz = m[6] * r[0] + m[7] * r[1] + m[8] * r[2];
    double ax, ay, az;
    gravity_itrs_lanes<MIXED>(gs, l, P, px, py, pz, ax, ay, az, mask);
    a[0] = m[0] * ax + m[3] * ay + m[6] * az;
    a[1] = m[1] * ax + m[4] * ay + m[7] * az;
    a[2] = m[2] * ax + m[5] * ay + m[8] * az;
}

// ---- gravity Jacobian (FP64) ----
// The column sums are functions of q = R/r and eps = z/r only, and Q(n,m) = q^n P(n,m)(eps) is
// homogeneous of degree n in q, so dQ/dq = n Q / q and dQ/deps follows the recursion
//   E(n) = q Q(n-1) + u E(n-1) - c w E(n-2),  E(m) = 0   (from Q(n) = u Q(n-1) - c w Q(n-2)).
// Three sums per table entry (of Q, n Q and E) give each column's value and both partials; the
// longitude dependence enters through (C1 + i S1)^m, whose partials are m (C1 + i S1)^(m-1) and
// i m (C1 + i S1)^(m-1). G, J, K, H and their partials in (q, eps, C1, S1) are then chained to
// the Earth-fixed position. Cost per (n, m) term: about 3 times one acceleration evaluation.
struct JacF {
    double v, q, e, c, s; // value and partials in q, eps, C1, S1
};

__device__ __forceinline__ void jac_warp_sum(double& x, int P, unsigned mask)
{
    for (int o = P >> 1; o > 0; o >>= 1)
        x += __shfl_xor_sync(mask, x, o);
}

// Acceleration a and Jacobian Jm[i][j] = d a_i / d p_j in the Earth-fixed frame.
// mask: the lanes of the object's group (the shuffles stay inside it).
__device__ __forceinline__ void gravity_jac_itrs_lanes(const GravSmem& gs, int l, int P, double x,
    double y, double z, double* a, double (*Jm)[3], unsigned mask)
{
    const int L = gs.L;
    const double r = sqrt(x * x + y * y + z * z);
    const double invr = 1.0 / r;
    const double eps = z / r;
    const double q = gs.radius / r;
    const double u = q * eps, w = q * q;
    const double C1 = x / r, S1 = y / r;
    JacF G { 0, 0, 0, 0, 0 }, J { 0, 0, 0, 0, 0 }, K { 0, 0, 0, 0, 0 }, H { 0, 0, 0, 0, 0 };
    double CP, SP, qP = 1.0, qm = 1.0;
    cpow(C1, S1, P, CP, SP);
    for (int i = 0; i < P; ++i)
        qP *= q;
    for (int i = 0; i < l; ++i)
        qm *= q;
    double Cm = 0, Sm = 0, Cp = 0, Sp = 0, Cq = 0, Sq = 0; // z^m, z^(m-1), z^(m-2)
    for (int m = l; m <= L; m += P) {
        if (m == l || m - P < 2) { // first column of the lane, or a zero power to restart
            cpow(C1, S1, m, Cm, Sm);
            if (m >= 1)
                cpow(C1, S1, m - 1, Cp, Sp);
            else
                Cp = Sp = 0.0;
            if (m >= 2)
                cpow(C1, S1, m - 2, Cq, Sq);
            else
                Cq = Sq = 0.0;
        } else {
            cmul(Cm, Sm, CP, SP, Cm, Sm);
            cmul(Cp, Sp, CP, SP, Cp, Sp);
            cmul(Cq, Sq, CP, SP, Cq, Sq);
        }
        const GravEntry64* e = lane_col64(gs, m);
        // sums of Q, n Q and E times (g1, g2, j1, j2, h1, h2)
        double s0[6], s1[6], s2[6];
        {
            const double2* p = reinterpret_cast<const double2*>(e);
            const double2 g = p[1], j = p[2], h = p[3];
            const double t[6] = { g.x, g.y, j.x, j.y, h.x, h.y };
            const double nq = (double)m * qm;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                s0[k] = t[k] * qm;
                s1[k] = t[k] * nq;
                s2[k] = 0.0;
            }
        }
        double Q1 = qm, Q2 = 0.0, E1 = 0.0, E2 = 0.0, dn = (double)m;
        for (int i = 1; i <= L - m; ++i) {
            const double2* p = reinterpret_cast<const double2*>(e + i);
            const double cw = p[0].x * w;
            const double Q = fma(u, Q1, -cw * Q2);
            const double E = fma(q, Q1, fma(u, E1, -cw * E2));
            dn += 1.0;
            const double nQ = dn * Q;
            const double2 g = p[1], j = p[2], h = p[3];
            const double t[6] = { g.x, g.y, j.x, j.y, h.x, h.y };
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                s0[k] = fma(t[k], Q, s0[k]);
                s1[k] = fma(t[k], nQ, s1[k]);
                s2[k] = fma(t[k], E, s2[k]);
            }
            Q2 = Q1;
            Q1 = Q;
            E2 = E1;
            E1 = E;
        }
        const double dm = (double)m, dm1 = dm - 1.0;
        // G = sum Re(z^m) g1 + Im(z^m) g2
        G.v += Cm * s0[0] + Sm * s0[1];
        G.q += Cm * s1[0] + Sm * s1[1];
        G.e += Cm * s2[0] + Sm * s2[1];
        G.c += dm * (Cp * s0[0] + Sp * s0[1]);
        G.s += dm * (-Sp * s0[0] + Cp * s0[1]);
        // J = sum m (Re(z^(m-1)) j1 + Im(z^(m-1)) j2)
        J.v += dm * (Cp * s0[2] + Sp * s0[3]);
        J.q += dm * (Cp * s1[2] + Sp * s1[3]);
        J.e += dm * (Cp * s2[2] + Sp * s2[3]);
        J.c += dm * dm1 * (Cq * s0[2] + Sq * s0[3]);
        J.s += dm * dm1 * (-Sq * s0[2] + Cq * s0[3]);
        // K = -sum m (Im(z^(m-1)) j1 - Re(z^(m-1)) j2)
        K.v -= dm * (Sp * s0[2] - Cp * s0[3]);
        K.q -= dm * (Sp * s1[2] - Cp * s1[3]);
        K.e -= dm * (Sp * s2[2] - Cp * s2[3]);
        K.c -= dm * dm1 * (Sq * s0[2] - Cq * s0[3]);
        K.s -= dm * dm1 * (Cq * s0[2] + Sq * s0[3]);
        // H = sum Re(z^(m-1)) h1 + Im(z^(m-1)) h2
        H.v += Cp * s0[4] + Sp * s0[5];
        H.q += Cp * s1[4] + Sp * s1[5];
        H.e += Cp * s2[4] + Sp * s2[5];
        H.c += dm1 * (Cq * s0[4] + Sq * s0[5]);
        H.s += dm1 * (-Sq * s0[4] + Cq * s0[5]);
        qm *= qP;
    }
    JacF* F[4] = { &G, &J, &K, &H };
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        jac_warp_sum(F[f]->v, P, mask);
        jac_warp_sum(F[f]->q, P, mask);
        jac_warp_sum(F[f]->e, P, mask);
        jac_warp_sum(F[f]->c, P, mask);
        jac_warp_sum(F[f]->s, P, mask);
        F[f]->q /= q; // sums of n Q: q dQ/dq
    }
    const double ph[3] = { C1, S1, eps };
    double gq[3], ge[3], gc[3], gsn[3]; // gradients of q, eps, C1, S1
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        gq[j] = -q * invr * ph[j];
        ge[j] = ((j == 2 ? 1.0 : 0.0) - eps * ph[j]) * invr;
        gc[j] = ((j == 0 ? 1.0 : 0.0) - C1 * ph[j]) * invr;
        gsn[j] = ((j == 1 ? 1.0 : 0.0) - S1 * ph[j]) * invr;
    }
    double dF[4][3];
#pragma unroll
    for (int f = 0; f < 4; ++f)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            dF[f][j] = F[f]->q * gq[j] + F[f]->e * ge[j] + F[f]->c * gc[j] + F[f]->s * gsn[j];
    // a = c (Lambda p^ - P), P = (J, K, H), Lambda = 1 + G + eps H, c = -GM / r^2
    const double Lambda = G.v + 1.0 + z * H.v / r;
    const double c = -gs.gm / (r * r);
    const double Pv[3] = { J.v, K.v, H.v };
    const double* dP[3] = { dF[1], dF[2], dF[3] };
    double dL[3];
#pragma unroll
    for (int j = 0; j < 3; ++j)
        dL[j] = dF[0][j] + eps * dF[3][j] + H.v * ge[j];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double base = Lambda * ph[i] - Pv[i];
        a[i] = c * base;
#pragma unroll
        for (int j = 0; j < 3; ++j)
            Jm[i][j] = -2.0 * c * ph[j] * invr * base
                + c * (dL[j] * ph[i] + Lambda * ((i == j ? 1.0 : 0.0) - ph[i] * ph[j]) * invr - dP[i][j]);
    }
}

// GCRS acceleration and Jacobian for the ITRS<-GCRS matrix M of gravity_gcrs: p = A r with
// A[i][k] = M[3 i + k], a = A^T a_itrs, J = A^T J_itrs A.
__device__ __forceinline__ void gravity_jac_gcrs_lanes(const GravSmem& gs, int l, int P,
    const double* __restrict__ M, const double* r, double* a, double (*Jg)[3], unsigned mask)
{
    double A[3][3];
#pragma unroll
    for (int i = 0; i < 9; ++i)
        A[i / 3][i % 3] = __ldg(M + i);
    double p[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        p[i] = A[i][0] * r[0] + A[i][1] * r[1] + A[i][2] * r[2];
    double ai[3], Ji[3][3];
    gravity_jac_itrs_lanes(gs, l, P, p[0], p[1], p[2], ai, Ji, mask);
    double T[3][3]; // J_itrs A
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            T[i][k] = Ji[i][0] * A[0][k] + Ji[i][1] * A[1][k] + Ji[i][2] * A[2][k];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        a[k] = A[0][k] * ai[0] + A[1][k] * ai[1] + A[2][k] * ai[2];
#pragma unroll
        for (int l2 = 0; l2 < 3; ++l2)
            Jg[k][l2] = A[0][k] * T[0][l2] + A[1][k] * T[1][l2] + A[2][k] * T[2][l2];
    }
}

} // namespace gpop
