// frames.cuh -- IAU 2006/2000A GCRS<->ITRS transformation for one epoch (equinox-based route with
// EOP polar motion), host and device. Follows lib/force_model/src/utility/ref_sys_trans.cu:24-376
// and the matrix chain of lib/force_model/src/time_points.cu:160-201 (IERS Conventions 2010, ch. 5;
// Astronomical Almanac 2010 for GAST).
#pragma once
#include "model.h"
#include <cmath>

#ifdef __CUDACC__
#define GPOP_HD __host__ __device__ __forceinline__
#else
#define GPOP_HD inline
#endif

namespace gpop {
namespace frames {

constexpr double kPi = 3.14159265358979324;
constexpr double kArcsPerRad = 3600.0 * 180.0 / kPi;
constexpr double kMjdJ2000 = 51544.5;
constexpr double kTtTai = 32.184;
constexpr double kUasToRad = kArcsPerRad * 1e6;

// Column-major 3x3 (element (row, col) at col*3 + row), the layout of gpu_utils.cuh:60.
GPOP_HD void rot_x(double a, double* p)
{
    double c = cos(a), s = sin(a);
    p[0] = 1.0; p[3] = 0.0; p[6] = 0.0;
    p[1] = 0.0; p[4] = c;   p[7] = s;
    p[2] = 0.0; p[5] = -s;  p[8] = c;
}
GPOP_HD void rot_y(double a, double* p)
{
    double c = cos(a), s = sin(a);
    p[0] = c;   p[3] = 0.0; p[6] = -s;
    p[1] = 0.0; p[4] = 1.0; p[7] = 0.0;
    p[2] = s;   p[5] = 0.0; p[8] = c;
}
GPOP_HD void rot_z(double a, double* p)
{
    double c = cos(a), s = sin(a);
    p[0] = c;   p[3] = s;   p[6] = 0.0;
    p[1] = -s;  p[4] = c;   p[7] = 0.0;
    p[2] = 0.0; p[5] = 0.0; p[8] = 1.0;
}
GPOP_HD void mat_mul(const double* A, const double* B, double* C)
{
    double t[9];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i)
            t[j * 3 + i] = A[i] * B[j * 3] + A[3 + i] * B[j * 3 + 1] + A[6 + i] * B[j * 3 + 2];
    for (int k = 0; k < 9; ++k)
        C[k] = t[k];
}

// Calendar date to MJD (Montenbruck & Gill, eqs. A.3-A.6; ref_sys_trans.cu:122-144).
GPOP_HD double calendar_to_mjd(int year, int mon, int day, int h, int min, double sec)
{
    if (mon <= 2) {
        --year;
        mon += 12;
    }
    long long key = 10000LL * year + 100LL * mon + day;
    int B;
    if (key <= 15821004LL)
        B = -2 + ((year + 4716) / 4) - 1179;
    else if (key >= 15821015LL)
        B = (year / 400) - (year / 100) + (year / 4);
    else
        return -1.0;
    long long mjd = 365LL * year - 679004LL + B + (int)(30.6001 * (mon + 1)) + day;
    double frac = (h + min / 60.0 + sec / 3600.0) / 24.0;
    return (double)mjd + frac;
}

// Fundamental arguments, IERS 2010 eqs. 5.43 (luni-solar, arcsec polynomials) and 5.44
// (planetary, radians), each reduced modulo 2 pi (ref_sys_trans.cu:164-233).
GPOP_HD void fundamental_args(double t, double* F)
{
    const double ls[5][5] = {
        { 134.96340251 * 3600.0, 1717915923.2178, 31.8792, 0.051635, -0.00024470 },
        { 357.52910918 * 3600.0, 129596581.0481, -0.5532, 0.000136, -0.00001149 },
        { 93.27209062 * 3600.0, 1739527262.8478, -12.7512, -0.001037, 0.00000417 },
        { 297.85019547 * 3600.0, 1602961601.2090, -6.3706, 0.006593, -0.00003169 },
        { 125.04455501 * 3600.0, -6962890.5431, 7.4722, 0.007702, -0.00005939 },
    };
    const double pl[9][3] = {
        { 4.402608842, 2608.7903141574, 0.0 }, { 3.176146697, 1021.3285546211, 0.0 },
        { 1.753470314, 628.3075849991, 0.0 }, { 6.203480913, 334.0612426700, 0.0 },
        { 0.599546497, 52.9690962641, 0.0 }, { 0.874016757, 21.3299104960, 0.0 },
        { 5.481293872, 7.4781598567, 0.0 }, { 5.311886287, 3.8133035638, 0.0 },
        { 0.0, 0.02438175, 0.00000538691 },
    };
    for (int a = 0; a < 5; ++a) {
        double v = ls[a][4];
        for (int i = 3; i >= 0; --i)
            v = v * t + ls[a][i];
        F[a] = fmod(v / kArcsPerRad, 2.0 * kPi);
    }
    for (int a = 0; a < 9; ++a) {
        double v = pl[a][2];
        for (int i = 1; i >= 0; --i)
            v = v * t + pl[a][i];
        F[5 + a] = fmod(v, 2.0 * kPi);
    }
}

// One nutation term's contribution (eq. 5.35 summand; ref_sys_trans.cu:241-254).
GPOP_HD double nutation_term(const NutTerm& term, const double* F)
{
    double arg = 0.0;
    for (int k = 13; k >= 0; --k)
        arg += F[k] * (double)term.args[k];
    return term.sin_uas / kUasToRad * sin(arg) + term.cos_uas / kUasToRad * cos(arg);
}

// IAU 2006 precession quantities eps_A, gamma-bar, phi-bar, psi-bar (eq. 5.40; :262-291).
GPOP_HD void precession(double t, double& epsA, double& gam, double& phi, double& psi)
{
    const double e[6] = { 84381.406, -46.836769, -0.0001831, 0.00200340, -0.000000576, -0.0000000434 };
    const double g[6] = { -0.052928, 10.556378, 0.4932044, -0.00031238, -0.000002788, 0.0000000260 };
    const double p[6] = { 84381.412819, -46.811016, 0.0511268, 0.00053289, -0.000000440, -0.0000000176 };
    const double s[6] = { -0.041775, 5038.481484, 1.5584175, -0.00018522, -0.000026452, -0.0000000148 };
    epsA = e[5];
    gam = g[5];
    phi = p[5];
    psi = s[5];
    for (int i = 4; i >= 0; --i) {
        epsA = epsA * t + e[i];
        gam = gam * t + g[i];
        phi = phi * t + p[i];
        psi = psi * t + s[i];
    }
    epsA /= kArcsPerRad;
    gam /= kArcsPerRad;
    phi /= kArcsPerRad;
    psi /= kArcsPerRad;
}

// Greenwich apparent sidereal time by the equation of the equinoxes (Astronomical Almanac 2010,
// pp. B6-B10; ref_sys_trans.cu:75-119).
GPOP_HD double gast(double mjd_ut1, double mjd_tt, double dpsi, double epsA, const double* F)
{
    const double T = (mjd_tt - kMjdJ2000) / 36525.0;
    const double Du = mjd_ut1 - kMjdJ2000;
    const double frac = Du - floor(Du);
    double gmst = 86400.0 * (0.7790572732640 + 0.00273781191135448 * Du + frac);
    const double c[6] = { 0.00096707, 307.47710227, 0.092772113, -0.0000000293, -0.00000199707, -2.453e-9 };
    double poly = c[5];
    for (int i = 4; i >= 0; --i)
        poly = poly * T + c[i];
    gmst += poly;
    gmst *= (kPi / 43200.0);
    const double l = F[0], lp = F[1], f = F[2], D = F[3], Om = F[4];
    double ee = 0.0;
    ee -= 0.00000087 * T * sin(Om);
    ee -= 0.00000063 * sin(l - Om);
    ee -= 0.00000063 * sin(l + Om);
    ee -= 0.00000126 * sin(lp - Om);
    ee -= 0.00000141 * sin(lp + Om);
    ee -= 0.00000172 * sin(3.0 * Om);
    ee += 0.00000198 * sin(2.0 * f + Om);
    ee += 0.00000202 * sin(2.0 * f + 3.0 * Om);
    ee -= 0.00000455 * sin(2.0 * f - 2.0 * D + 2.0 * Om);
    ee += 0.00001121 * sin(2.0 * f - 2.0 * D + Om);
    ee += 0.00001175 * sin(2.0 * f - 2.0 * D + 3.0 * Om);
    ee += 0.00006352 * sin(2.0 * Om);
    ee += 0.00264096 * sin(Om);
    ee *= (kPi / 43200.0) / 15.0;
    ee += dpsi * cos(epsA);
    return fmod(gmst + ee, 2.0 * kPi);
}

// EOP at a UTC MJD: binary search and linear interpolation, clamped at both ends
// (force_model/include/force_model/types.cuh:79-130).
GPOP_HD EopRec eop_at(const EopRec* rec, int n, double mjd)
{
    if (n <= 0)
        return EopRec { -1.0, 0.0, 0.0, 0.0 };
    if (mjd <= rec[0].mjd)
        return rec[0];
    if (mjd >= rec[n - 1].mjd)
        return rec[n - 1];
    int lo = 0, hi = n - 1;
    while (lo <= hi) {
        int mid = lo + (hi - lo) / 2;
        double cur = rec[mid].mjd;
        if (cur == mjd)
            return rec[mid];
        if (cur < mjd)
            lo = mid + 1;
        else
            hi = mid - 1;
    }
    const EopRec a = rec[hi], b = rec[lo];
    const double fr = (mjd - a.mjd) / (b.mjd - a.mjd);
    return EopRec { mjd, a.xp + fr * (b.xp - a.xp), a.yp + fr * (b.yp - a.yp), a.ut1 + fr * (b.ut1 - a.ut1) };
}

// TAI-UTC active at a UTC MJD (types.cuh:140-152).
GPOP_HD double leap_at(const double* mjd_tab, const double* val, int n, double mjd)
{
    if (n <= 0)
        return 0.0;
    for (int i = n - 1; i >= 0; --i)
        if (mjd >= mjd_tab[i])
            return val[i];
    return val[0];
}

// Builds M = Q R W from the nutation sums (dpsi, deps), the fundamental arguments F, TT and UT1.
GPOP_HD void assemble(double t, const double* F, double dpsi, double deps, double mjd_ut1,
    double mjd_tt, const EopRec& eop, double* M)
{
    double epsA, gam, phi, psib;
    precession(t, epsA, gam, phi, psib);
    double Q1[9], Q2[9], Q3[9], Q4[9], W1[9], W2[9], W3[9], R[9], A[9], B[9], Q[9], W[9];
    rot_z(-gam, Q1); // Fukushima-Williams, ch. 5.4.5, in the ITRS->GCRS direction
    rot_x(-phi, Q2);
    rot_z(psib + dpsi, Q3);
    rot_x(epsA + deps, Q4);
    const double sp = -47e-6 * t / kArcsPerRad; // eq. 5.13
    rot_z(-sp, W1); // eq. 5.3
    rot_y(eop.xp, W2);
    rot_x(eop.yp, W3);
    rot_z(-gast(mjd_ut1, mjd_tt, dpsi, epsA, F), R); // ch. 5.4.3
    mat_mul(Q1, Q2, A);
    mat_mul(Q3, Q4, B);
    mat_mul(A, B, Q);
    mat_mul(W1, W2, A);
    mat_mul(A, W3, W);
    mat_mul(Q, R, A);
    mat_mul(A, W, M);
}

} // namespace frames
} // namespace gpop
