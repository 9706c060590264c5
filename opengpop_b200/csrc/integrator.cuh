// integrator.cuh -- RK8 startup and mid-corrector device code (lib/gpu_startup/src/gpu_startup.cu),
// shared by the single-request, batched and variational kernels. A force model F provides
//   gen(r, v, step, k, a)  -- acceleration at RK8 stage k of startup step `step` (+-1..4)
//   prop(r, v, idx, a)     -- acceleration at propagation epoch index idx (t = (idx - 4) h)
// The state type T is double, or a value with a tangent (variational equations): the startup is
// linear in the state apart from the force evaluations, so only + - and scaling by constants are
// applied to T.
#pragma once
#include "gj8_tables.cuh"

namespace gpop {

// ---- RK8 startup and mid-corrector (lib/gpu_startup/src/gpu_startup.cu:55-318) ----
template <class T> struct StartupMatsT {
    T r[9][3], v[9][3], a[9][3], s[9][3], S[9][3];
};
using StartupMats = StartupMatsT<double>;

// RK8::step (gpu_startup.cu:108-144): stage state = base + h sum a_ki K_i; new column = base +
// h sum b_k K_k, for both position (K = stage velocity) and velocity (K = acceleration).
template <class F, class T>
__device__ void rk8_step(const F& f, double h, int step, StartupMatsT<T>& m)
{
    const double hh = step > 0 ? h : -h;
    const int base = 4 + step + (step > 0 ? -1 : 1);
    T Kx[10][3], Kv[10][3];
    T tx[3], tv[3];
    for (int j = 0; j < 3; ++j) {
        tx[j] = m.r[base][j];
        tv[j] = m.v[base][j];
        Kx[0][j] = tv[j];
    }
    f.gen(tx, tv, step, 0, Kv[0]);
    for (int k = 1; k <= 9; ++k) {
        for (int j = 0; j < 3; ++j) {
            T sx = 0.0, sv = 0.0;
            for (int i = 0; i < k; ++i) {
                sx = fma(c_RKA[k - 1][i], Kx[i][j], sx);
                sv = fma(c_RKA[k - 1][i], Kv[i][j], sv);
            }
            tx[j] = fma(hh, sx, m.r[base][j]);
            tv[j] = fma(hh, sv, m.v[base][j]);
        }
        f.gen(tx, tv, step, k, Kv[k]);
        for (int j = 0; j < 3; ++j)
            Kx[k][j] = tv[j];
    }
    const int col = 4 + step;
    for (int j = 0; j < 3; ++j) {
        T sx = 0.0, sv = 0.0;
        for (int k = 0; k < 10; ++k) {
            sx = fma(Kx[k][j], c_RKB[k], sx);
            sv = fma(Kv[k][j], c_RKB[k], sv);
        }
        m.v[col][j] = fma(hh, sv, m.v[base][j]);
        m.r[col][j] = fma(hh, sx, m.r[base][j]);
    }
}

// StartupCorrector::CalculateAccelerationMatrix (gpu_startup.cu:196-224)
template <class F, class T> __device__ void corrector_accel(const F& f, StartupMatsT<T>& m, bool epoch)
{
    for (int i = 0; i < 9; ++i)
        if (i != 4 || epoch)
            f.prop(m.r[i], m.v[i], i, m.a[i]);
}

// StartupCorrector::CalculateS0 (gpu_startup.cu:170-195), Berry & Healy eqs. 73, 75, 86
template <class T> __device__ inline void corrector_s0(double h, StartupMatsT<T>& m)
{
    const double hinv = 1 / h, h2inv = 1 / (h * h);
    for (int j = 0; j < 3; ++j) {
        T sb = 0.0, sa = 0.0;
        for (int k = 0; k < 9; ++k) {
            sb = fma(c_SA[4][k], m.a[k][j], sb);
            sa = fma(c_GJ[4][k], m.a[k][j], sa);
        }
        m.s[4][j] = fma(hinv, m.v[4][j], -sb);
        m.S[4][j] = fma(h2inv, m.r[4][j], -sa);
    }
}

// CalculateAllSKernel (gpu_startup/src/device/calculate_all_s.cu:19-47)
template <class T> __device__ inline void corrector_all_s(StartupMatsT<T>& m)
{
    for (int i = 1; i <= 4; ++i)
        for (int j = 0; j < 3; ++j) {
            m.s[4 + i][j] = m.s[4 + i - 1][j] + (m.a[4 + i - 1][j] + m.a[4 + i][j]) / 2;
            m.s[4 - i][j] = m.s[4 - i + 1][j] - (m.a[4 - i + 1][j] + m.a[4 - i][j]) / 2;
            m.S[4 + i][j] = m.s[4 + i - 1][j] + m.S[4 + i - 1][j] + m.a[4 + i - 1][j] / 2;
            m.S[4 - i][j] = -m.s[4 - i + 1][j] + m.S[4 - i + 1][j] + m.a[4 - i + 1][j] / 2;
        }
}

// StartupCorrector::Correct (gpu_startup.cu:247-294)
template <class F, class T> __device__ void corrector_correct(const F& f, double h, StartupMatsT<T>& m)
{
    corrector_s0(h, m);
    corrector_all_s(m);
    const double h2 = h * h;
    for (int c = 0; c < 9; ++c) {
        if (c == 4)
            continue; // the epoch column is restored
        for (int j = 0; j < 3; ++j) {
            T sv = 0.0, sr = 0.0;
            for (int k = 0; k < 9; ++k) {
                sv = fma(m.a[k][j], c_SA[c][k], sv);
                sr = fma(m.a[k][j], c_GJ[c][k], sr);
            }
            m.v[c][j] = h * (sv + m.s[c][j]);
            m.r[c][j] = h2 * (sr + m.S[c][j]);
        }
    }
    corrector_accel(f, m, false);
}

template <class F, class T>
__device__ void run_startup(const F& f, double h, int ncorr, const T* r0, const T* v0, StartupMatsT<T>& m)
{
    for (int c = 0; c < 9; ++c)
        for (int j = 0; j < 3; ++j)
            m.r[c][j] = m.v[c][j] = m.a[c][j] = m.s[c][j] = m.S[c][j] = 0.0;
    for (int j = 0; j < 3; ++j) {
        m.r[4][j] = r0[j];
        m.v[4][j] = v0[j];
    }
    for (int i = 1; i <= 4; ++i) { // StartupPredictor::Predict (gpu_startup.cu:162-165)
        rk8_step(f, h, i, m);
        rk8_step(f, h, -i, m);
    }
    if (ncorr <= 0)
        return;
    corrector_accel(f, m, true);
    for (int i = 0; i < ncorr; ++i)
        corrector_correct(f, h, m);
}

// ---- the same startup for two objects in lockstep (the split block's startup kernel) ----
// F2 provides gen2(r, v, step, k, a) and prop2(r, v, idx, a) over both objects at once
// ([2][3] arrays); those may hold block-wide barriers, so every thread of a block makes the same
// calls in the same order (the control flow below depends on no data). Per object the arithmetic
// is that of rk8_step, corrector_correct and run_startup. A thread that carries no objects
// (active false) makes the same force calls and skips the arithmetic around them.
template <class F2>
__device__ void rk8_step2(const F2& f, double h, int step, StartupMats (&m)[2], bool active)
{
    const double hh = step > 0 ? h : -h;
    const int base = 4 + step + (step > 0 ? -1 : 1);
    double Kx[2][10][3], Kv[2][10][3];
    double tx[2][3] = {}, tv[2][3] = {};
    for (int o = 0; o < 2 && active; ++o)
        for (int j = 0; j < 3; ++j) {
            tx[o][j] = m[o].r[base][j];
            tv[o][j] = m[o].v[base][j];
            Kx[o][0][j] = tv[o][j];
        }
    {
        double acc[2][3];
        f.gen2(tx, tv, step, 0, acc);
        for (int o = 0; o < 2 && active; ++o)
            for (int j = 0; j < 3; ++j)
                Kv[o][0][j] = acc[o][j];
    }
    for (int k = 1; k <= 9; ++k) {
        for (int o = 0; o < 2 && active; ++o)
            for (int j = 0; j < 3; ++j) {
                double sx = 0.0, sv = 0.0;
                for (int i = 0; i < k; ++i) {
                    sx = fma(c_RKA[k - 1][i], Kx[o][i][j], sx);
                    sv = fma(c_RKA[k - 1][i], Kv[o][i][j], sv);
                }
                tx[o][j] = fma(hh, sx, m[o].r[base][j]);
                tv[o][j] = fma(hh, sv, m[o].v[base][j]);
            }
        double acc[2][3];
        f.gen2(tx, tv, step, k, acc);
        for (int o = 0; o < 2 && active; ++o)
            for (int j = 0; j < 3; ++j) {
                Kv[o][k][j] = acc[o][j];
                Kx[o][k][j] = tv[o][j];
            }
    }
    const int col = 4 + step;
    for (int o = 0; o < 2 && active; ++o)
        for (int j = 0; j < 3; ++j) {
            double sx = 0.0, sv = 0.0;
            for (int k = 0; k < 10; ++k) {
                sx = fma(Kx[o][k][j], c_RKB[k], sx);
                sv = fma(Kv[o][k][j], c_RKB[k], sv);
            }
            m[o].v[col][j] = fma(hh, sv, m[o].v[base][j]);
            m[o].r[col][j] = fma(hh, sx, m[o].r[base][j]);
        }
}

template <class F2>
__device__ void corrector_accel2(const F2& f, StartupMats (&m)[2], bool epoch, bool active)
{
    for (int i = 0; i < 9; ++i) {
        if (i == 4 && !epoch)
            continue; // the same for every thread: no evaluation, no barrier
        double r[2][3] = {}, v[2][3] = {}, acc[2][3];
        for (int o = 0; o < 2 && active; ++o)
            for (int j = 0; j < 3; ++j) {
                r[o][j] = m[o].r[i][j];
                v[o][j] = m[o].v[i][j];
            }
        f.prop2(r, v, i, acc);
        for (int o = 0; o < 2 && active; ++o)
            for (int j = 0; j < 3; ++j)
                m[o].a[i][j] = acc[o][j];
    }
}

template <class F2>
__device__ void corrector_correct2(const F2& f, double h, StartupMats (&m)[2], bool active)
{
    const double h2 = h * h;
    for (int o = 0; o < 2 && active; ++o) {
        corrector_s0(h, m[o]);
        corrector_all_s(m[o]);
        for (int c = 0; c < 9; ++c) {
            if (c == 4)
                continue; // the epoch column is restored
            for (int j = 0; j < 3; ++j) {
                double sv = 0.0, sr = 0.0;
                for (int k = 0; k < 9; ++k) {
                    sv = fma(m[o].a[k][j], c_SA[c][k], sv);
                    sr = fma(m[o].a[k][j], c_GJ[c][k], sr);
                }
                m[o].v[c][j] = h * (sv + m[o].s[c][j]);
                m[o].r[c][j] = h2 * (sr + m[o].S[c][j]);
            }
        }
    }
    corrector_accel2(f, m, false, active);
}

template <class F2>
__device__ void run_startup2(const F2& f, double h, int ncorr, const double (&r0)[2][3],
    const double (&v0)[2][3], StartupMats (&m)[2], bool active)
{
    for (int o = 0; o < 2 && active; ++o) {
        for (int c = 0; c < 9; ++c)
            for (int j = 0; j < 3; ++j)
                m[o].r[c][j] = m[o].v[c][j] = m[o].a[c][j] = m[o].s[c][j] = m[o].S[c][j] = 0.0;
        for (int j = 0; j < 3; ++j) {
            m[o].r[4][j] = r0[o][j];
            m[o].v[4][j] = v0[o][j];
        }
    }
    for (int i = 1; i <= 4; ++i) {
        rk8_step2(f, h, i, m, active);
        rk8_step2(f, h, -i, m, active);
    }
    if (ncorr <= 0)
        return;
    corrector_accel2(f, m, true, active);
    for (int i = 0; i < ncorr; ++i)
        corrector_correct2(f, h, m, active);
}

} // namespace gpop
