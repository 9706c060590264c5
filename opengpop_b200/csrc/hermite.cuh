// hermite.cuh -- TCA refinement helpers: the 9-coefficient confluent Hermite interpolant of
// HermitePolynomial, ApproachFunc and the secant FindRoot (closest_approach/utility/
// interpolation.cuh:27-152), shared by the set-partitioned screen and the pair-list kernels.
#pragma once
#include <cuda_runtime.h>

namespace gpop {

struct Herm {
    double c[9];
};

// 9-coefficient confluent Hermite polynomial in Newton form through (p, v, a/2) at 0, dt, 2dt
// (Kincaid & Cheney, ch. 6.3; interpolation.cuh:32-64).
__device__ __forceinline__ void herm_build(Herm& H, double p0, double v0, double a0, double p1,
    double v1, double a1, double p2, double v2, double a2, double dt)
{
    const double t[9] = { 0.0, 0.0, 0.0, dt, dt, dt, 2.0 * dt, 2.0 * dt, 2.0 * dt };
    double* c = H.c;
    c[0] = c[1] = c[2] = p0;
    c[3] = c[4] = c[5] = p1;
    c[6] = c[7] = c[8] = p2;
#pragma unroll
    for (int j = 1; j < 9; j++)
#pragma unroll
        for (int i = 8; i >= j; i--) {
            if (t[i] == t[i - j]) {
                if (j == 1)
                    c[i] = (i < 3) ? v0 : (i < 6) ? v1 : v2;
                else if (j == 2)
                    c[i] = ((i < 3) ? a0 : (i < 6) ? a1 : a2) / 2.0;
            } else {
                c[i] = (c[i] - c[i - 1]) / (t[i] - t[i - j]);
            }
        }
}

__device__ __forceinline__ double herm_eval(const Herm& H, double dt, double t)
{
    const double z[9] = { 0.0, 0.0, 0.0, dt, dt, dt, 2.0 * dt, 2.0 * dt, 2.0 * dt };
    double res = H.c[0], term = 1.0;
#pragma unroll
    for (int i = 1; i < 9; ++i) {
        term *= (t - z[i - 1]);
        res += H.c[i] * term;
    }
    return res;
}

__device__ __forceinline__ double herm_deriv(const Herm& H, double dt, double t)
{
    const double z[9] = { 0.0, 0.0, 0.0, dt, dt, dt, 2.0 * dt, 2.0 * dt, 2.0 * dt };
    double res = 0.0, Nn = 1.0, dN = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        res += H.c[i] * dN;
        if (i < 8) {
            dN = dN * (t - z[i]) + Nn;
            Nn *= (t - z[i]);
        }
    }
    return res;
}

struct Pair6 {
    Herm A[3], B[3];
    double dt;
    __device__ double f(double t) const // ApproachFunc: (dr . dv)(t)
    {
        double s = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double d = herm_eval(A[c], dt, t) - herm_eval(B[c], dt, t);
            const double dd = herm_deriv(A[c], dt, t) - herm_deriv(B[c], dt, t);
            s += d * dd;
        }
        return s;
    }
};

// Secant iteration of FindRoot (interpolation.cuh:126-152): tol 1e-7, at most 100 iterations.
__device__ inline double find_root(const Pair6& P, double x0, double x1)
{
    const double tol = 1e-7;
    double f0 = P.f(x0), f1 = P.f(x1);
    for (int i = 0; i < 100; ++i) {
        if (fabs(f1 - f0) < 1e-14)
            return x1;
        const double xn = x1 - f1 * (x1 - x0) / (f1 - f0);
        const double fn = P.f(xn);
        if (fabs(xn - x1) < tol || fabs(fn) < tol)
            return xn;
        x0 = x1;
        f0 = f1;
        x1 = xn;
        f1 = fn;
    }
    return x1;
}


__device__ __forceinline__ double herm_deriv2(const Herm& H, double dt, double t)
{
    const double z[9] = { 0.0, 0.0, 0.0, dt, dt, dt, 2.0 * dt, 2.0 * dt, 2.0 * dt };
    // N_i(t) = prod_{k<i} (t - z_k): carry N, N' and N'' along the product
    double res = 0.0, Nn = 1.0, dN = 0.0, ddN = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        res += H.c[i] * ddN;
        if (i < 8) {
            ddN = ddN * (t - z[i]) + 2.0 * dN;
            dN = dN * (t - z[i]) + Nn;
            Nn *= (t - z[i]);
        }
    }
    return res;
}

} // namespace gpop
