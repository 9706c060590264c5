// tangent.cuh -- a value with one directional derivative (forward-mode tangent) for the
// variational equations. Only the operations the integrator applies to its state are defined:
// sums, differences and scaling by constants; products of two tangents do not occur (the force
// models supply a + J dr themselves).
#pragma once
#include <cuda_runtime.h>

namespace gpop {

struct Tan {
    double v; // value
    double d; // derivative along the lane's direction
    __host__ __device__ Tan() : v(0.0), d(0.0) {}
    __host__ __device__ Tan(double x) : v(x), d(0.0) {}
    __host__ __device__ Tan(double x, double dx) : v(x), d(dx) {}
};

__device__ __forceinline__ Tan operator+(Tan a, Tan b) { return Tan(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Tan operator-(Tan a, Tan b) { return Tan(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Tan operator-(Tan a) { return Tan(-a.v, -a.d); }
__device__ __forceinline__ Tan operator*(double c, Tan a) { return Tan(c * a.v, c * a.d); }
__device__ __forceinline__ Tan operator*(Tan a, double c) { return Tan(a.v * c, a.d * c); }
__device__ __forceinline__ Tan operator/(Tan a, double c) { return Tan(a.v / c, a.d / c); }
__device__ __forceinline__ Tan& operator+=(Tan& a, Tan b)
{
    a.v += b.v;
    a.d += b.d;
    return a;
}
// (the double overload keeps plain-double calls exact matches where these are visible)
__device__ __forceinline__ double fma(double a, double b, double c) { return ::fma(a, b, c); }
__device__ __forceinline__ Tan fma(double c, Tan a, Tan b) { return Tan(::fma(c, a.v, b.v), ::fma(c, a.d, b.d)); }
__device__ __forceinline__ Tan fma(Tan a, double c, Tan b) { return Tan(::fma(a.v, c, b.v), ::fma(a.d, c, b.d)); }

__device__ __forceinline__ double value(double x) { return x; }
__device__ __forceinline__ double value(Tan x) { return x.v; }

} // namespace gpop
