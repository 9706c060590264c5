// probe.cu -- FP64 / FP32 FMA throughput probes (libgpop_probe.so). Measurement utility for the
// roofline denominators of FP64-ALU-bound kernels: independent FMA chains per thread, every SM
// busy, timed with CUDA events by the caller.
#include <cuda_runtime.h>
#include <cstdint>

namespace {

__global__ void __launch_bounds__(256) fma64_kernel(double* out, int iters, double a, double b)
{
    double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-9, x2 = x0 + 2e-9, x3 = x0 + 3e-9;
    double x4 = x0 + 4e-9, x5 = x0 + 5e-9, x6 = x0 + 6e-9, x7 = x0 + 7e-9;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    double s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 12345.678)
        out[0] = s; // keeps the chains alive
}

__global__ void __launch_bounds__(256) fma32_kernel(float* out, int iters, float a, float b)
{
    float2 x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
        x[k] = make_float2(threadIdx.x * 1e-7f + k, threadIdx.x * 1e-7f - k);
    const float2 A = make_float2(a, a), B = make_float2(b, b);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
#pragma unroll
            for (int j = 0; j < 8; ++j)
                x[j] = __ffma2_rn(x[j], A, B);
        }
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k)
        s += x[k].x + x[k].y;
    if (s == 12345.678f)
        out[0] = s;
}

// Packed FP32 chains, FP64 chains, or both interleaved (6 + 6 per iteration): whether the FP64
// pipe can work beside the FMA pipe. Time with one block of 256 threads per SM.
__global__ void __launch_bounds__(256) mix_kernel(float* out, int mode, int iters, float a, float b,
    double da, double db)
{
    float2 x[6];
    double y[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        x[k] = make_float2(threadIdx.x * 1e-7f + k, k * 0.5f);
        y[k] = threadIdx.x * 1e-9 + k;
    }
    const float2 A = make_float2(a, a), B = make_float2(b, b);
    if (mode == 0) {
        for (int i = 0; i < iters; ++i)
#pragma unroll
            for (int k = 0; k < 6; ++k)
                x[k] = __ffma2_rn(x[k], A, B);
    } else if (mode == 1) {
        for (int i = 0; i < iters; ++i)
#pragma unroll
            for (int k = 0; k < 6; ++k)
                y[k] = fma(y[k], da, db);
    } else {
        for (int i = 0; i < iters; ++i)
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                x[k] = __ffma2_rn(x[k], A, B);
                y[k] = fma(y[k], da, db);
            }
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 6; ++k)
        s += x[k].x + x[k].y + (float)y[k];
    if (s == 12345.f)
        out[0] = s;
}

} // namespace

extern "C" __attribute__((visibility("default"))) int gpop_probe_mix(int mode, int blocks, int iters,
    void* scratch, void* stream)
{
    mix_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>((float*)scratch, mode, iters, 0.999f, 1e-4f,
        0.999999, 1e-7);
    return (int)cudaGetLastError();
}

extern "C" __attribute__((visibility("default"))) int gpop_probe_fma(int fp64, int blocks,
    int iters, void* scratch, void* stream, double* flops_out)
{
    const int threads = 256;
    if (fp64) {
        fma64_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>((double*)scratch, iters, 0.999999, 1e-7);
        *flops_out = 2.0 * 64.0 * (double)iters * blocks * threads;
    } else {
        fma32_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>((float*)scratch, iters, 0.999f, 1e-4f);
        *flops_out = 2.0 * 2.0 * 64.0 * (double)iters * blocks * threads;
    }
    return (int)cudaGetLastError();
}
