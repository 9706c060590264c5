// sampler.cu -- seeded on-device sampling of perturbed initial states (Monte Carlo ensembles), in
// place of the reference's PerturbationGenerator (lib/perturbation_generator/src/
// perturbation_generator.cu:21-79), which draws N(0, sigma^2) velocity perturbations of one object
// with curand. Here: Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC 2011) keyed by the seed and counted by the sample index, and the Box-Muller
// transform; every sample depends only on (seed, index), so ensembles are reproducible and can be
// generated in pieces.
#include "common.cuh"
#include "context.h"

#include <cmath>

using namespace gpop;

namespace {

struct U4 {
    uint32_t x, y, z, w;
};

// One Philox4x32 round and the key schedule of the published algorithm.
__device__ __forceinline__ U4 philox_round(U4 c, uint32_t k0, uint32_t k1)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    return U4 { hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0 };
}

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1)
{
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += W0;
            k1 += W1;
        }
        c = philox_round(c, k0, k1);
    }
    return c;
}

// (0, 1] from 53 bits of two words
__device__ __forceinline__ double unit53(uint32_t a, uint32_t b)
{
    const uint64_t x = ((uint64_t)a << 21) | (uint64_t)(b >> 11);
    return (double)(x + 1) * 0x1.0p-53;
}

// Sample i: counters (i, b, 0, 0), b = 0, 1, 2, give two 53-bit uniforms each and, by Box-Muller,
// two normals each: z0..z2 perturb the position, z3..z5 the velocity.
__global__ void sample_kernel(int64_t n, double r0, double r1, double r2, double v0, double v1, double v2,
    double sigma_r, double sigma_v, uint32_t k0, uint32_t k1, double* r, double* v)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double z[6];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        const U4 o = philox4x32_10(U4 { (uint32_t)i, (uint32_t)b, (uint32_t)(i >> 32), 0u }, k0, k1);
        const double u1 = unit53(o.x, o.y), u2 = unit53(o.z, o.w);
        const double rad = sqrt(-2.0 * log(u1));
        double sn, cs;
        sincospi(2.0 * u2, &sn, &cs);
        z[2 * b] = rad * cs;
        z[2 * b + 1] = rad * sn;
    }
    const double rr[3] = { r0, r1, r2 }, vv[3] = { v0, v1, v2 };
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        r[i * 3 + j] = rr[j] + sigma_r * z[j];
        v[i * 3 + j] = vv[j] + sigma_v * z[3 + j];
    }
}

} // namespace

extern "C" gpop_status gpop_sample_states(gpop_ctx* ctx, const double* r_nominal, const double* v_nominal,
    double sigma_r, double sigma_v, uint64_t seed, int64_t n, double* r_dev, double* v_dev, void* stream)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    if (!r_nominal || !v_nominal || n < 0 || (n > 0 && (!r_dev || !v_dev)) || !(sigma_r >= 0.0)
        || !(sigma_v >= 0.0) || !std::isfinite(sigma_r) || !std::isfinite(sigma_v))
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid sampling arguments");
    if (n == 0)
        return GPOP_OK;
    cudaError_t e = cudaSetDevice(ctx->cfg.device);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "cudaSetDevice");
    const int block = 256;
    sample_kernel<<<(unsigned)((n + block - 1) / block), block, 0, static_cast<cudaStream_t>(stream)>>>(n,
        r_nominal[0], r_nominal[1], r_nominal[2], v_nominal[0], v_nominal[1], v_nominal[2], sigma_r, sigma_v,
        (uint32_t)seed, (uint32_t)(seed >> 32), r_dev, v_dev);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return cuda_fail(ctx, e, "sampling kernel");
    ctx->launches++;
    return GPOP_OK;
}
