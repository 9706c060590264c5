// common.cuh -- device constants and helpers shared by the propagation and screening kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gpop {

// gpop_config.flags bit (GPOP_MIXED_COMPENSATED in gpop.h): compensated FP32 sums in mixed mode.
constexpr unsigned kFlagMixedCompensated = 1u << 3;

// Error bits a kernel may raise in the context's device error word.
enum : unsigned {
    kErrTmaTimeout = 1u, // the bounded wait on the gravity-table bulk copy gave up
    kErrBadInput = 2u, // a state with a non-finite component, or a position at the origin
    kErrTmaUnfinished = 4u, // a staging copy had still not landed when its block gave up and left
};

// ---- bulk-copy (TMA, cp.async.bulk) staging of a read-only table into shared memory ----
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Copies `bytes` (multiple of 16, both addresses 16-byte aligned) from global to shared memory with
// one elected thread issuing cp.async.bulk chunks that complete on an mbarrier. Every thread of the
// block waits with a bounded spin of first_spins polls; when that runs out the block raises
// kErrTmaTimeout and returns false after a second bounded wait for the copies still in flight
// (kErrTmaUnfinished if they have not landed by then either: the caller's results are void).
__device__ __forceinline__ bool stage_to_smem(void* smem_dst, const void* gsrc, uint32_t bytes,
    uint64_t* mbar, unsigned* err_word, uint32_t first_spins)
{
    const uint32_t bar = smem_u32(mbar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                     : "memory");
        const uint32_t chunk = 32768u;
        uint32_t dst = smem_u32(smem_dst);
        const char* src = static_cast<const char*>(gsrc);
        for (uint32_t off = 0; off < bytes; off += chunk) {
            uint32_t len = (bytes - off) < chunk ? (bytes - off) : chunk;
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                         "[%0], [%1], %2, [%3];" ::"r"(dst + off),
                         "l"(src + off), "r"(len), "r"(bar)
                         : "memory");
        }
    }
    // bounded wait on phase 0 (about a second at the sleep below before giving up)
    uint32_t done = 0;
    for (uint32_t it = 0; it < first_spins && !done; ++it) {
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
                     " selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(done)
                     : "r"(bar)
                     : "memory");
        if (!done)
            __nanosleep(64);
    }
    if (!done) {
        if (threadIdx.x == 0)
            atomicOr(err_word, kErrTmaTimeout);
        // give the copies in flight a second bounded window before the block leaves
        for (int it = 0; it < (1 << 22) && !done; ++it) {
            asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
                         " selp.u32 %0, 1, 0, p;\n}"
                         : "=r"(done)
                         : "r"(bar)
                         : "memory");
            if (!done)
                __nanosleep(64);
        }
        if (!done && threadIdx.x == 0)
            atomicOr(err_word, kErrTmaUnfinished);
        return false;
    }
    return true;
}

// Stores and loads of per-thread values parked in shared memory across a long computation. The
// asm keeps the compiler from forwarding the stored value (which would keep it in a register).
__device__ __forceinline__ void st_stage(double* p, double v)
{
    asm volatile("st.shared.f64 [%0], %1;" ::"r"(smem_u32(p)), "d"(v) : "memory");
}
__device__ __forceinline__ double ld_stage(const double* p)
{
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(smem_u32(p)) : "memory");
    return v;
}

} // namespace gpop
