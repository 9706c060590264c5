// noalloc.cu -- propagation entry point that allocates no device memory.
//
// Who needs it: callers that may not allocate device memory once they are running. Examples are
// conjunction-screening services that reserve their whole memory budget at start-up and forbid
// allocation afterwards (so a long-running process cannot fail or fragment half-way), and host
// applications whose device memory is already held by another allocator's pool, where a
// cudaMalloc would fail. gpop_propagate_device sizes its scratch (the per-object GJ8 state and the
// epoch tables) with cudaMalloc on demand; this variant keeps the same scratch in one fixed
// file-scope device array instead, so a call never allocates.
//
// Limits: at most GPOP_NOALLOC_MAX_OBJECTS objects and GPOP_NOALLOC_MAX_STEPS steps per call
// (about 4.5 MB of device memory, held by every GPU that loads the library until the process
// exits). Every call shares the one array and finds the previous call's contents in it; calls that
// overlap on the GPU (several streams, threads or contexts at once) race on it.
//
// Set-up: every call looks the array's device address up with cudaGetSymbolAddress, with the
// context's device current. The address belongs to the CUDA context that loaded the library's
// device code; a cudaDeviceReset (which test harnesses written for the reference call between
// cases) makes a new context whose array may lie elsewhere, so a cached address could go stale.
// The lookup is a host-side query that allocates nothing. The first call on a device also loads
// the device code, so that first call should come before any stream capture. Each call waits for
// its own work (it reads the device error word back) before it returns.
#include "common.cuh"
#include "context.h"

#include <algorithm>
#include <cmath>
#include <string>

using namespace gpop;

namespace {

constexpr int64_t kMaxObjects = GPOP_NOALLOC_MAX_OBJECTS;
constexpr int kMaxSteps = GPOP_NOALLOC_MAX_STEPS;
constexpr int kMaxEpochs = 4 + kMaxSteps + 1; // propagation table entries
// Scratch layout in doubles: state | generation matrices | propagation matrices | generation
// seconds | propagation seconds | error word
constexpr size_t kOffState = 0;
constexpr size_t kOffGen = kOffState + (size_t)kStateArrays * kMaxObjects;
constexpr size_t kOffProp = kOffGen + 80 * 9;
constexpr size_t kOffGenSec = kOffProp + (size_t)kMaxEpochs * 9;
constexpr size_t kOffPropSec = kOffGenSec + 80;
constexpr size_t kOffErr = kOffPropSec + kMaxEpochs;
constexpr size_t kScratchDoubles = kOffErr + 1;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

__device__ const double kNodesDev[10]
    = { 0.0, 4.0 / 27.0, 2.0 / 9.0, 1.0 / 3.0, 1.0 / 2.0, 2.0 / 3.0, 1.0 / 6.0, 1.0, 5.0 / 6.0, 1.0 };

// Seconds arguments of the epoch tables, computed on the device with the same arithmetic (and no
// contraction) as the host path: (sec - 4 h) + time from the table start.
__global__ void epoch_args_kernel(double sec, double h, int count, bool fix_q1, double* gen_sec,
    double* prop_sec)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double base = __dsub_rn(sec, __dmul_rn(4.0, h));
    if (i < 80) {
        const int sp = i / 10 - 4;
        const int k = i % 10;
        double from = __dmul_rn(__dadd_rn((double)(i / 10), kNodesDev[k]), h);
        if (fix_q1 && sp < 0)
            from = __dadd_rn(__dmul_rn(__dsub_rn((double)(sp + 1), kNodesDev[k]), h), __dmul_rn(4.0, h));
        gen_sec[i] = __dadd_rn(base, from);
    }
    if (i < count)
        prop_sec[i] = __dadd_rn(base, __dmul_rn((double)i, h));
}

// The scratch array's device address in the current CUDA context (the caller has made the
// context's device current). Host code must not use g_noalloc_scratch itself: there it names a
// host-side stand-in, not device memory.
gpop_status scratch_address(gpop_ctx* ctx, double** out)
{
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return cuda_fail(ctx, e, "cudaGetSymbolAddress(no-alloc scratch)");
    *out = static_cast<double*>(p);
    return GPOP_OK;
}

} // namespace

extern "C" gpop_status gpop_propagate_device_noalloc(gpop_ctx* ctx, const gpop_time* start,
    double h, int32_t steps, int64_t n, double* r_dev, double* v_dev, void* stream)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    if (n > kMaxObjects || steps > kMaxSteps)
        return fail(ctx, GPOP_ERR_INVALID_ARG,
            "no-alloc propagation is limited to " + std::to_string(kMaxObjects) + " objects and "
                + std::to_string(kMaxSteps) + " steps per call");
    if (n <= 0 || !r_dev || !v_dev || !(h != 0.0) || !std::isfinite(h) || steps < 0 || !start
        || start->month < 1 || start->month > 12 || start->day < 1 || start->day > 31
        || !std::isfinite(start->sec))
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid propagation arguments");
    cudaError_t e = cudaSetDevice(ctx->cfg.device);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "cudaSetDevice");
    if (steps == 0)
        return GPOP_OK;
    double* scratch = nullptr;
    gpop_status st = scratch_address(ctx, &scratch);
    if (st != GPOP_OK)
        return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned* err = reinterpret_cast<unsigned*>(scratch + kOffErr);
    // the error word must start at zero; everything else is fully written before it is read
    if ((e = cudaMemsetAsync(err, 0, sizeof(double), s)) != cudaSuccess)
        return cuda_fail(ctx, e, "clearing the no-alloc error word");
    const int count = 4 + std::max(steps, 4) + 1;
    epoch_args_kernel<<<(count + 255) / 256, 256, 0, s>>>(start->sec, h, count,
        (ctx->cfg.flags & GPOP_FIX_BACKWARD_RK8_EPOCH) != 0, scratch + kOffGenSec, scratch + kOffPropSec);
    if ((e = cudaGetLastError()) != cudaSuccess
        || (e = launch_frames(ctx->frames, start->year, start->month, start->day, start->hour,
                start->min, scratch + kOffGenSec, 80, scratch + kOffGen, nullptr, s))
            != cudaSuccess
        || (e = launch_frames(ctx->frames, start->year, start->month, start->day, start->hour,
                start->min, scratch + kOffPropSec, count, scratch + kOffProp, nullptr, s))
            != cudaSuccess)
        return cuda_fail(ctx, e, "epoch tables");
    const bool mixed = ctx->cfg.precision == GPOP_MIXED;
    // the same walk and tables as gpop_propagate_device (both built when the context was made)
    const TableSrc ts = ctx->table(mixed);
    const TableSrc lane_ts = ctx->lane_table(mixed);
    PropArgs a;
    a.n = n;
    a.h = h;
    a.ncorr = ctx->cfg.n_corrections;
    a.state = scratch + kOffState;
    a.gen_m = scratch + kOffGen;
    a.prop_m = scratch + kOffProp;
    a.kind = GPOP_FORCE_GRAVITY;
    a.flags = ctx->cfg.flags;
    a.err = err;
    a.r0 = r_dev;
    a.v0 = v_dev;
    if ((e = launch_startup(ts, a, ctx->num_sms, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "startup kernel");
    const int chunk = ctx->steps_per_launch;
    for (int b = 1; b <= steps; b += chunk) {
        a.step_begin = b;
        a.step_end = std::min(steps + 1, b + chunk);
        const bool last = a.step_end == steps + 1;
        a.out_r = last ? r_dev : nullptr;
        a.out_v = last ? v_dev : nullptr;
        if ((e = launch_gj8(ts, a, ctx->num_sms, s, ctx->block_override, ctx->walk_mode, &lane_ts))
            != cudaSuccess)
            return cuda_fail(ctx, e, "GJ8 kernel");
    }
    ctx->launches += 4 + (steps + chunk - 1) / chunk;
    unsigned word = 0;
    if ((e = cudaMemcpyAsync(&word, err, sizeof(unsigned), cudaMemcpyDeviceToHost, s)) != cudaSuccess
        || (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_fail(ctx, e, "no-alloc propagation");
    if (word & kErrTmaTimeout)
        return fail(ctx, GPOP_ERR_TIMEOUT,
            (word & kErrTmaUnfinished)
                ? "gravity table staging timed out on the device; a copy was still in flight when its block left"
                : "gravity table staging timed out on the device; every copy had landed when its block left");
    if (word & kErrBadInput)
        return fail(ctx, GPOP_ERR_INVALID_ARG,
            "an initial state is not finite or lies at the origin (the other objects were propagated)");
    if (word)
        return fail(ctx, GPOP_ERR_CUDA, "device error word " + std::to_string(word));
    return GPOP_OK;
}
