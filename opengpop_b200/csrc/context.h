// context.h -- the gpop_ctx object behind the C ABI.
#pragma once
#include "gpop.h"
#include "kernels.h"
#include "model.h"

#include <cstring>
#include <string>
#include <vector>

namespace gpop {

// Grow-only device buffer owned by a context.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes)
    {
        if (bytes <= cap)
            return cudaSuccess;
        if (p)
            cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess)
            cap = bytes;
        return e;
    }
    void release()
    {
        if (p)
            cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// Up to four CUDA events on one stream; seconds(a, b) after the stream has passed mark b.
struct DeviceTimer {
    cudaEvent_t ev[4] = {};
    int n = 0;
    void mark(cudaStream_t s)
    {
        if (n >= 4)
            return;
        if (cudaEventCreate(&ev[n]) == cudaSuccess)
            cudaEventRecord(ev[n], s);
        else
            ev[n] = nullptr;
        ++n;
    }
    double seconds(int a, int b) const
    {
        float ms = 0.f;
        if (a < n && b < n && ev[a] && ev[b] && cudaEventElapsedTime(&ms, ev[a], ev[b]) == cudaSuccess)
            return ms * 1e-3;
        return 0.0;
    }
    ~DeviceTimer()
    {
        for (int i = 0; i < n; ++i)
            if (ev[i])
                cudaEventDestroy(ev[i]);
    }
};

} // namespace gpop

struct BatchCache; // buffers and captured graph of the last batch (batch_api.cu)

struct gpop_ctx {
    gpop_config cfg {};
    std::string data_dir;
    std::string err;
    gpop::ModelData md;
    int num_sms = 148;
    int steps_per_launch = 64;
    int block_override = 0; // GJ8 block size chosen by the tuner (0 = default policy)
    int walk_mode = 0; // GJ8 triangle walk (WalkMode; 0 = default)
    // first staging wait of every kernel (TableSrc::wait_spins); GPOP_TEST_FIRST_WAIT_SPINS, a
    // test setting, lowers it so that a test can watch the wait give up
    uint32_t first_wait_spins = 1u << 22;
    // device-resident model data
    gpop::DevBuf t64, mixed, nut, eop, leap, err_word;
    uint32_t t64_bytes = 0, mixed_bytes = 0, mixed_off32 = 0;
    // the same tables in the lane layout (lane-split kernels)
    gpop::DevBuf lane64, lane_mixed;
    uint32_t lane64_bytes = 0, lane64_off32 = 0, lane_mixed_bytes = 0, lane_mixed_off32 = 0;
    gpop::FrameData frames {};
    int64_t launches = 0;
    // scratch
    gpop::DevBuf state, gen_m, prop_m, gen_sec, prop_sec, io_r, io_v;
    // batched propagation: cached plan and graph, its stream and pinned staging buffer
    BatchCache* batch = nullptr;
    cudaStream_t batch_stream = nullptr;
    void* batch_host = nullptr;
    size_t batch_host_cap = 0;
    // batched-kernel throughput (object-steps/s per SM) for the persistent grid's block shapes
    // (4 or 8 warps per SM) x degrees {8, 20, 36, 70} x lanes 1..32
    bool tuned = false;
    double eta[2][4][6] = {};
    int force_lpo = 0; // lanes per object fixed by the autotuner while it measures (0 = planner)
    int force_warps = 0; // warps per SM fixed by the autotuner while it measures (0 = planner)
    int batch_warps = 8; // warps per SM of the last planned batch
    double batch_seconds = 0; // device time of the last batch launch (CUDA events around the graph)

    gpop::TableSrc lane_table(bool mixed_mode) const
    {
        gpop::TableSrc ts;
        ts.L = md.degree;
        ts.radius = md.radius;
        ts.gm = md.gm;
        ts.mixed = mixed_mode;
        ts.lanes = true;
        ts.src = mixed_mode ? lane_mixed.p : lane64.p;
        ts.bytes = mixed_mode ? lane_mixed_bytes : lane64_bytes;
        ts.off32 = mixed_mode ? lane_mixed_off32 : lane64_off32;
        ts.wait_spins = first_wait_spins;
        return ts;
    }

    gpop::TableSrc table(bool mixed_mode) const
    {
        gpop::TableSrc ts;
        ts.L = md.degree;
        ts.radius = md.radius;
        ts.gm = md.gm;
        ts.mixed = mixed_mode;
        if (mixed_mode) {
            ts.src = mixed.p;
            ts.bytes = mixed_bytes;
            ts.off32 = mixed_off32;
        } else {
            ts.src = t64.p;
            ts.bytes = t64_bytes;
            ts.off32 = 0;
        }
        ts.wait_spins = first_wait_spins;
        return ts;
    }
};

// A propagation in progress (GpuPropagator): startup on the first step call, then GJ8 steps.
// The buffers either belong to the object or are borrowed from the context's scratch.
struct gpop_propagator {
    gpop_ctx* ctx = nullptr;
    int kind = 0;
    gpop_time start {};
    double h = 0;
    int ncorr = 7;
    int max_steps = 0;
    int64_t n = 0;
    double* r = nullptr;
    double* v = nullptr;
    int done = 0;
    bool started = false;
    bool mixed = false;
    gpop::DevBuf own_state, own_gen, own_prop;
    gpop::DevBuf *state = &own_state, *gen_m = &own_gen, *prop_m = &own_prop;
    ~gpop_propagator()
    {
        own_state.release();
        own_gen.release();
        own_prop.release();
    }
};

namespace gpop {
gpop_status fail(gpop_ctx* ctx, gpop_status st, const std::string& msg);
gpop_status cuda_fail(gpop_ctx* ctx, cudaError_t e, const char* what);
// Builds and fills the generation (80) and propagation (4 + max(steps,4) + 1) epoch tables.
gpop_status build_epoch_tables(gpop_ctx* ctx, const gpop_time* start, double h, int32_t steps,
    DevBuf& gen_m, DevBuf& prop_m, cudaStream_t s);
// Prepares a propagator (validates, builds epoch tables, sizes the state).
gpop_status propagator_init(gpop_propagator* p, cudaStream_t s);
// Runs `steps` more steps (startup first when needed).
gpop_status propagator_step(gpop_propagator* p, int steps, double* traj_r, double* traj_v,
    double* traj_a, cudaStream_t s);
// Reads and clears the device error word (synchronises the stream).
gpop_status check_device_errors(gpop_ctx* ctx, cudaStream_t s);
// Index of the first object of n (host [n][3] arrays) whose position or velocity has a component
// that is not finite, or, when `radius` is set, whose position is the origin (where gravity is
// undefined); -1 when every object is usable. The reference takes such states without a check.
int64_t first_bad_state(const double* r, const double* v, int64_t n, bool radius);
// GPOP_ERR_INVALID_ARG naming object i of `what`.
gpop_status bad_state(gpop_ctx* ctx, int64_t i, const char* what);
// Frees the batch cache, stream and staging buffer of a context.
void destroy_batch_cache(gpop_ctx* ctx);
} // namespace gpop
