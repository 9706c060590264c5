// api.cu -- C ABI: context life cycle, propagation, force model and integrator entry points.
#include "common.cuh"
#include "context.h"
#include "gpop.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <new>

using namespace gpop;

namespace gpop {

gpop_status fail(gpop_ctx* ctx, gpop_status st, const std::string& msg)
{
    if (ctx)
        ctx->err = msg;
    return st;
}

gpop_status cuda_fail(gpop_ctx* ctx, cudaError_t e, const char* what)
{
    return fail(ctx, GPOP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// RK8 stage nodes (force_model/constants.cuh:31-33)
static const double kNodes[10]
    = { 0.0, 4.0 / 27.0, 2.0 / 9.0, 1.0 / 3.0, 1.0 / 2.0, 2.0 / 3.0, 1.0 / 6.0, 1.0, 5.0 / 6.0, 1.0 };

// Seconds argument of the calendar conversion for table entry idx, in the reference's association:
// (sec - before * h) + time_from_table_start (time_points.cu:34-46).
static double sec_arg(const gpop_time& st, double h, int before, double from_start)
{
    return (st.sec - (double)before * h) + from_start;
}

gpop_status build_epoch_tables(gpop_ctx* ctx, const gpop_time* start, double h, int32_t steps,
    DevBuf& gen_m, DevBuf& prop_m, cudaStream_t s)
{
    const int count = 4 + std::max(steps, 4) + 1;
    std::vector<double> gen(80), prop(count);
    for (int idx = 0; idx < 80; ++idx) {
        const int sp = idx / 10 - 4; // s' of force_model.cu:69-71
        const int k = idx % 10;
        double from = ((double)(idx / 10) + kNodes[k]) * h;
        if ((ctx->cfg.flags & GPOP_FIX_BACKWARD_RK8_EPOCH) && sp < 0)
            from = ((double)(sp + 1) - kNodes[k]) * h + 4.0 * h; // true backward stage time
        gen[idx] = sec_arg(*start, h, 4, from);
    }
    for (int i = 0; i < count; ++i)
        prop[i] = sec_arg(*start, h, 4, (double)i * h);
    cudaError_t e;
    if ((e = ctx->gen_sec.ensure(80 * sizeof(double))) != cudaSuccess
        || (e = ctx->prop_sec.ensure(count * sizeof(double))) != cudaSuccess
        || (e = gen_m.ensure(80 * 9 * sizeof(double))) != cudaSuccess
        || (e = prop_m.ensure((size_t)count * 9 * sizeof(double))) != cudaSuccess)
        return cuda_fail(ctx, e, "allocating epoch tables");
    if ((e = cudaMemcpyAsync(ctx->gen_sec.p, gen.data(), 80 * sizeof(double), cudaMemcpyHostToDevice, s))
            != cudaSuccess
        || (e = cudaMemcpyAsync(ctx->prop_sec.p, prop.data(), count * sizeof(double),
                cudaMemcpyHostToDevice, s))
            != cudaSuccess)
        return cuda_fail(ctx, e, "uploading epoch arguments");
    if ((e = launch_frames(ctx->frames, start->year, start->month, start->day, start->hour, start->min,
             ctx->gen_sec.as<double>(), 80, gen_m.as<double>(), nullptr, s))
            != cudaSuccess
        || (e = launch_frames(ctx->frames, start->year, start->month, start->day, start->hour,
                start->min, ctx->prop_sec.as<double>(), count, prop_m.as<double>(), nullptr, s))
            != cudaSuccess)
        return cuda_fail(ctx, e, "frame kernel");
    ctx->launches += 2;
    // the host vectors die here: wait for the (pageable, hence staged) copies to have been consumed
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_fail(ctx, e, "frame kernel");
    return GPOP_OK;
}

gpop_status check_device_errors(gpop_ctx* ctx, cudaStream_t s)
{
    unsigned word = 0;
    cudaError_t e = cudaMemcpyAsync(&word, ctx->err_word.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "kernel execution");
    if (word) {
        cudaMemsetAsync(ctx->err_word.p, 0, sizeof(unsigned), s);
        cudaStreamSynchronize(s);
        if (word & kErrTmaTimeout)
            return fail(ctx, GPOP_ERR_TIMEOUT,
                (word & kErrTmaUnfinished)
                    ? "gravity table staging timed out on the device; a copy was still in flight when its block left"
                    : "gravity table staging timed out on the device; every copy had landed when its block left");
        if (word & kErrBadInput)
            return fail(ctx, GPOP_ERR_INVALID_ARG,
                "an initial state on the device is not finite or lies at the origin (the other "
                "objects were propagated)");
        return fail(ctx, GPOP_ERR_CUDA, "device error word " + std::to_string(word));
    }
    return GPOP_OK;
}

int64_t first_bad_state(const double* r, const double* v, int64_t n, bool radius)
{
    for (int64_t i = 0; i < n; ++i) {
        const double* p = r + 3 * i;
        const double* q = v + 3 * i;
        if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2]) || !std::isfinite(q[0])
            || !std::isfinite(q[1]) || !std::isfinite(q[2]))
            return i;
        if (radius && p[0] == 0.0 && p[1] == 0.0 && p[2] == 0.0)
            return i;
    }
    return -1;
}

gpop_status bad_state(gpop_ctx* ctx, int64_t i, const char* what)
{
    return fail(ctx, GPOP_ERR_INVALID_ARG,
        std::string(what) + " " + std::to_string(i) + ": position or velocity not finite, or position at the origin");
}

static bool valid_time(const gpop_time* t)
{
    return t && t->month >= 1 && t->month <= 12 && t->day >= 1 && t->day <= 31 && std::isfinite(t->sec);
}

gpop_status propagator_init(gpop_propagator* p, cudaStream_t s)
{
    gpop_ctx* ctx = p->ctx;
    if (p->n <= 0 || !p->r || !p->v || !(p->h != 0.0) || !std::isfinite(p->h) || p->max_steps < 0
        || p->ncorr < 1)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid propagation arguments");
    if (p->n > ((int64_t)1 << 31))
        return fail(ctx, GPOP_ERR_INVALID_ARG, "too many objects");
    cudaError_t e = cudaSetDevice(ctx->cfg.device);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "cudaSetDevice");
    if (p->kind == GPOP_FORCE_GRAVITY) {
        if (!valid_time(&p->start))
            return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid start time");
        gpop_status st = build_epoch_tables(ctx, &p->start, p->h, p->max_steps, *p->gen_m, *p->prop_m, s);
        if (st != GPOP_OK)
            return st;
    }
    if ((e = p->state->ensure((size_t)kStateArrays * p->n * sizeof(double))) != cudaSuccess)
        return fail(ctx, GPOP_ERR_NOMEM, std::string("propagation state: ") + cudaGetErrorString(e));
    return GPOP_OK;
}

gpop_status propagator_step(gpop_propagator* p, int steps, double* traj_r, double* traj_v,
    double* traj_a, cudaStream_t s)
{
    gpop_ctx* ctx = p->ctx;
    if (steps <= 0)
        return steps == 0 ? GPOP_OK : fail(ctx, GPOP_ERR_INVALID_ARG, "negative step count");
    if (p->done + steps > p->max_steps)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "more steps than the propagator was created for");
    cudaError_t e = cudaSetDevice(ctx->cfg.device);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "cudaSetDevice");
    const TableSrc ts = ctx->table(p->mixed);
    const TableSrc lane_ts = ctx->lane_table(p->mixed);
    PropArgs a;
    a.n = p->n;
    a.h = p->h;
    a.ncorr = p->ncorr;
    a.state = p->state->as<double>();
    a.gen_m = p->gen_m->as<double>();
    a.prop_m = p->prop_m->as<double>();
    a.kind = p->kind;
    a.flags = ctx->cfg.flags;
    a.err = ctx->err_word.as<unsigned>();
    a.r0 = p->r;
    a.v0 = p->v;
    if (!p->started) {
        if ((e = launch_startup(ts, a, ctx->num_sms, s)) != cudaSuccess)
            return cuda_fail(ctx, e, "startup kernel");
        ctx->launches++;
        p->started = true;
    }
    a.traj_r = traj_r;
    a.traj_v = traj_v;
    a.traj_a = traj_a;
    a.traj_step0 = p->done + 1;
    const int first = p->done + 1, end = p->done + steps + 1;
    const int chunk = ctx->steps_per_launch;
    for (int b = first; b < end; b += chunk) {
        a.step_begin = b;
        a.step_end = std::min(end, b + chunk);
        const bool last = a.step_end == end;
        a.out_r = last ? p->r : nullptr;
        a.out_v = last ? p->v : nullptr;
        if ((e = launch_gj8(ts, a, ctx->num_sms, s, ctx->block_override, ctx->walk_mode, &lane_ts))
            != cudaSuccess)
            return cuda_fail(ctx, e, "GJ8 kernel");
        ctx->launches++;
    }
    p->done += steps;
    return check_device_errors(ctx, s);
}

} // namespace gpop

static cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

extern "C" {

void gpop_config_default(gpop_config* cfg)
{
    if (!cfg)
        return;
    cfg->data_dir = nullptr;
    cfg->device = 0;
    cfg->gravity_degree = 0;
    cfg->n_corrections = 7;
    cfg->precision = GPOP_FP64;
    cfg->flags = 0;
}

const char* gpop_status_string(int32_t st)
{
    switch (st) {
    case GPOP_OK:
        return "ok";
    case GPOP_ERR_INVALID_ARG:
        return "invalid argument";
    case GPOP_ERR_CUDA:
        return "CUDA error";
    case GPOP_ERR_DATA:
        return "model data error";
    case GPOP_ERR_NOMEM:
        return "out of memory";
    case GPOP_ERR_TIMEOUT:
        return "device wait timed out";
    case GPOP_ERR_UNSUPPORTED:
        return "unsupported";
    case GPOP_ERR_STATE:
        return "call out of order";
    default:
        return "unknown status";
    }
}

gpop_status gpop_create(const gpop_config* cfg_in, gpop_ctx** out)
{
    if (!out)
        return GPOP_ERR_INVALID_ARG;
    *out = nullptr;
    gpop_config cfg;
    gpop_config_default(&cfg);
    if (cfg_in)
        cfg = *cfg_in;
    if (!cfg.data_dir)
        return GPOP_ERR_INVALID_ARG;
    if (cfg.n_corrections < 1 || cfg.n_corrections > 64 || (cfg.precision != GPOP_FP64 && cfg.precision != GPOP_MIXED))
        return GPOP_ERR_INVALID_ARG;
    gpop_ctx* ctx = new (std::nothrow) gpop_ctx();
    if (!ctx)
        return GPOP_ERR_NOMEM;
    ctx->cfg = cfg;
    ctx->data_dir = cfg.data_dir;
    ctx->cfg.data_dir = ctx->data_dir.c_str();
    *out = ctx; // handed out even on failure so gpop_last_error() can explain it
    std::string err;
    if (!load_model(ctx->data_dir, cfg.gravity_degree, ctx->md, err))
        return fail(ctx, GPOP_ERR_DATA, err);
    if (const char* spl = std::getenv("GPOP_STEPS_PER_LAUNCH"))
        ctx->steps_per_launch = std::max(1, atoi(spl));
    if (const char* wm = std::getenv("GPOP_WALK_MODE"))
        ctx->walk_mode = std::min((int)kWalkTwoPlain, std::max(0, atoi(wm)));
    if (const char* ws = std::getenv("GPOP_TEST_FIRST_WAIT_SPINS"))
        ctx->first_wait_spins = (uint32_t)std::min(1L << 22, std::max(0L, atol(ws)));
    cudaError_t e = cudaSetDevice(cfg.device);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "cudaSetDevice");
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, cfg.device);
    // gravity tables
    std::vector<GravEntry64> t64;
    std::vector<GravEntry32> t32;
    build_gravity_tables(ctx->md, t64, t32);
    const int L = ctx->md.degree;
    std::vector<GravEntry64> head(grav_entries(8));
    for (int m = 0; m <= 8; ++m)
        for (int n = m; n <= 8; ++n)
            head[grav_col_offset(m, 8) + (n - m)]
                = (n <= L) ? t64[grav_col_offset(m, L) + (n - m)] : GravEntry64 {};
    ctx->t64_bytes = (uint32_t)(t64.size() * sizeof(GravEntry64));
    ctx->mixed_off32 = (uint32_t)(head.size() * sizeof(GravEntry64));
    ctx->mixed_bytes = ctx->mixed_off32 + (uint32_t)(t32.size() * sizeof(GravEntry32));
    if (table_smem_bytes(ctx->table(false)) > 227 * 1024)
        return fail(ctx, GPOP_ERR_UNSUPPORTED, "gravity degree too high for the shared-memory table");
    std::vector<uint8_t> lane64, lane_mixed;
    if (L > kLaneMaxDegree)
        return fail(ctx, GPOP_ERR_UNSUPPORTED, "gravity degree too high for the lane-layout tables");
    build_lane_blob(t64.data(), L, nullptr, 0, lane64, ctx->lane64_off32);
    build_lane_blob(head.data(), 8, t32.data(), L, lane_mixed, ctx->lane_mixed_off32);
    ctx->lane64_bytes = (uint32_t)lane64.size();
    ctx->lane_mixed_bytes = (uint32_t)lane_mixed.size();
    if (table_smem_bytes(ctx->lane_table(false)) > 227 * 1024)
        return fail(ctx, GPOP_ERR_UNSUPPORTED, "gravity degree too high for the lane-layout table");
    // frame data
    std::vector<NutTerm> nut;
    nut.insert(nut.end(), ctx->md.lon0.begin(), ctx->md.lon0.end());
    nut.insert(nut.end(), ctx->md.lon1.begin(), ctx->md.lon1.end());
    nut.insert(nut.end(), ctx->md.obl0.begin(), ctx->md.obl0.end());
    nut.insert(nut.end(), ctx->md.obl1.begin(), ctx->md.obl1.end());
    std::vector<double> leap(ctx->md.leap_mjd);
    leap.insert(leap.end(), ctx->md.leap_val.begin(), ctx->md.leap_val.end());
    if ((e = ctx->t64.ensure(ctx->t64_bytes)) != cudaSuccess
        || (e = ctx->mixed.ensure(ctx->mixed_bytes)) != cudaSuccess
        || (e = ctx->nut.ensure(nut.size() * sizeof(NutTerm))) != cudaSuccess
        || (e = ctx->eop.ensure(ctx->md.eop.size() * sizeof(EopRec))) != cudaSuccess
        || (e = ctx->leap.ensure(leap.size() * sizeof(double))) != cudaSuccess
        || (e = ctx->err_word.ensure(sizeof(unsigned))) != cudaSuccess
        || (e = ctx->lane64.ensure(lane64.size())) != cudaSuccess
        || (e = ctx->lane_mixed.ensure(lane_mixed.size())) != cudaSuccess)
        return cuda_fail(ctx, e, "allocating model data");
    uint8_t* mixed = ctx->mixed.as<uint8_t>();
    if ((e = cudaMemcpy(ctx->t64.p, t64.data(), ctx->t64_bytes, cudaMemcpyHostToDevice)) != cudaSuccess
        || (e = cudaMemcpy(mixed, head.data(), ctx->mixed_off32, cudaMemcpyHostToDevice)) != cudaSuccess
        || (e = cudaMemcpy(mixed + ctx->mixed_off32, t32.data(), t32.size() * sizeof(GravEntry32),
                cudaMemcpyHostToDevice))
            != cudaSuccess
        || (e = cudaMemcpy(ctx->nut.p, nut.data(), nut.size() * sizeof(NutTerm), cudaMemcpyHostToDevice))
            != cudaSuccess
        || (e = cudaMemcpy(ctx->eop.p, ctx->md.eop.data(), ctx->md.eop.size() * sizeof(EopRec),
                cudaMemcpyHostToDevice))
            != cudaSuccess
        || (e = cudaMemcpy(ctx->leap.p, leap.data(), leap.size() * sizeof(double), cudaMemcpyHostToDevice))
            != cudaSuccess
        || (e = cudaMemset(ctx->err_word.p, 0, sizeof(unsigned))) != cudaSuccess
        || (e = cudaMemcpy(ctx->lane64.p, lane64.data(), lane64.size(), cudaMemcpyHostToDevice)) != cudaSuccess
        || (e = cudaMemcpy(ctx->lane_mixed.p, lane_mixed.data(), lane_mixed.size(), cudaMemcpyHostToDevice))
            != cudaSuccess)
        return cuda_fail(ctx, e, "uploading model data");
    FrameData& fd = ctx->frames;
    fd.nut = ctx->nut.as<NutTerm>();
    fd.n_lon0 = (int)ctx->md.lon0.size();
    fd.n_lon1 = (int)ctx->md.lon1.size();
    fd.n_obl0 = (int)ctx->md.obl0.size();
    fd.n_obl1 = (int)ctx->md.obl1.size();
    fd.eop = ctx->eop.as<EopRec>();
    fd.n_eop = (int)ctx->md.eop.size();
    fd.leap_mjd = ctx->leap.as<double>();
    fd.leap_val = ctx->leap.as<double>() + ctx->md.leap_mjd.size();
    fd.n_leap = (int)ctx->md.leap_mjd.size();
    ctx->err.clear();
    return GPOP_OK;
}

void gpop_destroy(gpop_ctx* ctx)
{
    if (!ctx)
        return;
    destroy_batch_cache(ctx);
    for (DevBuf* b : { &ctx->lane64, &ctx->lane_mixed, &ctx->t64, &ctx->mixed, &ctx->nut, &ctx->eop, &ctx->leap, &ctx->err_word,
             &ctx->state, &ctx->gen_m, &ctx->prop_m, &ctx->gen_sec, &ctx->prop_sec, &ctx->io_r,
             &ctx->io_v })
        b->release();
    delete ctx;
}

const char* gpop_last_error(const gpop_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }
int32_t gpop_gravity_degree(const gpop_ctx* ctx) { return ctx ? ctx->md.degree : -1; }
int64_t gpop_kernel_launches(const gpop_ctx* ctx) { return ctx ? ctx->launches : 0; }

// Startup + chunked GJ8 launches over device AoS buffers (in place), optional trajectory.
static gpop_status run_propagation(gpop_ctx* ctx, int kind, const gpop_time* start, double h,
    int32_t steps, int32_t ncorr, int64_t n, double* r_dev, double* v_dev, double* traj_r,
    double* traj_v, double* traj_a, cudaStream_t s)
{
    gpop_propagator p;
    p.ctx = ctx;
    p.kind = kind;
    if (start)
        p.start = *start;
    p.h = h;
    p.ncorr = ncorr;
    p.max_steps = steps;
    p.n = n;
    p.r = r_dev;
    p.v = v_dev;
    p.mixed = ctx->cfg.precision == GPOP_MIXED;
    p.state = &ctx->state; // borrow the context's scratch
    p.gen_m = &ctx->gen_m;
    p.prop_m = &ctx->prop_m;
    gpop_status st = propagator_init(&p, s);
    if (st == GPOP_OK && steps > 0)
        st = propagator_step(&p, steps, traj_r, traj_v, traj_a, s);
    return st;
}

gpop_status gpop_propagate_device(gpop_ctx* ctx, const gpop_time* start, double h, int32_t steps,
    int64_t n, double* r_dev, double* v_dev, void* stream)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    return run_propagation(ctx, GPOP_FORCE_GRAVITY, start, h, steps, ctx->cfg.n_corrections, n,
        r_dev, v_dev, nullptr, nullptr, nullptr, as_stream(stream));
}

gpop_status gpop_propagate_trajectory(gpop_ctx* ctx, const gpop_time* start, double h,
    int32_t steps, int64_t n, double* r_dev, double* v_dev, double* traj_r, double* traj_v,
    double* traj_a, void* stream)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    return run_propagation(ctx, GPOP_FORCE_GRAVITY, start, h, steps, ctx->cfg.n_corrections, n,
        r_dev, v_dev, traj_r, traj_v, traj_a, as_stream(stream));
}

gpop_status gpop_propagator_create(gpop_ctx* ctx, const gpop_time* start, double h,
    int32_t max_steps, int64_t n, double* r_dev, double* v_dev, gpop_propagator** out)
{
    if (!ctx || !out)
        return GPOP_ERR_INVALID_ARG;
    *out = nullptr;
    if (!start)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "missing start time");
    gpop_propagator* p = new (std::nothrow) gpop_propagator();
    if (!p)
        return fail(ctx, GPOP_ERR_NOMEM, "propagator");
    p->ctx = ctx;
    p->kind = GPOP_FORCE_GRAVITY;
    p->start = *start;
    p->h = h;
    p->ncorr = ctx->cfg.n_corrections;
    p->max_steps = max_steps;
    p->n = n;
    p->r = r_dev;
    p->v = v_dev;
    p->mixed = ctx->cfg.precision == GPOP_MIXED;
    gpop_status st = propagator_init(p, nullptr);
    if (st != GPOP_OK) {
        delete p;
        return st;
    }
    *out = p;
    return GPOP_OK;
}

gpop_status gpop_propagator_step(gpop_propagator* p, int32_t steps, double* traj_r, double* traj_v,
    double* traj_a, void* stream)
{
    if (!p)
        return GPOP_ERR_INVALID_ARG;
    return propagator_step(p, steps, traj_r, traj_v, traj_a, as_stream(stream));
}

int32_t gpop_propagator_steps_done(const gpop_propagator* p) { return p ? p->done : -1; }

int32_t gpop_walk_policy(int64_t n, int32_t num_sms, int32_t precision, int32_t* lanes_out)
{
    if (n <= 0 || num_sms <= 0 || (precision != GPOP_FP64 && precision != GPOP_MIXED))
        return -1;
    const int walk = default_walk(n, num_sms, true, precision == GPOP_FP64);
    if (lanes_out)
        *lanes_out = walk == kWalkLanes ? lanes_per_object(n, num_sms)
            : walk == kWalkLanesTwo     ? lane_pair_lanes(n, num_sms, precision == GPOP_FP64)
                                        : 1;
    return walk;
}

int32_t gpop_split_block(int64_t n, int32_t num_sms, int32_t degree)
{
    if (n <= 0 || num_sms <= 0 || degree < 0)
        return -1;
    return split_owner_warps(n, num_sms, degree);
}

void gpop_propagator_destroy(gpop_propagator* p) { delete p; }

gpop_status gpop_propagate_analytic(gpop_ctx* ctx, int32_t kind, double h, int32_t steps,
    int32_t ncorr, int64_t n, double* r_dev, double* v_dev, double* traj_r, double* traj_v,
    double* traj_a, void* stream)
{
    if (!ctx || kind < GPOP_FORCE_ZERO || kind > GPOP_FORCE_DAMPED)
        return ctx ? fail(ctx, GPOP_ERR_INVALID_ARG, "invalid analytic force kind") : GPOP_ERR_INVALID_ARG;
    return run_propagation(ctx, kind, nullptr, h, steps, ncorr, n, r_dev, v_dev, traj_r, traj_v,
        traj_a, as_stream(stream));
}

gpop_status gpop_propagate(gpop_ctx* ctx, const gpop_time* start, double h, int32_t steps, int64_t n,
    const double* r_in, const double* v_in, double* r_out, double* v_out)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    if (n <= 0 || !r_in || !v_in || !r_out || !v_out)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid buffers");
    const int64_t bad = first_bad_state(r_in, v_in, n, true);
    if (bad >= 0)
        return bad_state(ctx, bad, "object");
    cudaError_t e = cudaSetDevice(ctx->cfg.device);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "cudaSetDevice");
    const size_t bytes = (size_t)n * 3 * sizeof(double);
    if ((e = ctx->io_r.ensure(bytes)) != cudaSuccess || (e = ctx->io_v.ensure(bytes)) != cudaSuccess)
        return fail(ctx, GPOP_ERR_NOMEM, "state buffers");
    cudaStream_t s = nullptr;
    if ((e = cudaMemcpyAsync(ctx->io_r.p, r_in, bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess
        || (e = cudaMemcpyAsync(ctx->io_v.p, v_in, bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "copying state to the device");
    gpop_status st = run_propagation(ctx, GPOP_FORCE_GRAVITY, start, h, steps, ctx->cfg.n_corrections,
        n, ctx->io_r.as<double>(), ctx->io_v.as<double>(), nullptr, nullptr, nullptr, s);
    if (st != GPOP_OK)
        return st;
    if ((e = cudaMemcpyAsync(r_out, ctx->io_r.p, bytes, cudaMemcpyDeviceToHost, s)) != cudaSuccess
        || (e = cudaMemcpyAsync(v_out, ctx->io_v.p, bytes, cudaMemcpyDeviceToHost, s)) != cudaSuccess
        || (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_fail(ctx, e, "copying state to the host");
    return GPOP_OK;
}

gpop_status gpop_startup(gpop_ctx* ctx, int32_t kind, const gpop_time* start, double h,
    int32_t ncorr, const double* r0_dev, const double* v0_dev, double* r27, double* v27,
    double* a27, double* s27, double* S27, void* stream)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    if (kind < GPOP_FORCE_GRAVITY || kind > GPOP_FORCE_DAMPED || !r0_dev || !v0_dev || !r27 || !v27
        || !a27 || !s27 || !S27 || !(h != 0.0) || ncorr < 0)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid startup arguments");
    cudaStream_t s = as_stream(stream);
    cudaSetDevice(ctx->cfg.device);
    if (kind == GPOP_FORCE_GRAVITY) {
        if (!valid_time(start))
            return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid start time");
        gpop_status st = build_epoch_tables(ctx, start, h, 4, ctx->gen_m, ctx->prop_m, s);
        if (st != GPOP_OK)
            return st;
    }
    PropArgs a;
    a.n = 1;
    a.h = h;
    a.ncorr = ncorr;
    a.gen_m = ctx->gen_m.as<double>();
    a.prop_m = ctx->prop_m.as<double>();
    a.kind = kind;
    a.flags = ctx->cfg.flags;
    a.err = ctx->err_word.as<unsigned>();
    a.r0 = r0_dev;
    a.v0 = v0_dev;
    a.out27[0] = r27;
    a.out27[1] = v27;
    a.out27[2] = a27;
    a.out27[3] = s27;
    a.out27[4] = S27;
    cudaError_t e = launch_startup(ctx->table(ctx->cfg.precision == GPOP_MIXED), a, ctx->num_sms, s);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "startup kernel");
    ctx->launches++;
    return check_device_errors(ctx, s);
}

gpop_status gpop_corrector_unit(gpop_ctx* ctx, int32_t kind, double h, int32_t op, double* r27,
    double* v27, double* a27, double* s27, double* S27, void* stream)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    if (kind < GPOP_FORCE_ZERO || kind > GPOP_FORCE_DAMPED || op < 0 || op > 2 || !r27 || !v27
        || !a27 || !s27 || !S27)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid corrector arguments");
    cudaSetDevice(ctx->cfg.device);
    cudaError_t e = launch_corrector_unit(kind, h, op, r27, v27, a27, s27, S27, as_stream(stream));
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "corrector kernel");
    ctx->launches++;
    return check_device_errors(ctx, as_stream(stream));
}

gpop_status gpop_predict_unit(gpop_ctx* ctx, int32_t kind, double h, int32_t step, double* r3,
    double* v3, double* a27, double* s3, double* S3, void* stream)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    if (kind < GPOP_FORCE_ZERO || kind > GPOP_FORCE_DAMPED || !r3 || !v3 || !a27 || !s3 || !S3)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid predictor arguments");
    cudaSetDevice(ctx->cfg.device);
    cudaError_t e = launch_predict_unit(kind, h, step, r3, v3, a27, s3, S3, as_stream(stream));
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "predictor kernel");
    ctx->launches++;
    return check_device_errors(ctx, as_stream(stream));
}

gpop_status gpop_finalize_correction_unit(gpop_ctx* ctx, double h, double* r3, double* v3,
    const double* a27, const double* s3, const double* S3, void* stream)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    if (!r3 || !v3 || !a27 || !s3 || !S3)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid buffers");
    cudaSetDevice(ctx->cfg.device);
    cudaError_t e = launch_finalize_unit(h, r3, v3, a27, s3, S3, as_stream(stream));
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "finalize kernel");
    ctx->launches++;
    return check_device_errors(ctx, as_stream(stream));
}

gpop_status gpop_gravity(gpop_ctx* ctx, int64_t n, const double* r_dev, const double* frame9_dev,
    double* a_dev, int32_t precision, void* stream)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    if (n <= 0 || !r_dev || !a_dev || (precision != GPOP_FP64 && precision != GPOP_MIXED))
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid gravity arguments");
    cudaSetDevice(ctx->cfg.device);
    cudaError_t e = launch_gravity(ctx->table(precision == GPOP_MIXED), n, r_dev, frame9_dev, a_dev,
        ctx->err_word.as<unsigned>(), ctx->num_sms, as_stream(stream));
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "gravity kernel");
    ctx->launches++;
    return check_device_errors(ctx, as_stream(stream));
}

gpop_status gpop_frame_matrices(gpop_ctx* ctx, const gpop_time* start, double h, int32_t count,
    int32_t use_midpoints, int32_t before_epoch, double* m_dev, double* mjd_dev, void* stream)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    if (!valid_time(start) || count <= 0 || !m_dev)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid frame arguments");
    cudaSetDevice(ctx->cfg.device);
    std::vector<double> args(count);
    for (int i = 0; i < count; ++i) {
        double from = use_midpoints ? ((double)(i / 10) + kNodes[i % 10]) * h : (double)i * h;
        args[i] = sec_arg(*start, h, before_epoch, from);
    }
    cudaStream_t s = as_stream(stream);
    cudaError_t e = ctx->prop_sec.ensure(count * sizeof(double));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ctx->prop_sec.p, args.data(), count * sizeof(double), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = launch_frames(ctx->frames, start->year, start->month, start->day, start->hour, start->min,
            ctx->prop_sec.as<double>(), count, m_dev, mjd_dev, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "frame kernel");
    ctx->launches++;
    return GPOP_OK;
}

} // extern "C"
