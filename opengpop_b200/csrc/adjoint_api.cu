// adjoint_api.cu -- C ABI of the variational equations and the adjoint (FP64): state transition
// matrices, vector-Jacobian products of the propagation, and the gradient of the closest-approach
// miss distance of listed pairs with respect to both objects' initial states.
#include "common.cuh"
#include "context.h"
#include "variational.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

using namespace gpop;

namespace {

struct ScopedBufs {
    DevBuf b[12];
    ~ScopedBufs()
    {
        for (DevBuf& x : b)
            x.release();
    }
};

bool valid_start(const gpop_time* t)
{
    return t && t->month >= 1 && t->month <= 12 && t->day >= 1 && t->day <= 31 && std::isfinite(t->sec);
}

gpop_status check_common(gpop_ctx* ctx, const gpop_time* start, double h, int32_t steps, int64_t n,
    const void* r_in, const void* v_in)
{
    if (!valid_start(start) || !(h > 0.0) || !std::isfinite(h) || steps < 0 || n <= 0 || !r_in || !v_in)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid propagation arguments");
    if (n > (int64_t)1 << 24)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "too many objects");
    const int64_t bad = first_bad_state(static_cast<const double*>(r_in), static_cast<const double*>(v_in), n, true);
    if (bad >= 0)
        return bad_state(ctx, bad, "object");
    if (ctx->cfg.n_corrections < 1)
        return fail(ctx, GPOP_ERR_UNSUPPORTED, "the adjoint needs at least one corrector pass");
    cudaError_t e = cudaSetDevice(ctx->cfg.device);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "cudaSetDevice");
    return GPOP_OK;
}

gpop_status upload(gpop_ctx* ctx, DevBuf& d, const double* host, size_t count, cudaStream_t s)
{
    cudaError_t e = d.ensure(count * sizeof(double));
    if (e != cudaSuccess)
        return fail(ctx, GPOP_ERR_NOMEM, std::string("device buffer: ") + cudaGetErrorString(e));
    if ((e = cudaMemcpyAsync(d.p, host, count * sizeof(double), cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "upload");
    return GPOP_OK;
}

// FP64 propagation of n objects (device AoS r, v in place) that saves the GJ8 state after the
// startup and after every 64th step, and optionally the trajectory ([steps][3][n] r, v, a).
gpop_status forward_checkpointed(gpop_ctx* ctx, gpop_propagator& p, const gpop_time* start, double h,
    int32_t steps, int64_t n, double* r, double* v, DevBuf& ckpt, double* traj_r, double* traj_v,
    double* traj_a, cudaStream_t s)
{
    p.ctx = ctx;
    p.kind = GPOP_FORCE_GRAVITY;
    p.start = *start;
    p.h = h;
    p.ncorr = ctx->cfg.n_corrections;
    p.max_steps = steps;
    p.n = n;
    p.r = r;
    p.v = v;
    p.mixed = false;
    gpop_status st = propagator_init(&p, s);
    if (st != GPOP_OK)
        return st;
    const int nseg = (steps - 1) / kCheckpointSteps + 1;
    const size_t ck_elems = (size_t)kCheckpointArrays * n;
    cudaError_t e = ckpt.ensure(std::max(1, nseg) * ck_elems * sizeof(double));
    if (e != cudaSuccess)
        return fail(ctx, GPOP_ERR_NOMEM, std::string("checkpoints: ") + cudaGetErrorString(e));
    const double* state_ck = p.state->as<double>() + (size_t)kSs * n;
    auto tr = [&](double* base, int done) { return base ? base + (size_t)done * 3 * n : nullptr; };
    int done = std::min(steps, 4); // startup + the replayed steps: the GJ8 state is final here
    if ((st = propagator_step(&p, done, tr(traj_r, 0), tr(traj_v, 0), tr(traj_a, 0), s)) != GPOP_OK)
        return st;
    if ((e = cudaMemcpyAsync(ckpt.p, state_ck, ck_elems * sizeof(double), cudaMemcpyDeviceToDevice, s))
        != cudaSuccess)
        return cuda_fail(ctx, e, "checkpoint copy");
    for (int seg = 0; done < steps; ++seg) {
        const int target = std::min(steps, (seg + 1) * kCheckpointSteps);
        if ((st = propagator_step(&p, target - done, tr(traj_r, done), tr(traj_v, done), tr(traj_a, done), s))
            != GPOP_OK)
            return st;
        done = target;
        if (done < steps
            && (e = cudaMemcpyAsync(ckpt.as<double>() + (size_t)(seg + 1) * ck_elems, state_ck,
                    ck_elems * sizeof(double), cudaMemcpyDeviceToDevice, s))
                != cudaSuccess)
            return cuda_fail(ctx, e, "checkpoint copy");
    }
    return GPOP_OK;
}

// Reverse sweep for n_units seeded units over a checkpointed forward run.
gpop_status run_adjoint(gpop_ctx* ctx, gpop_propagator& p, int32_t steps, int64_t n_obj,
    const double* r0, const double* v0, const DevBuf& ckpt, int64_t n_units, const int* unit_obj,
    const int* seed_step0, const double* seeds, double* grad, DevBuf& scratch, cudaStream_t s)
{
    const size_t scr = (size_t)kCheckpointSteps * 3 * n_units;
    cudaError_t e = scratch.ensure(scr * sizeof(double));
    if (e != cudaSuccess)
        return fail(ctx, GPOP_ERR_NOMEM, std::string("adjoint scratch: ") + cudaGetErrorString(e));
    AdjArgs a;
    a.n_obj = n_obj;
    a.n_units = n_units;
    a.unit_obj = unit_obj;
    a.seed_step0 = seed_step0;
    a.seeds = seeds;
    a.steps = steps;
    a.h = p.h;
    a.ncorr = ctx->cfg.n_corrections;
    a.flags = ctx->cfg.flags;
    a.gen_m = p.gen_m->as<double>();
    a.prop_m = p.prop_m->as<double>();
    a.r0 = r0;
    a.v0 = v0;
    a.ckpt = ckpt.as<double>();
    a.scratch = scratch.as<double>();
    a.grad = grad;
    a.err = ctx->err_word.as<unsigned>();
    if ((e = launch_adjoint(ctx->lane_table(false), a, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "adjoint kernel");
    ctx->launches++;
    return check_device_errors(ctx, s);
}

} // namespace

extern "C" {

gpop_status gpop_gravity_jacobian(gpop_ctx* ctx, int64_t n, const double* r_dev, const double* frame9_dev,
    double* a_dev, double* jac_dev, void* stream)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    if (n < 0 || (n > 0 && (!r_dev || !jac_dev)))
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid Jacobian arguments");
    cudaError_t e = cudaSetDevice(ctx->cfg.device);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "cudaSetDevice");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if ((e = launch_jacobian(ctx->lane_table(false), n, r_dev, frame9_dev, a_dev, jac_dev,
             ctx->err_word.as<unsigned>(), s))
        != cudaSuccess)
        return cuda_fail(ctx, e, "Jacobian kernel");
    ctx->launches++;
    return check_device_errors(ctx, s);
}

gpop_status gpop_stm(gpop_ctx* ctx, const gpop_time* start, double h, int32_t steps, int64_t n,
    const double* r_in, const double* v_in, double* r_out, double* v_out, double* stm_out)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    gpop_status st = check_common(ctx, start, h, steps, n, r_in, v_in);
    if (st != GPOP_OK)
        return st;
    if (!stm_out)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "missing STM output");
    if (steps == 0) {
        for (int64_t o = 0; o < n; ++o)
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j < 6; ++j)
                    stm_out[(o * 6 + i) * 6 + j] = i == j ? 1.0 : 0.0;
        if (r_out)
            std::copy(r_in, r_in + 3 * n, r_out);
        if (v_out)
            std::copy(v_in, v_in + 3 * n, v_out);
        return GPOP_OK;
    }
    cudaStream_t s = nullptr;
    ScopedBufs B;
    DevBuf &gen = B.b[0], &prop = B.b[1], &dr = B.b[2], &dv = B.b[3], &dro = B.b[4], &dvo = B.b[5],
           &dphi = B.b[6];
    if ((st = build_epoch_tables(ctx, start, h, steps, gen, prop, s)) != GPOP_OK
        || (st = upload(ctx, dr, r_in, 3 * n, s)) != GPOP_OK || (st = upload(ctx, dv, v_in, 3 * n, s)) != GPOP_OK)
        return st;
    cudaError_t e;
    if ((e = dro.ensure(3 * n * sizeof(double))) != cudaSuccess || (e = dvo.ensure(3 * n * sizeof(double))) != cudaSuccess
        || (e = dphi.ensure(36 * n * sizeof(double))) != cudaSuccess)
        return fail(ctx, GPOP_ERR_NOMEM, std::string("STM buffers: ") + cudaGetErrorString(e));
    VarArgs a;
    a.n = n;
    a.steps = steps;
    a.h = h;
    a.ncorr = ctx->cfg.n_corrections;
    a.flags = ctx->cfg.flags;
    a.gen_m = gen.as<double>();
    a.prop_m = prop.as<double>();
    a.r0 = dr.as<double>();
    a.v0 = dv.as<double>();
    a.r_out = dro.as<double>();
    a.v_out = dvo.as<double>();
    a.phi = dphi.as<double>();
    a.err = ctx->err_word.as<unsigned>();
    if ((e = launch_stm(ctx->lane_table(false), a, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "STM kernel");
    ctx->launches++;
    if ((e = cudaMemcpyAsync(stm_out, dphi.p, 36 * n * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess
        || (r_out && (e = cudaMemcpyAsync(r_out, dro.p, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        || (v_out && (e = cudaMemcpyAsync(v_out, dvo.p, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess))
        return cuda_fail(ctx, e, "STM download");
    return check_device_errors(ctx, s);
}

gpop_status gpop_propagate_vjp(gpop_ctx* ctx, const gpop_time* start, double h, int32_t steps, int64_t n,
    const double* r_in, const double* v_in, const double* r_bar, const double* v_bar, double* grad_r0,
    double* grad_v0)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    gpop_status st = check_common(ctx, start, h, steps, n, r_in, v_in);
    if (st != GPOP_OK)
        return st;
    if (!grad_r0 || !grad_v0)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "missing gradient outputs");
    if (steps == 0) {
        for (int64_t i = 0; i < 3 * n; ++i) {
            grad_r0[i] = r_bar ? r_bar[i] : 0.0;
            grad_v0[i] = v_bar ? v_bar[i] : 0.0;
        }
        return GPOP_OK;
    }
    cudaStream_t s = nullptr;
    ScopedBufs B;
    DevBuf &dr = B.b[0], &dv = B.b[1], &dr0 = B.b[2], &dv0 = B.b[3], &ck = B.b[4], &scr = B.b[5],
           &dobj = B.b[6], &dstep = B.b[7], &dseed = B.b[8], &dgrad = B.b[9];
    if ((st = upload(ctx, dr, r_in, 3 * n, s)) != GPOP_OK || (st = upload(ctx, dv, v_in, 3 * n, s)) != GPOP_OK
        || (st = upload(ctx, dr0, r_in, 3 * n, s)) != GPOP_OK || (st = upload(ctx, dv0, v_in, 3 * n, s)) != GPOP_OK)
        return st;
    gpop_propagator p;
    if ((st = forward_checkpointed(ctx, p, start, h, steps, n, dr.as<double>(), dv.as<double>(), ck, nullptr,
             nullptr, nullptr, s))
        != GPOP_OK)
        return st;
    // seeds on the final state: node 0 at the last step
    std::vector<int> obj(n), step0(n, steps);
    std::vector<double> seeds((size_t)n * 27, 0.0);
    for (int64_t o = 0; o < n; ++o) {
        obj[o] = (int)o;
        for (int j = 0; j < 3; ++j) {
            seeds[o * 27 + j] = r_bar ? r_bar[o * 3 + j] : 0.0;
            seeds[o * 27 + 3 + j] = v_bar ? v_bar[o * 3 + j] : 0.0;
        }
    }
    cudaError_t e;
    if ((e = dobj.ensure(n * sizeof(int))) != cudaSuccess || (e = dstep.ensure(n * sizeof(int))) != cudaSuccess
        || (e = dgrad.ensure(6 * n * sizeof(double))) != cudaSuccess)
        return fail(ctx, GPOP_ERR_NOMEM, std::string("adjoint buffers: ") + cudaGetErrorString(e));
    if ((st = upload(ctx, dseed, seeds.data(), seeds.size(), s)) != GPOP_OK)
        return st;
    if ((e = cudaMemcpyAsync(dobj.p, obj.data(), n * sizeof(int), cudaMemcpyHostToDevice, s)) != cudaSuccess
        || (e = cudaMemcpyAsync(dstep.p, step0.data(), n * sizeof(int), cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "seed upload");
    if ((st = run_adjoint(ctx, p, steps, n, dr0.as<double>(), dv0.as<double>(), ck, n, dobj.as<int>(),
             dstep.as<int>(), dseed.as<double>(), dgrad.as<double>(), scr, s))
        != GPOP_OK)
        return st;
    std::vector<double> g(6 * n);
    if ((e = cudaMemcpy(g.data(), dgrad.p, 6 * n * sizeof(double), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(ctx, e, "gradient download");
    for (int64_t o = 0; o < n; ++o)
        for (int j = 0; j < 3; ++j) {
            grad_r0[o * 3 + j] = g[o * 6 + j];
            grad_v0[o * 3 + j] = g[o * 6 + 3 + j];
        }
    return GPOP_OK;
}

gpop_status gpop_miss_gradient(gpop_ctx* ctx, const gpop_time* start, double h, int32_t steps, int64_t n,
    const double* r_in, const double* v_in, int64_t n_pairs, const int32_t* pairs, double* tca,
    double* miss, double* grad)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    gpop_status st = check_common(ctx, start, h, steps, n, r_in, v_in);
    if (st != GPOP_OK)
        return st;
    if (steps < 1 || n_pairs <= 0 || !pairs || !tca || !miss || !grad)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid pair arguments");
    if (n_pairs > (int64_t)1 << 24)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "too many pairs");
    for (int64_t i = 0; i < n_pairs; ++i) {
        const int32_t a = pairs[2 * i], b = pairs[2 * i + 1];
        if (a < 0 || b < 0 || a >= n || b >= n || a == b)
            return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid pair " + std::to_string(i));
    }
    const size_t traj_bytes = (size_t)steps * 3 * n * sizeof(double);
    cudaStream_t s = nullptr;
    ScopedBufs B;
    DevBuf &dr = B.b[0], &dv = B.b[1], &dr0 = B.b[2], &dv0 = B.b[3], &ck = B.b[4], &scr = B.b[5],
           &traj = B.b[6], &dpairs = B.b[7], &units = B.b[8], &dseed = B.b[9], &out = B.b[10],
           &dgrad = B.b[11];
    if ((st = upload(ctx, dr, r_in, 3 * n, s)) != GPOP_OK || (st = upload(ctx, dv, v_in, 3 * n, s)) != GPOP_OK
        || (st = upload(ctx, dr0, r_in, 3 * n, s)) != GPOP_OK || (st = upload(ctx, dv0, v_in, 3 * n, s)) != GPOP_OK)
        return st;
    cudaError_t e;
    const int64_t U = 2 * n_pairs;
    if ((e = traj.ensure(3 * traj_bytes)) != cudaSuccess
        || (e = dpairs.ensure(2 * n_pairs * sizeof(int32_t))) != cudaSuccess
        || (e = units.ensure(2 * U * sizeof(int))) != cudaSuccess
        || (e = dseed.ensure(27 * U * sizeof(double))) != cudaSuccess
        || (e = out.ensure(n_pairs * (2 * sizeof(double) + sizeof(int)))) != cudaSuccess
        || (e = dgrad.ensure(6 * U * sizeof(double))) != cudaSuccess)
        return fail(ctx, GPOP_ERR_NOMEM, std::string("pair buffers: ") + cudaGetErrorString(e));
    double* tr = traj.as<double>();
    const size_t tn = (size_t)steps * 3 * n;
    gpop_propagator p;
    if ((st = forward_checkpointed(ctx, p, start, h, steps, n, dr.as<double>(), dv.as<double>(), ck, tr, tr + tn,
             tr + 2 * tn, s))
        != GPOP_OK)
        return st;
    if ((e = cudaMemcpyAsync(dpairs.p, pairs, 2 * n_pairs * sizeof(int32_t), cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "pair upload");
    PairArgs pa;
    pa.n_obj = n;
    pa.n_pairs = n_pairs;
    pa.pairs = dpairs.as<int>();
    pa.steps = steps;
    pa.h = h;
    pa.traj_r = tr;
    pa.traj_v = tr + tn;
    pa.traj_a = tr + 2 * tn;
    pa.tca = out.as<double>();
    pa.miss = out.as<double>() + n_pairs;
    pa.closest = reinterpret_cast<int*>(out.as<double>() + 2 * n_pairs);
    pa.unit_obj = units.as<int>();
    pa.seed_step0 = units.as<int>() + U;
    pa.seeds = dseed.as<double>();
    if ((e = launch_pair_approach(pa, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "pair approach kernel");
    ctx->launches++;
    traj.release(); // the reverse sweep needs only the checkpoints
    if ((st = run_adjoint(ctx, p, steps, n, dr0.as<double>(), dv0.as<double>(), ck, U, pa.unit_obj,
             pa.seed_step0, pa.seeds, dgrad.as<double>(), scr, s))
        != GPOP_OK)
        return st;
    std::vector<double> g(6 * U);
    if ((e = cudaMemcpy(g.data(), dgrad.p, 6 * U * sizeof(double), cudaMemcpyDeviceToHost)) != cudaSuccess
        || (e = cudaMemcpy(tca, pa.tca, n_pairs * sizeof(double), cudaMemcpyDeviceToHost)) != cudaSuccess
        || (e = cudaMemcpy(miss, pa.miss, n_pairs * sizeof(double), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(ctx, e, "result download");
    std::copy(g.begin(), g.end(), grad); // [pair][object a: r0 3, v0 3 | object b: r0 3, v0 3]
    return GPOP_OK;
}

} // extern "C"
