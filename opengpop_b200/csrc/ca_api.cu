// ca_api.cu -- closest-approach entry points (ClosestApproach, closest_approach.cu:47-209 and the
// record loop of exec/runner.cu:96-106).
#include "common.cuh"
#include "context.h"
#include "screen.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <new>

using namespace gpop;

struct gpop_ca {
    gpop_ctx* ctx = nullptr;
    int kind = GPOP_FORCE_GRAVITY;
    gpop_time start {};
    double h = 0;
    int64_t n = 0;
    // partition (PartitionParameters, partition_parameters.cuh:23-144)
    uint32_t num_sets = 0;
    uint64_t num_pairs = 0;
    std::vector<uint32_t> set_offsets, num_higher;
    std::vector<uint64_t> map_offsets;
    int num_tiles = 0;
    // rows (first objects) whose pairs this object screens and refines, and their pair range;
    // all of them unless gpop_ca_set_rows narrowed it
    int64_t row_lo = 0, row_hi = 0;
    int64_t pair_lo = 0, pair_hi = 0;
    DevBuf r, v, bound, base, tiles, min_d2, min_step, so, nh, mo;
    // trajectory store [step][3][n] for r, v and the exported acceleration
    DevBuf traj_r, traj_v, traj_a;
    int cap_steps = 0;
    int total_steps = 0;
    // per-pair results
    DevBuf dist, time, pos_a, pos_b, cand, count;
    bool refined = false;
    // propagation scratch
    DevBuf state, gen_m, prop_m;
    // cumulative device time (s) of propagation, screen and refinement (CUDA events)
    double t_prop = 0, t_screen = 0, t_refine = 0;

    ~gpop_ca()
    {
        for (DevBuf* b : { &r, &v, &bound, &base, &tiles, &min_d2, &min_step, &so, &nh, &mo, &traj_r,
                 &traj_v, &traj_a, &dist, &time, &pos_a, &pos_b, &cand, &count, &state, &gen_m, &prop_m })
            b->release();
    }
};

namespace {

constexpr int kTile = kScreenTileA; // rows of a screen tile (screen_kernel's block)

__global__ void gather_kernel(const int64_t* idx, int64_t count, const double* dist, const double* time,
    const double* pa, const double* pb, double* out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const int64_t p = idx[i];
    double* o = out + i * 8;
    o[0] = dist[p];
    o[1] = time[p];
    for (int c = 0; c < 3; ++c) {
        o[2 + c] = pa[p * 3 + c];
        o[5 + c] = pb[p * 3 + c];
    }
}

// Pair index -> (a, b) on the host (inverse of GetPartitionMapIdx).
void pair_objects(const gpop_ca* ca, uint64_t idx, uint32_t& a, uint32_t& b)
{
    auto it = std::upper_bound(ca->map_offsets.begin(), ca->map_offsets.begin() + (ca->num_sets - 1), idx);
    const size_t s = (size_t)(it - ca->map_offsets.begin()) - 1;
    const uint64_t rel = idx - ca->map_offsets[s];
    a = (uint32_t)(rel / ca->num_higher[s]) + ca->set_offsets[s];
    b = (uint32_t)(rel % ca->num_higher[s]) + ca->set_offsets[s + 1];
}

// Number of pairs whose first object precedes object a (GetPartitionMapIdx of (a, first b)).
int64_t pairs_before(const gpop_ca* ca, int64_t a)
{
    if (a >= ca->n)
        return (int64_t)ca->num_pairs;
    auto it = std::upper_bound(ca->set_offsets.begin(), ca->set_offsets.end(), (uint32_t)a);
    const size_t s = (size_t)(it - ca->set_offsets.begin()) - 1;
    if (s + 1 >= ca->num_sets)
        return (int64_t)ca->num_pairs;
    return (int64_t)(ca->map_offsets[s] + (uint64_t)(a - ca->set_offsets[s]) * ca->num_higher[s]);
}

// Tiles of the (a, b) staircase with a0 in [row_lo, row_hi), b-major (the screen's work list).
std::vector<int2> staircase_tiles(const gpop_ca* ca, int64_t row_lo, int64_t row_hi)
{
    const int64_t n = ca->n;
    std::vector<int> bound;
    for (int64_t a0 = row_lo; a0 < row_hi; a0 += kTile) {
        auto it = std::upper_bound(ca->set_offsets.begin(), ca->set_offsets.end(), (uint32_t)a0);
        const size_t s = (size_t)(it - ca->set_offsets.begin()) - 1;
        bound.push_back(s + 1 >= ca->num_sets ? (int)n : (int)ca->set_offsets[s + 1]);
    }
    std::vector<int2> tiles;
    for (int64_t b0 = 0; b0 < n; b0 += kScreenTileB)
        for (size_t t = 0; t < bound.size(); ++t)
            if (bound[t] < n && b0 + kScreenTileB > bound[t])
                tiles.push_back(make_int2((int)(row_lo + (int64_t)t * kTile), (int)b0));
    return tiles;
}

gpop_status refine(gpop_ca* ca, cudaStream_t s)
{
    gpop_ctx* ctx = ca->ctx;
    if (ca->refined)
        return GPOP_OK;
    const size_t P = ca->num_pairs;
    cudaError_t e;
    if ((e = ca->dist.ensure(P * 8)) != cudaSuccess || (e = ca->time.ensure(P * 8)) != cudaSuccess
        || (e = ca->pos_a.ensure(P * 24)) != cudaSuccess || (e = ca->pos_b.ensure(P * 24)) != cudaSuccess)
        return fail(ctx, GPOP_ERR_NOMEM, "per-pair results");
    RefineArgs a;
    a.n = ca->n;
    a.num_pairs = (int64_t)P;
    a.pair_lo = ca->pair_lo;
    a.pair_hi = ca->pair_hi;
    a.num_sets = (int)ca->num_sets;
    a.set_offsets = ca->so.as<uint32_t>();
    a.num_higher = ca->nh.as<uint32_t>();
    a.map_offsets = ca->mo.as<uint64_t>();
    a.traj_r = ca->traj_r.as<double>();
    a.traj_v = ca->traj_v.as<double>();
    a.traj_a = ca->traj_a.as<double>();
    a.min_d2 = ca->min_d2.as<double>();
    a.min_step = ca->min_step.as<uint32_t>();
    a.total_steps = (uint32_t)ca->total_steps;
    a.h = ca->h;
    a.dist = ca->dist.as<double>();
    a.time = ca->time.as<double>();
    a.pos_a = ca->pos_a.as<double>();
    a.pos_b = ca->pos_b.as<double>();
    DeviceTimer timer;
    timer.mark(s);
    if ((e = launch_refine(a, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "refine kernel");
    ctx->launches++;
    timer.mark(s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_fail(ctx, e, "refine kernel");
    ca->t_refine += timer.seconds(0, 1);
    ca->refined = true;
    return GPOP_OK;
}

constexpr int kExternalKind = -1; // trajectory supplied by gpop_ca_append

// AoS rows [steps][n][3] of r, v, a into the trajectory store's SoA rows [step][3][n].
__global__ void append_rows_kernel(int64_t n, int64_t count, const double* __restrict__ r,
    const double* __restrict__ v, const double* __restrict__ a, double* __restrict__ tr,
    double* __restrict__ tv, double* __restrict__ ta)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count)
        return;
    const int64_t s = t / n, i = t - s * n;
    for (int j = 0; j < 3; ++j) {
        const int64_t src = (s * n + i) * 3 + j, dst = (s * 3 + j) * n + i;
        tr[dst] = r[src];
        tv[dst] = v[src];
        ta[dst] = a[src];
    }
}

// Replaces the trajectory store by one of `cap` steps, keeping the rows already written.
cudaError_t resize_store(gpop_ca* ca, int cap)
{
    const size_t row = (size_t)ca->n * 3 * sizeof(double);
    DevBuf nr, nv, na;
    cudaError_t e;
    if ((e = nr.ensure(row * cap)) == cudaSuccess && (e = nv.ensure(row * cap)) == cudaSuccess
        && (e = na.ensure(row * cap)) == cudaSuccess && ca->total_steps > 0) {
        const size_t used = row * ca->total_steps;
        if ((e = cudaMemcpy(nr.p, ca->traj_r.p, used, cudaMemcpyDeviceToDevice)) == cudaSuccess
            && (e = cudaMemcpy(nv.p, ca->traj_v.p, used, cudaMemcpyDeviceToDevice)) == cudaSuccess)
            e = cudaMemcpy(na.p, ca->traj_a.p, used, cudaMemcpyDeviceToDevice);
    }
    if (e != cudaSuccess) {
        nr.release();
        nv.release();
        na.release();
        return e;
    }
    ca->traj_r.release();
    ca->traj_v.release();
    ca->traj_a.release();
    ca->traj_r = nr;
    ca->traj_v = nv;
    ca->traj_a = na;
    nr.p = nv.p = na.p = nullptr;
    ca->cap_steps = cap;
    return cudaSuccess;
}

// Grows the trajectory store to hold `need` steps. With `amortized` (steps appended a few at a
// time by a caller that reserved nothing) it first tries twice the present capacity, so that
// appends copy the store O(log steps) times instead of once per call.
gpop_status grow_store(gpop_ca* ca, int need, bool amortized = false)
{
    if (need <= ca->cap_steps)
        return GPOP_OK;
    if (amortized && ca->cap_steps > 0 && 2LL * ca->cap_steps > need && 2LL * ca->cap_steps <= INT32_MAX) {
        if (resize_store(ca, 2 * ca->cap_steps) == cudaSuccess)
            return GPOP_OK;
        cudaGetLastError(); // out of memory for the doubled store: try the exact size
    }
    const cudaError_t e = resize_store(ca, need);
    if (e == cudaErrorMemoryAllocation)
        return fail(ca->ctx, GPOP_ERR_NOMEM,
            "trajectory store (" + std::to_string((size_t)ca->n * 72 * need >> 20) + " MiB)");
    return e == cudaSuccess ? GPOP_OK : cuda_fail(ca->ctx, e, "growing the trajectory store");
}

// UpdateClosestApproachKernel over steps [total_steps, need) of the store (running minima).
gpop_status screen_steps(gpop_ca* ca, int need, cudaStream_t s)
{
    ScreenArgs a;
    a.n = ca->n;
    a.traj_r = ca->traj_r.as<double>();
    a.bound = ca->bound.as<int>();
    a.base = ca->base.as<int64_t>();
    a.tiles = ca->tiles.as<int2>();
    a.min_d2 = ca->min_d2.as<double>();
    a.min_step = ca->min_step.as<uint32_t>();
    a.step_lo = ca->total_steps;
    a.step_hi = need;
    a.step_offset = 0;
    a.init = ca->total_steps == 0 ? 1 : 0;
    const cudaError_t e = launch_screen(a, ca->num_tiles, s);
    if (e != cudaSuccess)
        return cuda_fail(ca->ctx, e, "screen kernel");
    ca->ctx->launches++;
    return GPOP_OK;
}

} // namespace

extern "C" {

gpop_status gpop_ca_create(gpop_ctx* ctx, const gpop_time* start, double h, int64_t n,
    const double* r_in, const double* v_in, const uint32_t* set_ids, gpop_ca** out)
{
    if (!ctx || !out)
        return GPOP_ERR_INVALID_ARG;
    *out = nullptr;
    // ClosestApproach::Initialize input checks (closest_approach.cu:56-81)
    if (n <= 0 || !r_in || !v_in || !set_ids)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "positions array is empty");
    if (n > (int64_t)INT32_MAX)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "too many objects");
    if (!start || !(h > 0.0) || !std::isfinite(h))
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid start time or step size");
    if (set_ids[0] == set_ids[n - 1])
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid setIndices: at least 2 sets are required");
    if (set_ids[0] != 0)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid setIndices: they must start at 0");
    // non-finite states are refused here; a position at the origin only where gravity is evaluated
    // (the startup kernel flags it, and gpop_ca_propagate fails)
    const int64_t bad = first_bad_state(r_in, v_in, n, false);
    if (bad >= 0)
        return bad_state(ctx, bad, "object");
    gpop_ca* ca = new (std::nothrow) gpop_ca();
    if (!ca)
        return fail(ctx, GPOP_ERR_NOMEM, "closest approach");
    ca->ctx = ctx;
    ca->start = *start;
    ca->h = h;
    ca->n = n;
    // PartitionParameters::Calculate (partition_parameters.cuh:94-135)
    ca->set_offsets.push_back(0);
    ca->map_offsets.push_back(0);
    uint32_t prev = set_ids[0], prev_change = 0;
    for (int64_t i = 1; i < n; ++i) {
        if (set_ids[i] < prev || set_ids[i] > prev + 1) {
            delete ca;
            return fail(ctx, GPOP_ERR_INVALID_ARG,
                "invalid setIndices: ids must be non-decreasing by at most 1 (failed to calculate "
                "partition parameters)");
        }
        if (set_ids[i] > prev) {
            const uint32_t size = (uint32_t)i - prev_change;
            const uint32_t higher = (uint32_t)(n - i);
            ca->set_offsets.push_back((uint32_t)i);
            ca->num_higher.push_back(higher);
            ca->map_offsets.push_back(ca->map_offsets.back() + (uint64_t)size * higher);
            prev_change = (uint32_t)i;
        }
        prev = set_ids[i];
    }
    ca->num_higher.push_back(0);
    ca->num_sets = (uint32_t)ca->set_offsets.size();
    ca->num_pairs = ca->map_offsets.back();
    // per-object bound and pair-index base; tiles of the (a, b) staircase, b-major
    std::vector<int> bound(n);
    std::vector<int64_t> base(n);
    for (int64_t a = 0; a < n; ++a) {
        const uint32_t s = set_ids[a];
        if (s + 1 >= ca->num_sets) {
            bound[a] = (int)n;
            base[a] = 0;
        } else {
            bound[a] = (int)ca->set_offsets[s + 1];
            base[a] = (int64_t)ca->map_offsets[s] + (int64_t)(a - ca->set_offsets[s]) * ca->num_higher[s]
                - (int64_t)ca->set_offsets[s + 1];
        }
    }
    const std::vector<int2> tiles = staircase_tiles(ca, 0, n);
    ca->num_tiles = (int)tiles.size();
    ca->row_hi = n;
    ca->pair_hi = (int64_t)ca->num_pairs;
    cudaError_t e = cudaSetDevice(ctx->cfg.device);
    const size_t P = ca->num_pairs;
    if (e != cudaSuccess || (e = ca->r.ensure(n * 24)) != cudaSuccess || (e = ca->v.ensure(n * 24)) != cudaSuccess
        || (e = ca->bound.ensure(n * sizeof(int))) != cudaSuccess
        || (e = ca->base.ensure(n * sizeof(int64_t))) != cudaSuccess
        || (e = ca->tiles.ensure(std::max<size_t>(1, tiles.size()) * sizeof(int2))) != cudaSuccess
        || (e = ca->min_d2.ensure(std::max<size_t>(1, P) * 8)) != cudaSuccess
        || (e = ca->min_step.ensure(std::max<size_t>(1, P) * 4)) != cudaSuccess
        || (e = ca->so.ensure(ca->num_sets * 4)) != cudaSuccess || (e = ca->nh.ensure(ca->num_sets * 4)) != cudaSuccess
        || (e = ca->mo.ensure(ca->num_sets * 8)) != cudaSuccess) {
        delete ca;
        return fail(ctx, GPOP_ERR_NOMEM, std::string("closest-approach buffers: ") + cudaGetErrorString(e));
    }
    if ((e = cudaMemcpy(ca->r.p, r_in, n * 24, cudaMemcpyHostToDevice)) != cudaSuccess
        || (e = cudaMemcpy(ca->v.p, v_in, n * 24, cudaMemcpyHostToDevice)) != cudaSuccess
        || (e = cudaMemcpy(ca->bound.p, bound.data(), n * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess
        || (e = cudaMemcpy(ca->base.p, base.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice)) != cudaSuccess
        || (!tiles.empty()
            && (e = cudaMemcpy(ca->tiles.p, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice))
                != cudaSuccess)
        || (e = cudaMemcpy(ca->so.p, ca->set_offsets.data(), ca->num_sets * 4, cudaMemcpyHostToDevice)) != cudaSuccess
        || (e = cudaMemcpy(ca->nh.p, ca->num_higher.data(), ca->num_sets * 4, cudaMemcpyHostToDevice)) != cudaSuccess
        || (e = cudaMemcpy(ca->mo.p, ca->map_offsets.data(), ca->num_sets * 8, cudaMemcpyHostToDevice)) != cudaSuccess) {
        delete ca;
        return cuda_fail(ctx, e, "closest-approach upload");
    }
    *out = ca;
    return GPOP_OK;
}

gpop_status gpop_ca_create_analytic(gpop_ctx* ctx, int32_t kind, double h, int64_t n,
    const double* r_in, const double* v_in, const uint32_t* set_ids, gpop_ca** out)
{
    if (!ctx || !out)
        return GPOP_ERR_INVALID_ARG;
    if (kind < GPOP_FORCE_ZERO || kind > GPOP_FORCE_DAMPED)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "invalid analytic force kind");
    const gpop_time t0 { 2000, 1, 1, 0, 0, 0.0 };
    gpop_status st = gpop_ca_create(ctx, &t0, h, n, r_in, v_in, set_ids, out);
    if (st == GPOP_OK)
        (*out)->kind = kind;
    return st;
}

gpop_status gpop_ca_create_external(gpop_ctx* ctx, double h, int64_t n, const double* r_in,
    const double* v_in, const uint32_t* set_ids, gpop_ca** out)
{
    if (!ctx || !out)
        return GPOP_ERR_INVALID_ARG;
    const gpop_time t0 { 2000, 1, 1, 0, 0, 0.0 };
    gpop_status st = gpop_ca_create(ctx, &t0, h, n, r_in, v_in, set_ids, out);
    if (st == GPOP_OK)
        (*out)->kind = kExternalKind;
    return st;
}

gpop_status gpop_ca_append(gpop_ca* ca, int32_t steps, const double* r_dev, const double* v_dev,
    const double* a_dev)
{
    if (!ca)
        return GPOP_ERR_INVALID_ARG;
    gpop_ctx* ctx = ca->ctx;
    if (ca->kind != kExternalKind)
        return fail(ctx, GPOP_ERR_STATE, "gpop_ca_append needs an object from gpop_ca_create_external");
    if (steps <= 0 || !r_dev || !v_dev || !a_dev)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "steps must be positive and the buffers given");
    cudaError_t e = cudaSetDevice(ctx->cfg.device);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "cudaSetDevice");
    cudaStream_t s = nullptr;
    const int need = ca->total_steps + steps;
    gpop_status st = grow_store(ca, need, true);
    if (st != GPOP_OK)
        return st;
    const size_t off = (size_t)ca->total_steps * 3 * ca->n;
    const int64_t count = (int64_t)steps * ca->n;
    append_rows_kernel<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(ca->n, count, r_dev, v_dev, a_dev,
        ca->traj_r.as<double>() + off, ca->traj_v.as<double>() + off, ca->traj_a.as<double>() + off);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return cuda_fail(ctx, e, "trajectory rows");
    ctx->launches++;
    DeviceTimer timer;
    timer.mark(s);
    if ((st = screen_steps(ca, need, s)) != GPOP_OK)
        return st;
    timer.mark(s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_fail(ctx, e, "screen kernel");
    ca->t_screen += timer.seconds(0, 1);
    ca->total_steps = need;
    ca->refined = false;
    return GPOP_OK;
}

int64_t gpop_ca_num_pairs(const gpop_ca* ca) { return ca ? (int64_t)ca->num_pairs : -1; }

gpop_status gpop_ca_reserve(gpop_ca* ca, int32_t total_steps)
{
    if (!ca)
        return GPOP_ERR_INVALID_ARG;
    if (total_steps < 0)
        return fail(ca->ctx, GPOP_ERR_INVALID_ARG, "negative step count");
    cudaError_t e = cudaSetDevice(ca->ctx->cfg.device);
    if (e != cudaSuccess)
        return cuda_fail(ca->ctx, e, "cudaSetDevice");
    return grow_store(ca, total_steps);
}

gpop_status gpop_ca_set_rows(gpop_ca* ca, int64_t row_begin, int64_t row_end)
{
    if (!ca)
        return GPOP_ERR_INVALID_ARG;
    gpop_ctx* ctx = ca->ctx;
    if (ca->total_steps != 0)
        return fail(ctx, GPOP_ERR_STATE, "gpop_ca_set_rows after the first propagation");
    if (row_begin < 0 || row_end > ca->n || row_end < row_begin
        || (row_begin % kTile != 0 && row_begin != ca->n) || (row_end % kTile != 0 && row_end != ca->n))
        return fail(ctx, GPOP_ERR_INVALID_ARG,
            "rows must satisfy 0 <= begin <= end <= n with begin and end multiples of 64 or n");
    const std::vector<int2> tiles = staircase_tiles(ca, row_begin, row_end);
    cudaError_t e = cudaSetDevice(ctx->cfg.device);
    if (e == cudaSuccess && (e = ca->tiles.ensure(std::max<size_t>(1, tiles.size()) * sizeof(int2))) == cudaSuccess
        && !tiles.empty())
        e = cudaMemcpy(ca->tiles.p, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "screen tiles");
    ca->num_tiles = (int)tiles.size();
    ca->row_lo = row_begin;
    ca->row_hi = row_end;
    ca->pair_lo = pairs_before(ca, row_begin);
    ca->pair_hi = std::max(ca->pair_lo, pairs_before(ca, row_end));
    return GPOP_OK;
}

gpop_status gpop_ca_pair_range(const gpop_ca* ca, int64_t* pair_begin, int64_t* pair_end)
{
    if (!ca || !pair_begin || !pair_end)
        return GPOP_ERR_INVALID_ARG;
    *pair_begin = ca->pair_lo;
    *pair_end = ca->pair_hi;
    return GPOP_OK;
}

gpop_status gpop_ca_propagate(gpop_ca* ca, int32_t steps)
{
    if (!ca)
        return GPOP_ERR_INVALID_ARG;
    gpop_ctx* ctx = ca->ctx;
    if (steps <= 0)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "number of steps must be positive");
    cudaError_t e = cudaSetDevice(ctx->cfg.device);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "cudaSetDevice");
    cudaStream_t s = nullptr;
    if (ca->kind == kExternalKind)
        return fail(ctx, GPOP_ERR_STATE, "this closest-approach object takes its trajectory from gpop_ca_append");
    const int need = ca->total_steps + steps;
    gpop_status gs = grow_store(ca, need);
    if (gs != GPOP_OK)
        return gs;
    // ClosestApproach::Propagate builds a new GpuPropagator from the current state for every
    // phase (closest_approach.cu:134-136): a fresh startup each call. The reference's force model
    // keeps the original start epoch for every phase; GPOP_FIX_PHASE_EPOCH advances it.
    gpop_propagator p;
    p.ctx = ctx;
    p.kind = ca->kind;
    p.start = ca->start;
    if (ctx->cfg.flags & GPOP_FIX_PHASE_EPOCH)
        p.start.sec += (double)ca->total_steps * ca->h;
    p.h = ca->h;
    p.ncorr = ctx->cfg.n_corrections;
    p.max_steps = steps;
    p.n = ca->n;
    p.r = ca->r.as<double>();
    p.v = ca->v.as<double>();
    p.mixed = ctx->cfg.precision == GPOP_MIXED;
    p.state = &ca->state;
    p.gen_m = &ca->gen_m;
    p.prop_m = &ca->prop_m;
    const size_t off = (size_t)ca->total_steps * 3 * ca->n;
    DeviceTimer timer;
    timer.mark(s);
    gpop_status st = propagator_init(&p, s);
    if (st == GPOP_OK)
        st = propagator_step(&p, steps, ca->traj_r.as<double>() + off, ca->traj_v.as<double>() + off,
            ca->traj_a.as<double>() + off, s);
    if (st != GPOP_OK)
        return st;
    timer.mark(s);
    if ((st = screen_steps(ca, need, s)) != GPOP_OK)
        return st;
    timer.mark(s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_fail(ctx, e, "screen kernel");
    ca->t_prop += timer.seconds(0, 1);
    ca->t_screen += timer.seconds(1, 2);
    ca->total_steps = need;
    ca->refined = false;
    return GPOP_OK;
}

gpop_status gpop_ca_find(gpop_ca* ca, double threshold, gpop_ca_record* out, int64_t capacity,
    int64_t* n_out)
{
    if (!ca || !n_out)
        return GPOP_ERR_INVALID_ARG;
    gpop_ctx* ctx = ca->ctx;
    if (ca->total_steps == 0)
        return fail(ctx, GPOP_ERR_STATE, "FindClosest before Propagate");
    cudaSetDevice(ctx->cfg.device);
    cudaStream_t s = nullptr;
    gpop_status st = refine(ca, s);
    if (st != GPOP_OK)
        return st;
    // the pairs of this object's rows (all pairs unless gpop_ca_set_rows narrowed them)
    const int64_t lo = ca->pair_lo, P = ca->pair_hi - ca->pair_lo;
    std::vector<int64_t> idx;
    cudaError_t e;
    if (threshold < 0.0) {
        *n_out = P;
        if (!out)
            return GPOP_OK;
        const int64_t k = std::min(P, capacity);
        idx.resize(k);
        for (int64_t i = 0; i < k; ++i)
            idx[i] = lo + i;
    } else {
        if ((e = ca->count.ensure(8)) != cudaSuccess || (e = ca->cand.ensure(std::max<int64_t>(1, P) * 8)) != cudaSuccess)
            return fail(ctx, GPOP_ERR_NOMEM, "candidate list");
        cudaMemsetAsync(ca->count.p, 0, 8, s);
        if ((e = launch_select(ca->dist.as<double>() + lo, P, threshold, ca->count.as<unsigned long long>(),
                 ca->cand.as<int64_t>(), P, s))
            != cudaSuccess)
            return cuda_fail(ctx, e, "select kernel");
        ctx->launches++;
        unsigned long long cnt = 0;
        if ((e = cudaMemcpy(&cnt, ca->count.p, 8, cudaMemcpyDeviceToHost)) != cudaSuccess)
            return cuda_fail(ctx, e, "select kernel");
        *n_out = (int64_t)cnt;
        if (!out)
            return GPOP_OK;
        idx.resize(cnt);
        if (cnt && (e = cudaMemcpy(idx.data(), ca->cand.p, cnt * 8, cudaMemcpyDeviceToHost)) != cudaSuccess)
            return cuda_fail(ctx, e, "candidate list");
        for (int64_t& i : idx)
            i += lo;
        std::sort(idx.begin(), idx.end()); // pair order = (object_index1, object_index2) order
        if ((int64_t)idx.size() > capacity)
            idx.resize(capacity);
    }
    const int64_t k = (int64_t)idx.size();
    if (k == 0)
        return GPOP_OK;
    DevBuf d_idx, d_rec;
    if ((e = d_idx.ensure(k * 8)) != cudaSuccess || (e = d_rec.ensure(k * 64)) != cudaSuccess) {
        d_idx.release();
        d_rec.release();
        return fail(ctx, GPOP_ERR_NOMEM, "record buffer");
    }
    std::vector<double> rec(k * 8);
    e = cudaMemcpy(d_idx.p, idx.data(), k * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        gather_kernel<<<(unsigned)((k + 255) / 256), 256, 0, s>>>(d_idx.as<int64_t>(), k, ca->dist.as<double>(),
            ca->time.as<double>(), ca->pos_a.as<double>(), ca->pos_b.as<double>(), d_rec.as<double>());
        e = cudaGetLastError();
        ctx->launches++;
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(rec.data(), d_rec.p, k * 64, cudaMemcpyDeviceToHost);
    d_idx.release();
    d_rec.release();
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "gathering records");
    for (int64_t i = 0; i < k; ++i) {
        gpop_ca_record& r = out[i];
        pair_objects(ca, (uint64_t)idx[i], r.object_index1, r.object_index2);
        r.distance = rec[i * 8];
        r.time = rec[i * 8 + 1];
        for (int c = 0; c < 3; ++c) {
            r.position_a[c] = rec[i * 8 + 2 + c];
            r.position_b[c] = rec[i * 8 + 5 + c];
        }
    }
    return GPOP_OK;
}

gpop_status gpop_ca_pairs(gpop_ca* ca, double* dist, double* time, double* pos_a, double* pos_b,
    uint32_t* closest_step)
{
    if (!ca)
        return GPOP_ERR_INVALID_ARG;
    gpop_ctx* ctx = ca->ctx;
    if (ca->total_steps == 0)
        return fail(ctx, GPOP_ERR_STATE, "FindClosest before Propagate");
    cudaSetDevice(ctx->cfg.device);
    gpop_status st = refine(ca, nullptr);
    if (st != GPOP_OK)
        return st;
    // entries [pair_lo, pair_hi) of the full-length arrays; the others are left as they are
    const size_t lo = (size_t)ca->pair_lo, P = (size_t)(ca->pair_hi - ca->pair_lo);
    cudaError_t e = cudaSuccess;
    if (P == 0)
        return GPOP_OK;
    if (dist && e == cudaSuccess)
        e = cudaMemcpy(dist + lo, ca->dist.as<double>() + lo, P * 8, cudaMemcpyDeviceToHost);
    if (time && e == cudaSuccess)
        e = cudaMemcpy(time + lo, ca->time.as<double>() + lo, P * 8, cudaMemcpyDeviceToHost);
    if (pos_a && e == cudaSuccess)
        e = cudaMemcpy(pos_a + 3 * lo, ca->pos_a.as<double>() + 3 * lo, P * 24, cudaMemcpyDeviceToHost);
    if (pos_b && e == cudaSuccess)
        e = cudaMemcpy(pos_b + 3 * lo, ca->pos_b.as<double>() + 3 * lo, P * 24, cudaMemcpyDeviceToHost);
    if (closest_step && e == cudaSuccess)
        e = cudaMemcpy(closest_step + lo, ca->min_step.as<uint32_t>() + lo, P * 4, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? GPOP_OK : cuda_fail(ctx, e, "copying pair results");
}

gpop_status gpop_ca_trajectory(gpop_ca* ca, double* r_host, double* v_host, double* a_host,
    int32_t* steps_out)
{
    if (!ca || !steps_out)
        return GPOP_ERR_INVALID_ARG;
    *steps_out = ca->total_steps;
    const size_t bytes = (size_t)ca->total_steps * 3 * ca->n * sizeof(double);
    if (bytes == 0)
        return GPOP_OK;
    cudaSetDevice(ca->ctx->cfg.device);
    cudaError_t e = cudaSuccess;
    if (r_host)
        e = cudaMemcpy(r_host, ca->traj_r.p, bytes, cudaMemcpyDeviceToHost);
    if (v_host && e == cudaSuccess)
        e = cudaMemcpy(v_host, ca->traj_v.p, bytes, cudaMemcpyDeviceToHost);
    if (a_host && e == cudaSuccess)
        e = cudaMemcpy(a_host, ca->traj_a.p, bytes, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? GPOP_OK : cuda_fail(ca->ctx, e, "copying the trajectory");
}

gpop_status gpop_ca_device_seconds(const gpop_ca* ca, double* out3)
{
    if (!ca || !out3)
        return GPOP_ERR_INVALID_ARG;
    out3[0] = ca->t_prop;
    out3[1] = ca->t_screen;
    out3[2] = ca->t_refine;
    return GPOP_OK;
}

void gpop_ca_destroy(gpop_ca* ca) { delete ca; }

} // extern "C"
