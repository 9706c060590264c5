// batch_api.cu -- batched propagation entry points: planner, autotuner and the captured launch.
#include "batch.cuh"
#include "common.cuh"
#include "context.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <new>
#include <numeric>
#include <queue>
#include <tuple>

using namespace gpop;

namespace {

// Persistent grid: one block per SM of 4 or 8 warps (the block shapes the planner chooses from);
// the two-object path needs the registers of 8 warps at most.
constexpr int kWarpOptions[2] = { 4, 8 };
inline int warp_index(int W) { return W == kWarpOptions[0] ? 0 : 1; }
constexpr int kDegrees[4] = { 8, 20, 36, 70 };
const double kNodesH[10] = { 0.0, 4.0 / 27.0, 2.0 / 9.0, 1.0 / 3.0, 1.0 / 2.0, 2.0 / 3.0, 1.0 / 6.0, 1.0, 5.0 / 6.0, 1.0 };

int terms(int L) { return (L + 1) * (L + 2) / 2 - 3; }

// Object-steps per second per SM of the batched kernel at degree L with P lanes per object, with
// W warps per SM. Measured by gpop_tune; before tuning a model is used: cost proportional to the
// terms walked, with a per-lane overhead for the column split and the shuffles, and three
// quarters of the throughput with four warps (one per scheduler) as with eight.
double eta(const gpop_ctx* ctx, int W, int L, int P)
{
    const int wi = warp_index(W);
    int lp = 0;
    while ((1 << lp) < P)
        ++lp;
    if (ctx->tuned) {
        // interpolate in the number of terms between the tuned degrees
        int i = 0;
        while (i < 3 && kDegrees[i + 1] <= L)
            ++i;
        const int j = std::min(i + 1, 3);
        const double t0 = terms(kDegrees[i]), t1 = terms(kDegrees[j]), t = terms(std::max(L, 2));
        const double c0 = 1.0 / ctx->eta[wi][i][lp], c1 = 1.0 / ctx->eta[wi][j][lp];
        const double f = (t1 > t0) ? std::min(1.0, std::max(0.0, (t - t0) / (t1 - t0))) : 0.0;
        return 1.0 / (c0 + f * (c1 - c0));
    }
    const bool mixed = ctx->cfg.precision == GPOP_MIXED;
    const double base70 = mixed ? 6.5e5 : 4.5e5; // object-steps/s per SM at 70x70, one lane
    const double cost = (terms(std::max(L, 2)) + 60.0) / (terms(70) + 60.0);
    return base70 / cost / (1.0 + 0.12 * lp) * (wi == 0 ? 0.75 : 1.0);
}

// Speed of single-lane items in a batch of single-lane items (two-column walk on the plain table)
// over their speed in mixed batches, which is what the tuner measures (65,536 objects at 70x70 on
// B200: 135.6 / 115.0 M object-steps/s mixed precision, 69.7 / 66.8 M FP64).
constexpr double kPairWalkGainMixed = 1.15;
constexpr double kPairWalkGainFp64 = 1.04;

// Makespan of the persistent launch: work items taken longest first by the first free warp (the
// queue order), simulated with a heap of warp loads.
inline double lpt_makespan(std::vector<std::pair<double, int64_t>>& groups, double warps)
{
    std::sort(groups.begin(), groups.end(),
        [](const std::pair<double, int64_t>& a, const std::pair<double, int64_t>& b) { return a.first > b.first; });
    std::priority_queue<double, std::vector<double>, std::greater<double>> load;
    for (int w = 0; w < (int)warps; ++w)
        load.push(0.0);
    double span = 0.0;
    for (const auto& g : groups)
        for (int64_t i = 0; i < g.second; ++i) {
            const double t = load.top() + g.first;
            load.pop();
            load.push(t);
            span = std::max(span, t);
        }
    return span;
}

// Lanes per object: small requests fill their warp with lanes (the warp is theirs either way).
// Then every request whose work item outlasts the makespan bound -- the larger of the average warp
// load and the shortest possible item of the longest request -- doubles its lanes while that
// shortens the item -- except that a batch whose items fit one wave of warps keeps them in one
// wave (lanes cost efficiency; a second wave of split items costs more). Measured on B200:
// 4,096 uneven requests 8.7 s; one 65,536-object request at 70x70 keeps one lane per object
// (136 M object-steps/s with the two-column walk on the plain table; 75 M with two lanes per
// object and the one-column walk).
template <class ItemTime>
double choose_lanes(const std::vector<int64_t>& n, const std::vector<int>& steps, double warps,
    const ItemTime& item_time, std::vector<int>& lpo, bool fixed, double pair_gain)
{
    const size_t R = n.size();
    auto items_of = [&](size_t r, int P) { return (n[r] + batch_item_objects(P) - 1) / batch_item_objects(P); };
    if (!fixed) {
        for (size_t r = 0; r < R; ++r) {
            int P = 1;
            while (P < 32 && n[r] * (int64_t)(2 * P) <= 32)
                P *= 2;
            lpo[r] = P;
        }
        double crit = 0.0;
        for (size_t r = 0; r < R; ++r)
            if (steps[r] > 0)
                crit = std::max(crit, item_time(r, 32));
        for (int iter = 0; iter < 8; ++iter) {
            double total = 0.0;
            int64_t count = 0;
            for (size_t r = 0; r < R; ++r)
                if (steps[r] > 0) {
                    total += (double)items_of(r, lpo[r]) * item_time(r, lpo[r]);
                    count += items_of(r, lpo[r]);
                }
            const double bound = std::max(total / warps, crit);
            bool changed = false;
            for (size_t r = 0; r < R; ++r)
                while (steps[r] > 0 && lpo[r] < 32 && item_time(r, lpo[r]) > bound
                    && item_time(r, 2 * lpo[r]) < item_time(r, lpo[r])
                    && (count > (int64_t)warps
                        || count - items_of(r, lpo[r]) + items_of(r, 2 * lpo[r]) <= (int64_t)warps)) {
                    count += items_of(r, 2 * lpo[r]) - items_of(r, lpo[r]);
                    lpo[r] *= 2;
                    changed = true;
                }
            if (!changed)
                break;
        }
    }
    auto span_of = [&](const std::vector<int>& lp) {
        std::vector<std::pair<double, int64_t>> groups;
        for (size_t r = 0; r < R; ++r)
            if (steps[r] > 0)
                groups.push_back({ item_time(r, lp[r]), items_of(r, lp[r]) });
        return lpt_makespan(groups, warps);
    };
    const double span = span_of(lpo);
    if (!fixed) {
        // A batch of single-lane items runs the two-column walk, faster than the rates measured
        // for single-lane items in mixed batches: keep one lane per object unless the lanes plan
        // is shorter even so (64 requests of 1,024 objects at 70x70: lanes on some requests left
        // the makespan as it was and cost the whole batch the faster kernel, 114 against 136 M
        // object-steps/s).
        std::vector<int> ones(R, 1);
        bool all_one = true;
        for (size_t r = 0; r < R; ++r)
            all_one = all_one && (steps[r] <= 0 || lpo[r] == 1);
        if (!all_one) {
            const double span1 = span_of(ones) / pair_gain;
            if (span1 <= span) {
                lpo = ones;
                return span1;
            }
        } else {
            return span / pair_gain;
        }
    }
    return span;
}

struct Plan {
    std::vector<int> lpo;
    std::vector<BatchItem> items;
    double est = 0.0;
    int warps_per_sm = 8; // block shape of the persistent grid
};

// The plan: for each block shape (warps per SM), lanes per object and the simulated makespan with
// that shape's rates; the shape with the shorter makespan wins (four warps give a batch with at
// most one item per scheduler a whole scheduler per item).
Plan make_plan(const gpop_ctx* ctx, const std::vector<int64_t>& n, const std::vector<int>& steps,
    const std::vector<int>& L)
{
    const size_t R = n.size();
    Plan p;
    p.est = -1.0;
    for (int W : kWarpOptions) {
        if (ctx->force_warps > 0 && W != ctx->force_warps)
            continue;
        std::vector<int> lpo(R, 1);
        const double warps = (double)ctx->num_sms * W;
        auto item_time = [&](size_t r, int P) { // seconds for one warp to run its group through all steps
            return (double)steps[r] * W * batch_item_objects(P) / eta(ctx, W, L[r], P);
        };
        const bool fixed = ctx->force_lpo > 0; // autotuner: fixed lanes per object
        if (fixed)
            lpo.assign(R, ctx->force_lpo);
        const double est = choose_lanes(n, steps, warps, item_time, lpo, fixed,
            ctx->cfg.precision == GPOP_MIXED ? kPairWalkGainMixed : kPairWalkGainFp64);
        if (p.est < 0.0 || est < p.est) {
            p.est = est;
            p.lpo = lpo;
            p.warps_per_sm = W;
        }
    }
    std::vector<std::pair<double, BatchItem>> items;
    for (size_t r = 0; r < R; ++r) {
        if (steps[r] <= 0)
            continue;
        const int per = batch_item_objects(p.lpo[r]);
        const double t = (double)steps[r] * p.warps_per_sm * per / eta(ctx, p.warps_per_sm, L[r], p.lpo[r]);
        for (int64_t f = 0; f < n[r]; f += per) {
            items.push_back({ t, BatchItem { (int)r, (int)f, (int)std::min<int64_t>(per, n[r] - f) } });
        }
    }
    std::stable_sort(items.begin(), items.end(),
        [](const std::pair<double, BatchItem>& a, const std::pair<double, BatchItem>& b) { return a.first > b.first; });
    for (auto& it : items)
        p.items.push_back(it.second);
    return p;
}

struct TableKey {
    int y, mo, d, hh, mi;
    double sec, h;
    bool operator<(const TableKey& o) const
    {
        return std::tie(y, mo, d, hh, mi, sec, h) < std::tie(o.y, o.mo, o.d, o.hh, o.mi, o.sec, o.h);
    }
};

// Why request q cannot run (empty when it can): bad arguments, or an object whose position or
// velocity is not finite or whose position is the origin.
std::string request_problem(const gpop_request& q)
{
    const gpop_time& t = q.start;
    if (q.n <= 0 || !q.r_in || !q.v_in || !q.r_out || !q.v_out || q.steps < 0 || !(q.h > 0.0)
        || !std::isfinite(q.h) || t.month < 1 || t.month > 12 || t.day < 1 || t.day > 31 || !std::isfinite(t.sec))
        return "invalid arguments";
    if (q.n > (int64_t)1 << 24)
        return "too many objects";
    const int64_t bad = first_bad_state(q.r_in, q.v_in, q.n, true);
    if (bad >= 0)
        return "object " + std::to_string(bad) + " has a position or velocity that is not finite, or a position at the origin";
    return std::string();
}

gpop_status validate(gpop_ctx* ctx, const gpop_request* reqs, int32_t n_req)
{
    if (!reqs || n_req <= 0)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "empty batch");
    for (int32_t i = 0; i < n_req; ++i) {
        const std::string why = request_problem(reqs[i]);
        if (!why.empty())
            return fail(ctx, GPOP_ERR_INVALID_ARG, "request " + std::to_string(i) + ": " + why);
    }
    return GPOP_OK;
}

} // namespace

// Buffers and captured graph of the last batch (replayed when the next batch has the same shape).
struct BatchCache {
    std::vector<int64_t> sig;
    cudaGraphExec_t exec = nullptr;
    DevBuf reqs, items, obj_req, state, io, tables, sec, cal, epoch_req, queue;
    std::vector<double> host_io;
    ~BatchCache()
    {
        if (exec)
            cudaGraphExecDestroy(exec);
        for (DevBuf* b : { &reqs, &items, &obj_req, &state, &io, &tables, &sec, &cal, &epoch_req, &queue })
            b->release();
    }
};

namespace gpop {
void destroy_batch_cache(gpop_ctx* ctx)
{
    delete ctx->batch;
    ctx->batch = nullptr;
    if (ctx->batch_stream)
        cudaStreamDestroy(ctx->batch_stream);
    ctx->batch_stream = nullptr;
    if (ctx->batch_host)
        cudaFreeHost(ctx->batch_host);
    ctx->batch_host = nullptr;
    ctx->batch_host_cap = 0;
}
} // namespace gpop

extern "C" {

gpop_status gpop_batch_plan(gpop_ctx* ctx, const gpop_request* reqs, int32_t n_req,
    int32_t* lanes_per_object, double* est_seconds)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    gpop_status st = validate(ctx, reqs, n_req);
    if (st != GPOP_OK)
        return st;
    std::vector<int64_t> n(n_req);
    std::vector<int> steps(n_req), L(n_req);
    for (int i = 0; i < n_req; ++i) {
        n[i] = reqs[i].n;
        steps[i] = reqs[i].steps;
        L[i] = (reqs[i].degree > 0 && reqs[i].degree < ctx->md.degree) ? reqs[i].degree : ctx->md.degree;
    }
    Plan p = make_plan(ctx, n, steps, L);
    if (lanes_per_object)
        std::copy(p.lpo.begin(), p.lpo.end(), lanes_per_object);
    if (est_seconds)
        *est_seconds = p.est;
    return GPOP_OK;
}

} // extern "C"

// The batch proper, over requests that have passed request_problem.
static gpop_status run_batch(gpop_ctx* ctx, const gpop_request* reqs, int32_t n_req)
{
    cudaError_t e = cudaSetDevice(ctx->cfg.device);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "cudaSetDevice");
    // ---- layout: objects of the requests that take steps, one epoch table per (start, h) ----
    std::vector<int64_t> n(n_req);
    std::vector<int> steps(n_req), L(n_req);
    std::vector<int64_t> obj0(n_req, -1);
    int64_t N = 0;
    std::map<TableKey, int> table_of;
    std::vector<TableKey> tables;
    std::vector<int> table_len; // propagation entries of each table
    std::vector<int> req_table(n_req, -1);
    for (int i = 0; i < n_req; ++i) {
        const gpop_request& q = reqs[i];
        n[i] = q.n;
        steps[i] = q.steps;
        L[i] = (q.degree > 0 && q.degree < ctx->md.degree) ? q.degree : ctx->md.degree;
        if (q.steps == 0)
            continue;
        obj0[i] = N;
        N += q.n;
        TableKey k { q.start.year, q.start.month, q.start.day, q.start.hour, q.start.min, q.start.sec, q.h };
        auto it = table_of.find(k);
        int t;
        if (it == table_of.end()) {
            t = (int)tables.size();
            table_of[k] = t;
            tables.push_back(k);
            table_len.push_back(0);
        } else {
            t = it->second;
        }
        table_len[t] = std::max(table_len[t], 4 + std::max(q.steps, 4) + 1);
        req_table[i] = t;
    }
    for (int i = 0; i < n_req; ++i) // zero-step requests return their input (exec/runner.cu:48-51)
        if (reqs[i].steps == 0) {
            std::copy(reqs[i].r_in, reqs[i].r_in + 3 * reqs[i].n, reqs[i].r_out);
            std::copy(reqs[i].v_in, reqs[i].v_in + 3 * reqs[i].n, reqs[i].v_out);
        }
    if (N == 0)
        return GPOP_OK;
    Plan plan = make_plan(ctx, n, steps, L);
    ctx->batch_warps = plan.warps_per_sm;
    // epoch table offsets (in matrices): [gen 80 | prop len] per table
    std::vector<int64_t> t_off(tables.size());
    int64_t E = 0;
    for (size_t t = 0; t < tables.size(); ++t) {
        t_off[t] = E;
        E += 80 + table_len[t];
    }
    // Two-object items walk the gravity columns two at a time only in batches that hold nothing
    // else: beside many-lane items the larger kernel code slows the many-lane items (4,096 uneven
    // requests: 174 -> 165 M object-steps/s), while a batch of 64-object items gains (one
    // 65,536-object 70x70 request: mixed 97 -> 115 M). The autotuner's fixed-lane runs keep the
    // one-column walk, so its single-lane figures hold for uneven batches.
    bool pair_walk = ctx->force_lpo == 0;
    for (int i = 0; i < n_req; ++i)
        pair_walk = pair_walk && plan.lpo[i] == 1;
    // shape signature: the graph is replayed only for an identical plan and layout
    std::vector<int64_t> sig { (int64_t)ctx->cfg.precision, (int64_t)ctx->cfg.flags, N, E, (int64_t)n_req,
        (int64_t)pair_walk, (int64_t)plan.warps_per_sm };
    for (int i = 0; i < n_req; ++i) {
        sig.push_back(n[i]);
        sig.push_back(steps[i]);
        sig.push_back(L[i]);
        sig.push_back(plan.lpo[i]);
        int64_t hb;
        std::memcpy(&hb, &reqs[i].h, 8);
        sig.push_back(hb);
        int64_t sb;
        std::memcpy(&sb, &reqs[i].start.sec, 8);
        sig.push_back(sb);
        sig.push_back(((int64_t)reqs[i].start.year << 32) | (reqs[i].start.month << 24) | (reqs[i].start.day << 16)
            | (reqs[i].start.hour << 8) | reqs[i].start.min);
    }
    if (!ctx->batch)
        ctx->batch = new (std::nothrow) BatchCache();
    BatchCache* bc = ctx->batch;
    if (!bc)
        return fail(ctx, GPOP_ERR_NOMEM, "batch cache");
    const bool replay = bc->exec && bc->sig == sig;
    cudaStream_t s = ctx->batch_stream;
    if (!s && (e = cudaStreamCreateWithFlags(&ctx->batch_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return cuda_fail(ctx, e, "batch stream");
    s = ctx->batch_stream;
    // ---- inputs: one pinned staging buffer [r0 | v0 | r_out | v_out] ----
    const size_t io_bytes = (size_t)N * 3 * 4 * sizeof(double);
    if ((e = bc->io.ensure(io_bytes)) != cudaSuccess)
        return fail(ctx, GPOP_ERR_NOMEM, "batch state buffers");
    if (ctx->batch_host_cap < io_bytes) {
        if (ctx->batch_host)
            cudaFreeHost(ctx->batch_host);
        ctx->batch_host = nullptr;
        ctx->batch_host_cap = 0;
        if ((e = cudaMallocHost(&ctx->batch_host, io_bytes)) != cudaSuccess)
            return fail(ctx, GPOP_ERR_NOMEM, "pinned staging buffer");
        ctx->batch_host_cap = io_bytes;
    }
    double* host = static_cast<double*>(ctx->batch_host);
    for (int i = 0; i < n_req; ++i) {
        if (obj0[i] < 0)
            continue;
        std::copy(reqs[i].r_in, reqs[i].r_in + 3 * n[i], host + 3 * obj0[i]);
        std::copy(reqs[i].v_in, reqs[i].v_in + 3 * n[i], host + 3 * N + 3 * obj0[i]);
    }
    double* dio = bc->io.as<double>();
    if ((e = cudaMemcpyAsync(dio, host, (size_t)N * 6 * sizeof(double), cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "batch upload");
    if (!replay) {
        if (bc->exec) {
            cudaGraphExecDestroy(bc->exec);
            bc->exec = nullptr;
        }
        // request descriptors, items, epoch arguments
        std::vector<BatchReq> rq(n_req);
        std::vector<int> obj_req(N);
        std::vector<double> sec(E);
        std::vector<int> epoch_req(E), cal(5 * tables.size());
        if ((e = bc->tables.ensure((size_t)E * 9 * sizeof(double))) != cudaSuccess
            || (e = bc->sec.ensure((size_t)E * sizeof(double))) != cudaSuccess
            || (e = bc->epoch_req.ensure((size_t)E * sizeof(int))) != cudaSuccess
            || (e = bc->cal.ensure(cal.size() * sizeof(int) + 4)) != cudaSuccess
            || (e = bc->reqs.ensure(n_req * sizeof(BatchReq))) != cudaSuccess
            || (e = bc->items.ensure(std::max<size_t>(1, plan.items.size()) * sizeof(BatchItem))) != cudaSuccess
            || (e = bc->obj_req.ensure((size_t)N * sizeof(int))) != cudaSuccess
            || (e = bc->state.ensure((size_t)kStateArrays * N * sizeof(double))) != cudaSuccess
            || (e = bc->queue.ensure(sizeof(int))) != cudaSuccess)
            return fail(ctx, GPOP_ERR_NOMEM, std::string("batch buffers: ") + cudaGetErrorString(e));
        for (size_t t = 0; t < tables.size(); ++t) {
            const TableKey& k = tables[t];
            cal[5 * t] = k.y;
            cal[5 * t + 1] = k.mo;
            cal[5 * t + 2] = k.d;
            cal[5 * t + 3] = k.hh;
            cal[5 * t + 4] = k.mi;
            const double base = k.sec - 4.0 * k.h; // (sec - before h) + time from table start
            for (int idx = 0; idx < 80; ++idx) {
                const int sp = idx / 10 - 4;
                double from = ((double)(idx / 10) + kNodesH[idx % 10]) * k.h;
                if ((ctx->cfg.flags & GPOP_FIX_BACKWARD_RK8_EPOCH) && sp < 0)
                    from = ((double)(sp + 1) - kNodesH[idx % 10]) * k.h + 4.0 * k.h;
                sec[t_off[t] + idx] = base + from;
                epoch_req[t_off[t] + idx] = (int)t;
            }
            for (int i = 0; i < table_len[t]; ++i) {
                sec[t_off[t] + 80 + i] = base + (double)i * k.h;
                epoch_req[t_off[t] + 80 + i] = (int)t;
            }
        }
        double* dtab = bc->tables.as<double>();
        for (int i = 0; i < n_req; ++i) {
            rq[i].obj0 = std::max<int64_t>(0, obj0[i]);
            rq[i].n = (int)n[i];
            rq[i].steps = steps[i];
            rq[i].L = L[i];
            rq[i].lpo = plan.lpo[i];
            rq[i].h = reqs[i].h;
            if (req_table[i] >= 0) {
                rq[i].gen_m = dtab + t_off[req_table[i]] * 9;
                rq[i].prop_m = dtab + (t_off[req_table[i]] + 80) * 9;
                for (int64_t o = 0; o < n[i]; ++o)
                    obj_req[obj0[i] + o] = i;
            }
        }
        if ((e = cudaMemcpyAsync(bc->sec.p, sec.data(), E * sizeof(double), cudaMemcpyHostToDevice, s)) != cudaSuccess
            || (e = cudaMemcpyAsync(bc->epoch_req.p, epoch_req.data(), E * sizeof(int), cudaMemcpyHostToDevice, s))
                != cudaSuccess
            || (e = cudaMemcpyAsync(bc->cal.p, cal.data(), cal.size() * sizeof(int), cudaMemcpyHostToDevice, s))
                != cudaSuccess
            || (e = cudaMemcpyAsync(bc->reqs.p, rq.data(), n_req * sizeof(BatchReq), cudaMemcpyHostToDevice, s))
                != cudaSuccess
            || (e = cudaMemcpyAsync(bc->items.p, plan.items.data(), plan.items.size() * sizeof(BatchItem),
                    cudaMemcpyHostToDevice, s))
                != cudaSuccess
            || (e = cudaMemcpyAsync(bc->obj_req.p, obj_req.data(), N * sizeof(int), cudaMemcpyHostToDevice, s))
                != cudaSuccess
            || (e = cudaStreamSynchronize(s)) != cudaSuccess) // the host vectors go out of scope
            return cuda_fail(ctx, e, "batch plan upload");
        // ---- capture: frames, startup, queue reset, persistent GJ8 ----
        const bool mixed = ctx->cfg.precision == GPOP_MIXED;
        TableSrc ts = ctx->table(mixed);
        BatchArgs a;
        a.reqs = bc->reqs.as<BatchReq>();
        a.n_req = n_req;
        a.items = bc->items.as<BatchItem>();
        a.n_items = (int)plan.items.size();
        a.next_item = bc->queue.as<int>();
        a.obj_req = bc->obj_req.as<int>();
        a.n_obj = N;
        a.ncorr = ctx->cfg.n_corrections;
        a.flags = ctx->cfg.flags;
        a.state = bc->state.as<double>();
        a.r0 = dio;
        a.v0 = dio + 3 * N;
        a.r_out = dio + 6 * N;
        a.v_out = dio + 9 * N;
        a.err = ctx->err_word.as<unsigned>();
        a.Ltab = ctx->md.degree;
        a.pair_walk = pair_walk;
        cudaGraph_t graph = nullptr;
        if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
            return cuda_fail(ctx, e, "graph capture");
        cudaError_t le = launch_frames_batch(ctx->frames, bc->cal.as<int>(), bc->epoch_req.as<int>(),
            bc->sec.as<double>(), (int)E, dtab, s);
        if (le == cudaSuccess)
            le = launch_batch_startup(ts, a, ctx->num_sms, s);
        if (le == cudaSuccess)
            le = cudaMemsetAsync(bc->queue.p, 0, sizeof(int), s);
        if (le == cudaSuccess)
            le = launch_batch_gj8(ctx->lane_table(mixed), ctx->table(mixed), a, ctx->num_sms,
                32 * plan.warps_per_sm, s);
        e = cudaStreamEndCapture(s, &graph);
        if (le != cudaSuccess || e != cudaSuccess) {
            if (graph)
                cudaGraphDestroy(graph);
            return cuda_fail(ctx, le != cudaSuccess ? le : e, "capturing the batch launch");
        }
        e = cudaGraphInstantiate(&bc->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            bc->exec = nullptr;
            return cuda_fail(ctx, e, "instantiating the batch graph");
        }
        bc->sig = sig;
    }
    DeviceTimer timer;
    timer.mark(s);
    if ((e = cudaGraphLaunch(bc->exec, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "batch graph launch");
    ctx->launches += 3;
    timer.mark(s);
    if ((e = cudaMemcpyAsync(host + 6 * N, dio + 6 * N, (size_t)N * 6 * sizeof(double), cudaMemcpyDeviceToHost, s))
        != cudaSuccess)
        return cuda_fail(ctx, e, "batch download");
    const gpop_status st = check_device_errors(ctx, s);
    if (st != GPOP_OK)
        return st;
    ctx->batch_seconds = timer.seconds(0, 1);
    for (int i = 0; i < n_req; ++i) {
        if (obj0[i] < 0)
            continue;
        std::copy(host + 6 * N + 3 * obj0[i], host + 6 * N + 3 * (obj0[i] + n[i]), reqs[i].r_out);
        std::copy(host + 9 * N + 3 * obj0[i], host + 9 * N + 3 * (obj0[i] + n[i]), reqs[i].v_out);
    }
    return GPOP_OK;
}

extern "C" {

gpop_status gpop_propagate_batch_status(gpop_ctx* ctx, const gpop_request* reqs, int32_t n_req,
    int32_t* status)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    if (!reqs || n_req <= 0)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "empty batch");
    // a request that cannot run is refused alone; the others run as one batch
    std::vector<gpop_request> good;
    std::vector<int32_t> good_idx;
    good.reserve(n_req);
    int32_t first_bad = -1, refused = 0;
    std::string why_first;
    for (int32_t i = 0; i < n_req; ++i) {
        const std::string why = request_problem(reqs[i]);
        if (why.empty()) {
            good.push_back(reqs[i]);
            good_idx.push_back(i);
        } else {
            ++refused;
            if (first_bad < 0) {
                first_bad = i;
                why_first = why;
            }
        }
        if (status)
            status[i] = why.empty() ? GPOP_OK : GPOP_ERR_INVALID_ARG;
    }
    if (!good.empty()) {
        const gpop_status st = run_batch(ctx, good.data(), (int32_t)good.size());
        if (st != GPOP_OK) {
            if (status)
                for (int32_t i : good_idx)
                    status[i] = st;
            return st;
        }
    }
    if (first_bad >= 0)
        return fail(ctx, GPOP_ERR_INVALID_ARG,
            "request " + std::to_string(first_bad) + ": " + why_first + " (" + std::to_string(refused) + " of "
                + std::to_string(n_req) + " requests refused; the others were propagated)");
    return GPOP_OK;
}

gpop_status gpop_propagate_batch(gpop_ctx* ctx, const gpop_request* reqs, int32_t n_req)
{
    return gpop_propagate_batch_status(ctx, reqs, n_req, nullptr);
}

double gpop_batch_device_seconds(const gpop_ctx* ctx) { return ctx ? ctx->batch_seconds : -1.0; }

int32_t gpop_batch_warps_per_sm(const gpop_ctx* ctx) { return ctx ? ctx->batch_warps : -1; }

gpop_status gpop_tune(gpop_ctx* ctx, const char* cache_path)
{
    if (!ctx)
        return GPOP_ERR_INVALID_ARG;
    const bool mixed = ctx->cfg.precision == GPOP_MIXED;
    if (cache_path) { // "<precision> <warps per SM> <L> <P> <eta>" lines
        std::ifstream f(cache_path);
        if (f.is_open()) {
            int prec, W, Lc, P;
            double val;
            int found = 0;
            while (f >> prec >> W >> Lc >> P >> val)
                for (int wi = 0; wi < 2; ++wi)
                    for (int i = 0; i < 4; ++i)
                        for (int lp = 0; lp < 6; ++lp)
                            if (prec == (int)mixed && W == kWarpOptions[wi] && Lc == kDegrees[i]
                                && P == (1 << lp) && val > 0) {
                                ctx->eta[wi][i][lp] = val;
                                ++found;
                            }
            if (found == 48) {
                ctx->tuned = true;
                return GPOP_OK;
            }
        }
    }
    // Calibration: for each block shape (warps per SM), one request per (degree, lanes) that fills
    // every warp of the persistent grid, on near-circular orbits. The captured graph is replayed
    // at two durations (fastest of three replays each); the difference (32 GJ8 steps) removes the
    // frames, startup and launch overheads.
    const gpop_time t0 { 2024, 1, 1, 0, 0, 0.0 };
    const bool saved = ctx->tuned;
    double measured[2][4][6];
    auto replay_ms = [&](gpop_request& q, int steps, float& ms) -> gpop_status {
        q.steps = steps;
        ctx->tuned = false;
        gpop_status st = gpop_propagate_batch(ctx, &q, 1); // builds the plan and the graph
        if (st != GPOP_OK)
            return st;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaError_t e = cudaEventCreate(&e0);
        if (e == cudaSuccess)
            e = cudaEventCreate(&e1);
        ms = 1e30f;
        for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) { // the fastest of three replays
            float t = 0.f;
            if ((e = cudaEventRecord(e0, ctx->batch_stream)) == cudaSuccess
                && (e = cudaGraphLaunch(ctx->batch->exec, ctx->batch_stream)) == cudaSuccess
                && (e = cudaEventRecord(e1, ctx->batch_stream)) == cudaSuccess
                && (e = cudaEventSynchronize(e1)) == cudaSuccess
                && (e = cudaEventElapsedTime(&t, e0, e1)) == cudaSuccess)
                ms = std::min(ms, t);
            ctx->launches += 3;
        }
        if (e0)
            cudaEventDestroy(e0);
        if (e1)
            cudaEventDestroy(e1);
        if (e != cudaSuccess)
            return cuda_fail(ctx, e, "timing the batch graph");
        return check_device_errors(ctx, ctx->batch_stream);
    };
    for (int wi = 0; wi < 2; ++wi) {
        const int W = kWarpOptions[wi];
        for (int i = 0; i < 4; ++i) {
            const int Lc = std::min(kDegrees[i], ctx->md.degree);
            for (int lp = 0; lp < 6; ++lp) {
                const int P = 1 << lp;
                const int64_t nobj = (int64_t)ctx->num_sms * W * batch_item_objects(P);
                std::vector<double> r(3 * nobj), v(3 * nobj), ro(3 * nobj), vo(3 * nobj);
                for (int64_t o = 0; o < nobj; ++o) {
                    const double ang = 0.001 * (double)o, a = 7.0e6 + 10.0 * (double)(o % 97);
                    const double sp = std::sqrt(ctx->md.gm / a), inc = 0.3 + 1e-4 * (double)(o % 31);
                    r[3 * o] = a * std::cos(ang);
                    r[3 * o + 1] = a * std::sin(ang) * std::cos(inc);
                    r[3 * o + 2] = a * std::sin(ang) * std::sin(inc);
                    v[3 * o] = -sp * std::sin(ang);
                    v[3 * o + 1] = sp * std::cos(ang) * std::cos(inc);
                    v[3 * o + 2] = sp * std::cos(ang) * std::sin(inc);
                }
                gpop_request q { t0, 30.0, 0, Lc, nobj, r.data(), v.data(), ro.data(), vo.data() };
                // pin the lanes and the block shape: the planner keeps them for a request that
                // fills the grid exactly
                float ms_short = 0.f, ms_long = 0.f;
                ctx->force_lpo = P;
                ctx->force_warps = W;
                gpop_status st = replay_ms(q, 8, ms_short);
                if (st == GPOP_OK)
                    st = replay_ms(q, 40, ms_long);
                ctx->force_lpo = 0;
                ctx->force_warps = 0;
                if (st != GPOP_OK) {
                    ctx->tuned = saved;
                    return st;
                }
                const double dt = std::max(1e-6, (double)(ms_long - ms_short) * 1e-3);
                measured[wi][i][lp] = (double)nobj * 32.0 / dt / ctx->num_sms;
            }
        }
    }
    for (int wi = 0; wi < 2; ++wi)
        for (int i = 0; i < 4; ++i)
            for (int lp = 0; lp < 6; ++lp)
                ctx->eta[wi][i][lp] = measured[wi][i][lp];
    ctx->tuned = true;
    if (cache_path) {
        std::ofstream f(cache_path);
        for (int wi = 0; wi < 2; ++wi)
            for (int i = 0; i < 4; ++i)
                for (int lp = 0; lp < 6; ++lp)
                    f << (int)mixed << " " << kWarpOptions[wi] << " " << kDegrees[i] << " " << (1 << lp)
                      << " " << ctx->eta[wi][i][lp] << "\n";
    }
    return GPOP_OK;
}

} // extern "C"
