// batch.cu -- one persistent launch for many independent propagation requests.
//
// Requests differ in object count, duration, step size and gravity degree. A request's objects
// advance one step at a time, so its duration sets a critical path that a larger batch cannot
// shorten; the planner (batch_api.cu) therefore gives long requests several lanes per object:
// the lanes of an object split the gravity columns (lane l of P takes m = l, l + P, ...) and add
// their sums with warp shuffles. Warps pull work items (a request's group of 32 / P objects, all of
// its steps) from a global queue ordered longest first, so the grid stays busy until the end.
#include "batch.cuh"
#include "common.cuh"
#include "frames.cuh"
#include "gravity.cuh"
#include "integrator.cuh"
#include "lanes.cuh"

#include <type_traits>

namespace gpop {

// Force model of one request (startup kernel, one lane per object).
template <bool MIXED> struct ForceReq {
    GravSmem g;
    const double* gen_m;
    const double* prop_m;
    __device__ __forceinline__ void prop(const double* r, const double*, int idx, double* a) const
    {
        gravity_gcrs1<MIXED>(g, prop_m + (size_t)idx * 9, r, a);
    }
    __device__ __forceinline__ void gen(const double* r, const double*, int step, int k, double* a) const
    {
        const int s = step > 0 ? step - 1 : step;
        gravity_gcrs1<MIXED>(g, gen_m + (size_t)((s + 4) * 10 + k) * 9, r, a);
    }
};

template <bool MIXED>
__device__ __forceinline__ bool stage_batch_table(uint8_t* smem, const TableSrc& ts, unsigned* err, GravSmem& g)
{
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem);
    uint8_t* tab = smem + 128;
    const bool ok = stage_to_smem(tab, ts.src, ts.bytes, mbar, err, ts.wait_spins);
    g.L = ts.L;
    g.Lt = ts.L;
    g.radius = ts.radius;
    g.gm = ts.gm;
    g.t64 = reinterpret_cast<const GravEntry64*>(tab);
    g.t32 = reinterpret_cast<const GravEntry32*>(tab + ts.off32);
    return ok;
}

template <bool MIXED>
__global__ void __launch_bounds__(256) batch_startup_kernel(TableSrc ts, BatchArgs a)
{
    extern __shared__ __align__(128) uint8_t smem[];
    GravSmem g0;
    if (!stage_batch_table<MIXED>(smem, ts, a.err, g0))
        return;
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= a.n_obj)
        return;
    const BatchReq rq = a.reqs[a.obj_req[o]];
    ForceReq<MIXED> f;
    f.g = g0;
    f.g.L = rq.L;
    f.gen_m = rq.gen_m;
    f.prop_m = rq.prop_m;
    double r0[3], v0[3];
    for (int j = 0; j < 3; ++j) {
        r0[j] = a.r0[o * 3 + j];
        v0[j] = a.v0[o * 3 + j];
    }
    StartupMats m;
    run_startup(f, rq.h, a.ncorr, r0, v0, m);
    const int64_t n = a.n_obj;
    double* st = a.state;
    const bool fix_q3 = (a.flags & 2u) != 0;
    for (int j = 0; j < 3; ++j) {
        st[(kR + j) * n + o] = m.r[8][j];
        st[(kV + j) * n + o] = m.v[8][j];
        st[(kSs + j) * n + o] = m.s[8][j];
        st[(kSb + j) * n + o] = m.S[8][j];
        for (int c = 0; c < 9; ++c)
            st[(kHist + c * 3 + j) * n + o] = m.a[c][j];
        for (int k = 0; k < 4; ++k) {
            st[(kRep + k * 6 + j) * n + o] = m.r[5 + k][j];
            st[(kRep + k * 6 + 3 + j) * n + o] = m.v[5 + k][j];
            st[(kRepA + k * 3 + j) * n + o] = fix_q3 ? m.a[5 + k][j] : m.a[8][j];
        }
    }
}

// Two objects per lane may walk the gravity columns two at a time (as gj8_kernel does), in
// batches whose items all have one lane per object (BatchArgs::pair_walk).
#ifndef GPOP_BATCH_PAIRS
#define GPOP_BATCH_PAIRS 1
#endif
constexpr bool kBatchPairs = GPOP_BATCH_PAIRS != 0;
// Two-object items park the corrector's constants (s1, s2, prev, a7: 12 doubles per object) in
// shared memory while the gravity walk runs, as gj8_kernel does, when that fits beside the table.
#ifndef GPOP_BATCH_STAGE
#define GPOP_BATCH_STAGE 1
#endif
constexpr bool kBatchStage = GPOP_BATCH_STAGE != 0;
constexpr int kBatchStageDoubles = 24; // two objects x 12
// Batches of single-lane items stage the plain table and run gj8_kernel's gravity walk (no lane
// code in that kernel).
#ifndef GPOP_BATCH_PLAIN
#define GPOP_BATCH_PLAIN 1
#endif
constexpr bool kBatchPlain = GPOP_BATCH_PLAIN != 0;

// One work item on one warp: K = 2 objects per lane for single-lane items (up to 64 objects),
// else one object per group of P lanes (up to 32 / P objects).
template <bool MIXED, int K, bool STAGE, bool PAIRS>
__device__ __forceinline__ void run_item(const GravSmem& g0, const BatchArgs& a, const BatchItem& it,
    const BatchReq& rq, int lane, double* stage)
{
    constexpr bool kStage = K == 2 && STAGE;
    // staged value q (0..3: s1, s2, prev, a7) of object k, axis j
    auto slot = [&](int q, int k, int j) { return stage + (size_t)((q * K + k) * 3 + j) * blockDim.x; };
    const int64_t n = a.n_obj;
    double* st = a.state;
    const int P = K == 1 ? rq.lpo : 1;
    const int sl = lane % P;
    int64_t o[K];
    bool valid[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int slot = K == 1 ? lane / P : lane + 32 * k;
        valid[k] = slot < it.count;
        o[k] = rq.obj0 + it.first + (valid[k] ? slot : 0); // idle slots shadow slot 0
    }
    const bool lead = sl == 0;
    GravSmem g = g0;
    g.L = rq.L;
    const double h = rq.h;
    double r[K][3], v[K][3], s[K][3], S[K][3];
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            r[k][j] = st[(kR + j) * n + o[k]];
            v[k][j] = st[(kV + j) * n + o[k]];
            s[k][j] = st[(kSs + j) * n + o[k]];
            S[k][j] = st[(kSb + j) * n + o[k]];
        }
    for (int step = 1; step <= rq.steps; ++step) {
        if (step <= 4) {
#pragma unroll
            for (int k = 0; k < K; ++k)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    r[k][j] = st[(kRep + (step - 1) * 6 + j) * n + o[k]];
                    v[k][j] = st[(kRep + (step - 1) * 6 + 3 + j) * n + o[k]];
                }
            continue;
        }
        const int ring0 = (step - 5) % 9;
        double s1[K][3], s2[K][3], prev[K][3], a7[K][3], a8[K][3];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double hist[9][3];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                int sl9 = ring0 + c;
                sl9 -= sl9 >= 9 ? 9 : 0;
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    hist[c][j] = st[(kHist + sl9 * 3 + j) * n + o[k]];
            }
#pragma unroll
            for (int j = 0; j < 3; ++j) { // predictor, as in gj8_kernel
                double vt = 0.0, rt = 0.0;
#pragma unroll
                for (int c = 0; c < 9; ++c) {
                    vt = fma(hist[c][j], c_SA[9][c], vt);
                    rt = fma(hist[c][j], c_GJ[9][c], rt);
                }
                S[k][j] += s[k][j] + hist[8][j] / 2;
                v[k][j] = (vt + s[k][j] + hist[8][j] / 2) * h;
                r[k][j] = (rt + S[k][j]) * h * h;
                double c1 = 0.0, c2 = 0.0;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    c1 = fma(hist[c + 1][j], c_SA[8][c], c1);
                    c2 = fma(hist[c + 1][j], c_GJ[8][c], c2);
                }
                s1[k][j] = c1;
                s2[k][j] = c2;
                prev[k][j] = s[k][j];
                a7[k][j] = hist[8][j];
                if constexpr (kStage) {
                    st_stage(slot(0, k, j), s1[k][j]);
                    st_stage(slot(1, k, j), s2[k][j]);
                    st_stage(slot(2, k, j), prev[k][j]);
                    st_stage(slot(3, k, j), a7[k][j]);
                }
            }
        }
        const double* M = rq.prop_m + (size_t)(step + 4) * 9;
        for (int itc = 0; itc < a.ncorr; ++itc) {
            if constexpr (K == 2 && PAIRS && kBatchPlain) {
                gravity_gcrs<MIXED, 2>(g, M, r, a8); // the plain table: gj8_kernel's walk
            } else if constexpr (K == 2 && PAIRS) {
                // two objects per lane: the two-column walk on the lane-layout tables (mixed
                // needs degree > 8 for it)
                if (!MIXED || g.L > kMixedSplit)
                    gravity_gcrs<MIXED, 2, true>(g, M, r, a8);
                else
                    gravity_gcrs_lk<MIXED, K>(g, sl, P, M, r, a8, 0xffffffffu);
            } else {
                gravity_gcrs_lk<MIXED, K>(g, sl, P, M, r, a8, 0xffffffffu);
            }
#pragma unroll
            for (int k = 0; k < K; ++k)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    if constexpr (kStage) {
                        s1[k][j] = ld_stage(slot(0, k, j));
                        s2[k][j] = ld_stage(slot(1, k, j));
                        prev[k][j] = ld_stage(slot(2, k, j));
                        a7[k][j] = ld_stage(slot(3, k, j));
                    }
                    s[k][j] = prev[k][j] + (a8[k][j] + a7[k][j]) / 2;
                    v[k][j] = h * (s1[k][j] + a8[k][j] * c_SA[8][8] + s[k][j]);
                    r[k][j] = h * h * (s2[k][j] + a8[k][j] * c_GJ[8][8] + S[k][j]);
                }
        }
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (lead && valid[k])
                for (int j = 0; j < 3; ++j)
                    st[(kHist + ring0 * 3 + j) * n + o[k]] = a8[k][j];
        __syncwarp(); // the ring write precedes the other lanes' loads of the next step
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (lead && valid[k])
            for (int j = 0; j < 3; ++j) {
                st[(kR + j) * n + o[k]] = r[k][j];
                st[(kV + j) * n + o[k]] = v[k][j];
                st[(kSs + j) * n + o[k]] = s[k][j];
                st[(kSb + j) * n + o[k]] = S[k][j];
                a.r_out[o[k] * 3 + j] = rq.steps > 0 ? r[k][j] : a.r0[o[k] * 3 + j];
                a.v_out[o[k] * 3 + j] = rq.steps > 0 ? v[k][j] : a.v0[o[k] * 3 + j];
            }
}

// Persistent GJ8 kernel: warps pull work items until the queue is empty. One 256-thread block per
// SM: the two-object path needs the registers of 8 warps.
template <bool MIXED, bool STAGE, bool PAIRS>
__global__ void __launch_bounds__(256, 1) batch_gj8_kernel(TableSrc ts, BatchArgs a)
{
    extern __shared__ __align__(128) uint8_t smem[];
    constexpr bool kPlain = PAIRS && kBatchPlain;
    GravSmem g0;
    if constexpr (kPlain) {
        if (!stage_batch_table<MIXED>(smem, ts, a.err, g0))
            return;
    } else {
        if (!bind_lane_table(smem, ts, a.err, g0))
            return;
    }
    const int lane = threadIdx.x & 31;
    double* stage = reinterpret_cast<double*>(smem + stage_offset(ts)) + threadIdx.x;
    for (;;) {
        int item = 0;
        if (lane == 0)
            item = atomicAdd(a.next_item, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= a.n_items)
            break;
        const BatchItem it = a.items[item];
        const BatchReq rq = a.reqs[it.req];
        if constexpr (kPlain) { // every item has one lane per object
            run_item<MIXED, 2, STAGE, PAIRS>(g0, a, it, rq, lane, stage);
        } else {
            if (rq.lpo == 1)
                run_item<MIXED, 2, STAGE, PAIRS>(g0, a, it, rq, lane, stage);
            else
                run_item<MIXED, 1, false, false>(g0, a, it, rq, lane, stage);
        }
    }
}

template <class K> static cudaError_t set_smem(K kernel, size_t bytes)
{
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t launch_batch_startup(const TableSrc& ts, const BatchArgs& a, int num_sms, cudaStream_t s)
{
    if (a.n_obj <= 0)
        return cudaSuccess;
    LaunchShape ls = pick_shape(a.n_obj, 256, num_sms);
    const size_t smem = table_smem_bytes(ts);
    cudaError_t e;
    if (ts.mixed) {
        if ((e = set_smem(batch_startup_kernel<true>, smem)) != cudaSuccess)
            return e;
        batch_startup_kernel<true><<<ls.grid, ls.block, smem, s>>>(ts, a);
    } else {
        if ((e = set_smem(batch_startup_kernel<false>, smem)) != cudaSuccess)
            return e;
        batch_startup_kernel<false><<<ls.grid, ls.block, smem, s>>>(ts, a);
    }
    return cudaGetLastError();
}

template <bool MIXED, bool STAGE, bool PAIRS>
static cudaError_t launch_batch_gj8_k(const TableSrc& ts, const BatchArgs& a, int blocks, int block,
    size_t smem, cudaStream_t s)
{
    cudaError_t e = set_smem(batch_gj8_kernel<MIXED, STAGE, PAIRS>, smem);
    if (e != cudaSuccess)
        return e;
    batch_gj8_kernel<MIXED, STAGE, PAIRS><<<blocks, block, smem, s>>>(ts, a);
    return cudaGetLastError();
}

template <bool MIXED>
static cudaError_t launch_batch_gj8_m(const TableSrc& lane_ts, const TableSrc& plain_ts, const BatchArgs& a,
    int blocks, int block, cudaStream_t s)
{
    const bool pairs = kBatchPairs && a.pair_walk;
    const TableSrc& ts = pairs && kBatchPlain ? plain_ts : lane_ts;
    const size_t staged = stage_offset(ts) + (size_t)kBatchStageDoubles * 8 * block;
    const bool stage = kBatchStage && staged <= max_smem_optin();
    const size_t smem = stage ? staged : table_smem_bytes(ts);
    if (stage)
        return pairs ? launch_batch_gj8_k<MIXED, true, true>(ts, a, blocks, block, smem, s)
                     : launch_batch_gj8_k<MIXED, true, false>(ts, a, blocks, block, smem, s);
    return pairs ? launch_batch_gj8_k<MIXED, false, true>(ts, a, blocks, block, smem, s)
                 : launch_batch_gj8_k<MIXED, false, false>(ts, a, blocks, block, smem, s);
}

cudaError_t launch_batch_gj8(const TableSrc& lane_ts, const TableSrc& plain_ts, const BatchArgs& a,
    int blocks, int block, cudaStream_t s)
{
    if (a.n_items <= 0)
        return cudaSuccess;
    return lane_ts.mixed ? launch_batch_gj8_m<true>(lane_ts, plain_ts, a, blocks, block, s)
                         : launch_batch_gj8_m<false>(lane_ts, plain_ts, a, blocks, block, s);
}

// ---- epoch tables of many requests: epoch e uses calendar cal[5 * epoch_req[e]] ----
__device__ __forceinline__ double warp_sum_b(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ double series_sum_b(const NutTerm* terms, int count, const double* F, int lane)
{
    double acc = 0.0;
    for (int i = lane; i < count; i += 32)
        acc += frames::nutation_term(terms[i], F);
    return warp_sum_b(acc);
}

__global__ void __launch_bounds__(256) frames_batch_kernel(FrameData fd, const int* __restrict__ cal,
    const int* __restrict__ epoch_req, const double* __restrict__ sec_args, int count,
    double* __restrict__ m_out)
{
    const int e = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (e >= count)
        return;
    const int* c = cal + 5 * epoch_req[e];
    const double mjd_utc = frames::calendar_to_mjd(c[0], c[1], c[2], c[3], c[4], sec_args[e]);
    const EopRec eop = frames::eop_at(fd.eop, fd.n_eop, mjd_utc);
    const double mjd_ut1 = mjd_utc + eop.ut1 / 86400.0;
    const double mjd_tt
        = mjd_utc + (frames::leap_at(fd.leap_mjd, fd.leap_val, fd.n_leap, mjd_utc) + frames::kTtTai) / 86400.0;
    const double t = (mjd_tt - frames::kMjdJ2000) / 36525.0;
    double F[14];
    frames::fundamental_args(t, F);
    const NutTerm* lon1 = fd.nut + fd.n_lon0;
    const NutTerm* obl0 = lon1 + fd.n_lon1;
    const NutTerm* obl1 = obl0 + fd.n_obl0;
    const double dpsi = series_sum_b(fd.nut, fd.n_lon0, F, lane) + series_sum_b(lon1, fd.n_lon1, F, lane) * t;
    const double deps = series_sum_b(obl0, fd.n_obl0, F, lane) + series_sum_b(obl1, fd.n_obl1, F, lane) * t;
    if (lane == 0) {
        double M[9];
        frames::assemble(t, F, dpsi, deps, mjd_ut1, mjd_tt, eop, M);
        for (int k = 0; k < 9; ++k)
            m_out[(size_t)e * 9 + k] = M[k];
    }
}

cudaError_t launch_frames_batch(const FrameData& fd, const int* cal, const int* epoch_req,
    const double* sec_args, int count, double* m_out, cudaStream_t s)
{
    if (count <= 0)
        return cudaSuccess;
    const int threads = 256;
    const int blocks = (int)(((int64_t)count * 32 + threads - 1) / threads);
    frames_batch_kernel<<<blocks, threads, 0, s>>>(fd, cal, epoch_req, sec_args, count, m_out);
    return cudaGetLastError();
}

} // namespace gpop
