// propagate.cu -- RK8 startup, fused GJ8 predict-evaluate-correct steps, and the gravity kernel.
//
// One thread owns one object for a whole range of steps (objects never interact), so a launch runs
// many steps with no grid-wide synchronisation. The GJ8 acceleration history lives in a 9-slot
// ring in global memory (SoA, coalesced); the working state of a step stays in registers.
#include "common.cuh"
#include "gravity.cuh"
#include "gj8_tables.cuh"
#include "integrator.cuh"
#include "lanes.cuh"
#include "kernels.h"

#include <type_traits>

namespace gpop {

// ---- force models seen by the integrator (IForceModel, iforce_model.cuh:19-33) ----
// COMP: mixed precision with compensated FP32 sums (GPOP_MIXED_COMPENSATED).
template <bool MIXED, bool COMP = false> struct ForceGravity {
    static constexpr bool kTable = true;
    static constexpr bool kMixed = MIXED;
    static constexpr bool kComp = COMP;
    GravSmem g;
    const double* gen_m;
    const double* prop_m;
    // ForceModel::ComputePropagationAcceleration (force_model.cu:91-109): epoch index idx
    __device__ __forceinline__ void prop(const double* r, const double*, int idx, double* a) const
    {
        gravity_gcrs1<MIXED, COMP>(g, prop_m + (size_t)idx * 9, r, a);
    }
    template <int K>
    __device__ __forceinline__ void prop_k(const double (&r)[K][3], const double (&)[K][3], int idx,
        double (&a)[K][3]) const
    {
        gravity_gcrs<MIXED, K, false, COMP>(g, prop_m + (size_t)idx * 9, r, a);
    }
    // ForceModel::ComputeGenerationAcceleration (force_model.cu:59-89): table (s'+4)*10 + k
    __device__ __forceinline__ void gen(const double* r, const double*, int step, int k, double* a) const
    {
        const int s = step > 0 ? step - 1 : step;
        gravity_gcrs1<MIXED, COMP>(g, gen_m + (size_t)((s + 4) * 10 + k) * 9, r, a);
    }
};

// Analytic accelerations of the reference's tests (unit_tests/include/gpu_test_helpers.cuh) with the
// mock's time rules (unit_tests/include/mock_force_model.cuh:65-106).
struct ForceAnalytic {
    static constexpr bool kTable = false;
    static constexpr bool kMixed = false;
    int kind;
    double h;
    __device__ void eval(const double* p, const double* v, double t, double* a) const
    {
        double val = 0.0;
        switch (kind) {
        case 2:
            a[0] = 1;
            a[1] = 2;
            a[2] = 3;
            return;
        case 3:
            val = -3 * 2 * t + 7 * 6 * t * t * t * t * t;
            break;
        case 4:
            val = 56 * pow(t, 6) - 42 * pow(t, 5) + 60 * pow(t, 4) - 100 * pow(t, 3)
                - 120 * pow(t, 2) + 6 * t - 2;
            break;
        case 5:
            val = 72 * pow(t, 7) + 56 * pow(t, 6) - 42 * pow(t, 5) + 60 * pow(t, 4)
                - 100 * pow(t, 3) - 120 * pow(t, 2) + 6 * t - 2;
            break;
        case 6:
            val = exp(-t);
            break;
        case 7:
            for (int i = 0; i < 3; ++i)
                a[i] = -2 * p[i] - 2 * v[i];
            return;
        default:
            val = 0.0;
        }
        a[0] = a[1] = a[2] = val;
    }
    __device__ __forceinline__ void prop(const double* r, const double* v, int idx, double* a) const
    {
        eval(r, v, (double)(idx - 4) * h, a);
    }
    template <int K>
    __device__ __forceinline__ void prop_k(const double (&r)[K][3], const double (&v)[K][3], int idx,
        double (&a)[K][3]) const
    {
#pragma unroll
        for (int k = 0; k < K; ++k)
            eval(r[k], v[k], (double)(idx - 4) * h, a[k]);
    }
    __device__ __forceinline__ void gen(const double* r, const double* v, int step, int k, double* a) const
    {
        const int dir = step > 0 ? -1 : 1;
        eval(r, v, (double)(step + dir) * h + (-dir) * c_RKC[k] * h, a);
    }
};

// ---- table staging ----
size_t table_smem_bytes(const TableSrc& ts) { return 128 + (size_t)ts.bytes; }

template <bool MIXED>
__device__ __forceinline__ bool bind_table(uint8_t* smem, const TableSrc& ts, unsigned* err, GravSmem& g)
{
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem);
    uint8_t* tab = smem + 128;
    bool ok = stage_to_smem(tab, ts.src, ts.bytes, mbar, err, ts.wait_spins);
    g.L = ts.L;
    g.Lt = ts.L;
    g.radius = ts.radius;
    g.gm = ts.gm;
    g.t64 = reinterpret_cast<const GravEntry64*>(tab);
    g.t32 = reinterpret_cast<const GravEntry32*>(tab + ts.off32);
    return ok;
}

template <class F>
__global__ void __launch_bounds__(256) startup_kernel(F f, TableSrc ts, PropArgs a)
{
    extern __shared__ __align__(128) uint8_t smem[];
    if constexpr (F::kTable) {
        if (!bind_table<F::kMixed>(smem, ts, a.err, f.g))
            return;
    }
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n)
        return;
    double r0[3], v0[3];
    for (int j = 0; j < 3; ++j) {
        r0[j] = a.r0[i * 3 + j];
        v0[j] = a.v0[i * 3 + j];
    }
    // a state the force model cannot take (the reference propagates it into NaNs) fails the call;
    // the object still runs, so every other object's result is written as usual
    bool usable = true;
    for (int j = 0; j < 3; ++j)
        usable = usable && isfinite(r0[j]) && isfinite(v0[j]);
    if (F::kTable && r0[0] == 0.0 && r0[1] == 0.0 && r0[2] == 0.0)
        usable = false;
    if (!usable && a.err)
        atomicOr(a.err, kErrBadInput);
    StartupMats m;
    run_startup(f, a.h, a.ncorr, r0, v0, m);
    if (a.out27[0]) {
        for (int c = 0; c < 9; ++c)
            for (int j = 0; j < 3; ++j) {
                const int64_t o = i * 27 + c * 3 + j;
                a.out27[0][o] = m.r[c][j];
                a.out27[1][o] = m.v[c][j];
                a.out27[2][o] = m.a[c][j];
                a.out27[3][o] = m.s[c][j];
                a.out27[4][o] = m.S[c][j];
            }
    }
    if (a.state) {
        const int64_t n = a.n;
        double* st = a.state;
        const bool fix_q3 = (a.flags & 2u) != 0;
        for (int j = 0; j < 3; ++j) {
            // GpuPropagator::Step at step 1 (gpu_propagator.cu:31-47): s, S from column 8; the
            // caller's buffers hold column 8 after the corrector (gpu_startup.cu:59-61).
            st[(kR + j) * n + i] = m.r[8][j];
            st[(kV + j) * n + i] = m.v[8][j];
            st[(kSs + j) * n + i] = m.s[8][j];
            st[(kSb + j) * n + i] = m.S[8][j];
            for (int c = 0; c < 9; ++c)
                st[(kHist + c * 3 + j) * n + i] = m.a[c][j];
            for (int k = 0; k < 4; ++k) { // replay of steps 1..4 (CopyStartupStateKernel)
                st[(kRep + k * 6 + j) * n + i] = m.r[5 + k][j];
                st[(kRep + k * 6 + 3 + j) * n + i] = m.v[5 + k][j];
                st[(kRepA + k * 3 + j) * n + i] = fix_q3 ? m.a[5 + k][j] : m.a[8][j];
            }
        }
    }
}

// ---- GJ8 step (prediction.cu:49-74 + gpu_propagator.cu:86-119) ----
// K objects per thread: object k of thread g is g + k * (threads in the grid); every gravity
// evaluation of a step runs the K objects in lockstep on the same table entries.
//
// With a gravity table, the corrector's constants of a step (s1, s2, prev, a7: 12 doubles per
// object) and S wait in shared memory while the gravity walk runs, which leaves the walk the
// registers they would hold (two objects, 65,536 objects at 70x70 on B200, with the paired column
// walks: mixed 125.5 -> 131.5 M object-steps/s, FP64 72.3 -> 73.8 M).
// Largest block of the one-object-per-thread kernel (its register budget is 65,536 / this; at 256
// the FP64 two-column walk fits without spills).
#ifndef GPOP_ONE_OBJECT_BLOCK
#define GPOP_ONE_OBJECT_BLOCK 256
#endif
constexpr int kOneObjectBlock = GPOP_ONE_OBJECT_BLOCK;

#ifndef GPOP_STAGE_CORRECTOR
#define GPOP_STAGE_CORRECTOR 1
#endif
#ifndef GPOP_STAGE_FP64
#define GPOP_STAGE_FP64 1
#endif
constexpr int kStageDoubles = 15; // per object: s1, s2, prev, a7, S (3 each)
template <class F> constexpr bool stage_corrector()
{
    return F::kTable && (F::kMixed || GPOP_STAGE_FP64 != 0) && GPOP_STAGE_CORRECTOR != 0;
}


// ---- column-split block (gj8_kernel with SPLIT) ----
// With two objects per thread, a block of 5 to 7 warps loads the four schedulers of an SM
// unevenly (65,536 objects: 7 warps, spread 2-2-2-1, so the SM takes as long as for 8 warps). The
// split block has 8 warps: S owner warps carry two objects per thread through the step and walk
// the high columns of their objects (split_high); warp S + b walks the low columns (split_low) of
// the objects of owner warps b, b + (8 - S), ... Per evaluation the owners publish each object's
// Earth-fixed position and walk start values, a barrier, both walks, the low totals are
// published, a barrier, and the owners add them to their own. The exchange lives in shared memory
// when it fits beside the table and the corrector state (kSplitSmem), else in the state arrays
// kX0.. (per object). Every thread of the block takes the same barriers: the loops over steps and
// evaluations are the same for all threads and none leaves early.
constexpr int kSplitWarps = 8;
constexpr int kSplitBlock = 32 * kSplitWarps;
enum SplitMode : int { kSplitNone = 0, kSplitGlobal = 1, kSplitSmem = 2 };
// exchanged values per object: x y z | q u w C1 S1 | low totals G H J K
constexpr int kXchValues = 12;
constexpr size_t kSplitSmemBytes = (size_t)kXchValues * 2 * kSplitBlock * sizeof(double);
static_assert(kXchValues == kStateArrays - kX0, "the state carries one exchange array per value");

// Owner thread t of a split launch over objects [lo, lo + cnt) carries objects lo + t and
// lo + t + (owner threads in the grid); an idle slot shadows the thread's first object (or the
// last one) and never stores.
__device__ __forceinline__ void split_objects(int64_t t, int64_t gown, int64_t lo, int64_t cnt,
    int64_t (&obj)[2], bool (&live)[2])
{
    const int64_t shadow = t < cnt ? t : cnt - 1;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int64_t o = t + k * gown;
        live[k] = o < cnt;
        obj[k] = lo + (live[k] ? o : shadow);
    }
}

// Exchange value v of a slot: in shared memory slot k * kSplitBlock + (owner thread of the block),
// in the state arrays the object itself.
template <int SPLIT> struct Exchange {
    double* base;
    int64_t stride;
    __device__ __forceinline__ double* at(int v, int64_t slot) const { return base + v * stride + slot; }
    __device__ __forceinline__ void put(int v, int64_t slot, double x) const
    {
        if constexpr (SPLIT == kSplitSmem)
            *at(v, slot) = x;
        else
            __stcg(at(v, slot), x);
    }
    __device__ __forceinline__ double get(int v, int64_t slot) const
    {
        if constexpr (SPLIT == kSplitSmem)
            return *at(v, slot);
        else
            return __ldcg(at(v, slot));
    }
};

// One gravity evaluation of a split block: a8 (owners) = GCRS accelerations at the GCRS positions r.
template <bool MIXED, int SPLIT>
__device__ __forceinline__ void split_eval(const GravSmem& g, const double* __restrict__ M,
    const PropArgs& a, bool owner, const bool (&live)[2], const int64_t (&obj)[2],
    const double (&r)[2][3], double (&a8)[2][3], double* xsmem)
{
    constexpr int K = 2;
    const int S = a.split_owners;
    const int64_t n = a.n; // the state's stride
    const int64_t cnt = (a.obj_hi < 0 ? n : a.obj_hi) - a.obj_lo; // objects of this launch
    const int tau = (int)threadIdx.x; // owner thread of the block (owners only)
    Exchange<SPLIT> X;
    if constexpr (SPLIT == kSplitSmem) {
        X.base = xsmem;
        X.stride = 2 * kSplitBlock;
    } else {
        X.base = a.state + (int64_t)kX0 * n;
        X.stride = n;
    }
    // slot of value k of owner thread t whose object k is ok
    auto slot = [](int k, int t, int64_t ok) -> int64_t {
        if constexpr (SPLIT == kSplitSmem)
            return (int64_t)k * kSplitBlock + t;
        else
            return ok;
    };
    double m[9];
#pragma unroll
    for (int i = 0; i < 9; ++i)
        m[i] = __ldg(M + i);
    if (owner) {
        double x[K], y[K], z[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            x[k] = m[0] * r[k][0] + m[1] * r[k][1] + m[2] * r[k][2];
            y[k] = m[3] * r[k][0] + m[4] * r[k][1] + m[5] * r[k][2];
            z[k] = m[6] * r[k][0] + m[7] * r[k][1] + m[8] * r[k][2];
        }
        WalkStart ws;
        walk_start(g.radius, x, y, z, ws);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!live[k])
                continue;
            const int64_t sl = slot(k, tau, obj[k]);
            X.put(0, sl, x[k]);
            X.put(1, sl, y[k]);
            X.put(2, sl, z[k]);
            X.put(3, sl, ws.q[k]);
            X.put(4, sl, ws.u[k]);
            X.put(5, sl, ws.w[k]);
            X.put(6, sl, ws.C1[k]);
            X.put(7, sl, ws.S1[k]);
        }
    }
    __syncthreads();
    SplitTotals hi;
    if (owner) {
        // the start values are read back rather than held across the barrier; an idle slot walks
        // the thread's first object again
        WalkStart ws;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int64_t sl = live[k] ? slot(k, tau, obj[k]) : slot(0, tau, obj[0]);
            ws.q[k] = X.get(3, sl);
            ws.u[k] = X.get(4, sl);
            ws.w[k] = X.get(5, sl);
            ws.C1[k] = X.get(6, sl);
            ws.S1[k] = X.get(7, sl);
        }
        split_high<MIXED>(g, ws, hi);
    } else {
        const int64_t gown = (int64_t)gridDim.x * 32 * S;
        const int lane = (int)(threadIdx.x & 31);
        const int nb = kSplitWarps - S;
        for (int w = (int)(threadIdx.x >> 5) - S; w < S; w += nb) {
            const int t = w * 32 + lane; // the owner thread whose objects this lane walks
            int64_t o[K];
            bool lv[K];
            split_objects((int64_t)blockIdx.x * 32 * S + t, gown, a.obj_lo, cnt, o, lv);
            if (!lv[0])
                continue; // no object (then the second slot is empty too)
            WalkStart ws;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int64_t sl = lv[k] ? slot(k, t, o[k]) : slot(0, t, o[0]);
                ws.q[k] = X.get(3, sl);
                ws.u[k] = X.get(4, sl);
                ws.w[k] = X.get(5, sl);
                ws.C1[k] = X.get(6, sl);
                ws.S1[k] = X.get(7, sl);
            }
            SplitTotals lo;
            split_low<MIXED>(g, ws, lo);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if (!lv[k])
                    continue;
                const int64_t sl = slot(k, t, o[k]);
                X.put(8, sl, lo.G[k]);
                X.put(9, sl, lo.H[k]);
                X.put(10, sl, lo.J[k]);
                X.put(11, sl, lo.K[k]);
            }
        }
    }
    __syncthreads();
    // The rotation and the positions are read again rather than held through the walk, and every
    // thread writes a8 (zero for an idle slot or a walk-only thread), so that no earlier value
    // lives through the walks.
#pragma unroll
    for (int i = 0; i < 9; ++i)
        m[i] = __ldg(M + i);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (!live[k]) {
            a8[k][0] = a8[k][1] = a8[k][2] = 0.0;
            continue;
        }
        const int64_t sl = slot(k, tau, obj[k]);
        const double x = X.get(0, sl), y = X.get(1, sl), z = X.get(2, sl);
        const double rk = sqrt(x * x + y * y + z * z);
        double ax, ay, az;
        assemble_itrs(g.gm, x, y, z, rk, X.get(8, sl) + hi.G[k], X.get(9, sl) + hi.H[k],
            X.get(10, sl) + hi.J[k], X.get(11, sl) + hi.K[k], ax, ay, az);
        a8[k][0] = m[0] * ax + m[3] * ay + m[6] * az;
        a8[k][1] = m[1] * ax + m[4] * ay + m[7] * az;
        a8[k][2] = m[2] * ax + m[5] * ay + m[8] * az;
    }
}

template <class F, int K, bool STAGE, int SPLIT = kSplitNone>
__global__ void __launch_bounds__(K == 1 ? kOneObjectBlock : 256, 1) gj8_kernel(F f, TableSrc ts, PropArgs a)
{
    extern __shared__ __align__(128) uint8_t smem[];
    constexpr bool kStage = STAGE && stage_corrector<F>();
    static_assert(SPLIT == kSplitNone || (K == 2 && F::kTable),
        "the split block carries two objects per thread");
    double* stage = nullptr;
    if constexpr (F::kTable) {
        bool ok = bind_table<F::kMixed>(smem, ts, a.err, f.g);
        if constexpr (SPLIT != kSplitNone)
            ok = __syncthreads_and(ok); // the block leaves as one: barriers follow
        if (!ok)
            return;
        stage = reinterpret_cast<double*>(smem + stage_offset(ts)) + threadIdx.x;
    }
    // staged value q (0..4: s1, s2, prev, a7, S) of object k, axis j
    auto slot = [&](int q, int k, int j) { return stage + (size_t)((q * K + k) * 3 + j) * blockDim.x; };
    const int64_t n = a.n; // the state's stride; this launch runs objects [lo, lo + cnt)
    const int64_t lo = a.obj_lo, cnt = (a.obj_hi < 0 ? n : a.obj_hi) - lo;
    int64_t obj[K];
    bool live[K];
    // split block: owner warps carry objects; the other warps walk low columns and run the step on
    // a shadow of the block's first objects (never stored), so that no value lives on only for them
    bool owner = true;
    double* xsmem = nullptr; // split block: the exchange in shared memory, after the staged state
    if constexpr (SPLIT != kSplitNone) {
        if constexpr (SPLIT == kSplitSmem)
            xsmem = reinterpret_cast<double*>(smem + stage_offset(ts)
                + (kStage ? (size_t)kStageDoubles * K * 8 * blockDim.x : 0));
        const int S = a.split_owners;
        owner = (int)(threadIdx.x >> 5) < S;
        const int64_t gown = (int64_t)gridDim.x * 32 * S;
        split_objects((int64_t)blockIdx.x * 32 * S + (owner ? threadIdx.x : 0), gown, lo, cnt, obj,
            live);
        if (!owner)
            live[0] = live[1] = false;
    } else {
        const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        const int64_t G = (int64_t)gridDim.x * blockDim.x;
        if (g >= cnt)
            return;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int64_t o = g + k * G;
            live[k] = o < cnt;
            obj[k] = lo + (live[k] ? o : g); // idle slots shadow object lo + g and never store
        }
    }
    double* st = a.state;
    const double h = a.h;
    double r[K][3], v[K][3], s[K][3], S[K][3];
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            r[k][j] = st[(kR + j) * n + obj[k]];
            v[k][j] = st[(kV + j) * n + obj[k]];
            s[k][j] = st[(kSs + j) * n + obj[k]];
            S[k][j] = st[(kSb + j) * n + obj[k]];
        }
    for (int step = a.step_begin; step < a.step_end; ++step) {
        double ae[K][3];
        if (step <= 4) {
#pragma unroll
            for (int k = 0; k < K; ++k)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    r[k][j] = st[(kRep + (step - 1) * 6 + j) * n + obj[k]];
                    v[k][j] = st[(kRep + (step - 1) * 6 + 3 + j) * n + obj[k]];
                    ae[k][j] = st[(kRepA + (step - 1) * 3 + j) * n + obj[k]];
                }
        } else {
            const int ring0 = (step - 5) % 9;
            double s1[K][3], s2[K][3], prev[K][3], a7[K][3], a8[K][3];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                double hist[9][3];
#pragma unroll
                for (int c = 0; c < 9; ++c) {
                    int slot = ring0 + c;
                    slot -= slot >= 9 ? 9 : 0;
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        hist[c][j] = st[(kHist + slot * 3 + j) * n + obj[k]];
                }
                // Predictor (FinalizePredictionKernel, gpu_integrator/src/device/dev_functions.cu:34-50)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    double vt = 0.0, rt = 0.0;
#pragma unroll
                    for (int c = 0; c < 9; ++c) {
                        vt = fma(hist[c][j], c_SA[9][c], vt);
                        rt = fma(hist[c][j], c_GJ[9][c], rt);
                    }
                    S[k][j] += s[k][j] + hist[8][j] / 2;
                    v[k][j] = (vt + s[k][j] + hist[8][j] / 2) * h;
                    r[k][j] = (rt + S[k][j]) * h * h;
                    // corrector partial sums over the shifted history (gpu_propagator.cu:92-100)
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
                        st_stage(slot(4, k, j), S[k][j]);
                    }
                }
            }
            const int idx = step + 4;
            if constexpr (SPLIT != kSplitNone)
                split_eval<F::kMixed, SPLIT>(f.g, f.prop_m + (size_t)idx * 9, a, owner, live, obj, r,
                    a8, xsmem);
            else
                f.template prop_k<K>(r, v, idx, a8);
            // Corrector: the first pass reuses the predictor's evaluation at the unchanged
            // position (bit-identical to the reference's repeated call).
            for (int it = 0; it < a.ncorr; ++it) {
                if (it > 0) {
                    if constexpr (SPLIT != kSplitNone)
                        split_eval<F::kMixed, SPLIT>(f.g, f.prop_m + (size_t)idx * 9, a, owner, live,
                            obj, r, a8, xsmem);
                    else
                        f.template prop_k<K>(r, v, idx, a8);
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
                            S[k][j] = ld_stage(slot(4, k, j));
                        }
                        s[k][j] = prev[k][j] + (a8[k][j] + a7[k][j]) / 2;
                        v[k][j] = h * (s1[k][j] + a8[k][j] * c_SA[8][8] + s[k][j]);
                        r[k][j] = h * h * (s2[k][j] + a8[k][j] * c_GJ[8][8] + S[k][j]);
                    }
            }
#pragma unroll
            for (int k = 0; k < K; ++k)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    if (live[k])
                        st[(kHist + ring0 * 3 + j) * n + obj[k]] = a8[k][j];
                    ae[k][j] = a8[k][j];
                }
        }
        const int64_t t = step - a.traj_step0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!live[k])
                continue;
            if (a.traj_r)
                for (int j = 0; j < 3; ++j)
                    a.traj_r[(t * 3 + j) * n + obj[k]] = r[k][j];
            if (a.traj_v)
                for (int j = 0; j < 3; ++j)
                    a.traj_v[(t * 3 + j) * n + obj[k]] = v[k][j];
            if (a.traj_a)
                for (int j = 0; j < 3; ++j)
                    a.traj_a[(t * 3 + j) * n + obj[k]] = ae[k][j];
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (!live[k])
            continue;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            st[(kR + j) * n + obj[k]] = r[k][j];
            st[(kV + j) * n + obj[k]] = v[k][j];
            st[(kSs + j) * n + obj[k]] = s[k][j];
            st[(kSb + j) * n + obj[k]] = S[k][j];
            if (a.out_r)
                a.out_r[obj[k] * 3 + j] = r[k][j];
            if (a.out_v)
                a.out_v[obj[k] * 3 + j] = v[k][j];
        }
    }
}

// ---- RK8 startup in the split block (the sizes where the GJ8 steps take it) ----
// run_startup2 over two objects per owner thread; each of its 145 gravity evaluations per object
// is one split_eval, so the walk-only warps take the low columns here too. Outputs and the
// bad-input flag as startup_kernel.
template <bool MIXED, int SPLIT> struct SplitForce2 {
    const ForceGravity<MIXED>& f;
    const PropArgs& a;
    bool owner;
    const bool (&live)[2];
    const int64_t (&obj)[2];
    double* xsmem;
    __device__ __forceinline__ void gen2(const double (&r)[2][3], const double (&)[2][3], int step,
        int k, double (&acc)[2][3]) const
    {
        const int st = step > 0 ? step - 1 : step; // ForceModel::ComputeGenerationAcceleration
        split_eval<MIXED, SPLIT>(f.g, f.gen_m + (size_t)((st + 4) * 10 + k) * 9, a, owner, live, obj,
            r, acc, xsmem);
    }
    __device__ __forceinline__ void prop2(const double (&r)[2][3], const double (&)[2][3], int idx,
        double (&acc)[2][3]) const
    {
        split_eval<MIXED, SPLIT>(f.g, f.prop_m + (size_t)idx * 9, a, owner, live, obj, r, acc, xsmem);
    }
};

template <bool MIXED, int SPLIT>
__global__ void __launch_bounds__(kSplitBlock, 1) startup_split_kernel(ForceGravity<MIXED> f, TableSrc ts,
    PropArgs a)
{
    extern __shared__ __align__(128) uint8_t smem[];
    bool ok = bind_table<MIXED>(smem, ts, a.err, f.g);
    ok = __syncthreads_and(ok); // the block leaves as one: barriers follow
    if (!ok)
        return;
    double* xsmem = SPLIT == kSplitSmem ? reinterpret_cast<double*>(smem + stage_offset(ts)) : nullptr;
    const int S = a.split_owners;
    const bool owner = (int)(threadIdx.x >> 5) < S;
    const int64_t n = a.n;
    int64_t obj[2];
    bool live[2];
    split_objects((int64_t)blockIdx.x * 32 * S + (owner ? threadIdx.x : 0), (int64_t)gridDim.x * 32 * S,
        0, n, obj, live);
    if (!owner)
        live[0] = live[1] = false;
    double r0[2][3], v0[2][3];
    for (int k = 0; k < 2; ++k)
        for (int j = 0; j < 3; ++j) {
            r0[k][j] = a.r0[obj[k] * 3 + j];
            v0[k][j] = a.v0[obj[k] * 3 + j];
        }
    for (int k = 0; k < 2; ++k) { // as startup_kernel: the call fails, the object still runs
        if (!live[k])
            continue;
        bool usable = true;
        for (int j = 0; j < 3; ++j)
            usable = usable && isfinite(r0[k][j]) && isfinite(v0[k][j]);
        if (r0[k][0] == 0.0 && r0[k][1] == 0.0 && r0[k][2] == 0.0)
            usable = false;
        if (!usable && a.err)
            atomicOr(a.err, kErrBadInput);
    }
    StartupMats m[2];
    const SplitForce2<MIXED, SPLIT> F { f, a, owner, live, obj, xsmem };
    run_startup2(F, a.h, a.ncorr, r0, v0, m, owner); // the walk-only warps skip the arithmetic
    const bool fix_q3 = (a.flags & 2u) != 0;
    double* st = a.state;
    for (int k = 0; k < 2; ++k) {
        if (!live[k])
            continue;
        const int64_t i = obj[k];
        if (a.out27[0]) {
            for (int c = 0; c < 9; ++c)
                for (int j = 0; j < 3; ++j) {
                    const int64_t o = i * 27 + c * 3 + j;
                    a.out27[0][o] = m[k].r[c][j];
                    a.out27[1][o] = m[k].v[c][j];
                    a.out27[2][o] = m[k].a[c][j];
                    a.out27[3][o] = m[k].s[c][j];
                    a.out27[4][o] = m[k].S[c][j];
                }
        }
        if (st) {
            for (int j = 0; j < 3; ++j) {
                st[(kR + j) * n + i] = m[k].r[8][j];
                st[(kV + j) * n + i] = m[k].v[8][j];
                st[(kSs + j) * n + i] = m[k].s[8][j];
                st[(kSb + j) * n + i] = m[k].S[8][j];
                for (int c = 0; c < 9; ++c)
                    st[(kHist + c * 3 + j) * n + i] = m[k].a[c][j];
                for (int q = 0; q < 4; ++q) {
                    st[(kRep + q * 6 + j) * n + i] = m[k].r[5 + q][j];
                    st[(kRep + q * 6 + 3 + j) * n + i] = m[k].v[5 + q][j];
                    st[(kRepA + q * 3 + j) * n + i] = fix_q3 ? m[k].a[5 + q][j] : m[k].a[8][j];
                }
            }
        }
    }
}

// ---- GJ8 step with P lanes per group of K objects (few objects) ----
// Same step as gj8_kernel; the P lanes of a group split the gravity columns of its K objects
// (lanes.cuh, lane-layout table) and hold identical state; lane 0 of the group stores. Object k
// of group g is g + k * (groups in the grid). Used when the objects alone leave most warp slots of
// the GPU empty. MAXT bounds the block (and so the registers a thread may hold): 512 for the many
// lanes of few objects, 384 for two lanes per object, which then keeps its table loads in flight.
// STAGE: the corrector's constants of a step (s1, s2, prev, a7, S) wait in shared memory during
// the gravity walks, one copy per lane group written by its lead lane, as in gj8_kernel (two
// objects per lane group, FP64, 18,944 objects at four lanes: the walk at 254 registers waited on
// its table loads, short_scoreboard 1.43 per issued instruction, FP64 pipe 59 % busy).
template <bool MIXED, int K, int MAXT = (K == 1 ? 512 : 256), bool STAGE = false>
__global__ void __launch_bounds__(MAXT, 1) gj8_lanes_kernel(TableSrc ts, PropArgs a, int P)
{
    extern __shared__ __align__(128) uint8_t smem[];
    GravSmem g;
    if (!bind_lane_table(smem, ts, a.err, g))
        return;
    double* stage = nullptr;
    if constexpr (STAGE)
        stage = reinterpret_cast<double*>(smem + stage_offset(ts)) + threadIdx.x / P;
    // staged value q (0..4: s1, s2, prev, a7, S) of object k, axis j, of this lane's group
    auto slot = [&](int q, int k, int j) { return stage + (size_t)((q * K + k) * 3 + j) * (blockDim.x / P); };
    const int64_t grp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / P;
    const int64_t groups = ((int64_t)gridDim.x * blockDim.x) / P;
    const int lane = (int)(threadIdx.x & 31);
    const int l = lane & (P - 1);
    const int64_t n = a.n; // the state's stride; this launch runs objects [lo, hi)
    const int64_t lo = a.obj_lo, hi = a.obj_hi < 0 ? n : a.obj_hi;
    if (grp >= hi - lo)
        return; // whole groups leave: shuffles name the group only
    const unsigned mask = P == 32 ? 0xffffffffu : ((1u << P) - 1u) << (lane & ~(P - 1));
    const bool lead = l == 0;
    int64_t obj[K];
    bool live[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int64_t o = lo + grp + k * groups;
        live[k] = o < hi;
        obj[k] = live[k] ? o : lo + grp; // idle slots shadow the group's first object and never store
    }
    double* st = a.state;
    const double h = a.h;
    double r[K][3], v[K][3], s[K][3], S[K][3];
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            r[k][j] = st[(kR + j) * n + obj[k]];
            v[k][j] = st[(kV + j) * n + obj[k]];
            s[k][j] = st[(kSs + j) * n + obj[k]];
            S[k][j] = st[(kSb + j) * n + obj[k]];
        }
    for (int step = a.step_begin; step < a.step_end; ++step) {
        double ae[K][3];
        if (step <= 4) {
#pragma unroll
            for (int k = 0; k < K; ++k)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    r[k][j] = st[(kRep + (step - 1) * 6 + j) * n + obj[k]];
                    v[k][j] = st[(kRep + (step - 1) * 6 + 3 + j) * n + obj[k]];
                    ae[k][j] = st[(kRepA + (step - 1) * 3 + j) * n + obj[k]];
                }
        } else {
            const int ring0 = (step - 5) % 9;
            double s1[K][3], s2[K][3], prev[K][3], a7[K][3], a8[K][3];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                double hist[9][3];
#pragma unroll
                for (int c = 0; c < 9; ++c) {
                    int slot = ring0 + c;
                    slot -= slot >= 9 ? 9 : 0;
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        hist[c][j] = st[(kHist + slot * 3 + j) * n + obj[k]];
                }
#pragma unroll
                for (int j = 0; j < 3; ++j) { // as gj8_kernel
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
                    if constexpr (STAGE) {
                        if (lead) {
                            st_stage(slot(0, k, j), s1[k][j]);
                            st_stage(slot(1, k, j), s2[k][j]);
                            st_stage(slot(2, k, j), prev[k][j]);
                            st_stage(slot(3, k, j), a7[k][j]);
                            st_stage(slot(4, k, j), S[k][j]);
                        }
                    }
                }
            }
            if constexpr (STAGE)
                __syncwarp(mask); // the lead's stores precede the group's loads
            const double* M = a.prop_m + (size_t)(step + 4) * 9;
            for (int it = 0; it < a.ncorr; ++it) {
                // two columns at a time for one object per group at up to 384 threads a block (FP64
                // 1,024 objects: 18.8 against 17.4 M object-steps/s); with two objects per group,
                // or the 128 registers of 512-thread blocks, that spills (-9 %)
                gravity_gcrs_lk<MIXED, K, K == 1 && MAXT <= 384>(g, l, P, M, r, a8, mask);
#pragma unroll
                for (int k = 0; k < K; ++k)
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        if constexpr (STAGE) {
                            s1[k][j] = ld_stage(slot(0, k, j));
                            s2[k][j] = ld_stage(slot(1, k, j));
                            prev[k][j] = ld_stage(slot(2, k, j));
                            a7[k][j] = ld_stage(slot(3, k, j));
                            S[k][j] = ld_stage(slot(4, k, j));
                        }
                        s[k][j] = prev[k][j] + (a8[k][j] + a7[k][j]) / 2;
                        v[k][j] = h * (s1[k][j] + a8[k][j] * c_SA[8][8] + s[k][j]);
                        r[k][j] = h * h * (s2[k][j] + a8[k][j] * c_GJ[8][8] + S[k][j]);
                    }
            }
#pragma unroll
            for (int k = 0; k < K; ++k)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    if (lead && live[k])
                        st[(kHist + ring0 * 3 + j) * n + obj[k]] = a8[k][j];
                    ae[k][j] = a8[k][j];
                }
        }
        __syncwarp(mask); // the group's ring write precedes its next step's loads
        if (lead) {
            const int64_t t = step - a.traj_step0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if (!live[k])
                    continue;
                for (int j = 0; j < 3; ++j) {
                    if (a.traj_r)
                        a.traj_r[(t * 3 + j) * n + obj[k]] = r[k][j];
                    if (a.traj_v)
                        a.traj_v[(t * 3 + j) * n + obj[k]] = v[k][j];
                    if (a.traj_a)
                        a.traj_a[(t * 3 + j) * n + obj[k]] = ae[k][j];
                }
            }
        }
    }
    if (!lead)
        return;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (!live[k])
            continue;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            st[(kR + j) * n + obj[k]] = r[k][j];
            st[(kV + j) * n + obj[k]] = v[k][j];
            st[(kSs + j) * n + obj[k]] = s[k][j];
            st[(kSb + j) * n + obj[k]] = S[k][j];
            if (a.out_r)
                a.out_r[obj[k] * 3 + j] = r[k][j];
            if (a.out_v)
                a.out_v[obj[k] * 3 + j] = v[k][j];
        }
    }
}

template <bool MIXED>
__global__ void __launch_bounds__(512, 1) gravity_kernel(TableSrc ts, int64_t n, const double* r,
    const double* m9, double* a, unsigned* err)
{
    extern __shared__ __align__(128) uint8_t smem[];
    GravSmem g;
    if (!bind_table<MIXED>(smem, ts, err, g))
        return;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double p[3] = { r[i * 3], r[i * 3 + 1], r[i * 3 + 2] };
    if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2]) || (p[0] == 0.0 && p[1] == 0.0 && p[2] == 0.0))
        atomicOr(err, kErrBadInput);
    double acc[3];
    if (m9) {
        gravity_gcrs1<MIXED>(g, m9, p, acc);
    } else {
        gravity_itrs1<MIXED>(g, p[0], p[1], p[2], acc[0], acc[1], acc[2]);
    }
    a[i * 3] = acc[0];
    a[i * 3 + 1] = acc[1];
    a[i * 3 + 2] = acc[2];
}

// ---- single-object unit kernels for the integrator's known-answer tests ----
__global__ void corrector_unit_kernel(ForceAnalytic f, int op, double* r27, double* v27,
    double* a27, double* s27, double* S27)
{
    StartupMats m;
    for (int c = 0; c < 9; ++c)
        for (int j = 0; j < 3; ++j) {
            m.r[c][j] = r27[c * 3 + j];
            m.v[c][j] = v27[c * 3 + j];
            m.a[c][j] = m.s[c][j] = m.S[c][j] = 0.0;
        }
    corrector_accel(f, m, true);
    if (op == 1)
        corrector_s0(f.h, m);
    else if (op == 2)
        corrector_correct(f, f.h, m);
    for (int c = 0; c < 9; ++c)
        for (int j = 0; j < 3; ++j) {
            r27[c * 3 + j] = m.r[c][j];
            v27[c * 3 + j] = m.v[c][j];
            a27[c * 3 + j] = m.a[c][j];
            s27[c * 3 + j] = m.s[c][j];
            S27[c * 3 + j] = m.S[c][j];
        }
}

__global__ void predict_unit_kernel(ForceAnalytic f, int step, double* r, double* v, double* a27,
    double* s, double* S)
{
    const double h = f.h;
    double vt[3], rt[3];
    for (int j = 0; j < 3; ++j) {
        double sv = 0.0, sr = 0.0;
        for (int k = 0; k < 9; ++k) {
            sv = fma(a27[k * 3 + j], c_SA[9][k], sv);
            sr = fma(a27[k * 3 + j], c_GJ[9][k], sr);
        }
        vt[j] = sv;
        rt[j] = sr;
    }
    for (int j = 0; j < 3; ++j) {
        S[j] += s[j] + a27[24 + j] / 2;
        v[j] = (vt[j] + s[j] + a27[24 + j] / 2) * h;
        r[j] = (rt[j] + S[j]) * h * h;
    }
    for (int k = 0; k < 8; ++k)
        for (int j = 0; j < 3; ++j)
            a27[k * 3 + j] = a27[(k + 1) * 3 + j];
    double a8[3];
    f.prop(r, v, step + 4, a8);
    for (int j = 0; j < 3; ++j)
        a27[24 + j] = a8[j];
}

__global__ void finalize_unit_kernel(double h, double* r, double* v, const double* a27,
    const double* s, const double* S)
{
    for (int j = 0; j < 3; ++j) {
        v[j] = h * (v[j] + a27[24 + j] * c_SA[8][8] + s[j]);
        r[j] = h * h * (r[j] + a27[24 + j] * c_GJ[8][8] + S[j]);
    }
}

// ---- launchers ----
// Blocks of exactly the threads each SM needs (a multiple of 2, at least 32), so that one block per
// SM covers n on every SM: rounding the block up to whole warps left SMs idle (65,536 objects at
// two per thread: 147 of 148 SMs; the last warp of a block may be partial). When an SM needs more
// than max_block threads, its share is cut into equal blocks, one per wave, so that every wave
// fills every SM (the startup of 65,536 objects: two waves of 222-thread blocks instead of a full
// wave of 256-thread blocks and one on 108 SMs).
LaunchShape pick_shape(int64_t n, int max_block, int num_sms)
{
    LaunchShape ls;
    int64_t per_sm = (n + num_sms - 1) / num_sms;
    const int64_t waves = per_sm > max_block ? (per_sm + max_block - 1) / max_block : 1;
    int64_t block = (((per_sm + waves - 1) / waves + 1) / 2) * 2;
    if (block < 32)
        block = 32;
    if (block > max_block)
        block = max_block;
    ls.block = (int)block;
    ls.grid = (int)((n + block - 1) / block);
    return ls;
}

size_t max_smem_optin()
{
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess
        || cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return 0;
    return (size_t)v;
}

template <class K> static cudaError_t set_smem(K kernel, size_t bytes)
{
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <bool MIXED>
static cudaError_t launch_startup_split(const TableSrc& ts, const PropArgs& a, int S, int num_sms,
    cudaStream_t s)
{
    PropArgs b = a;
    b.split_owners = S;
    b.obj_lo = 0;
    b.obj_hi = -1;
    ForceGravity<MIXED> f {};
    f.gen_m = a.gen_m;
    f.prop_m = a.prop_m;
    cudaError_t e;
    const size_t xbytes = stage_offset(ts) + kSplitSmemBytes;
    if (xbytes <= max_smem_optin()) { // the exchange in shared memory beside the table
        if ((e = set_smem(startup_split_kernel<MIXED, kSplitSmem>, xbytes)) != cudaSuccess)
            return e;
        startup_split_kernel<MIXED, kSplitSmem><<<num_sms, kSplitBlock, xbytes, s>>>(f, ts, b);
    } else {
        const size_t bytes = table_smem_bytes(ts);
        if ((e = set_smem(startup_split_kernel<MIXED, kSplitGlobal>, bytes)) != cudaSuccess)
            return e;
        startup_split_kernel<MIXED, kSplitGlobal><<<num_sms, kSplitBlock, bytes, s>>>(f, ts, b);
    }
    return cudaGetLastError();
}

cudaError_t launch_startup(const TableSrc& ts, const PropArgs& a, int num_sms, cudaStream_t s)
{
    if (a.n <= 0)
        return cudaSuccess;
    // the sizes whose GJ8 steps take the split block start in it too (the exchange may use the
    // state arrays, so only when the state is there)
    if (a.kind == 0 && a.state && !(ts.mixed && (a.flags & kFlagMixedCompensated))) {
        const int S = split_owner_warps(a.n, num_sms, ts.L);
        if (S > 0)
            return ts.mixed ? launch_startup_split<true>(ts, a, S, num_sms, s)
                            : launch_startup_split<false>(ts, a, S, num_sms, s);
    }
    LaunchShape ls = pick_shape(a.n, 256, num_sms);
    if (a.kind == 0) {
        size_t smem = table_smem_bytes(ts);
        if (ts.mixed && (a.flags & kFlagMixedCompensated)) {
            ForceGravity<true, true> f {};
            f.gen_m = a.gen_m;
            f.prop_m = a.prop_m;
            cudaError_t e = set_smem(startup_kernel<ForceGravity<true, true>>, smem);
            if (e != cudaSuccess)
                return e;
            startup_kernel<<<ls.grid, ls.block, smem, s>>>(f, ts, a);
        } else if (ts.mixed) {
            ForceGravity<true> f {};
            f.gen_m = a.gen_m;
            f.prop_m = a.prop_m;
            cudaError_t e = set_smem(startup_kernel<ForceGravity<true>>, smem);
            if (e != cudaSuccess)
                return e;
            startup_kernel<<<ls.grid, ls.block, smem, s>>>(f, ts, a);
        } else {
            ForceGravity<false> f {};
            f.gen_m = a.gen_m;
            f.prop_m = a.prop_m;
            cudaError_t e = set_smem(startup_kernel<ForceGravity<false>>, smem);
            if (e != cudaSuccess)
                return e;
            startup_kernel<<<ls.grid, ls.block, smem, s>>>(f, ts, a);
        }
    } else {
        ForceAnalytic f { a.kind, a.h };
        startup_kernel<<<ls.grid, ls.block, 0, s>>>(f, ts, a);
    }
    return cudaGetLastError();
}

#ifndef GPOP_SPLIT_BLOCK
#define GPOP_SPLIT_BLOCK 1
#endif

// Owner warps of a split block for n objects at two per thread and one block per SM: the sets of
// 64 objects an SM carries, when that is 5 to 7 (a plain block of that many warps leaves one or
// two schedulers with a warp less); 0 otherwise. The split needs the FP32 tail (L > 8).
int split_owner_warps(int64_t n, int num_sms, int L)
{
    if (!GPOP_SPLIT_BLOCK || L <= kMixedSplit || num_sms <= 0)
        return 0;
    const int64_t per_sm = (n + num_sms - 1) / num_sms;
    const int64_t sets = (per_sm + 63) / 64;
    return sets >= 5 && sets < kSplitWarps ? (int)sets : 0;
}

template <class F, int K>
static cudaError_t launch_gj8_k(F f, const TableSrc& ts, const PropArgs& a, int num_sms,
    cudaStream_t s, int block_override, bool split = true)
{
    const int64_t cnt = (a.obj_hi < 0 ? a.n : a.obj_hi) - a.obj_lo; // objects of this launch
    if constexpr (K == 2 && F::kTable) {
        if constexpr (!F::kComp) {
            const int S = block_override > 0 || !split ? 0 : split_owner_warps(cnt, num_sms, ts.L);
            if (S > 0) {
                PropArgs b = a;
                b.split_owners = S;
                const size_t staged = stage_offset(ts) + (size_t)kStageDoubles * K * 8 * kSplitBlock;
                const size_t optin = max_smem_optin();
                cudaError_t e;
                if (stage_corrector<F>() && staged + kSplitSmemBytes <= optin) {
                    // mixed at 70x70: table, corrector state and exchange all in shared memory
                    const size_t bytes = staged + kSplitSmemBytes;
                    if ((e = set_smem(gj8_kernel<F, K, true, kSplitSmem>, bytes)) != cudaSuccess)
                        return e;
                    gj8_kernel<F, K, true, kSplitSmem><<<num_sms, kSplitBlock, bytes, s>>>(f, ts, b);
                } else if (stage_corrector<F>() && staged <= optin) {
                    // FP64 at 70x70: the exchange goes through the state arrays (L2)
                    if ((e = set_smem(gj8_kernel<F, K, true, kSplitGlobal>, staged)) != cudaSuccess)
                        return e;
                    gj8_kernel<F, K, true, kSplitGlobal><<<num_sms, kSplitBlock, staged, s>>>(f, ts, b);
                } else {
                    const size_t bytes = table_smem_bytes(ts);
                    if ((e = set_smem(gj8_kernel<F, K, false, kSplitGlobal>, bytes)) != cudaSuccess)
                        return e;
                    gj8_kernel<F, K, false, kSplitGlobal><<<num_sms, kSplitBlock, bytes, s>>>(f, ts, b);
                }
                return cudaGetLastError();
            }
        }
    }
    const int64_t threads = (cnt + K - 1) / K;
    LaunchShape ls = pick_shape(threads, K == 1 ? kOneObjectBlock : 256, num_sms);
    if (block_override > 0) {
        ls.block = block_override;
        ls.grid = (int)((threads + block_override - 1) / block_override);
    }
    if constexpr (F::kTable) {
        // the corrector state is parked in shared memory when it fits beside the table
        const size_t staged = stage_offset(ts) + (size_t)kStageDoubles * K * 8 * ls.block;
        if (stage_corrector<F>() && staged <= max_smem_optin()) {
            cudaError_t e = set_smem(gj8_kernel<F, K, true>, staged);
            if (e != cudaSuccess)
                return e;
            gj8_kernel<F, K, true><<<ls.grid, ls.block, staged, s>>>(f, ts, a);
        } else {
            const size_t smem = table_smem_bytes(ts);
            cudaError_t e = set_smem(gj8_kernel<F, K, false>, smem);
            if (e != cudaSuccess)
                return e;
            gj8_kernel<F, K, false><<<ls.grid, ls.block, smem, s>>>(f, ts, a);
        }
    } else {
        gj8_kernel<F, K, false><<<ls.grid, ls.block, 0, s>>>(f, ts, a);
    }
    return cudaGetLastError();
}

template <class F>
static cudaError_t launch_gj8_f(F f, const TableSrc& ts, const PropArgs& a, int num_sms,
    cudaStream_t s, int block_override, int walk)
{
    if (walk == kWalkTwoObjects || walk == kWalkTwoPlain)
        return launch_gj8_k<F, 2>(f, ts, a, num_sms, s, block_override, walk == kWalkTwoObjects);
    return launch_gj8_k<F, 1>(f, ts, a, num_sms, s, block_override);
}

#ifndef GPOP_LANES_BLOCK_MID
#define GPOP_LANES_BLOCK_MID 384
#endif
constexpr int kLanesBlockMid = GPOP_LANES_BLOCK_MID; // blocks up to this size take the MAXT = 384 kernel

// The most lanes that keep every object in one wave of blocks of at most kLanesBlockMid threads,
// so that the lane kernel runs with the registers of its 384-thread variant: fewer lanes with
// more registers beat more lanes with 128 (B200, 70x70, FP64 / mixed M object-steps/s: 2,048
// objects 19.0 / 26.1 against 16.2 / 21.2 with 512-thread blocks; 4,096: 25.6 / 36.1 against
// 21.8 / 33.6; 9,472: 31.6 / 49.4 against 29.6 / 46.5; 16,000: 42.2 / 63.7 against 30.2 / 53.1).
int lanes_per_object(int64_t n, int num_sms)
{
    int P = 1;
    while (P < 32 && n * 2 * P <= (int64_t)num_sms * kLanesBlockMid)
        P *= 2;
    return P;
}

// Two objects per lane group (K = 2) share every table entry a lane loads and give each lane two
// independent recursions. Measured on B200 at 70x70 (LEO objects, M object-steps/s, the corrector
// constants staged per group), lanes per group in brackets, against the walk taken before (one
// object per lane group; in mixed precision above 128 objects per SM two objects per thread):
//   FP64   1,200: 15.6 (32) / 11.4     4,096: 38.4 (16) / 28.7    9,472: 53.4 (8) / 33.9
//         14,000: 48.7 (8) / 34.3     18,944: 60.1 (4) / 51.7    20,000: 53.3 (4) / 46.7
//         22,000: 52.6 (4) / 48.0     outside: 1,024: 17.0 (32) / 17.4; 24,000: 50.6 (8) / 52.0
//   mixed  3,000: 35.7 (16) / 33.8     4,096: 47.9 (16) / 37.5    6,000: 47.7 (8) / 42.9
//          8,000: 62.4 (8) / 44.3      9,472: 69.5 (8) / 50.0    12,000: 59.4 (4) / 50.9
//         18,944: 88.3 (4) / 73.0     20,000: 73.5 (4) / 68.4
//                                     outside: 2,048: 29.5 (16) / 29.0; 24,000: 76.0 (2) / 81.8
// P is the most lanes whose groups fit one wave of 8 warps per SM, doubled once, up to 8 lanes,
// when the groups still fit one and a half waves (FP64) or 1.2 waves (mixed); the groups past one
// wave run in a second launch with more lanes. Before the staging, FP64 12,000 objects ran at 41.6
// with 8 lanes against 38.7 with 4, and 6,000 at 34.4 with 8 against 31.4 with 16; staged, mixed
// 12,000 runs at 59.4 with 4 against 54.9 with 8.
int lane_pair_lanes(int64_t n, int num_sms, bool fp64_gravity)
{
    const int64_t sms = num_sms;
    if (n <= 0 || sms <= 0 || n < sms * (fp64_gravity ? 8 : 16) || n > sms * 150)
        return 0;
    const int64_t wave = sms * 512; // objects of one wave of 8 warps per SM at one lane per group
    int P = 2;
    while (P < 32 && n * 2 * P <= wave)
        P *= 2;
    if (2 * P <= 8 && n * 2 * P * 10 <= wave * (fp64_gravity ? 15 : 12))
        P *= 2;
    return P;
}

// Default walk (measured on B200 at 70x70, LEO objects, mixed / FP64 M object-steps/s):
// - up to 128 objects per SM, lanes (P from lanes_per_object, blocks of at most 384 threads):
//   18,900 objects 74.7 / 49.4 against 65.0 / 47.0 with two lanes per pair of objects; 9,472:
//   49.4 / 31.6 against 34.0 / 20.8 with two objects per thread;
// - FP64 up to 192 per SM keeps two lanes per object (20,000: 42.0 against 39.1 with one object
//   per thread; 24,000: 50.0 against 46.4; 28,000: 57.7 against 54.1);
// - above, two objects per thread (20,000 mixed: 64.5 against 63.7 with two lanes per object;
//   37,000: 120 / 64 against 104 / 62 with two lanes per pair), except that FP64 takes one
//   object per thread up to 256 per SM, where two objects per thread leave at most one warp
//   per scheduler (30,000: 57.2 against 52.7; 37,000: 65.1 against 64.5).
// One or two objects per thread when no lane-layout table is at hand.
int default_walk(int64_t n, int num_sms, bool lanes, bool fp64_gravity)
{
    if (lanes && lane_pair_lanes(n, num_sms, fp64_gravity) > 0)
        return kWalkLanesTwo;
    if (lanes && (n <= (int64_t)num_sms * 128 || (fp64_gravity && 2 * n <= (int64_t)num_sms * kLanesBlockMid)))
        return kWalkLanes;
    if (n >= (int64_t)num_sms * 128)
        return fp64_gravity && n <= (int64_t)num_sms * 256 ? kWalkOneObject : kWalkTwoObjects;
    return kWalkOneObject;
}

// The lane kernel over objects [lo, hi) (of a.n) with P lanes per group of K objects: whole lane
// groups per block (a multiple of P, at least a warp), sized so that every SM gets a block
// (rounding up to whole warps left SMs idle: 20,000 objects with two lanes ran on 139 of 148 SMs
// with 288-thread blocks, on 148 with 272).
static cudaError_t launch_lanes_range(const TableSrc& lt, const PropArgs& a0, int K, int P, int64_t lo,
    int64_t hi, int num_sms, cudaStream_t s)
{
    PropArgs a = a0;
    a.obj_lo = lo;
    a.obj_hi = hi;
    const int64_t groups = (hi - lo + K - 1) / K;
    const int64_t threads = groups * P;
    const int64_t per_sm = (threads + num_sms - 1) / num_sms; // spread over every SM
    const int cap = K == 1 ? 512 : 256;
    const int block = (int)std::min<int64_t>(cap, std::max<int64_t>(32, ((per_sm + P - 1) / P) * P));
    const unsigned grid = (unsigned)((threads + block - 1) / block);
    const size_t smem = table_smem_bytes(lt);
    // two objects per lane group: the corrector's constants parked in shared memory, one copy per
    // group (gj8_lanes_kernel STAGE), when they fit beside the table
#ifndef GPOP_STAGE_LANES
#define GPOP_STAGE_LANES 1
#endif
    const size_t staged = GPOP_STAGE_LANES ? stage_offset(lt) + (size_t)kStageDoubles * K * 8 * (block / P)
                                           : (size_t)1 << 40;
    cudaError_t e;
    if (lt.mixed) {
        if (K == 1 && block <= kLanesBlockMid) {
            if ((e = set_smem(gj8_lanes_kernel<true, 1, kLanesBlockMid>, smem)) != cudaSuccess)
                return e;
            gj8_lanes_kernel<true, 1, kLanesBlockMid><<<grid, block, smem, s>>>(lt, a, P);
        } else if (K == 1) {
            if ((e = set_smem(gj8_lanes_kernel<true, 1>, smem)) != cudaSuccess)
                return e;
            gj8_lanes_kernel<true, 1><<<grid, block, smem, s>>>(lt, a, P);
        } else {
            if (staged <= max_smem_optin()) {
                if ((e = set_smem(gj8_lanes_kernel<true, 2, 256, true>, staged)) != cudaSuccess)
                    return e;
                gj8_lanes_kernel<true, 2, 256, true><<<grid, block, staged, s>>>(lt, a, P);
            } else {
                if ((e = set_smem(gj8_lanes_kernel<true, 2>, smem)) != cudaSuccess)
                    return e;
                gj8_lanes_kernel<true, 2><<<grid, block, smem, s>>>(lt, a, P);
            }
        }
    } else {
        if (K == 1 && block <= kLanesBlockMid) {
            if ((e = set_smem(gj8_lanes_kernel<false, 1, kLanesBlockMid>, smem)) != cudaSuccess)
                return e;
            gj8_lanes_kernel<false, 1, kLanesBlockMid><<<grid, block, smem, s>>>(lt, a, P);
        } else if (K == 1) {
            if ((e = set_smem(gj8_lanes_kernel<false, 1>, smem)) != cudaSuccess)
                return e;
            gj8_lanes_kernel<false, 1><<<grid, block, smem, s>>>(lt, a, P);
        } else {
            if (staged <= max_smem_optin()) {
                if ((e = set_smem(gj8_lanes_kernel<false, 2, 256, true>, staged)) != cudaSuccess)
                    return e;
                gj8_lanes_kernel<false, 2, 256, true><<<grid, block, staged, s>>>(lt, a, P);
            } else {
                if ((e = set_smem(gj8_lanes_kernel<false, 2>, smem)) != cudaSuccess)
                    return e;
                gj8_lanes_kernel<false, 2><<<grid, block, smem, s>>>(lt, a, P);
            }
        }
    }
    return cudaGetLastError();
}

cudaError_t launch_gj8(const TableSrc& ts, const PropArgs& a, int num_sms, cudaStream_t s,
    int block_override, int walk, const TableSrc* lane_ts)
{
    // objects [lo, hi) of the n the state holds
    const int64_t lo = a.obj_lo, hi = a.obj_hi < 0 ? a.n : a.obj_hi, cnt = hi - lo;
    if (cnt <= 0 || lo < 0 || hi > a.n || a.step_end <= a.step_begin)
        return cudaSuccess;
    const bool forced = walk > 0;
    const bool comp = a.kind == 0 && ts.mixed && (a.flags & kFlagMixedCompensated);
    if (walk <= 0)
        walk = default_walk(cnt, num_sms, lane_ts && a.kind == 0 && !comp, a.kind == 0 && !ts.mixed);
    if (comp) { // compensated sums: the plain walks only
        ForceGravity<true, true> f {};
        f.gen_m = a.gen_m;
        f.prop_m = a.prop_m;
        return launch_gj8_f(f, ts, a, num_sms, s, block_override,
            walk == kWalkTwoObjects || walk == kWalkTwoPlain ? walk : kWalkOneObject);
    }
    if (walk == kWalkTwoObjects && a.kind == 0 && block_override <= 0) {
        // More objects than one wave of 8 warps per SM holds at two per thread: whole waves of
        // 256-thread blocks, then the rest with the walk its own size takes (100,000 objects ran as
        // two waves of 169-thread blocks, 6 warps per SM spread 2-2-1-1).
        const int64_t wave = (int64_t)num_sms * 512;
        if (cnt > wave) {
            const int64_t full = cnt / wave * wave;
            PropArgs b = a;
            b.obj_hi = lo + full;
            cudaError_t e = launch_gj8(ts, b, num_sms, s, block_override, kWalkTwoPlain, lane_ts);
            if (e != cudaSuccess || full == cnt)
                return e;
            PropArgs c = a;
            c.obj_lo = lo + full;
            return launch_gj8(ts, c, num_sms, s, block_override, forced ? walk : 0, lane_ts);
        }
    }
    if ((walk == kWalkLanes || walk == kWalkLanesTwo) && a.kind == 0 && lane_ts) {
        const int K = walk == kWalkLanesTwo ? 2 : 1;
        if (K == 2) {
            // the groups of one wave of 8 warps per SM, then the rest with more lanes each
            const int pp = lane_pair_lanes(cnt, num_sms, !lane_ts->mixed);
            const int P = pp > 0 ? pp : 2;
            const int64_t main_objects = std::min<int64_t>(cnt, (int64_t)num_sms * 256 / P * 2);
            cudaError_t e = launch_lanes_range(*lane_ts, a, 2, P, lo, lo + main_objects, num_sms, s);
            if (e != cudaSuccess || main_objects >= cnt)
                return e;
            const int64_t rest_groups = (cnt - main_objects + 1) / 2;
            int P2 = 1; // the fewest lanes that give the rest over half a wave of threads (<= 32)
            while (P2 < 32 && rest_groups * 2 * P2 <= (int64_t)num_sms * 256)
                P2 *= 2;
            return launch_lanes_range(*lane_ts, a, 2, P2, lo + main_objects, hi, num_sms, s);
        }
        const int P = lanes_per_object(cnt, num_sms);
        // A block of 8 warps and a bit leaves three warps on one scheduler of every SM: the
        // objects of 8 warps per SM run in one launch, the rest, with more lanes each, in a second
        // one (20,000 objects, FP64: 4.69e7 object-steps/s against 4.38e7 in one).
        const int64_t per_sm = ((cnt * P + num_sms - 1) / num_sms + P - 1) / P * P;
        const int64_t main_objects = (int64_t)num_sms * 256 / P;
        if (per_sm > 256 && per_sm <= 288 && main_objects < cnt) {
            cudaError_t e = launch_lanes_range(*lane_ts, a, 1, P, lo, lo + main_objects, num_sms, s);
            if (e != cudaSuccess)
                return e;
            const int P2 = lanes_per_object(cnt - main_objects, num_sms);
            return launch_lanes_range(*lane_ts, a, 1, P2, lo + main_objects, hi, num_sms, s);
        }
        return launch_lanes_range(*lane_ts, a, K, P, lo, hi, num_sms, s);
    }
    if (walk == kWalkLanes || walk == kWalkLanesTwo)
        walk = kWalkOneObject;
    if (a.kind == 0) {
        if (ts.mixed) {
            ForceGravity<true> f {};
            f.gen_m = a.gen_m;
            f.prop_m = a.prop_m;
            return launch_gj8_f(f, ts, a, num_sms, s, block_override, walk);
        }
        ForceGravity<false> f {};
        f.gen_m = a.gen_m;
        f.prop_m = a.prop_m;
        return launch_gj8_f(f, ts, a, num_sms, s, block_override, walk);
    }
    ForceAnalytic f { a.kind, a.h };
    return launch_gj8_f(f, ts, a, num_sms, s, block_override, walk);
}

cudaError_t launch_gravity(const TableSrc& ts, int64_t n, const double* r, const double* m9,
    double* a, unsigned* err, int num_sms, cudaStream_t s)
{
    if (n <= 0)
        return cudaSuccess;
    LaunchShape ls = pick_shape(n, 512, num_sms);
    size_t smem = table_smem_bytes(ts);
    if (ts.mixed) {
        cudaError_t e = set_smem(gravity_kernel<true>, smem);
        if (e != cudaSuccess)
            return e;
        gravity_kernel<true><<<ls.grid, ls.block, smem, s>>>(ts, n, r, m9, a, err);
    } else {
        cudaError_t e = set_smem(gravity_kernel<false>, smem);
        if (e != cudaSuccess)
            return e;
        gravity_kernel<false><<<ls.grid, ls.block, smem, s>>>(ts, n, r, m9, a, err);
    }
    return cudaGetLastError();
}

cudaError_t launch_corrector_unit(int kind, double h, int op, double* r27, double* v27, double* a27,
    double* s27, double* S27, cudaStream_t s)
{
    corrector_unit_kernel<<<1, 1, 0, s>>>(ForceAnalytic { kind, h }, op, r27, v27, a27, s27, S27);
    return cudaGetLastError();
}

cudaError_t launch_predict_unit(int kind, double h, int step, double* r3, double* v3, double* a27,
    double* s3, double* S3, cudaStream_t s)
{
    predict_unit_kernel<<<1, 1, 0, s>>>(ForceAnalytic { kind, h }, step, r3, v3, a27, s3, S3);
    return cudaGetLastError();
}

cudaError_t launch_finalize_unit(double h, double* r3, double* v3, const double* a27,
    const double* s3, const double* S3, cudaStream_t s)
{
    finalize_unit_kernel<<<1, 1, 0, s>>>(h, r3, v3, a27, s3, S3);
    return cudaGetLastError();
}

} // namespace gpop
