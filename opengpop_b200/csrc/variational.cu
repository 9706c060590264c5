// variational.cu -- forward variational equations (6x6 STM), the adjoint (reverse sweep) of the
// GJ8 propagation, and the closest approach of listed pairs with miss-distance seeds.
//
// Every object (STM) or adjoint unit runs on kVarLanes = 8 lanes of a warp. The lanes split the
// gravity columns (lanes.cuh) and share the acceleration and its Jacobian; lane d < 6 carries the
// tangent of initial-state direction d. The integrator is the same discrete map as the forward
// propagation (startup: integrator.cuh; GJ8 step: gpu_propagator.cu:28-119 as in gj8_kernel),
// so the tangents and adjoints are the derivatives of that map with one simplification: the
// Jacobian of a GJ8 step's corrector passes is taken once, at the step's last evaluation point
// (the corrector converges, so the passes' iterates differ by far less than the truncation error);
// the startup is differentiated exactly. Forward tangents and the reverse sweep make the same
// choice, so they are exact transposes of each other.
//
// Adjoint of one GJ8 step n (K = number of corrector passes, iterates r(0..K-1), a(i) = f(r(i))):
//   S' = S + s + h8/2,  r(0) = h^2 (sum_c GJ[9][c] h_c + S'),  s1 = sum_c SA[8][c] h_(c+1),
//   s2 = sum_c GJ[8][c] h_(c+1),  r(i+1) = h^2 (s2 + GJ[8][8] a(i) + S'),
//   s_n = s + (a(K-1) + h8)/2,  v_n = h (s1 + SA[8][8] a(K-1) + s_n),  history <- (h_1..h_8, a(K-1)).
// The reverse pass below applies the transposes of these maps in the opposite order, with J^T at
// the last evaluation point r(K-1), recomputed from the checkpoint of the step's 64-step segment.
#include "common.cuh"
#include "gj8_tables.cuh"
#include "gravity.cuh"
#include "hermite.cuh"
#include "integrator.cuh"
#include "lanes.cuh"
#include "tangent.cuh"
#include "variational.cuh"

namespace gpop {

namespace {

// Tangent force: a(r) and J(r) dr, epoch tables as in ForceGravity (force_model.cu:59-109).
struct LaneForceTan {
    GravSmem g;
    int l, P;
    unsigned mask;
    const double* gen_m;
    const double* prop_m;
    __device__ __forceinline__ void eval(const double* M, const Tan* r, Tan* a) const
    {
        const double rv[3] = { r[0].v, r[1].v, r[2].v };
        double av[3], J[3][3];
        gravity_jac_gcrs_lanes(g, l, P, M, rv, av, J, mask);
#pragma unroll
        for (int i = 0; i < 3; ++i)
            a[i] = Tan(av[i], J[i][0] * r[0].d + J[i][1] * r[1].d + J[i][2] * r[2].d);
    }
    __device__ __forceinline__ void prop(const Tan* r, const Tan*, int idx, Tan* a) const
    {
        eval(prop_m + (size_t)idx * 9, r, a);
    }
    __device__ __forceinline__ void gen(const Tan* r, const Tan*, int step, int k, Tan* a) const
    {
        const int s = step > 0 ? step - 1 : step;
        eval(gen_m + (size_t)((s + 4) * 10 + k) * 9, r, a);
    }
};

// One GJ8 step (predict, then ncorr evaluate-correct passes) on a history held in logical order
// (hist[8] newest). eval(r, a, pass) evaluates the force at r for corrector pass `pass`.
template <class T, class Eval>
__device__ __forceinline__ void gj8_step(const Eval& eval, double h, int ncorr, T (&hist)[9][3],
    T (&s)[3], T (&S)[3], T (&r)[3], T (&v)[3])
{
    T s1[3], s2[3], prev[3], a7[3], a8[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) { // Predictor::Predict (dev_functions.cu:20-50)
        T vt = 0.0, rt = 0.0;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            vt = fma(hist[c][j], c_SA[9][c], vt);
            rt = fma(hist[c][j], c_GJ[9][c], rt);
        }
        S[j] += s[j] + hist[8][j] / 2;
        v[j] = (vt + s[j] + hist[8][j] / 2) * h;
        r[j] = (rt + S[j]) * h * h;
        T c1 = 0.0, c2 = 0.0;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            c1 = fma(hist[c + 1][j], c_SA[8][c], c1);
            c2 = fma(hist[c + 1][j], c_GJ[8][c], c2);
        }
        s1[j] = c1;
        s2[j] = c2;
        prev[j] = s[j];
        a7[j] = hist[8][j];
        a8[j] = 0.0;
    }
    for (int it = 0; it < ncorr; ++it) { // GpuPropagator::Correct (gpu_propagator.cu:61-119)
        eval(r, a8, it);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            s[j] = prev[j] + (a8[j] + a7[j]) / 2;
            v[j] = h * (s1[j] + a8[j] * c_SA[8][8] + s[j]);
            r[j] = h * h * (s2[j] + a8[j] * c_GJ[8][8] + S[j]);
        }
    }
#pragma unroll
    for (int c = 0; c < 8; ++c)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            hist[c][j] = hist[c + 1][j];
#pragma unroll
    for (int j = 0; j < 3; ++j)
        hist[8][j] = a8[j];
}

__device__ __forceinline__ bool stage_table64(uint8_t* smem, const TableSrc& ts, unsigned* err, GravSmem& g)
{
    return bind_lane_table(smem, ts, err, g); // FP64 lane-layout table
}

} // namespace

// ---- forward variational equations ----
__global__ void __launch_bounds__(256, 1) stm_kernel(TableSrc ts, VarArgs a)
{
    extern __shared__ __align__(128) uint8_t smem[];
    GravSmem g;
    if (!stage_table64(smem, ts, a.err, g))
        return;
    const int P = kVarLanes;
    const int64_t gid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / P;
    const int l = (int)(threadIdx.x % P);
    if (gid >= a.n)
        return; // the lanes of a group share gid; shuffles stay inside the group
    const int64_t o = gid;
    const unsigned mask = 0xffu << (threadIdx.x & 24);
    const int dir = l < 6 ? l : -1;
    LaneForceTan f { g, l, P, mask, a.gen_m, a.prop_m };
    Tan r0[3], v0[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        r0[j] = Tan(a.r0[o * 3 + j], dir == j ? 1.0 : 0.0);
        v0[j] = Tan(a.v0[o * 3 + j], dir == 3 + j ? 1.0 : 0.0);
    }
    // primal state (every lane) and the tangent of this lane's direction
    double hist[9][3], s[3], S[3], r[3], v[3], dh[9][3], ds[3], dS[3], dr[3], dv[3];
    {
        StartupMatsT<Tan> m; // the startup: exact tangents, Jacobian at every evaluation
        run_startup(f, a.h, a.ncorr, r0, v0, m);
        const int rep = a.steps < 4 ? a.steps : 4; // steps 1..4 replay the startup columns
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            for (int c = 0; c < 9; ++c) {
                hist[c][j] = m.a[c][j].v;
                dh[c][j] = m.a[c][j].d;
            }
            s[j] = m.s[8][j].v;
            ds[j] = m.s[8][j].d;
            S[j] = m.S[8][j].v;
            dS[j] = m.S[8][j].d;
            r[j] = m.r[4 + rep][j].v;
            dr[j] = m.r[4 + rep][j].d;
            v[j] = m.v[4 + rep][j].v;
            dv[j] = m.v[4 + rep][j].d;
        }
    }
    for (int step = 5; step <= a.steps; ++step) {
        const double* M = a.prop_m + (size_t)(step + 4) * 9;
        // primal passes; the Jacobian at the last evaluation point serves every pass of the
        // tangent step (as in the reverse sweep)
        double rl[3];
        auto evalp = [&](const double* rr, double* aa, int it) {
            if (it == a.ncorr - 1)
                for (int j = 0; j < 3; ++j)
                    rl[j] = rr[j];
            gravity_gcrs_lanes<false>(g, l, P, M, rr, aa, mask);
        };
        gj8_step<double>(evalp, a.h, a.ncorr, hist, s, S, r, v);
        double av[3], J[3][3];
        gravity_jac_gcrs_lanes(g, l, P, M, rl, av, J, mask);
        auto evalt = [&](const double* rr, double* aa, int) {
#pragma unroll
            for (int i = 0; i < 3; ++i)
                aa[i] = J[i][0] * rr[0] + J[i][1] * rr[1] + J[i][2] * rr[2];
        };
        gj8_step<double>(evalt, a.h, a.ncorr, dh, ds, dS, dr, dv);
    }
    if (l == 0 && a.r_out)
        for (int j = 0; j < 3; ++j) {
            a.r_out[o * 3 + j] = r[j];
            a.v_out[o * 3 + j] = v[j];
        }
    if (dir >= 0)
        for (int i = 0; i < 3; ++i) {
            a.phi[(o * 6 + i) * 6 + dir] = dr[i];
            a.phi[(o * 6 + 3 + i) * 6 + dir] = dv[i];
        }
}

// ---- adjoint ----
namespace {

// Reverse of one GJ8 step (see the header comment). hb: history adjoints in logical order after
// the step on entry, before it on exit; sb, Sb: adjoints of s and S likewise.
// iter: the step's last evaluation point r(K-1) (3 values, stride apart); its Jacobian stands for
// every corrector pass (the corrector converges: the iterates differ by far less than the step's
// truncation error, and the forward tangents make the same choice).
__device__ __forceinline__ void gj8_reverse_step(const GravSmem& g, int l, int P, unsigned mask,
    const double* M, double h, int ncorr, const double* iter, int64_t stride, const double* seed,
    double (&hb)[9][3], double (&sb)[3], double (&Sb)[3])
{
    const double h2 = h * h;
    double abar[3], s1b[3], s2b[3], Spb[3], prevb[3], a7b[3];
#pragma unroll
    for (int j = 0; j < 3; ++j)
        abar[j] = hb[8][j] + (seed ? seed[6 + j] : 0.0);
#pragma unroll
    for (int c = 8; c >= 1; --c)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            hb[c][j] = hb[c - 1][j];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        hb[0][j] = 0.0;
        const double rb = seed ? seed[j] : 0.0, vb = seed ? seed[3 + j] : 0.0;
        const double sK = sb[j] + h * vb; // s_n feeds v_n = h (s1 + SA88 a + s_n)
        s1b[j] = h * vb;
        abar[j] += h * c_SA[8][8] * vb + sK / 2;
        prevb[j] = sK;
        a7b[j] = sK / 2;
        s2b[j] = h2 * rb;
        abar[j] += h2 * c_GJ[8][8] * rb;
        Spb[j] = Sb[j] + h2 * rb;
    }
    double J[3][3];
    {
        double ri[3], av[3];
#pragma unroll
        for (int j = 0; j < 3; ++j)
            ri[j] = iter[(int64_t)j * stride];
        gravity_jac_gcrs_lanes(g, l, P, M, ri, av, J, mask);
    }
    for (int it = ncorr - 1; it >= 0; --it) {
        double rb[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
            rb[k] = J[0][k] * abar[0] + J[1][k] * abar[1] + J[2][k] * abar[2];
        if (it >= 1) {
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                s2b[j] += h2 * rb[j];
                Spb[j] += h2 * rb[j];
                abar[j] = h2 * c_GJ[8][8] * rb[j];
            }
        } else {
#pragma unroll
            for (int j = 0; j < 3; ++j) {
#pragma unroll
                for (int c = 0; c < 9; ++c)
                    hb[c][j] += h2 * c_GJ[9][c] * rb[j];
                Spb[j] += h2 * rb[j];
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
#pragma unroll
        for (int c = 0; c < 8; ++c)
            hb[c + 1][j] += c_SA[8][c] * s1b[j] + c_GJ[8][c] * s2b[j];
        hb[8][j] += a7b[j] + Spb[j] / 2; // a7 = h8, and S' = S + s + h8/2
        Sb[j] = Spb[j];
        sb[j] = prevb[j] + Spb[j];
    }
}

} // namespace

__global__ void __launch_bounds__(256, 1) adjoint_kernel(TableSrc ts, AdjArgs a)
{
    extern __shared__ __align__(128) uint8_t smem[];
    GravSmem g;
    if (!stage_table64(smem, ts, a.err, g))
        return;
    const int P = kVarLanes;
    const int64_t gid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / P;
    const int l = (int)(threadIdx.x % P);
    if (gid >= a.n_units)
        return; // groups run independently: every shuffle and warp sync names the group only
    const int64_t u = gid;
    const unsigned mask = 0xffu << (threadIdx.x & 24);
    const int64_t o = a.unit_obj[u];
    const int64_t n = a.n_obj, U = a.n_units;
    const int N = a.steps, K = a.ncorr;
    const int k0 = a.seed_step0[u];
    const int kend = k0 + 2 < N ? k0 + 2 : N;
    const double* seeds = a.seeds + u * 27;
    double hb[9][3], sb[3], Sb[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        for (int c = 0; c < 9; ++c)
            hb[c][j] = 0.0;
        sb[j] = Sb[j] = 0.0;
    }
    if (kend >= 5) {
        for (int seg = (kend - 1) / kCheckpointSteps; seg >= 0; --seg) {
            const int lo = seg == 0 ? 5 : seg * kCheckpointSteps + 1;
            const int hi = (seg + 1) * kCheckpointSteps < kend ? (seg + 1) * kCheckpointSteps : kend;
            if (lo > hi)
                continue;
            // recompute the segment from its checkpoint, keeping every corrector iterate
            const double* ck = a.ckpt + (size_t)seg * kCheckpointArrays * n;
            double hist[9][3], s[3], S[3], r[3], v[3];
            const int ring0 = (lo - 5) % 9;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                s[j] = ck[(0 + j) * n + o]; // arrays kSs, kSb, kHist relative to kSs
                S[j] = ck[(3 + j) * n + o];
                for (int c = 0; c < 9; ++c) {
                    const int slot = (ring0 + c) % 9;
                    hist[c][j] = ck[(6 + slot * 3 + j) * n + o];
                }
            }
            for (int step = lo; step <= hi; ++step) {
                const double* M = a.prop_m + (size_t)(step + 4) * 9;
                double* it_base = a.scratch + (size_t)(step - lo) * 3 * U + u;
                auto eval = [&](const double* rr, double* aa, int it) {
                    if (l == 0 && it == K - 1)
#pragma unroll
                        for (int j = 0; j < 3; ++j)
                            it_base[(int64_t)j * U] = rr[j];
                    gravity_gcrs_lanes<false>(g, l, P, M, rr, aa, mask);
                };
                gj8_step<double>(eval, a.h, K, hist, s, S, r, v);
            }
            __syncwarp(mask);
            for (int step = hi; step >= lo; --step) {
                const double* M = a.prop_m + (size_t)(step + 4) * 9;
                const double* it_base = a.scratch + (size_t)(step - lo) * 3 * U + u;
                const int node = step - k0;
                const double* seed = (node >= 0 && node < 3) ? seeds + node * 9 : nullptr;
                gj8_reverse_step(g, l, P, mask, M, a.h, K, it_base, U, seed, hb, sb, Sb);
            }
            __syncwarp(mask); // the next segment overwrites the iterates
        }
    }
    // startup: forward tangents of its outputs along direction l, dotted with their adjoints
    const int dir = l < 6 ? l : -1;
    LaneForceTan ft { g, l, P, mask, a.gen_m, a.prop_m };
    Tan r0[3], v0[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        r0[j] = Tan(a.r0[o * 3 + j], dir == j ? 1.0 : 0.0);
        v0[j] = Tan(a.v0[o * 3 + j], dir == 3 + j ? 1.0 : 0.0);
    }
    StartupMatsT<Tan> m;
    run_startup(ft, a.h, K, r0, v0, m);
    double gsum = 0.0; // history, s and S adjoints are those of the step-5 inputs (zero if none)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        for (int c = 0; c < 9; ++c)
            gsum += hb[c][j] * m.a[c][j].d;
        gsum += sb[j] * m.s[8][j].d + Sb[j] * m.S[8][j].d;
    }
    const bool fix_q3 = (a.flags & 2u) != 0;
    for (int node = 0; node < 3; ++node) { // seeds on the replayed steps 1..4
        const int step = k0 + node;
        if (step < 1 || step > 4 || step > N)
            continue;
        const double* sd = seeds + node * 9;
        for (int j = 0; j < 3; ++j) {
            gsum += sd[j] * m.r[4 + step][j].d + sd[3 + j] * m.v[4 + step][j].d;
            gsum += sd[6 + j] * (fix_q3 ? m.a[4 + step][j].d : m.a[8][j].d);
        }
    }
    if (dir >= 0)
        a.grad[u * 6 + dir] = gsum;
}

// ---- closest approach of listed pairs, with the seeds of d(miss) ----
__global__ void __launch_bounds__(128) pair_approach_kernel(PairArgs a)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n_pairs)
        return;
    const int64_t oa = a.pairs[2 * p], ob = a.pairs[2 * p + 1], n = a.n_obj;
    const int N = a.steps;
    const double h = a.h;
    // running minimum of the sampled distance (UpdateClosestApproachKernel, device.cu:56-91)
    double best = __longlong_as_double(0x7ff0000000000000ll); // +inf
    int bk = -1;
    for (int k = 0; k < N; ++k) {
        double d2 = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double d = a.traj_r[((int64_t)k * 3 + c) * n + oa] - a.traj_r[((int64_t)k * 3 + c) * n + ob];
            d2 += d * d;
        }
        if (d2 < best) {
            best = d2;
            bk = k;
        }
    }
    double seed[27];
#pragma unroll
    for (int i = 0; i < 27; ++i)
        seed[i] = 0.0;
    double tca, miss;
    int step0;
    if (bk <= 0 || bk >= N - 1) {
        // first or last sample: not refined (device.cu:100-110); miss = the sampled distance
        const int k = bk < 0 ? 0 : bk;
        tca = k == 0 ? 0.0 : (double)N * h;
        double D[3], d2 = 0.0;
        for (int c = 0; c < 3; ++c) {
            D[c] = a.traj_r[((int64_t)k * 3 + c) * n + oa] - a.traj_r[((int64_t)k * 3 + c) * n + ob];
            d2 += D[c] * D[c];
        }
        miss = sqrt(d2);
        step0 = k + 1;
        if (miss > 0.0)
            for (int c = 0; c < 3; ++c)
                seed[c] = D[c] / miss;
    } else {
        // Hermite through trajectory indices bk-1, bk, bk+1 (steps bk .. bk+2), secant TCA
        // (CalculateClosestApproachesKernel, device.cu:111-173)
        Pair6 H;
        H.dt = h;
        for (int c = 0; c < 3; ++c) {
            double qa[9], qb[9];
            for (int node = 0; node < 3; ++node) {
                const int64_t base = ((int64_t)(bk - 1 + node) * 3 + c) * n;
                qa[node * 3 + 0] = a.traj_r[base + oa];
                qa[node * 3 + 1] = a.traj_v[base + oa];
                qa[node * 3 + 2] = a.traj_a[base + oa];
                qb[node * 3 + 0] = a.traj_r[base + ob];
                qb[node * 3 + 1] = a.traj_v[base + ob];
                qb[node * 3 + 2] = a.traj_a[base + ob];
            }
            herm_build(H.A[c], qa[0], qa[1], qa[2], qa[3], qa[4], qa[5], qa[6], qa[7], qa[8], h);
            herm_build(H.B[c], qb[0], qb[1], qb[2], qb[3], qb[4], qb[5], qb[6], qb[7], qb[8], h);
        }
        const double t = find_root(H, 0.0, h);
        tca = t + (double)bk * h;
        double D[3], D1[3], D2[3], d2 = 0.0, f = 0.0, ft = 0.0;
        for (int c = 0; c < 3; ++c) {
            D[c] = herm_eval(H.A[c], h, t) - herm_eval(H.B[c], h, t);
            D1[c] = herm_deriv(H.A[c], h, t) - herm_deriv(H.B[c], h, t);
            D2[c] = herm_deriv2(H.A[c], h, t) - herm_deriv2(H.B[c], h, t);
            d2 += D[c] * D[c];
            f += D[c] * D1[c];
            ft += D1[c] * D1[c] + D[c] * D2[c];
        }
        miss = sqrt(d2);
        step0 = bk;
        if (miss > 0.0) {
            // miss = |D(t*)|, f(t*) = D . D' = 0 defines t*: d miss = (D . dD + f dt*) / miss,
            // dt* = -(D' . dD + D . dD') / f_t (implicit function at the computed root). The
            // interpolant is linear in the node data, so dD = sum_i beta_i(t*) d(data_i).
            for (int i = 0; i < 9; ++i) {
                Herm B;
                double e[9];
                for (int k = 0; k < 9; ++k)
                    e[k] = k == i ? 1.0 : 0.0;
                herm_build(B, e[0], e[1], e[2], e[3], e[4], e[5], e[6], e[7], e[8], h);
                const double beta = herm_eval(B, h, t), dbeta = herm_deriv(B, h, t);
                for (int c = 0; c < 3; ++c) {
                    const double df = beta * D1[c] + D[c] * dbeta;
                    const double dt = ft != 0.0 ? -df / ft : 0.0;
                    // node i/3, kind i%3 (r, v, a) -> seed layout [node][r3 | v3 | a3]
                    seed[(i / 3) * 9 + (i % 3) * 3 + c] = (D[c] * beta + f * dt) / miss;
                }
            }
        }
    }
    a.tca[p] = tca;
    a.miss[p] = miss;
    a.closest[p] = bk;
    a.unit_obj[2 * p] = (int)oa;
    a.unit_obj[2 * p + 1] = (int)ob;
    a.seed_step0[2 * p] = step0;
    a.seed_step0[2 * p + 1] = step0;
    for (int i = 0; i < 27; ++i) {
        a.seeds[(2 * p) * 27 + i] = seed[i];
        a.seeds[(2 * p + 1) * 27 + i] = -seed[i];
    }
}

// ---- launchers ----
static size_t var_smem(const TableSrc& ts) { return 128 + (size_t)ts.bytes; }

cudaError_t launch_stm(const TableSrc& ts, const VarArgs& a, cudaStream_t s)
{
    if (a.n <= 0)
        return cudaSuccess;
    const size_t smem = var_smem(ts);
    cudaError_t e = cudaFuncSetAttribute(stm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    const int block = 256;
    const int64_t blocks = (a.n * kVarLanes + block - 1) / block;
    stm_kernel<<<(unsigned)blocks, block, smem, s>>>(ts, a);
    return cudaGetLastError();
}

cudaError_t launch_adjoint(const TableSrc& ts, const AdjArgs& a, cudaStream_t s)
{
    if (a.n_units <= 0)
        return cudaSuccess;
    const size_t smem = var_smem(ts);
    cudaError_t e
        = cudaFuncSetAttribute(adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    const int block = 256;
    const int64_t blocks = (a.n_units * kVarLanes + block - 1) / block;
    adjoint_kernel<<<(unsigned)blocks, block, smem, s>>>(ts, a);
    return cudaGetLastError();
}

cudaError_t launch_pair_approach(const PairArgs& a, cudaStream_t s)
{
    if (a.n_pairs <= 0)
        return cudaSuccess;
    pair_approach_kernel<<<(unsigned)((a.n_pairs + 127) / 128), 128, 0, s>>>(a);
    return cudaGetLastError();
}

// ---- acceleration Jacobian of many positions (one group of kVarLanes lanes each) ----
__global__ void __launch_bounds__(256, 1) jacobian_kernel(TableSrc ts, int64_t n, const double* r,
    const double* M, double* acc, double* jac, unsigned* err)
{
    extern __shared__ __align__(128) uint8_t smem[];
    GravSmem g;
    if (!stage_table64(smem, ts, err, g))
        return;
    const int P = kVarLanes;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / P;
    const int l = (int)(threadIdx.x % P);
    if (i >= n)
        return;
    const unsigned mask = 0xffu << (threadIdx.x & 24);
    const double ri[3] = { r[i * 3], r[i * 3 + 1], r[i * 3 + 2] };
    double a[3], J[3][3];
    if (M)
        gravity_jac_gcrs_lanes(g, l, P, M, ri, a, J, mask);
    else
        gravity_jac_itrs_lanes(g, l, P, ri[0], ri[1], ri[2], a, J, mask);
    if (l == 0)
        for (int k = 0; k < 3; ++k) {
            if (acc)
                acc[i * 3 + k] = a[k];
            for (int m = 0; m < 3; ++m)
                jac[(i * 3 + k) * 3 + m] = J[k][m];
        }
}

cudaError_t launch_jacobian(const TableSrc& ts, int64_t n, const double* r, const double* M,
    double* acc, double* jac, unsigned* err, cudaStream_t s)
{
    if (n <= 0)
        return cudaSuccess;
    const size_t smem = var_smem(ts);
    cudaError_t e
        = cudaFuncSetAttribute(jacobian_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    const int block = 256;
    jacobian_kernel<<<(unsigned)((n * kVarLanes + block - 1) / block), block, smem, s>>>(ts, n, r, M, acc,
        jac, err);
    return cudaGetLastError();
}

} // namespace gpop
