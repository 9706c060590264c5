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

#include <type_traits>

namespace gpop {

__device__ __forceinline__ void cmul(double ac, double as, double bc, double bs, double& rc, double& rs)
{
    const double c = ac * bc - as * bs;
    const double s = as * bc + ac * bs;
    rc = c;
    rs = s;
}

// (C1 + i S1)^p by binary powering (p >= 0).
__device__ __forceinline__ void cpow(double c1, double s1, int p, double& rc, double& rs)
{
    double xc = 1.0, xs = 0.0, bc = c1, bs = s1;
    while (p > 0) {
        if (p & 1)
            cmul(xc, xs, bc, bs, xc, xs);
        p >>= 1;
        if (p)
            cmul(bc, bs, bc, bs, bc, bs);
    }
    rc = xc;
    rs = xs;
}

// Gravity in the Earth-fixed frame with the columns split over the P lanes of an object
// (lane l takes columns l, l + P, ...); the per-object totals are added across the P lanes.
template <bool MIXED>
__device__ __forceinline__ void gravity_itrs_lanes(const GravSmem& gs, int l, int P, double x,
    double y, double z, double& ax, double& ay, double& az)
{
    const int L = gs.L, Lt = gs.Lt;
    const double r = sqrt(x * x + y * y + z * z);
    const double eps = z / r;
    const double q = gs.radius / r;
    const double u = q * eps, w = q * q;
    const float uf = (float)u, wf = (float)w;
    const double C1 = x / r, S1 = y / r;
    double CP, SP, Cm, Sm, Cp, Sp, CPm1, SPm1;
    cpow(C1, S1, P, CP, SP); // step between this lane's columns
    cpow(C1, S1, l, Cm, Sm);
    if (l > 0)
        cpow(C1, S1, l - 1, Cp, Sp);
    else
        Cp = Sp = 0.0; // column 0 has no J, K or H part
    cpow(C1, S1, P - 1, CPm1, SPm1); // (C + iS)_{P-1}: the m-1 values of column P
    double qm = 1.0, qP = 1.0;
    for (int i = 0; i < l; ++i)
        qm *= q;
    for (int i = 0; i < P; ++i)
        qP *= q;
    double G = 0.0, H = 0.0, J = 0.0, KK = 0.0;
    for (int m = l; m <= L; m += P) {
        ColSums64<1> s;
        s.zero();
        double Q1[1] = { qm }, Q2[1] = { 0.0 };
        const double uu[1] = { u }, ww[1] = { w };
        if constexpr (!MIXED) {
            const GravEntry64* e = gs.t64 + grav_col_offset(m, Lt);
            s.add(e, Q1);
            column64<1>(e, 1, L - m, uu, ww, Q1, Q2, s);
        } else {
            ColSums32<1> f;
            f.zero();
            const GravEntry32* e32 = gs.t32 + grav_col_offset(m, Lt);
            float Q1f[1], Q2f[1];
            const float ufa[1] = { uf }, wfa[1] = { wf };
            if (m <= kMixedSplit) {
                const int top = L < kMixedSplit ? L : kMixedSplit;
                const GravEntry64* e = gs.t64 + grav_col_offset(m, kMixedSplit);
                s.add(e, Q1);
                column64<1>(e, 1, top - m, uu, ww, Q1, Q2, s);
                Q1f[0] = (float)Q1[0];
                Q2f[0] = (float)Q2[0];
                column32k<1>(e32, kMixedSplit + 1 - m, L - m, ufa, wfa, Q1f, Q2f, f);
            } else {
                const float4* p = reinterpret_cast<const float4*>(e32);
                const float4 a = p[0], b = p[1];
                const float Qm = (float)qm;
                const float2 QQ = make_float2(Qm, Qm);
                f.g[0] = __fmul2_rn(QQ, make_float2(a.z, a.w));
                f.j[0] = __fmul2_rn(QQ, make_float2(b.x, b.y));
                f.h[0] = __fmul2_rn(QQ, make_float2(b.z, b.w));
                Q1f[0] = Qm;
                Q2f[0] = 0.f;
                column32k<1>(e32, 1, L - m, ufa, wfa, Q1f, Q2f, f);
            }
            s.g1[0] += (double)f.g[0].x;
            s.g2[0] += (double)f.g[0].y;
            s.j1[0] += (double)f.j[0].x;
            s.j2[0] += (double)f.j[0].y;
            s.h1[0] += (double)f.h[0].x;
            s.h2[0] += (double)f.h[0].y;
        }
        const double dm = (double)m; // eq. 4-11
        G += Cm * s.g1[0] + Sm * s.g2[0];
        J += dm * (Cp * s.j1[0] + Sp * s.j2[0]);
        KK -= dm * (Sp * s.j1[0] - Cp * s.j2[0]);
        H += Cp * s.h1[0] + Sp * s.h2[0];
        if (m == 0) {
            Cp = CPm1;
            Sp = SPm1;
        } else {
            cmul(Cp, Sp, CP, SP, Cp, Sp);
        }
        cmul(Cm, Sm, CP, SP, Cm, Sm);
        qm *= qP;
    }
    for (int o = P >> 1; o > 0; o >>= 1) {
        G += __shfl_xor_sync(0xffffffffu, G, o);
        H += __shfl_xor_sync(0xffffffffu, H, o);
        J += __shfl_xor_sync(0xffffffffu, J, o);
        KK += __shfl_xor_sync(0xffffffffu, KK, o);
    }
    const double Gt = G + 1.0; // eq. 4-13
    const double Lambda = Gt + z * H / r;
    const double c = -gs.gm / (r * r);
    ax = c * (Lambda * x / r - J);
    ay = c * (Lambda * y / r - KK);
    az = c * (Lambda * z / r - H);
}

template <bool MIXED>
__device__ __forceinline__ void gravity_gcrs_lanes(const GravSmem& gs, int l, int P,
    const double* __restrict__ M, const double* r, double* a)
{
    double m[9];
#pragma unroll
    for (int i = 0; i < 9; ++i)
        m[i] = __ldg(M + i);
    const double px = m[0] * r[0] + m[1] * r[1] + m[2] * r[2];
    const double py = m[3] * r[0] + m[4] * r[1] + m[5] * r[2];
    const double pz = m[6] * r[0] + m[7] * r[1] + m[8] * r[2];
    double ax, ay, az;
    gravity_itrs_lanes<MIXED>(gs, l, P, px, py, pz, ax, ay, az);
    a[0] = m[0] * ax + m[3] * ay + m[6] * az;
    a[1] = m[1] * ax + m[4] * ay + m[7] * az;
    a[2] = m[2] * ax + m[5] * ay + m[8] * az;
}

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
    const bool ok = stage_to_smem(tab, ts.src, ts.bytes, mbar, err);
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

// Persistent GJ8 kernel: warps pull work items until the queue is empty.
template <bool MIXED>
__global__ void __launch_bounds__(512, 1) batch_gj8_kernel(TableSrc ts, BatchArgs a)
{
    extern __shared__ __align__(128) uint8_t smem[];
    GravSmem g0;
    if (!stage_batch_table<MIXED>(smem, ts, a.err, g0))
        return;
    const int lane = threadIdx.x & 31;
    const int64_t n = a.n_obj;
    double* st = a.state;
    for (;;) {
        int item = 0;
        if (lane == 0)
            item = atomicAdd(a.next_item, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= a.n_items)
            break;
        const BatchItem it = a.items[item];
        const BatchReq rq = a.reqs[it.req];
        const int P = rq.lpo;
        const int slot = lane / P, sl = lane % P;
        const bool valid = slot < it.count;
        const int64_t o = rq.obj0 + it.first + (valid ? slot : 0); // idle slots shadow slot 0
        const bool store = valid && sl == 0;
        GravSmem g = g0;
        g.L = rq.L;
        const double h = rq.h;
        double r[3], v[3], s[3], S[3];
        for (int j = 0; j < 3; ++j) {
            r[j] = st[(kR + j) * n + o];
            v[j] = st[(kV + j) * n + o];
            s[j] = st[(kSs + j) * n + o];
            S[j] = st[(kSb + j) * n + o];
        }
        for (int step = 1; step <= rq.steps; ++step) {
            if (step <= 4) {
                for (int j = 0; j < 3; ++j) {
                    r[j] = st[(kRep + (step - 1) * 6 + j) * n + o];
                    v[j] = st[(kRep + (step - 1) * 6 + 3 + j) * n + o];
                }
                continue;
            }
            const int ring0 = (step - 5) % 9;
            double hist[9][3];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                int sl9 = ring0 + c;
                sl9 -= sl9 >= 9 ? 9 : 0;
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    hist[c][j] = st[(kHist + sl9 * 3 + j) * n + o];
            }
            double s1[3], s2[3], prev[3], a7[3], a8[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) { // predictor, as in gj8_kernel
                double vt = 0.0, rt = 0.0;
#pragma unroll
                for (int c = 0; c < 9; ++c) {
                    vt = fma(hist[c][j], c_SA[9][c], vt);
                    rt = fma(hist[c][j], c_GJ[9][c], rt);
                }
                S[j] += s[j] + hist[8][j] / 2;
                v[j] = (vt + s[j] + hist[8][j] / 2) * h;
                r[j] = (rt + S[j]) * h * h;
                double c1 = 0.0, c2 = 0.0;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    c1 = fma(hist[c + 1][j], c_SA[8][c], c1);
                    c2 = fma(hist[c + 1][j], c_GJ[8][c], c2);
                }
                s1[j] = c1;
                s2[j] = c2;
                prev[j] = s[j];
                a7[j] = hist[8][j];
            }
            const double* M = rq.prop_m + (size_t)(step + 4) * 9;
            for (int itc = 0; itc < a.ncorr; ++itc) {
                gravity_gcrs_lanes<MIXED>(g, sl, P, M, r, a8);
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    s[j] = prev[j] + (a8[j] + a7[j]) / 2;
                    v[j] = h * (s1[j] + a8[j] * c_SA[8][8] + s[j]);
                    r[j] = h * h * (s2[j] + a8[j] * c_GJ[8][8] + S[j]);
                }
            }
            if (store)
                for (int j = 0; j < 3; ++j)
                    st[(kHist + ring0 * 3 + j) * n + o] = a8[j];
        }
        if (store) {
            for (int j = 0; j < 3; ++j) {
                st[(kR + j) * n + o] = r[j];
                st[(kV + j) * n + o] = v[j];
                st[(kSs + j) * n + o] = s[j];
                st[(kSb + j) * n + o] = S[j];
                a.r_out[o * 3 + j] = rq.steps > 0 ? r[j] : a.r0[o * 3 + j];
                a.v_out[o * 3 + j] = rq.steps > 0 ? v[j] : a.v0[o * 3 + j];
            }
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

cudaError_t launch_batch_gj8(const TableSrc& ts, const BatchArgs& a, int blocks, int block, cudaStream_t s)
{
    if (a.n_items <= 0)
        return cudaSuccess;
    const size_t smem = table_smem_bytes(ts);
    cudaError_t e;
    if (ts.mixed) {
        if ((e = set_smem(batch_gj8_kernel<true>, smem)) != cudaSuccess)
            return e;
        batch_gj8_kernel<true><<<blocks, block, smem, s>>>(ts, a);
    } else {
        if ((e = set_smem(batch_gj8_kernel<false>, smem)) != cudaSuccess)
            return e;
        batch_gj8_kernel<false><<<blocks, block, smem, s>>>(ts, a);
    }
    return cudaGetLastError();
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
