// The per-evaluation path of the C++ mirror: GpuPropagator (with GpuStartup and Predictor) driven
// by IForceModel implementations that are not the library's ForceModel, the way the reference's
// own tests drive it with mock force models. Prints JSON lines for tests/test_cpp_generic.py.
//  - Hooks: forwards every hook to a library ForceModel, so the per-evaluation path computes the
//    same gravity as the fused path; its results are printed beside the fused path's.
//  - Oscillator: a = -w^2 r computed on the host in the hooks (a force with a closed-form
//    solution); counts the hook calls.
//  - Poly: a polynomial in time with the reference mock's time rules (exact solution).
//  - ClosestApproach over the library's ForceModel and over Hooks, two phases.
#include "gpop.hpp"

#include <cmath>
#include <cstdio>
#include <vector>

static void print_vec(const char* key, const double* x, size_t n)
{
    std::printf("{\"%s\": [", key);
    for (size_t i = 0; i < n; ++i)
        std::printf("%s%.17g", i ? ", " : "", x[i]);
    std::printf("]}\n");
}

// Any IForceModel other than ForceModel takes the per-evaluation path; this one delegates.
struct Hooks : IForceModel {
    ForceModel& inner;
    explicit Hooks(ForceModel& m) : inner(m) { }
    void PreInitialize() override { inner.PreInitialize(); }
    void InitializeGeneration(int b, int a) override { inner.InitializeGeneration(b, a); }
    void ComputeGenerationAcceleration(double* p, double* v, double* k, int step, int kIndex) override
    {
        inner.ComputeGenerationAcceleration(p, v, k, step, kIndex);
    }
    void InitializePropagation(int b, int a) override { inner.InitializePropagation(b, a); }
    void ComputePropagationAcceleration(double* p, double* v, double* a, int step, int col) override
    {
        inner.ComputePropagationAcceleration(p, v, a, step, col);
    }
};

// a = -w^2 r, evaluated on the host from the device positions.
struct Oscillator : IForceModel {
    unsigned n;
    double w2;
    long gen_calls = 0, prop_calls = 0, pre = 0, init_gen = 0, init_prop = 0;
    Oscillator(unsigned count, double w) : n(count), w2(w * w) { }
    void eval(const double* devPosition, double* devOut, int stride, int slot)
    {
        std::vector<double> p(3 * n), a(3 * n);
        cudaMemcpy(p.data(), devPosition, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost);
        for (size_t i = 0; i < 3 * n; ++i)
            a[i] = -w2 * p[i];
        cudaMemcpy2D(devOut + 3 * slot, sizeof(double) * stride, a.data(), sizeof(double) * 3, sizeof(double) * 3, n,
            cudaMemcpyHostToDevice);
    }
    void PreInitialize() override { ++pre; }
    void InitializeGeneration(int, int) override { ++init_gen; }
    void ComputeGenerationAcceleration(double* p, double*, double* k, int, int kIndex) override
    {
        ++gen_calls;
        eval(p, k, 30, kIndex);
    }
    void InitializePropagation(int, int) override { ++init_prop; }
    void ComputePropagationAcceleration(double* p, double*, double* a, int, int col) override
    {
        ++prop_calls;
        eval(p, a, 27, col);
    }
};

// a = -6 t + 42 t^5 on every axis, with time from the hook arguments by the rules of the reference's
// mock force model (unit_tests/include/mock_force_model.cuh:65-106): RK8 stage k of startup step s
// at (s - 1 + c_k) h for s > 0 and (s + 1 - c_k) h for s < 0, propagation epoch index i at (i - 4) h.
// From r = v = 0 the solution is r = -t^3 + t^7, which GJ8 and RK8 integrate exactly.
struct Poly : IForceModel {
    unsigned n;
    double h;
    explicit Poly(unsigned count, double step) : n(count), h(step) { }
    static double f(double t) { return -6 * t + 42 * t * t * t * t * t; }
    void write(double t, double* devOut, int stride, int slot)
    {
        std::vector<double> a(3 * n, f(t));
        cudaMemcpy2D(devOut + 3 * slot, sizeof(double) * stride, a.data(), sizeof(double) * 3, sizeof(double) * 3, n,
            cudaMemcpyHostToDevice);
    }
    void PreInitialize() override { }
    void InitializeGeneration(int, int) override { }
    void ComputeGenerationAcceleration(double*, double*, double* k, int step, int kIndex) override
    {
        static const double c[10] = { 0.0, 4.0 / 27.0, 2.0 / 9.0, 1.0 / 3.0, 1.0 / 2.0, 2.0 / 3.0, 1.0 / 6.0, 1.0,
            5.0 / 6.0, 1.0 };
        const int dir = step > 0 ? -1 : 1;
        write((double)(step + dir) * h + (-dir) * c[kIndex] * h, k, 30, kIndex);
    }
    void InitializePropagation(int, int) override { }
    void ComputePropagationAcceleration(double*, double*, double* a, int stepNum, int col) override
    {
        write((double)(stepNum - 4) * h, a, 27, col);
    }
};

int main(int argc, char** argv)
{
    if (argc > 1)
        ForceModel::DataDirectory() = argv[1];
    const unsigned n = 16;
    std::vector<double> r(3 * n), v(3 * n);
    for (unsigned i = 0; i < n; ++i) { // circular orbits at 7000 km + 25 km i, spread in phase
        const double a = 7.0e6 + 2.5e4 * i, ph = 0.4 * i, inc = 0.1 + 0.12 * i;
        const double sp = std::sqrt(3.986004415e14 / a);
        const double ri[3] = { a * std::cos(ph), a * std::sin(ph) * std::cos(inc), a * std::sin(ph) * std::sin(inc) };
        const double vi[3] = { -sp * std::sin(ph), sp * std::cos(ph) * std::cos(inc), sp * std::cos(ph) * std::sin(inc) };
        for (int j = 0; j < 3; ++j) {
            r[3 * i + j] = ri[j];
            v[3 * i + j] = vi[j];
        }
    }
    FullPerturbationParameters params { { 2024, 1, 1, 0, 0, 0.0 } };
    const double h = 30.0;
    const int steps = 40;
    double *dr = nullptr, *dv = nullptr, *da = nullptr;
    cudaMalloc((void**)&dr, sizeof(double) * 3 * n);
    cudaMalloc((void**)&dv, sizeof(double) * 3 * n);
    cudaMalloc((void**)&da, sizeof(double) * 3 * n);
    std::vector<double> out(3 * n), outv(3 * n), acc(3 * n);
    {
        // fused path
        ForceModel fm(nullptr, n, h, &params);
        cudaMemcpy(dr, r.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice);
        cudaMemcpy(dv, v.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice);
        GpuPropagator prop(dr, dv, n, nullptr, h, &params, fm, steps);
        for (int s = 1; s <= steps; ++s)
            prop.Step(nullptr, nullptr, s == steps ? da : nullptr);
        prop.CopyStateToHost(out.data(), outv.data());
        cudaMemcpy(acc.data(), da, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost);
        print_vec("fused_r", out.data(), out.size());
        print_vec("fused_v", outv.data(), outv.size());
        print_vec("fused_a", acc.data(), acc.size());
    }
    {
        // the same model behind another IForceModel: the per-evaluation path
        ForceModel fm(nullptr, n, h, &params);
        Hooks hooks(fm);
        cudaMemcpy(dr, r.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice);
        cudaMemcpy(dv, v.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice);
        GpuPropagator prop(dr, dv, n, nullptr, h, &params, hooks, steps);
        for (int s = 1; s <= steps; ++s)
            prop.Step(s == steps ? out.data() : nullptr, s == steps ? outv.data() : nullptr,
                s == steps ? da : nullptr);
        cudaMemcpy(acc.data(), da, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost);
        print_vec("generic_r", out.data(), out.size());
        print_vec("generic_v", outv.data(), outv.size());
        print_vec("generic_a", acc.data(), acc.size());
    }
    {
        // harmonic oscillator, w = 1, h = 0.05: r(t) = r0 cos t + v0 sin t
        const unsigned m = 4;
        const double w = 1.0, hh = 0.05;
        const int osteps = 200;
        std::vector<double> r0(3 * m), v0(3 * m), ro(3 * m), vo(3 * m);
        for (unsigned i = 0; i < 3 * m; ++i) {
            r0[i] = 1.0 + 0.1 * i;
            v0[i] = 0.5 - 0.07 * i;
        }
        cudaMemcpy(dr, r0.data(), sizeof(double) * 3 * m, cudaMemcpyHostToDevice);
        cudaMemcpy(dv, v0.data(), sizeof(double) * 3 * m, cudaMemcpyHostToDevice);
        Oscillator osc(m, w);
        GpuPropagator prop(dr, dv, m, nullptr, hh, &params, osc, osteps, 7);
        for (int s = 1; s <= osteps; ++s)
            prop.Step();
        prop.CopyStateToHost(ro.data(), vo.data());
        print_vec("osc_r0", r0.data(), r0.size());
        print_vec("osc_v0", v0.data(), v0.size());
        print_vec("osc_r", ro.data(), ro.size());
        print_vec("osc_v", vo.data(), vo.size());
        std::printf("{\"osc_calls\": [%ld, %ld, %ld, %ld, %ld]}\n", osc.pre, osc.init_gen, osc.gen_calls,
            osc.init_prop, osc.prop_calls);
        std::printf("{\"osc_t\": %.17g}\n", hh * osteps);
    }
    {
        // the polynomial mock: 60 steps of 0.1 from rest
        const unsigned m = 3;
        const double hh = 0.1;
        const int psteps = 60;
        std::vector<double> zero(3 * m, 0.0), ro(3 * m), vo(3 * m);
        cudaMemcpy(dr, zero.data(), sizeof(double) * 3 * m, cudaMemcpyHostToDevice);
        cudaMemcpy(dv, zero.data(), sizeof(double) * 3 * m, cudaMemcpyHostToDevice);
        Poly poly(m, hh);
        GpuPropagator prop(dr, dv, m, nullptr, hh, &params, poly, psteps);
        for (int s = 1; s <= psteps; ++s)
            prop.Step();
        prop.CopyStateToHost(ro.data(), vo.data());
        print_vec("poly_r", ro.data(), ro.size());
        print_vec("poly_v", vo.data(), vo.size());
        std::printf("{\"poly_t\": %.17g}\n", hh * psteps);
    }
    {
        // ClosestApproach: fused (ForceModel) and per-evaluation (Hooks) over two phases; every
        // pair's Get(a, b) as rows (a, b, distance, time)
        const unsigned m = 8;
        std::vector<std::array<double, 3>> pr(m), pv(m);
        for (unsigned i = 0; i < m; ++i)
            for (int j = 0; j < 3; ++j) {
                pr[i][j] = r[3 * i + j];
                pv[i][j] = v[3 * i + j];
            }
        const std::vector<unsigned> sets { 0, 0, 0, 1, 1, 2, 2, 2 };
        ForceModel fm(nullptr, m, h, &params);
        Hooks hooks(fm);
        for (int which = 0; which < 2; ++which) {
            ClosestApproach ca(nullptr, &params, which == 0 ? static_cast<IForceModel&>(fm) : hooks, h);
            ca.Initialize(pr, pv, sets);
            ca.Propagate(30);
            ca.Propagate(20);
            ClosestApproachData data;
            ca.FindClosest(data);
            std::vector<double> rows;
            for (unsigned a = 0; a < m; ++a)
                for (unsigned b = 0; b < m; ++b) {
                    const Approach x = data.Get(a, b);
                    rows.insert(rows.end(), { (double)a, (double)b, x.distance, x.time });
                }
            print_vec(which == 0 ? "ca_fused" : "ca_generic", rows.data(), rows.size());
        }
    }
    cudaFree(dr);
    cudaFree(dv);
    cudaFree(da);
    return 0;
}
