// Drives the C++ mirror classes of include/gpop.hpp the way exec/runner.cu and the reference's
// applications do, and prints their results as JSON lines for tests/test_cpp_shim.py to compare
// with the C ABI called directly.
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

int main(int argc, char** argv)
{
    if (argc > 1)
        ForceModel::DataDirectory() = argv[1];
    const unsigned n = 8;
    std::vector<std::array<double, 3>> r(n), v(n);
    for (unsigned i = 0; i < n; ++i) { // circular orbits at 7000 km + 10 km i, spread in phase
        const double a = 7.0e6 + 1.0e4 * i, ph = 0.3 * i, inc = 0.2 + 0.1 * i;
        const double sp = std::sqrt(3.986004415e14 / a);
        r[i] = { a * std::cos(ph), a * std::sin(ph) * std::cos(inc), a * std::sin(ph) * std::sin(inc) };
        v[i] = { -sp * std::sin(ph), sp * std::cos(ph) * std::cos(inc), sp * std::cos(ph) * std::sin(inc) };
    }
    FullPerturbationParameters params { { 2024, 1, 1, 0, 0, 0.0 } };
    const double h = 30.0;
    const int steps = 100;
    ForceModel fm(nullptr, n, h, &params);
    fm.PreInitialize();
    double *dr = nullptr, *dv = nullptr, *dacc = nullptr, *dmat = nullptr;
    cudaMalloc((void**)&dr, sizeof(double) * 3 * n);
    cudaMalloc((void**)&dv, sizeof(double) * 3 * n);
    cudaMalloc((void**)&dacc, sizeof(double) * 3 * n);
    cudaMalloc((void**)&dmat, sizeof(double) * 27 * n);
    cudaMemcpy(dr, r.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice);
    cudaMemcpy(dv, v.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice);
    // per-evaluation hook: acceleration column 2 of a [N][3 x 9] matrix at propagation epoch 5
    fm.InitializePropagation(4, 10);
    cudaMemset(dmat, 0, sizeof(double) * 27 * n);
    fm.ComputePropagationAcceleration(dr, dv, dmat, 5, 2);
    std::vector<double> mat(27 * n);
    cudaMemcpy(mat.data(), dmat, sizeof(double) * 27 * n, cudaMemcpyDeviceToHost);
    print_vec("acc_matrix", mat.data(), mat.size());
    {
        GpuPropagator prop(dr, dv, n, nullptr, h, &params, fm, steps);
        std::vector<double> hr(3 * n), hv(3 * n);
        for (int s = 0; s < steps; ++s)
            prop.Step(s == steps - 1 ? hr.data() : nullptr, s == steps - 1 ? hv.data() : nullptr,
                s == steps - 1 ? dacc : nullptr);
        print_vec("r_end", hr.data(), hr.size());
        print_vec("v_end", hv.data(), hv.size());
        std::vector<double> acc(3 * n);
        cudaMemcpy(acc.data(), dacc, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost);
        print_vec("acc_last", acc.data(), acc.size());
    }
    ClosestApproach ca(nullptr, &params, fm, h);
    std::vector<unsigned> sets { 0, 0, 0, 1, 1, 2, 2, 2 };
    ca.Initialize(r, v, sets);
    ca.Propagate(60);
    ca.Propagate(40);
    ClosestApproachData data;
    ca.FindClosest(data);
    std::vector<double> rec;
    for (unsigned a = 0; a < n; ++a)
        for (unsigned b = 0; b < n; ++b) {
            const Approach ap = data.Get(a, b);
            rec.insert(rec.end(), { (double)a, (double)b, ap.distance, ap.time, ap.positionA[0], ap.positionB[2] });
        }
    print_vec("approaches", rec.data(), rec.size());
    cudaFree(dr);
    cudaFree(dv);
    cudaFree(dacc);
    cudaFree(dmat);
    return 0;
}
