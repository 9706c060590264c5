// gpop_propagate_device_noalloc across a cudaDeviceReset: a context made after the reset must find
// the scratch array of the new CUDA context, and give the same bits as before the reset.
// Usage: noalloc_reset_check <data_dir>. Prints "ok" and exits 0 on success.
#include <cuda_runtime.h>
#include <gpop.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

static bool run_once(const char* data_dir, const std::vector<double>& r0, const std::vector<double>& v0,
    std::vector<double>& r_out, std::vector<double>& v_out)
{
    gpop_config cfg;
    gpop_config_default(&cfg);
    cfg.data_dir = data_dir;
    gpop_ctx* ctx = nullptr;
    if (gpop_create(&cfg, &ctx) != GPOP_OK) {
        std::printf("create: %s\n", ctx ? gpop_last_error(ctx) : "no context");
        gpop_destroy(ctx);
        return false;
    }
    const size_t bytes = r0.size() * sizeof(double);
    double *r = nullptr, *v = nullptr;
    bool ok = cudaMalloc(&r, bytes) == cudaSuccess && cudaMalloc(&v, bytes) == cudaSuccess
        && cudaMemcpy(r, r0.data(), bytes, cudaMemcpyHostToDevice) == cudaSuccess
        && cudaMemcpy(v, v0.data(), bytes, cudaMemcpyHostToDevice) == cudaSuccess;
    gpop_time t0 = { 2024, 1, 1, 0, 0, 0.0 };
    if (ok) {
        const gpop_status st = gpop_propagate_device_noalloc(ctx, &t0, 30.0, 60, (int64_t)(r0.size() / 3),
            r, v, nullptr);
        if (st != GPOP_OK) {
            std::printf("noalloc: %s\n", gpop_last_error(ctx));
            ok = false;
        }
    }
    ok = ok && cudaMemcpy(r_out.data(), r, bytes, cudaMemcpyDeviceToHost) == cudaSuccess
        && cudaMemcpy(v_out.data(), v, bytes, cudaMemcpyDeviceToHost) == cudaSuccess;
    cudaFree(r);
    cudaFree(v);
    gpop_destroy(ctx);
    return ok;
}

int main(int argc, char** argv)
{
    if (argc < 2)
        return 2;
    const int n = 64;
    std::vector<double> r0(3 * n), v0(3 * n);
    for (int i = 0; i < n; ++i) {
        const double a = 6.9e6 + 2.0e4 * i, ph = 0.37 * i, inc = 0.1 + 0.045 * i;
        const double sp = std::sqrt(3.986004415e14 / a);
        r0[3 * i] = a * std::cos(ph);
        r0[3 * i + 1] = a * std::sin(ph) * std::cos(inc);
        r0[3 * i + 2] = a * std::sin(ph) * std::sin(inc);
        v0[3 * i] = -sp * std::sin(ph);
        v0[3 * i + 1] = sp * std::cos(ph) * std::cos(inc);
        v0[3 * i + 2] = sp * std::cos(ph) * std::sin(inc);
    }
    std::vector<double> ra(3 * n), va(3 * n), rb(3 * n), vb(3 * n);
    if (!run_once(argv[1], r0, v0, ra, va))
        return 1;
    if (cudaDeviceReset() != cudaSuccess) {
        std::printf("cudaDeviceReset failed\n");
        return 1;
    }
    if (!run_once(argv[1], r0, v0, rb, vb))
        return 1;
    if (std::memcmp(ra.data(), rb.data(), ra.size() * sizeof(double)) != 0
        || std::memcmp(va.data(), vb.data(), va.size() * sizeof(double)) != 0) {
        std::printf("results differ across the reset\n");
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
