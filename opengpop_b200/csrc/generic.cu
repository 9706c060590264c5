// generic.cu -- the integrator pieces between force evaluations, for n objects, with the
// accelerations supplied by the caller. This is the path the reference's classes take with an
// arbitrary IForceModel (lib/gpu_startup/src/gpu_startup.cu, lib/gpu_integrator/src/prediction.cu,
// lib/gpu_propagator/src/gpu_propagator.cu): the host calls the model's virtual hooks between these
// kernels, and the hooks read and write the reference's AoS buffers:
//   stage state x, v            [n][3]
//   RK8 stage matrices Kx, Kv   [n][10][3] (the generation hook writes Kv slot k)
//   startup matrices R, V, A, s, S and the GJ8 acceleration history A  [n][9][3] (the
//   propagation hook writes column i)
//   GJ8 vectors r, v, s, S      [n][3]
// Each kernel repeats the arithmetic of the fused device code (integrator.cuh, gj8_kernel) term for
// term, so with the library's own gravity behind the hooks the results are those of the fused path.
// One thread per object; nothing here allocates.
#include "common.cuh"
#include "context.h"
#include "gj8_tables.cuh"

#include <cmath>

using namespace gpop;

namespace {

constexpr int kBlock = 256;

inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

// RK8::step stage k (gpu_startup.cu:108-135): stage state = base + h sum_i a_ki K_i (K = stage
// velocity for x, acceleration for v); Kx_k is the stage velocity.
__global__ void rk8_stage_kernel(int64_t n, double h, int step, int k, const double* __restrict__ R27,
    const double* __restrict__ V27, double* __restrict__ Kx30, const double* __restrict__ Kv30,
    double* __restrict__ tx, double* __restrict__ tv)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double hh = step > 0 ? h : -h;
    const int base = 4 + step + (step > 0 ? -1 : 1);
    const double* rb = R27 + i * 27 + base * 3;
    const double* vb = V27 + i * 27 + base * 3;
    double* kx = Kx30 + i * 30;
    const double* kv = Kv30 + i * 30;
    for (int j = 0; j < 3; ++j) {
        double x, v;
        if (k == 0) {
            x = rb[j];
            v = vb[j];
        } else {
            double sx = 0.0, sv = 0.0;
            for (int s = 0; s < k; ++s) {
                sx = fma(c_RKA[k - 1][s], kx[s * 3 + j], sx);
                sv = fma(c_RKA[k - 1][s], kv[s * 3 + j], sv);
            }
            x = fma(hh, sx, rb[j]);
            v = fma(hh, sv, vb[j]);
        }
        tx[i * 3 + j] = x;
        tv[i * 3 + j] = v;
        kx[k * 3 + j] = v;
    }
}

// RK8::step end (gpu_startup.cu:136-144): column 4 + step = base + h sum_k b_k K_k.
__global__ void rk8_finish_kernel(int64_t n, double h, int step, double* __restrict__ R27,
    double* __restrict__ V27, const double* __restrict__ Kx30, const double* __restrict__ Kv30)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double hh = step > 0 ? h : -h;
    const int base = 4 + step + (step > 0 ? -1 : 1);
    const int col = 4 + step;
    double* r = R27 + i * 27;
    double* v = V27 + i * 27;
    const double* kx = Kx30 + i * 30;
    const double* kv = Kv30 + i * 30;
    for (int j = 0; j < 3; ++j) {
        double sx = 0.0, sv = 0.0;
        for (int k = 0; k < 10; ++k) {
            sx = fma(kx[k * 3 + j], c_RKB[k], sx);
            sv = fma(kv[k * 3 + j], c_RKB[k], sv);
        }
        v[col * 3 + j] = fma(hh, sv, v[base * 3 + j]);
        r[col * 3 + j] = fma(hh, sx, r[base * 3 + j]);
    }
}

// GpuStartup before StartupPredictor::Predict: epoch column 4 = (r, v), everything else zero.
__global__ void startup_init_kernel(int64_t n, const double* __restrict__ r, const double* __restrict__ v,
    double* R27, double* V27, double* A27, double* s27, double* S27)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    for (int c = 0; c < 27; ++c) {
        R27[i * 27 + c] = V27[i * 27 + c] = 0.0;
        if (A27)
            A27[i * 27 + c] = 0.0;
        if (s27)
            s27[i * 27 + c] = 0.0;
        if (S27)
            S27[i * 27 + c] = 0.0;
    }
    for (int j = 0; j < 3; ++j) {
        R27[i * 27 + 12 + j] = r[i * 3 + j];
        V27[i * 27 + 12 + j] = v[i * 3 + j];
    }
}

// StartupCorrector::Correct without its force evaluations (gpu_startup.cu:247-290): s0 and S0
// (eqs. 73, 75, 86), all s and S, and the new state columns (eqs. 74, 87) except the epoch's.
__global__ void startup_correct_kernel(int64_t n, double h, double* __restrict__ R27,
    double* __restrict__ V27, const double* __restrict__ A27, double* __restrict__ s27,
    double* __restrict__ S27)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double* r = R27 + i * 27;
    double* v = V27 + i * 27;
    const double* a = A27 + i * 27;
    double* s = s27 + i * 27;
    double* S = S27 + i * 27;
    const double hinv = 1 / h, h2inv = 1 / (h * h);
    for (int j = 0; j < 3; ++j) {
        double sb = 0.0, sa = 0.0;
        for (int k = 0; k < 9; ++k) {
            sb = fma(c_SA[4][k], a[k * 3 + j], sb);
            sa = fma(c_GJ[4][k], a[k * 3 + j], sa);
        }
        s[12 + j] = fma(hinv, v[12 + j], -sb);
        S[12 + j] = fma(h2inv, r[12 + j], -sa);
    }
    for (int q = 1; q <= 4; ++q)
        for (int j = 0; j < 3; ++j) {
            const int up = (4 + q) * 3 + j, upm = (4 + q - 1) * 3 + j;
            const int dn = (4 - q) * 3 + j, dnp = (4 - q + 1) * 3 + j;
            s[up] = s[upm] + (a[upm] + a[up]) / 2;
            s[dn] = s[dnp] - (a[dnp] + a[dn]) / 2;
            S[up] = s[upm] + S[upm] + a[upm] / 2;
            S[dn] = -s[dnp] + S[dnp] + a[dnp] / 2;
        }
    const double h2 = h * h;
    for (int c = 0; c < 9; ++c) {
        if (c == 4)
            continue;
        for (int j = 0; j < 3; ++j) {
            double sv = 0.0, sr = 0.0;
            for (int k = 0; k < 9; ++k) {
                sv = fma(a[k * 3 + j], c_SA[c][k], sv);
                sr = fma(a[k * 3 + j], c_GJ[c][k], sr);
            }
            v[c * 3 + j] = h * (sv + s[c * 3 + j]);
            r[c * 3 + j] = h2 * (sr + S[c * 3 + j]);
        }
    }
}

// Predictor::Predict without its force evaluation (prediction.cu:49-70, FinalizePredictionKernel
// and MoveAccelerationsKernel), plus the parts of GpuPropagator::Correct that do not depend on
// the new acceleration (gpu_propagator.cu:86-100): prev = s and the corrector sums over the
// shifted history.
__global__ void gj8_predict_kernel(int64_t n, double h, double* __restrict__ r, double* __restrict__ v,
    double* __restrict__ A27, const double* __restrict__ s3, double* __restrict__ S3,
    double* __restrict__ prev3, double* __restrict__ sum1, double* __restrict__ sum2)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double* a = A27 + i * 27;
    for (int j = 0; j < 3; ++j) {
        double vt = 0.0, rt = 0.0;
        for (int c = 0; c < 9; ++c) {
            vt = fma(a[c * 3 + j], c_SA[9][c], vt);
            rt = fma(a[c * 3 + j], c_GJ[9][c], rt);
        }
        const double s = s3[i * 3 + j];
        S3[i * 3 + j] += s + a[24 + j] / 2;
        v[i * 3 + j] = (vt + s + a[24 + j] / 2) * h;
        r[i * 3 + j] = (rt + S3[i * 3 + j]) * h * h;
        double c1 = 0.0, c2 = 0.0;
        for (int c = 0; c < 8; ++c) {
            c1 = fma(a[(c + 1) * 3 + j], c_SA[8][c], c1);
            c2 = fma(a[(c + 1) * 3 + j], c_GJ[8][c], c2);
        }
        sum1[i * 3 + j] = c1;
        sum2[i * 3 + j] = c2;
        prev3[i * 3 + j] = s;
    }
    for (int c = 0; c < 8; ++c)
        for (int j = 0; j < 3; ++j)
            a[c * 3 + j] = a[(c + 1) * 3 + j];
}

// One corrector pass after its force evaluation (UpdateSmallSKernel, FinalizeCorrectionKernel:
// gpu_propagator/src/device/*.cu): s = prev + (a8 + a7) / 2, then v and r.
__global__ void gj8_correct_kernel(int64_t n, double h, double* __restrict__ r, double* __restrict__ v,
    const double* __restrict__ A27, double* __restrict__ s3, const double* __restrict__ S3,
    const double* __restrict__ prev3, const double* __restrict__ sum1, const double* __restrict__ sum2)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double* a = A27 + i * 27;
    for (int j = 0; j < 3; ++j) {
        const double a8 = a[24 + j], a7 = a[21 + j];
        const double s = prev3[i * 3 + j] + (a8 + a7) / 2;
        s3[i * 3 + j] = s;
        v[i * 3 + j] = h * (sum1[i * 3 + j] + a8 * c_SA[8][8] + s);
        r[i * 3 + j] = h * h * (sum2[i * 3 + j] + a8 * c_GJ[8][8] + S3[i * 3 + j]);
    }
}

// Column col of an [n][cols][3] matrix to an [n][3] vector, or back.
__global__ void column_kernel(int64_t n, double* m, int cols, int col, double* v3, int to_matrix)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    for (int j = 0; j < 3; ++j) {
        double* e = m + (i * cols + col) * 3 + j;
        if (to_matrix)
            *e = v3[i * 3 + j];
        else
            v3[i * 3 + j] = *e;
    }
}

__global__ void coefficient_kernel(double* a90, double* b90)
{
    const int t = threadIdx.x; // t = 10 k + c: history column k, ordinate row c
    if (t >= 90)
        return;
    const int k = t / 10, c = t % 10;
    if (a90)
        a90[t] = c_GJ[c][k];
    if (b90)
        b90[t] = c_SA[c][k];
}

gpop_status finish(gpop_ctx* ctx, const char* what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, what);
    if (ctx)
        ctx->launches++;
    return GPOP_OK;
}

gpop_status check_n(gpop_ctx* ctx, int64_t n, double h)
{
    if (n < 0 || !(h > 0) || !std::isfinite(h))
        return fail(ctx, GPOP_ERR_INVALID_ARG, "n must be >= 0 and h positive");
    if (ctx) {
        const cudaError_t e = cudaSetDevice(ctx->cfg.device);
        if (e != cudaSuccess)
            return cuda_fail(ctx, e, "cudaSetDevice");
    }
    return GPOP_OK;
}

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

} // namespace

extern "C" gpop_status gpop_rk8_stage(gpop_ctx* ctx, int64_t n, double h, int32_t step, int32_t k,
    const double* R27, const double* V27, double* Kx30, const double* Kv30, double* x_dev,
    double* v_dev, void* stream)
{
    gpop_status st = check_n(ctx, n, h);
    if (st != GPOP_OK)
        return st;
    if (step == 0 || step < -4 || step > 4 || k < 0 || k > 9)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "step must be in +-1..4 and k in 0..9");
    if (n == 0)
        return GPOP_OK;
    if (!R27 || !V27 || !Kx30 || (k > 0 && !Kv30) || !x_dev || !v_dev)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "null buffer");
    rk8_stage_kernel<<<blocks_for(n), kBlock, 0, as_stream(stream)>>>(n, h, step, k, R27, V27, Kx30,
        Kv30, x_dev, v_dev);
    return finish(ctx, "RK8 stage kernel");
}

extern "C" gpop_status gpop_rk8_finish(gpop_ctx* ctx, int64_t n, double h, int32_t step, double* R27,
    double* V27, const double* Kx30, const double* Kv30, void* stream)
{
    gpop_status st = check_n(ctx, n, h);
    if (st != GPOP_OK)
        return st;
    if (step == 0 || step < -4 || step > 4)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "step must be in +-1..4");
    if (n == 0)
        return GPOP_OK;
    if (!R27 || !V27 || !Kx30 || !Kv30)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "null buffer");
    rk8_finish_kernel<<<blocks_for(n), kBlock, 0, as_stream(stream)>>>(n, h, step, R27, V27, Kx30, Kv30);
    return finish(ctx, "RK8 finish kernel");
}

extern "C" gpop_status gpop_startup_init(gpop_ctx* ctx, int64_t n, const double* r_dev,
    const double* v_dev, double* R27, double* V27, double* A27, double* s27, double* S27, void* stream)
{
    gpop_status st = check_n(ctx, n, 1.0);
    if (st != GPOP_OK)
        return st;
    if (n == 0)
        return GPOP_OK;
    if (!r_dev || !v_dev || !R27 || !V27)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "null buffer");
    startup_init_kernel<<<blocks_for(n), kBlock, 0, as_stream(stream)>>>(n, r_dev, v_dev, R27, V27, A27,
        s27, S27);
    return finish(ctx, "startup init kernel");
}

extern "C" gpop_status gpop_startup_correct(gpop_ctx* ctx, int64_t n, double h, double* R27,
    double* V27, const double* A27, double* s27, double* S27, void* stream)
{
    gpop_status st = check_n(ctx, n, h);
    if (st != GPOP_OK)
        return st;
    if (n == 0)
        return GPOP_OK;
    if (!R27 || !V27 || !A27 || !s27 || !S27)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "null buffer");
    startup_correct_kernel<<<blocks_for(n), kBlock, 0, as_stream(stream)>>>(n, h, R27, V27, A27, s27, S27);
    return finish(ctx, "startup corrector kernel");
}

extern "C" gpop_status gpop_gj8_predict(gpop_ctx* ctx, int64_t n, double h, double* r_dev,
    double* v_dev, double* A27, const double* s3, double* S3, double* prev3, double* sum1,
    double* sum2, void* stream)
{
    gpop_status st = check_n(ctx, n, h);
    if (st != GPOP_OK)
        return st;
    if (n == 0)
        return GPOP_OK;
    if (!r_dev || !v_dev || !A27 || !s3 || !S3 || !prev3 || !sum1 || !sum2)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "null buffer");
    gj8_predict_kernel<<<blocks_for(n), kBlock, 0, as_stream(stream)>>>(n, h, r_dev, v_dev, A27, s3, S3,
        prev3, sum1, sum2);
    return finish(ctx, "GJ8 predictor kernel");
}

extern "C" gpop_status gpop_gj8_correct(gpop_ctx* ctx, int64_t n, double h, double* r_dev,
    double* v_dev, const double* A27, double* s3, const double* S3, const double* prev3,
    const double* sum1, const double* sum2, void* stream)
{
    gpop_status st = check_n(ctx, n, h);
    if (st != GPOP_OK)
        return st;
    if (n == 0)
        return GPOP_OK;
    if (!r_dev || !v_dev || !A27 || !s3 || !S3 || !prev3 || !sum1 || !sum2)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "null buffer");
    gj8_correct_kernel<<<blocks_for(n), kBlock, 0, as_stream(stream)>>>(n, h, r_dev, v_dev, A27, s3, S3,
        prev3, sum1, sum2);
    return finish(ctx, "GJ8 corrector kernel");
}

extern "C" gpop_status gpop_matrix_column(gpop_ctx* ctx, int64_t n, double* m_dev, int32_t cols,
    int32_t col, double* v3_dev, int32_t to_matrix, void* stream)
{
    gpop_status st = check_n(ctx, n, 1.0);
    if (st != GPOP_OK)
        return st;
    if (cols <= 0 || col < 0 || col >= cols)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "column outside the matrix");
    if (n == 0)
        return GPOP_OK;
    if (!m_dev || !v3_dev)
        return fail(ctx, GPOP_ERR_INVALID_ARG, "null buffer");
    column_kernel<<<blocks_for(n), kBlock, 0, as_stream(stream)>>>(n, m_dev, cols, col, v3_dev, to_matrix);
    return finish(ctx, "matrix column kernel");
}

extern "C" gpop_status gpop_gj8_coefficients(gpop_ctx* ctx, double* a90_dev, double* b90_dev, void* stream)
{
    if (ctx) {
        const cudaError_t e = cudaSetDevice(ctx->cfg.device);
        if (e != cudaSuccess)
            return cuda_fail(ctx, e, "cudaSetDevice");
    }
    if (!a90_dev && !b90_dev)
        return GPOP_OK;
    coefficient_kernel<<<1, 96, 0, as_stream(stream)>>>(a90_dev, b90_dev);
    return finish(ctx, "coefficient kernel");
}
