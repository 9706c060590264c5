// ref_driver.cu -- TEST INFRASTRUCTURE ONLY: a C driver over the reference's own CUDA libraries
// (compiled from the reference sources by oracle/ref/build.sh into oracle/_ref/). It mirrors the
// reference runner (exec/runner.cu:11-119) without the progress bar, with an explicit step size,
// and times the step loop with CUDA events. The reference opens its data files at ../../data/
// relative to the working directory (gravity_source.cu:63, time_points.cu:77-109): the caller
// chdir()s into a directory two levels below a data/ copy before calling in.
#include "closest_approach/closest_approach.cuh"
#include "force_model/force_model.cuh"
#include "force_model/time_points/time_points.cuh"
#include "gpu_propagator/gpu_propagator.cuh"

#include <cstring>
#include <vector>

extern "C" {

// propagate(): returns 0 on success; r/v [n][3] host buffers; elapsed_ms = step loop only.
int ref_propagate(int year, int month, int day, int hour, int min, double sec, double h, int steps,
    int n, const double* r_in, const double* v_in, double* r_out, double* v_out, double* elapsed_ms)
{
    FullPerturbationParameters params { TimeData { year, month, day, hour, min, sec } };
    cublasHandle_t handle;
    if (cublasCreate(&handle) != CUBLAS_STATUS_SUCCESS)
        return 1;
    double *devR = nullptr, *devV = nullptr;
    cudaMalloc(&devR, (size_t)n * 3 * sizeof(double));
    cudaMalloc(&devV, (size_t)n * 3 * sizeof(double));
    cudaMemcpy(devR, r_in, (size_t)n * 3 * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(devV, v_in, (size_t)n * 3 * sizeof(double), cudaMemcpyHostToDevice);
    {
        ForceModel forceModel(&handle, n, h, &params);
        GpuPropagator propagator(devR, devV, n, &handle, h, &params, forceModel, steps, 7);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
        for (int i = 0; i < steps; i++)
            propagator.Step(nullptr, nullptr);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        *elapsed_ms = ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        propagator.CopyStateToHost(r_out, v_out);
    }
    cudaFree(devR);
    cudaFree(devV);
    cublasDestroy(handle);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// closestApproach(): one record per cross-set pair i < j in the runner's order
// (exec/runner.cu:96-106); out arrays hold num_pairs entries (positions 3 each).
int ref_closest_approach(int year, int month, int day, int hour, int min, double sec, double h,
    int steps, int n, const double* r_in, const double* v_in, const unsigned* set_ids,
    int* obj1, int* obj2, double* dist, double* time, double* pos_a, double* pos_b,
    long long* num_out, double* elapsed_ms)
{
    FullPerturbationParameters params { TimeData { year, month, day, hour, min, sec } };
    cublasHandle_t handle;
    if (cublasCreate(&handle) != CUBLAS_STATUS_SUCCESS)
        return 1;
    std::vector<std::array<double, 3>> r(n), v(n);
    std::memcpy(r.data(), r_in, (size_t)n * 24);
    std::memcpy(v.data(), v_in, (size_t)n * 24);
    std::vector<unsigned> ids(set_ids, set_ids + n);
    long long k = 0;
    {
        ForceModel forceModel(&handle, n, h, &params);
        ClosestApproach ca(&handle, &params, forceModel, h);
        ca.Initialize(r, v, ids);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
        ca.Propagate(steps, false);
        ClosestApproachData data;
        ca.FindClosest(data);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        *elapsed_ms = ms;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j)
                if (ids[i] != ids[j]) {
                    Approach a = data.Get(i, j);
                    obj1[k] = i;
                    obj2[k] = j;
                    dist[k] = a.distance;
                    time[k] = a.time;
                    for (int c = 0; c < 3; ++c) {
                        pos_a[k * 3 + c] = a.positionA[c];
                        pos_b[k * 3 + c] = a.positionB[c];
                    }
                    ++k;
                }
    }
    *num_out = k;
    cublasDestroy(handle);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// FMTimePoints::Initialize + CalculateParameters (time_points.cu:26-71,126-201: the per-epoch
// TimePointParamsKernel and the seven batched DGEMMs of ComputeITRStoGCRS): count ITRS->GCRS
// matrices (column-major, 9 each) and UTC MJDs into host buffers.
int ref_frame_matrices(int year, int month, int day, int hour, int min, double sec, double h,
    int count, int use_midpoints, int before_epoch, double* m_out, double* mjd_out)
{
    cublasHandle_t handle;
    if (cublasCreate(&handle) != CUBLAS_STATUS_SUCCESS)
        return 1;
    int rc = 0;
    {
        FMTimePoints tp(&handle, h, TimeData { year, month, day, hour, min, sec });
        tp.Initialize();
        tp.CalculateParameters(count, use_midpoints != 0, before_epoch);
        TimePointParameters p = tp.GetParametersDev(0);
        if (cudaMemcpy(m_out, p.ITRS_to_GCRS, (size_t)count * 9 * sizeof(double), cudaMemcpyDeviceToHost)
                != cudaSuccess
            || cudaMemcpy(mjd_out, p.mjd, (size_t)count * sizeof(double), cudaMemcpyDeviceToHost)
                != cudaSuccess)
            rc = 2;
    }
    cublasDestroy(handle);
    return rc == 0 && cudaGetLastError() == cudaSuccess ? 0 : 2;
}

} // extern "C"
