/*
 * gpop.hpp -- C++ mirror of the reference's class interfaces over the C ABI of gpop.h.
 *
 * The reference's callers (exec/runner.cu and applications built on its libraries) construct
 * ForceModel, GpuPropagator and ClosestApproach objects. This header gives the same class names,
 * constructor signatures and methods (lib/force_model/include/force_model/force_model.cuh:27-40,
 * iforce_model.cuh:19-33, gpu_propagator.cuh:26-59, closest_approach.cuh:36-88,
 * closest_approach/types.cuh:113-172, common/types/types/Parameters.hpp:19-26), so such code
 * compiles against libgpop.so instead. Differences:
 *  - errors throw std::runtime_error (the reference calls exit());
 *  - the cublasHandle_t* arguments are accepted and ignored;
 *  - GpuPropagator and ClosestApproach run the fused library path and therefore require the
 *    library's ForceModel; another IForceModel implementation is rejected with
 *    std::invalid_argument (the reference would call its virtual methods per evaluation);
 *  - the data directory is ForceModel::DataDirectory (default: $GPOP_DATA_DIR, else the
 *    reference's "../../data").
 * Header-only; link with -lgpop -lcudart.
 */
#ifndef GPOP_HPP
#define GPOP_HPP

#include "gpop.h"

#include <cuda_runtime_api.h>

#include <array>
#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

typedef struct cublasContext* cublasHandle_t;

/* TimeData, FullPerturbationParameters (common/types/types/Parameters.hpp:19-26) */
struct TimeData {
    int Year, Month, Day, Hour, Min;
    double Sec;
};

struct FullPerturbationParameters {
    TimeData StartTimeUTC;
};

namespace gpop_cpp {
inline void check(gpop_ctx* ctx, gpop_status st, const char* what)
{
    if (st != GPOP_OK)
        throw std::runtime_error(std::string(what) + ": " + gpop_status_string(st) + ": "
            + (ctx ? gpop_last_error(ctx) : ""));
}
inline void check_cuda(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
inline gpop_time to_time(const TimeData& t) { return gpop_time { t.Year, t.Month, t.Day, t.Hour, t.Min, t.Sec }; }
} // namespace gpop_cpp

/* IForceModel (force_model/iforce_model.cuh:19-33): the five device-pointer hooks. */
struct IForceModel {
    virtual ~IForceModel() = default;
    virtual void PreInitialize() = 0;
    virtual void InitializeGeneration(int beforeEpoch, int afterEpoch) = 0;
    virtual void ComputeGenerationAcceleration(
        double* devPosition, double* devVelocity, double* devKMatrix, int stepNum, int kIndex)
        = 0;
    virtual void InitializePropagation(int beforeEpoch, int afterEpoch) = 0;
    virtual void ComputePropagationAcceleration(double* devPosition, double* devVelocity,
        double* devAcceleration, int stepNum, int returnColumnIndex)
        = 0;
};

/* ForceModel (force_model.cuh:27-40, force_model.cu:23-109): 70x70 (or the file's degree)
 * gravity in the GCRS with per-epoch frame matrices. The per-evaluation hooks run the library's
 * gravity kernel; GpuPropagator and ClosestApproach use the fused path through context(). */
class ForceModel : public IForceModel {
public:
    static std::string& DataDirectory()
    {
        static std::string dir = std::getenv("GPOP_DATA_DIR") ? std::getenv("GPOP_DATA_DIR") : "../../data";
        return dir;
    }

    ForceModel(cublasHandle_t*, unsigned numEntities, double stepSize, FullPerturbationParameters* params)
        : _n(numEntities), _h(stepSize), _params(params)
    {
    }
    ~ForceModel() override
    {
        if (_frames)
            cudaFree(_frames);
        if (_tmp)
            cudaFree(_tmp);
        for (auto& kv : _contexts)
            gpop_destroy(kv.second);
    }
    ForceModel(const ForceModel&) = delete;
    ForceModel& operator=(const ForceModel&) = delete;

    void PreInitialize() override { context(7); }

    // RK8 midpoint epochs: (before + after) * 10 matrices (force_model.cu:47-51)
    void InitializeGeneration(int beforeEpoch, int afterEpoch) override
    {
        frames((beforeEpoch + afterEpoch) * 10, 1, beforeEpoch);
    }
    // step epochs: before + after + 1 matrices (force_model.cu:53-57)
    void InitializePropagation(int beforeEpoch, int afterEpoch) override
    {
        frames(beforeEpoch + afterEpoch + 1, 0, beforeEpoch);
    }
    // K matrix [N][3 x 10], column kIndex; table entry (stepNum' + 4) * 10 + kIndex with
    // stepNum' = stepNum - 1 for positive steps (force_model.cu:59-89)
    void ComputeGenerationAcceleration(
        double* devPosition, double*, double* devKMatrix, int stepNum, int kIndex) override
    {
        if (kIndex < 0 || kIndex >= 10)
            throw std::invalid_argument("kIndex must be between 0 and 9");
        const int s = stepNum > 0 ? stepNum - 1 : stepNum;
        evaluate(devPosition, (s + 4) * 10 + kIndex, devKMatrix + 3 * kIndex, 30);
    }
    // acceleration matrix [N][3 x 9], column returnColumnIndex; table entry stepNum
    // (force_model.cu:91-109)
    void ComputePropagationAcceleration(
        double* devPosition, double*, double* devAcceleration, int stepNum, int returnColumnIndex) override
    {
        evaluate(devPosition, stepNum, devAcceleration + 3 * returnColumnIndex, 27);
    }

    // The library context (FP64, numCorrections corrector passes), created on first use and kept
    // until the ForceModel is destroyed (propagators built on it may still be alive).
    gpop_ctx* context(int numCorrections)
    {
        for (auto& kv : _contexts)
            if (kv.first == numCorrections) {
                _ctx = kv.second;
                _ncorr = numCorrections;
                return _ctx;
            }
        gpop_config cfg;
        gpop_config_default(&cfg);
        cfg.data_dir = DataDirectory().c_str();
        cfg.n_corrections = numCorrections;
        gpop_ctx* c = nullptr;
        const gpop_status st = gpop_create(&cfg, &c);
        if (st != GPOP_OK) {
            const std::string msg = c ? gpop_last_error(c) : "";
            if (c)
                gpop_destroy(c);
            throw std::runtime_error("ForceModel: " + msg);
        }
        _contexts.push_back({ numCorrections, c });
        _ctx = c;
        _ncorr = numCorrections;
        return _ctx;
    }
    const FullPerturbationParameters* params() const { return _params; }
    double stepSize() const { return _h; }

private:
    unsigned _n;
    double _h;
    FullPerturbationParameters* _params;
    std::vector<std::pair<int, gpop_ctx*>> _contexts;
    gpop_ctx* _ctx = nullptr; // the most recently used of _contexts
    int _ncorr = 0;
    double* _frames = nullptr;
    int _count = 0;
    double* _tmp = nullptr;

    void frames(int count, int midpoints, int before)
    {
        gpop_ctx* c = context(_ncorr ? _ncorr : 7);
        if (_frames)
            cudaFree(_frames);
        _frames = nullptr;
        gpop_cpp::check_cuda(cudaMalloc(reinterpret_cast<void**>(&_frames), sizeof(double) * 9 * (size_t)count), "frame table");
        _count = count;
        const gpop_time t = gpop_cpp::to_time(_params->StartTimeUTC);
        gpop_cpp::check(c, gpop_frame_matrices(c, &t, _h, count, midpoints, before, _frames, nullptr, nullptr),
            "frame matrices");
    }
    void evaluate(const double* devPosition, int index, double* dst, int dst_stride)
    {
        if (!_frames || index < 0 || index >= _count)
            throw std::out_of_range("ForceModel: epoch index outside the initialized table");
        gpop_ctx* c = context(_ncorr ? _ncorr : 7);
        if (!_tmp)
            gpop_cpp::check_cuda(cudaMalloc(reinterpret_cast<void**>(&_tmp), sizeof(double) * 3 * _n), "acceleration buffer");
        gpop_cpp::check(c, gpop_gravity(c, _n, devPosition, _frames + (size_t)index * 9, _tmp, GPOP_FP64, nullptr),
            "gravity");
        gpop_cpp::check_cuda(cudaMemcpy2D(dst, sizeof(double) * dst_stride, _tmp, sizeof(double) * 3,
                                 sizeof(double) * 3, _n, cudaMemcpyDeviceToDevice),
            "acceleration column");
    }
};

namespace gpop_cpp {
inline ForceModel& library_model(IForceModel& m)
{
    ForceModel* f = dynamic_cast<ForceModel*>(&m);
    if (!f)
        throw std::invalid_argument("only the library's ForceModel runs on the fused propagation path");
    return *f;
}
} // namespace gpop_cpp

/* GpuPropagator (gpu_propagator.cuh:26-59): caller-owned device r, v ([N][3]) updated in place by
 * every Step(); the first Step() runs the startup. */
class GpuPropagator {
public:
    GpuPropagator(double* epochPositions, double* epochVelocities, unsigned numSatellites, cublasHandle_t*,
        double timeStep, FullPerturbationParameters* params, IForceModel& forceModel, int maxSteps,
        int numCorrections = 7)
        : _r(epochPositions), _v(epochVelocities), _n(numSatellites)
    {
        ForceModel& fm = gpop_cpp::library_model(forceModel);
        _ctx = fm.context(numCorrections);
        const gpop_time t = gpop_cpp::to_time(params->StartTimeUTC);
        gpop_cpp::check(_ctx,
            gpop_propagator_create(_ctx, &t, timeStep, maxSteps, numSatellites, _r, _v, &_p), "GpuPropagator");
    }
    ~GpuPropagator() { FreeAllMemory(); }
    GpuPropagator(const GpuPropagator&) = delete;
    GpuPropagator& operator=(const GpuPropagator&) = delete;

    // One step; optionally copies r, v to the host and the step's acceleration to
    // devAccelerationVector ([N][3]).
    void Step(double* hostPositions = nullptr, double* hostVelocities = nullptr,
        double* devAccelerationVector = nullptr)
    {
        if (!_p)
            throw std::runtime_error("GpuPropagator: memory already freed");
        double* acc = nullptr;
        if (devAccelerationVector) {
            if (!_acc)
                gpop_cpp::check_cuda(cudaMalloc(reinterpret_cast<void**>(&_acc), sizeof(double) * 3 * _n), "acceleration buffer");
            acc = _acc;
        }
        gpop_cpp::check(_ctx, gpop_propagator_step(_p, 1, nullptr, nullptr, acc, nullptr), "Step");
        if (acc) // [3][N] -> [N][3]
            for (int c = 0; c < 3; ++c)
                gpop_cpp::check_cuda(cudaMemcpy2D(devAccelerationVector + c, sizeof(double) * 3,
                                         _acc + (size_t)c * _n, sizeof(double), sizeof(double), _n,
                                         cudaMemcpyDeviceToDevice),
                    "acceleration copy");
        if (hostPositions || hostVelocities)
            CopyStateToHost(hostPositions, hostVelocities);
    }
    void CopyStateToHost(double* hostPositions, double* hostVelocities) const
    {
        if (hostPositions)
            gpop_cpp::check_cuda(
                cudaMemcpy(hostPositions, _r, sizeof(double) * 3 * _n, cudaMemcpyDeviceToHost), "copy r");
        if (hostVelocities)
            gpop_cpp::check_cuda(
                cudaMemcpy(hostVelocities, _v, sizeof(double) * 3 * _n, cudaMemcpyDeviceToHost), "copy v");
    }
    void FreeAllMemory()
    {
        if (_p)
            gpop_propagator_destroy(_p);
        _p = nullptr;
        if (_acc)
            cudaFree(_acc);
        _acc = nullptr;
    }

private:
    double* _r;
    double* _v;
    unsigned _n;
    gpop_ctx* _ctx = nullptr;
    gpop_propagator* _p = nullptr;
    double* _acc = nullptr;
};

/* Approach, ClosestApproachData (closest_approach/types.cuh:113-172) */
struct Approach {
    double distance;
    double time;
    double positionA[3];
    double positionB[3];
};

class ClosestApproachData {
    friend class ClosestApproach;
    std::vector<double> _d, _t, _pa, _pb;
    std::vector<uint32_t> _set, _offset, _higher;
    std::vector<uint64_t> _map;

public:
    // The closest approach of objA and objB; {-1, -1, ...} when not populated or not a screened
    // pair, zeros when objA == objB (types.cuh:153-169).
    Approach Get(unsigned objA, unsigned objB) const
    {
        const Approach bad { -1.0, -1.0, { -1.0, -1.0, -1.0 }, { -1.0, -1.0, -1.0 } };
        if (_d.empty())
            return bad;
        if (objA == objB)
            return { 0.0, 0.0, { 0.0, 0.0, 0.0 }, { 0.0, 0.0, 0.0 } };
        if (objA >= _set.size() || objB >= _set.size())
            return bad;
        const unsigned a = objA < objB ? objA : objB, b = objA < objB ? objB : objA;
        const uint32_t s = _set[a];
        if (_set[b] <= s)
            return bad;
        const uint64_t idx = _map[s] + (uint64_t)(a - _offset[s]) * _higher[s] + (b - _offset[s + 1]);
        return { _d[idx], _t[idx], { _pa[3 * idx], _pa[3 * idx + 1], _pa[3 * idx + 2] },
            { _pb[3 * idx], _pb[3 * idx + 1], _pb[3 * idx + 2] } };
    }
};

/* ClosestApproach (closest_approach.cuh:36-88) */
class ClosestApproach {
public:
    ClosestApproach(cublasHandle_t*, FullPerturbationParameters* params, IForceModel& forceModel, double stepSize)
        : _params(params), _model(&gpop_cpp::library_model(forceModel)), _h(stepSize)
    {
        if (!(stepSize > 0))
            throw std::invalid_argument("ClosestApproach: step size must be positive");
    }
    ~ClosestApproach()
    {
        if (_ca)
            gpop_ca_destroy(_ca);
    }
    ClosestApproach(const ClosestApproach&) = delete;
    ClosestApproach& operator=(const ClosestApproach&) = delete;

    void Initialize(const std::vector<std::array<double, 3>>& positions,
        const std::vector<std::array<double, 3>>& velocities, const std::vector<unsigned>& setIndices)
    {
        if (positions.size() != velocities.size() || positions.size() != setIndices.size())
            throw std::invalid_argument("ClosestApproach: sizes of positions, velocities and setIndices differ");
        _ctx = _model->context(7);
        if (_ca)
            gpop_ca_destroy(_ca);
        _ca = nullptr;
        const gpop_time t = gpop_cpp::to_time(_params->StartTimeUTC);
        gpop_cpp::check(_ctx,
            gpop_ca_create(_ctx, &t, _h, (int64_t)positions.size(), positions.data()->data(),
                velocities.data()->data(), setIndices.data(), &_ca),
            "ClosestApproach::Initialize");
        _set.assign(setIndices.begin(), setIndices.end());
    }
    void Propagate(int numSteps, bool = false)
    {
        gpop_cpp::check(_ctx, gpop_ca_propagate(_ca, numSteps), "ClosestApproach::Propagate");
    }
    void FindClosest(ClosestApproachData& out)
    {
        const int64_t P = gpop_ca_num_pairs(_ca);
        out._d.assign(P, 0.0);
        out._t.assign(P, 0.0);
        out._pa.assign(3 * P, 0.0);
        out._pb.assign(3 * P, 0.0);
        gpop_cpp::check(_ctx, gpop_ca_pairs(_ca, out._d.data(), out._t.data(), out._pa.data(), out._pb.data(), nullptr),
            "ClosestApproach::FindClosest");
        // PartitionParameters (partition_parameters.cuh:94-135): set offsets, objects above each
        // set, first pair index of each set
        out._set = _set;
        out._offset.assign(1, 0);
        out._higher.clear();
        out._map.assign(1, 0);
        for (size_t i = 1; i < _set.size(); ++i)
            if (_set[i] != _set[i - 1]) {
                const uint32_t size = (uint32_t)i - out._offset.back();
                out._higher.push_back((uint32_t)(_set.size() - i));
                out._offset.push_back((uint32_t)i);
                out._map.push_back(out._map.back() + (uint64_t)size * out._higher.back());
            }
        out._higher.push_back(0);
    }

private:
    FullPerturbationParameters* _params;
    ForceModel* _model;
    double _h;
    gpop_ctx* _ctx = nullptr;
    gpop_ca* _ca = nullptr;
    std::vector<uint32_t> _set;
};

#endif
