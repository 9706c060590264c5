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
 *  - GpuPropagator runs the fused library path with the library's ForceModel; with any other
 *    IForceModel it calls the model's virtual hooks per evaluation as the reference does (GpuStartup,
 *    Predictor and the corrector, with the integrator arithmetic in the library's kernels);
 *  - ClosestApproach does the same per phase, feeding the library's screen and refinement step
 *    by step (that path makes a library context from ForceModel::DataDirectory());
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
#include <memory>
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
// A device array of doubles owned by one of the classes below.
struct DevArray {
    double* p = nullptr;
    DevArray() = default;
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    ~DevArray() { release(); }
    void alloc(size_t count, const char* what)
    {
        release();
        check_cuda(cudaMalloc(reinterpret_cast<void**>(&p), sizeof(double) * (count ? count : 1)), what);
    }
    void release()
    {
        if (p)
            cudaFree(p);
        p = nullptr;
    }
};
inline void check_step(gpop_status st, const char* what) { check(nullptr, st, what); }
} // namespace gpop_cpp

/* FullStartupData (gpu_startup/include/gpu_startup/gpu_startup.cuh): the startup's device matrices
 * ([N][9][3]: s, S, accelerations, positions, velocities) and the Gauss-Jackson / summed-Adams
 * ordinate tables (devA, devB: 90 doubles, entry 10 k + c). The GpuStartup that returned them
 * owns them. */
struct FullStartupData {
    double* devBigS;
    double* devSmallS;
    double* devAccelerationMatrix;
    double* devPositionMatrix;
    double* devVelocityMatrix;
    double* devA;
    double* devB;
};

/* GpuStartup (gpu_startup.cuh:95-120, gpu_startup.cu:33-68, 146-318): RK8 four steps either side
 * of the epoch, then the mid-corrector, for any IForceModel: the model's hooks are called per
 * evaluation in the reference's order and with its arguments, the integrator arithmetic between
 * them runs in the library's kernels. devPositions, devVelocities: the epoch state [N][3]. */
class GpuStartup {
public:
    GpuStartup(double* devPositions, double* devVelocities, unsigned numSatellites, cublasHandle_t*,
        double timeStep, IForceModel& forceModel, int maxPropagationSteps, int numCorrections = 7)
        : _r(devPositions), _v(devVelocities), _n(numSatellites), _h(timeStep), _model(forceModel),
          _maxSteps(maxPropagationSteps), _ncorr(numCorrections)
    {
        if (numSatellites == 0 || numCorrections <= 0 || !(timeStep > 0))
            throw std::invalid_argument("GpuStartup: need objects, corrector passes and a positive step");
        const size_t n = numSatellites;
        for (gpop_cpp::DevArray* m : { &_R, &_V, &_A, &_s, &_S })
            m->alloc(27 * n, "startup matrices");
        _Kx.alloc(30 * n, "RK8 stages");
        _Kv.alloc(30 * n, "RK8 stages");
        _x.alloc(3 * n, "stage state");
        _vt.alloc(3 * n, "stage state");
        _ta.alloc(90, "GJ8 tables");
        _tb.alloc(90, "GJ8 tables");
        forceModel.PreInitialize();
    }
    GpuStartup(const GpuStartup&) = delete;
    GpuStartup& operator=(const GpuStartup&) = delete;

    FullStartupData Startup()
    {
        using gpop_cpp::check_step;
        _model.InitializeGeneration(4, 4);
        check_step(gpop_startup_init(nullptr, _n, _r, _v, _R.p, _V.p, _A.p, _s.p, _S.p, nullptr), "startup");
        for (int i = 1; i <= 4; ++i) // StartupPredictor::Predict: steps 1, -1, 2, -2, ...
            for (int step : { i, -i }) {
                for (int k = 0; k < 10; ++k) {
                    check_step(gpop_rk8_stage(nullptr, _n, _h, step, k, _R.p, _V.p, _Kx.p, _Kv.p, _x.p, _vt.p,
                                   nullptr),
                        "RK8 stage");
                    _model.ComputeGenerationAcceleration(_x.p, _vt.p, _Kv.p, step, k);
                }
                check_step(gpop_rk8_finish(nullptr, _n, _h, step, _R.p, _V.p, _Kx.p, _Kv.p, nullptr), "RK8 step");
            }
        _model.InitializePropagation(4, _maxSteps);
        accelerations(true); // StartupCorrector: CalculateAccelerationMatrix(true)
        for (int c = 0; c < _ncorr; ++c) {
            check_step(gpop_startup_correct(nullptr, _n, _h, _R.p, _V.p, _A.p, _s.p, _S.p, nullptr), "corrector");
            accelerations(false);
        }
        check_step(gpop_gj8_coefficients(nullptr, _ta.p, _tb.p, nullptr), "GJ8 tables");
        return FullStartupData { _S.p, _s.p, _A.p, _R.p, _V.p, _ta.p, _tb.p };
    }

private:
    double* _r;
    double* _v;
    int64_t _n;
    double _h;
    IForceModel& _model;
    int _maxSteps, _ncorr;
    gpop_cpp::DevArray _R, _V, _A, _s, _S, _Kx, _Kv, _x, _vt, _ta, _tb;

    // StartupCorrector::CalculateAccelerationMatrix (gpu_startup.cu:196-224): column i of the
    // acceleration matrix at column i of the state, epoch column only when asked
    void accelerations(bool epoch)
    {
        using gpop_cpp::check_step;
        for (int i = 0; i < 9; ++i) {
            if (i == 4 && !epoch)
                continue;
            check_step(gpop_matrix_column(nullptr, _n, _R.p, 9, i, _x.p, 0, nullptr), "state column");
            check_step(gpop_matrix_column(nullptr, _n, _V.p, 9, i, _vt.p, 0, nullptr), "state column");
            _model.ComputePropagationAcceleration(_x.p, _vt.p, _A.p, i, i);
        }
    }
};

/* Predictor (gpu_integrator/include/gpu_integrator/prediction.cuh:23-46): the GJ8 predictor, then
 * the model's acceleration at the predicted state into column 8 of the acceleration matrix. devA,
 * devB are accepted for the reference's signature; the library's kernels carry the same tables. */
class Predictor {
public:
    Predictor(IForceModel& forceModel, cublasHandle_t*, int numSatellites, double stepSize)
        : _model(forceModel), _n(numSatellites), _h(stepSize)
    {
        if (numSatellites <= 0 || !(stepSize > 0))
            throw std::invalid_argument("Predictor: need objects and a positive step");
        _prev.alloc(3 * (size_t)numSatellites, "corrector vectors");
        _sum1.alloc(3 * (size_t)numSatellites, "corrector vectors");
        _sum2.alloc(3 * (size_t)numSatellites, "corrector vectors");
    }
    Predictor(const Predictor&) = delete;
    Predictor& operator=(const Predictor&) = delete;

    void SetPointers(double* devPositionVector, double* devVelocityVector, double* devAccelerationMatrix,
        double* /*devA*/, double* /*devB*/, double* devSmallSVector, double* devBigSVector)
    {
        _r = devPositionVector;
        _v = devVelocityVector;
        _a = devAccelerationMatrix;
        _s = devSmallSVector;
        _S = devBigSVector;
    }
    void Predict(int stepNum)
    {
        if (!_r || !_v || !_a || !_s || !_S)
            throw std::runtime_error("Predictor: SetPointers first");
        gpop_cpp::check_step(
            gpop_gj8_predict(nullptr, _n, _h, _r, _v, _a, _s, _S, _prev.p, _sum1.p, _sum2.p, nullptr), "predictor");
        _model.ComputePropagationAcceleration(_r, _v, _a, stepNum + 4, 8);
    }
    // One corrector pass of GpuPropagator::Correct after the model wrote column 8 (the sums of the
    // pass come from the last Predict).
    void CorrectPass()
    {
        gpop_cpp::check_step(
            gpop_gj8_correct(nullptr, _n, _h, _r, _v, _a, _s, _S, _prev.p, _sum1.p, _sum2.p, nullptr), "corrector");
    }

private:
    IForceModel& _model;
    int64_t _n;
    double _h;
    double *_r = nullptr, *_v = nullptr, *_a = nullptr, *_s = nullptr, *_S = nullptr;
    gpop_cpp::DevArray _prev, _sum1, _sum2;
};

/* GpuPropagator (gpu_propagator.cuh:26-59): caller-owned device r, v ([N][3]) updated in place by
 * every Step(); the first Step() runs the startup. With the library's ForceModel the steps run in
 * the fused kernels; with any other IForceModel they follow the reference's per-evaluation path:
 * GpuStartup, then per step Predictor::Predict and numCorrections corrector passes, each after a
 * call of the model's ComputePropagationAcceleration (gpu_propagator.cu:29-117). */
class GpuPropagator {
public:
    GpuPropagator(double* epochPositions, double* epochVelocities, unsigned numSatellites, cublasHandle_t*,
        double timeStep, FullPerturbationParameters* params, IForceModel& forceModel, int maxSteps,
        int numCorrections = 7)
        : _r(epochPositions), _v(epochVelocities), _n(numSatellites)
    {
        if (ForceModel* fm = dynamic_cast<ForceModel*>(&forceModel)) {
            _ctx = fm->context(numCorrections);
            const gpop_time t = gpop_cpp::to_time(params->StartTimeUTC);
            gpop_cpp::check(_ctx,
                gpop_propagator_create(_ctx, &t, timeStep, maxSteps, numSatellites, _r, _v, &_p), "GpuPropagator");
            return;
        }
        _model = &forceModel;
        _ncorr = numCorrections;
        _startup.reset(new GpuStartup(epochPositions, epochVelocities, numSatellites, nullptr, timeStep,
            forceModel, maxSteps, numCorrections));
        _predictor.reset(new Predictor(forceModel, nullptr, (int)numSatellites, timeStep));
        _gs.alloc(3 * (size_t)numSatellites, "s vector");
        _gS.alloc(3 * (size_t)numSatellites, "S vector");
    }
    ~GpuPropagator() { FreeAllMemory(); }
    GpuPropagator(const GpuPropagator&) = delete;
    GpuPropagator& operator=(const GpuPropagator&) = delete;

    // One step; optionally copies r, v to the host and the step's acceleration to
    // devAccelerationVector ([N][3]).
    void Step(double* hostPositions = nullptr, double* hostVelocities = nullptr,
        double* devAccelerationVector = nullptr)
    {
        if (_model) {
            generic_step(devAccelerationVector);
        } else {
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
        }
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
        _predictor.reset();
        _startup.reset();
        _gs.release();
        _gS.release();
        _freed = _model != nullptr;
    }

private:
    double* _r;
    double* _v;
    unsigned _n;
    gpop_ctx* _ctx = nullptr;
    gpop_propagator* _p = nullptr;
    double* _acc = nullptr;
    // the per-evaluation path (any IForceModel other than the library's)
    IForceModel* _model = nullptr;
    int _ncorr = 0;
    int _step = 1;
    bool _freed = false;
    std::unique_ptr<GpuStartup> _startup;
    std::unique_ptr<Predictor> _predictor;
    FullStartupData _data {};
    gpop_cpp::DevArray _gs, _gS;

    void generic_step(double* devAccelerationVector)
    {
        using gpop_cpp::check_step;
        if (_freed || !_startup)
            throw std::runtime_error("GpuPropagator: memory already freed");
        if (_step == 1) { // startup; s and S of the last startup column (CopySKernel)
            _data = _startup->Startup();
            check_step(gpop_matrix_column(nullptr, _n, _data.devSmallS, 9, 8, _gs.p, 0, nullptr), "s vector");
            check_step(gpop_matrix_column(nullptr, _n, _data.devBigS, 9, 8, _gS.p, 0, nullptr), "S vector");
            _predictor->SetPointers(_r, _v, _data.devAccelerationMatrix, _data.devA, _data.devB, _gs.p, _gS.p);
        }
        if (_step <= 4) { // CopyStartupStateKernel: the startup's column step + 4
            check_step(gpop_matrix_column(nullptr, _n, _data.devPositionMatrix, 9, _step + 4, _r, 0, nullptr), "state");
            check_step(gpop_matrix_column(nullptr, _n, _data.devVelocityMatrix, 9, _step + 4, _v, 0, nullptr), "state");
        } else {
            _predictor->Predict(_step);
            for (int i = 0; i < _ncorr; ++i) {
                _model->ComputePropagationAcceleration(_r, _v, _data.devAccelerationMatrix, _step + 4, 8);
                _predictor->CorrectPass();
            }
        }
        if (devAccelerationVector) // MoveColumnToVectorKernel: column 8
            check_step(gpop_matrix_column(nullptr, _n, _data.devAccelerationMatrix, 9, 8, devAccelerationVector, 0,
                           nullptr),
                "acceleration");
        gpop_cpp::check_cuda(cudaDeviceSynchronize(), "step");
        ++_step;
    }
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

/* ClosestApproach (closest_approach.cuh:36-88). With the library's ForceModel each phase runs in
 * the fused kernels; with any other IForceModel each phase is a per-evaluation GpuPropagator whose
 * steps (positions, velocities and exported accelerations) feed the library's screen one step at a
 * time (closest_approach.cu:129-157). The screen and refinement then need a library context, which
 * is made from ForceModel::DataDirectory(). */
class ClosestApproach {
public:
    ClosestApproach(cublasHandle_t*, FullPerturbationParameters* params, IForceModel& forceModel, double stepSize)
        : _params(params), _model(dynamic_cast<ForceModel*>(&forceModel)), _h(stepSize)
    {
        if (!(stepSize > 0))
            throw std::invalid_argument("ClosestApproach: step size must be positive");
        if (!_model)
            _any = &forceModel;
    }
    ~ClosestApproach()
    {
        if (_ca)
            gpop_ca_destroy(_ca);
        if (_own)
            gpop_destroy(_own);
    }
    ClosestApproach(const ClosestApproach&) = delete;
    ClosestApproach& operator=(const ClosestApproach&) = delete;

    void Initialize(const std::vector<std::array<double, 3>>& positions,
        const std::vector<std::array<double, 3>>& velocities, const std::vector<unsigned>& setIndices)
    {
        if (positions.size() != velocities.size() || positions.size() != setIndices.size())
            throw std::invalid_argument("ClosestApproach: sizes of positions, velocities and setIndices differ");
        if (_ca)
            gpop_ca_destroy(_ca);
        _ca = nullptr;
        _steps = 0;
        const int64_t n = (int64_t)positions.size();
        if (_model) {
            _ctx = _model->context(7);
            const gpop_time t = gpop_cpp::to_time(_params->StartTimeUTC);
            gpop_cpp::check(_ctx,
                gpop_ca_create(_ctx, &t, _h, n, positions.data()->data(), velocities.data()->data(),
                    setIndices.data(), &_ca),
                "ClosestApproach::Initialize");
        } else {
            if (!_own) {
                gpop_config cfg;
                gpop_config_default(&cfg);
                cfg.data_dir = ForceModel::DataDirectory().c_str();
                const gpop_status st = gpop_create(&cfg, &_own);
                if (st != GPOP_OK) {
                    const std::string msg = _own ? gpop_last_error(_own) : "";
                    if (_own)
                        gpop_destroy(_own);
                    _own = nullptr;
                    throw std::runtime_error("ClosestApproach: " + msg);
                }
            }
            _ctx = _own;
            gpop_cpp::check(_ctx,
                gpop_ca_create_external(_ctx, _h, n, positions.data()->data(), velocities.data()->data(),
                    setIndices.data(), &_ca),
                "ClosestApproach::Initialize");
            _dr.alloc(3 * (size_t)n, "positions");
            _dv.alloc(3 * (size_t)n, "velocities");
            _da.alloc(3 * (size_t)n, "accelerations");
            gpop_cpp::check_cuda(cudaMemcpy(_dr.p, positions.data()->data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice),
                "positions");
            gpop_cpp::check_cuda(cudaMemcpy(_dv.p, velocities.data()->data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice),
                "velocities");
        }
        _set.assign(setIndices.begin(), setIndices.end());
    }
    void Propagate(int numSteps, bool = false)
    {
        if (!_ca)
            throw std::runtime_error("ClosestApproach: Initialize first");
        if (_model) {
            gpop_cpp::check(_ctx, gpop_ca_propagate(_ca, numSteps), "ClosestApproach::Propagate");
            return;
        }
        if (numSteps <= 0)
            throw std::invalid_argument("ClosestApproach: number of steps must be positive");
        // a new propagator from the current state for every phase; the store is sized once for
        // the phase's steps, which are screened one at a time
        gpop_cpp::check(_ctx, gpop_ca_reserve(_ca, _steps + numSteps), "ClosestApproach::Propagate");
        GpuPropagator prop(_dr.p, _dv.p, (unsigned)_set.size(), nullptr, _h, _params, *_any, numSteps);
        for (int step = 0; step < numSteps; ++step, ++_steps) {
            prop.Step(nullptr, nullptr, _da.p);
            gpop_cpp::check(_ctx, gpop_ca_append(_ca, 1, _dr.p, _dv.p, _da.p), "ClosestApproach::Propagate");
        }
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
    ForceModel* _model; // the library's model (fused path), or null
    IForceModel* _any = nullptr; // any other model (per-evaluation path)
    double _h;
    gpop_ctx* _ctx = nullptr;
    gpop_ctx* _own = nullptr; // the context of the per-evaluation path
    gpop_ca* _ca = nullptr;
    std::vector<uint32_t> _set;
    int _steps = 0; // steps screened so far (per-evaluation path)
    gpop_cpp::DevArray _dr, _dv, _da;
};

#endif
