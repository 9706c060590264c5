// variational.cuh -- state transition matrices (forward variational equations) and the adjoint of
// the GJ8 propagation with respect to the initial state, plus the closest approach of explicit
// object pairs with the gradient of its miss distance (FP64 throughout).
#pragma once
#include "kernels.h"

#include <cstdint>

namespace gpop {

constexpr int kVarLanes = 8; // lanes per object: 6 tangent directions + 2 that only share gravity
constexpr int kCheckpointSteps = 64; // GJ8 state saved every 64 steps for the reverse sweep
constexpr int kCheckpointArrays = 33; // s, S and the 9-slot history (state arrays kSs .. kHist + 26)

struct VarArgs {
    int64_t n = 0; // objects
    int steps = 0; // >= 1
    double h = 0;
    int ncorr = 7;
    uint32_t flags = 0;
    const double* gen_m = nullptr;
    const double* prop_m = nullptr;
    const double* r0 = nullptr; // AoS [n][3]
    const double* v0 = nullptr;
    double* r_out = nullptr; // AoS [n][3] (may be NULL)
    double* v_out = nullptr;
    double* phi = nullptr; // [n][6][6], phi[i][j] = d x_N,i / d x_0,j with x = (r, v)
    unsigned* err = nullptr;
};

// One adjoint unit: an object with cotangents ("seeds") on its trajectory (r, v, a) at up to three
// consecutive steps step0, step0 + 1, step0 + 2 (1-based; steps beyond the run are ignored).
struct AdjArgs {
    int64_t n_obj = 0;
    int64_t n_units = 0;
    const int* unit_obj = nullptr;
    const int* seed_step0 = nullptr;
    const double* seeds = nullptr; // [n_units][3 nodes][r 3 | v 3 | a 3]
    int steps = 0;
    double h = 0;
    int ncorr = 7;
    uint32_t flags = 0;
    const double* gen_m = nullptr;
    const double* prop_m = nullptr;
    const double* r0 = nullptr; // AoS [n_obj][3] initial state
    const double* v0 = nullptr;
    const double* ckpt = nullptr; // [segments][kCheckpointArrays][n_obj]; segment 0 = after startup
    double* scratch = nullptr; // [kCheckpointSteps][3][n_units] last evaluation point of each step
    double* grad = nullptr; // [n_units][6] d(seeded sum) / d(r0, v0)
    unsigned* err = nullptr;
};

// Closest approach of listed pairs over a stored trajectory ([steps][3][n] r, v, a) and the seeds
// of the miss-distance adjoint (units 2p and 2p + 1 = the pair's two objects).
struct PairArgs {
    int64_t n_obj = 0;
    int64_t n_pairs = 0;
    const int* pairs = nullptr; // [n_pairs][2]
    int steps = 0;
    double h = 0;
    const double* traj_r = nullptr;
    const double* traj_v = nullptr;
    const double* traj_a = nullptr;
    double* tca = nullptr; // [n_pairs]
    double* miss = nullptr;
    int* closest = nullptr; // trajectory index of the sampled minimum
    int* unit_obj = nullptr; // [2 n_pairs]
    int* seed_step0 = nullptr;
    double* seeds = nullptr; // [2 n_pairs][27]
};

cudaError_t launch_stm(const TableSrc& ts64, const VarArgs& a, cudaStream_t s);
cudaError_t launch_adjoint(const TableSrc& ts64, const AdjArgs& a, cudaStream_t s);
cudaError_t launch_pair_approach(const PairArgs& a, cudaStream_t s);
// Acceleration (may be NULL) and 3x3 Jacobian [n][3][3] at GCRS positions r [n][3] with the frame
// matrix M of gravity_gcrs (NULL = Earth-fixed positions, no rotation).
cudaError_t launch_jacobian(const TableSrc& ts64, int64_t n, const double* r, const double* M,
    double* acc, double* jac, unsigned* err, cudaStream_t s);

} // namespace gpop
