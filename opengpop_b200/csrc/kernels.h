// kernels.h -- host launchers of the device kernels (implemented in the .cu files).
#pragma once
#include "model.h"
#include <cstdint>
#include <cuda_runtime.h>

namespace gpop {

// Gravity table as staged into shared memory by each block.
struct TableSrc {
    const void* src = nullptr; // device: FP64 table, or [FP64 head (n <= 8) | FP32 table]
    uint32_t bytes = 0;
    uint32_t off32 = 0; // byte offset of the FP32 table (mixed mode)
    int L = 0;
    double radius = 0, gm = 0;
    bool mixed = false;
    bool lanes = false; // lane layout (build_lane_blob): column bases, FP64 at kLaneOff64, FP32 at off32
    // spins of the first bounded wait on the staging copy (2^22, about a second; a test setting
    // lowers it to make the wait give up on purpose)
    uint32_t wait_spins = 1u << 22;
};

// Byte offset, in a kernel's dynamic shared memory, of what follows a staged table (the 128-byte
// mbarrier slot and the table, rounded up to 16 bytes).
inline __host__ __device__ size_t stage_offset(const TableSrc& ts)
{
    return (128 + (size_t)ts.bytes + 15) & ~(size_t)15;
}

// Per-object propagation state, SoA: array k (n doubles each) at state + k * n.
enum StateSlot : int {
    kR = 0, kV = 3, kSs = 6, kSb = 9, kHist = 12, kRep = 39, kRepA = 63,
    kX0 = 75, // split block exchange (12 values per object) when it does not fit in shared memory
    kStateArrays = 87
};

struct PropArgs {
    int64_t n = 0;
    double h = 0;
    int ncorr = 7;
    double* state = nullptr; // kStateArrays * n
    const double* gen_m = nullptr; // 80 x 9
    const double* prop_m = nullptr; // (steps + 5) x 9, index i <-> (i - 4) h
    int kind = 0; // gpop_force_kind (0 = gravity)
    uint32_t flags = 0;
    unsigned* err = nullptr;
    // startup inputs (AoS [n][3]) and optional full startup matrices ([n][27] each)
    const double* r0 = nullptr;
    const double* v0 = nullptr;
    double* out27[5] = { nullptr, nullptr, nullptr, nullptr, nullptr };
    // GJ8 range and outputs
    int step_begin = 1, step_end = 1; // steps [begin, end), 1-based
    double* traj_r = nullptr; // [steps][3][n], indexed by step - traj_step0
    double* traj_v = nullptr;
    double* traj_a = nullptr;
    int traj_step0 = 1;
    double* out_r = nullptr; // AoS [n][3] written at the end of the range (may be NULL)
    double* out_v = nullptr;
    int64_t obj_lo = 0, obj_hi = -1; // lane kernel: objects [obj_lo, obj_hi) of n (-1: n)
    int split_owners = 0; // split block (gj8_kernel with SPLIT): owner warps of its 8
};

struct LaunchShape {
    int block = 0, grid = 0;
    size_t smem = 0;
};

size_t table_smem_bytes(const TableSrc& ts);
LaunchShape pick_shape(int64_t n, int max_block, int num_sms);
// Dynamic shared memory one block of the current device may opt in to (0 if it cannot be read).
size_t max_smem_optin();

cudaError_t launch_startup(const TableSrc& ts, const PropArgs& a, int num_sms, cudaStream_t s);
// How many objects a GJ8 thread carries through the gravity triangle walk (0 = by problem size).
// kWalkLanes: P lanes per object split the gravity columns (few objects; P from lanes_per_object).
// kWalkLanesTwo: P lanes per group of two objects (P from lane_pair_lanes, else 2), the default
// in the bands lane_pair_lanes names.
// kWalkTwoPlain: two objects per thread in a plain block, never the split block (for comparisons).
enum WalkMode : int {
    kWalkOneObject = 1, kWalkTwoObjects = 2, kWalkLanes = 3, kWalkLanesTwo = 4, kWalkTwoPlain = 5
};
// Lanes per object (1..32, a power of 2): the most that keep n objects in one wave of blocks of at
// most 384 threads, one per SM.
int lanes_per_object(int64_t n, int num_sms);
// Lanes per group of two objects (a power of 2 up to 32) where the default walk carries two objects
// per lane group, 0 elsewhere.
int lane_pair_lanes(int64_t n, int num_sms, bool fp64_gravity);
// The walk launch_gj8 takes for n objects when none is forced (lanes: a lane-layout table is at
// hand and the force is the gravity model; fp64_gravity: the FP64 build of it).
int default_walk(int64_t n, int num_sms, bool lanes, bool fp64_gravity);
// Owner warps of the split block two objects per thread take for n objects (0: a plain block).
int split_owner_warps(int64_t n, int num_sms, int L);
// lane_ts: the lane-layout table of the same precision (NULL: no lane-split walk).
cudaError_t launch_gj8(const TableSrc& ts, const PropArgs& a, int num_sms, cudaStream_t s,
    int block_override = 0, int walk = 0, const TableSrc* lane_ts = nullptr);
cudaError_t launch_gravity(const TableSrc& ts, int64_t n, const double* r, const double* m9,
    double* a, unsigned* err, int num_sms, cudaStream_t s);
cudaError_t launch_corrector_unit(int kind, double h, int op, double* r27, double* v27, double* a27,
    double* s27, double* S27, cudaStream_t s);
cudaError_t launch_predict_unit(int kind, double h, int step, double* r3, double* v3, double* a27,
    double* s3, double* S3, cudaStream_t s);
cudaError_t launch_finalize_unit(double h, double* r3, double* v3, const double* a27,
    const double* s3, const double* S3, cudaStream_t s);

// Frame matrices: epoch e uses calendar (y, mo, d, hh, mi) and seconds argument sec_args[e].
struct FrameData {
    const NutTerm* nut = nullptr; // [lon0 | lon1 | obl0 | obl1]
    int n_lon0 = 0, n_lon1 = 0, n_obl0 = 0, n_obl1 = 0;
    const EopRec* eop = nullptr;
    int n_eop = 0;
    const double* leap_mjd = nullptr;
    const double* leap_val = nullptr;
    int n_leap = 0;
};
cudaError_t launch_frames(const FrameData& fd, int y, int mo, int d, int hh, int mi,
    const double* sec_args, int count, double* m_out, double* mjd_out, cudaStream_t s);

} // namespace gpop
