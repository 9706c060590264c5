// batch.cuh -- batched propagation of many independent requests (uneven object counts, durations,
// step sizes and gravity degrees) in one persistent launch.
#pragma once
#include "kernels.h"

#include <cstdint>

namespace gpop {

// One request after planning. Objects of all requests are flattened: request r owns objects
// [obj0, obj0 + n) of the batch state arrays.
struct BatchReq {
    int64_t obj0 = 0;
    int n = 0;
    int steps = 0;
    int L = 0; // gravity degree (<= the context's table degree)
    int lpo = 1; // lanes per object in the GJ8 walk (1, 2, 4, ..., 32)
    double h = 0;
    const double* gen_m = nullptr; // 80 x 9
    const double* prop_m = nullptr; // (steps + 5) x 9
};

// Work item: objects [first, first + count) of request req, all its steps, on one warp.
struct BatchItem {
    int req;
    int first;
    int count; // <= batch_item_objects(lpo)
};

// Objects per work item: two per lane with one lane per object, else 32 / lpo.
inline int batch_item_objects(int lpo) { return lpo == 1 ? 64 : 32 / lpo; }

struct BatchArgs {
    const BatchReq* reqs = nullptr;
    int n_req = 0;
    const BatchItem* items = nullptr;
    int n_items = 0;
    int* next_item = nullptr; // work-queue head (zeroed before the launch)
    const int* obj_req = nullptr; // request of each flattened object (startup kernel)
    int64_t n_obj = 0;
    int ncorr = 7;
    uint32_t flags = 0;
    double* state = nullptr; // kStateArrays x n_obj SoA
    const double* r0 = nullptr; // AoS [n_obj][3]
    const double* v0 = nullptr;
    double* r_out = nullptr; // AoS [n_obj][3]
    double* v_out = nullptr;
    unsigned* err = nullptr;
    int Ltab = 0; // degree of the staged table layout
    bool pair_walk = false; // two-object items walk two gravity columns at a time
};

cudaError_t launch_batch_startup(const TableSrc& ts, const BatchArgs& a, int num_sms, cudaStream_t s);
// lane_ts: the lane-layout table; plain_ts: the same model in the plain layout (batches of
// single-lane items). blocks: persistent grid size; block: threads per block.
cudaError_t launch_batch_gj8(const TableSrc& lane_ts, const TableSrc& plain_ts, const BatchArgs& a,
    int blocks, int block, cudaStream_t s);
cudaError_t launch_frames_batch(const FrameData& fd, const int* cal, const int* epoch_req,
    const double* sec_args, int count, double* m_out, cudaStream_t s);

} // namespace gpop
