// screen.h -- closest-approach screen / refinement launch arguments.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gpop {

// Screen tile: 64 rows (first objects) x kScreenTileB columns (second objects); each thread holds
// 4 rows x kScreenSubB columns of pairs. Measured on B200 (20,000 objects, 2,000 against all, 8,640
// steps): 4 columns 0.207 s, 8 columns 0.224 s (238 registers, 144 KB of staging).
#ifndef GPOP_SCREEN_SUBB
#define GPOP_SCREEN_SUBB 4
#endif
constexpr int kScreenSubB = GPOP_SCREEN_SUBB;
constexpr int kScreenTileA = 64;
constexpr int kScreenTileB = 16 * kScreenSubB;

struct ScreenArgs {
    int64_t n = 0; // objects
    const double* traj_r = nullptr; // trajectory store positions [step][3][n]
    const int* bound = nullptr; // per object a: first b of a higher set (n if none)
    const int64_t* base = nullptr; // per object a: pair index of (a, b) = base[a] + b
    const int2* tiles = nullptr; // (a0, b0) of each 64 x 64 tile
    double* min_d2 = nullptr; // per pair running minimum of the squared distance
    uint32_t* min_step = nullptr; // per pair step of that minimum
    int step_lo = 0, step_hi = 0; // store rows screened by this launch
    int64_t step_offset = 0; // screened-step number of store row 0
    int init = 0; // 1: ignore the stored minima (first phase)
};

struct RefineArgs {
    int64_t n = 0;
    int64_t num_pairs = 0;
    int64_t pair_lo = 0, pair_hi = 0; // pairs refined by this launch: [pair_lo, pair_hi)
    int num_sets = 0;
    const uint32_t* set_offsets = nullptr;
    const uint32_t* num_higher = nullptr;
    const uint64_t* map_offsets = nullptr;
    const double* traj_r = nullptr;
    const double* traj_v = nullptr;
    const double* traj_a = nullptr;
    const double* min_d2 = nullptr;
    const uint32_t* min_step = nullptr;
    uint32_t total_steps = 0;
    double h = 0;
    double* dist = nullptr;
    double* time = nullptr;
    double* pos_a = nullptr;
    double* pos_b = nullptr;
};

cudaError_t launch_screen(const ScreenArgs& a, int num_tiles, cudaStream_t s);
cudaError_t launch_refine(const RefineArgs& a, cudaStream_t s);
cudaError_t launch_select(const double* dist, int64_t num_pairs, double threshold,
    unsigned long long* count, int64_t* out, int64_t capacity, cudaStream_t s);

} // namespace gpop
