// screen.cu -- pairwise closest-approach screen and TCA refinement
// (lib/closest_approach/src/device.cu:56-173, utility/interpolation.cuh:27-152).
//
// Screen: the reference launches one thread per pair per step (UpdateClosestApproachKernel), each
// copying up to 54 doubles of node states on every new minimum and racing on a shared "last" array.
// Here a block owns a 64 x 64 tile of (a, b) object pairs and walks every step of a phase: the
// positions of its 128 objects are staged into shared memory 16 steps at a time from the
// trajectory store (asynchronous copies, double-buffered, so the next chunk loads while this one
// is screened), each thread keeps the running minimum of the squared distance and its step for a
// 4 x 4 micro-tile in registers, and writes once at the end. Squared distances are compared
// with the reference's strict "<", so the first step attaining the minimum wins as in the
// reference (sqrt is monotonic). Node states for the refinement are read back from the trajectory
// store, so "before" is always the previous step's state (no race).
#include "kernels.h"
#include "screen.h"
#include "hermite.cuh"

#include <cfloat>
#include <cstdint>

namespace gpop {

constexpr int kTileA = kScreenTileA; // rows (first objects) per tile
constexpr int kTileB = kScreenTileB; // columns (second objects) per tile
constexpr int kSub = 4; // rows per thread
constexpr int kSubB = kScreenSubB; // columns per thread (strided by 16)
constexpr int kRow = kTileA + kTileB; // doubles per staged (step, axis) row: a tile, then b tile
constexpr int kStepChunk = 16; // steps staged per pass
// shared memory: two chunk buffers of [step][axis][a tile | b tile] doubles
constexpr int kChunkDoubles = kStepChunk * 3 * kRow;
constexpr size_t kScreenSmem = 2 * (size_t)kChunkDoubles * sizeof(double);


__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Issues the asynchronous copies of steps [k0, k0 + kc) of the a and b tiles into buf
// (cp.async, 8 bytes each: rows start on any double, so no 16-byte alignment is assumed).
// Objects past n read object n - 1 (their pairs are masked).
__device__ __forceinline__ void stage_chunk(double* buf, const double* __restrict__ traj, int64_t N,
    int a0, int b0, int k0, int kc)
{
    for (int e = threadIdx.x; e < kc * 3 * kRow; e += blockDim.x) {
        const int w = e % kRow; // place in the row: a tile then b tile
        const int c = (e / kRow) % 3;
        const int k = e / (3 * kRow);
        int64_t obj = w < kTileA ? a0 + w : b0 + (w - kTileA);
        obj = obj < N ? obj : N - 1;
        const double* src = traj + ((int64_t)(k0 + k) * 3 + c) * N + obj;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(buf + e)), "l"(src)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Running minimum of the squared distance per pair: the thread's 4 x 4 pairs are
// a = a0 + ty*4 + i (contiguous, read as broadcast double2 pairs) and b = b0 + tx + 16 j (strided, so
// the 16 lanes of a half warp read 16 consecutive doubles: no bank conflicts). The running minimum
// is compared in FP64 (one compare on the FP64 pipe; an integer compare of the bit patterns, which
// orders non-negative doubles the same way, measured 9 % slower on B200: it loads the ALU pipe
// that the three selects of the minimum already use).
__global__ void __launch_bounds__(256) screen_kernel(ScreenArgs a)
{
    extern __shared__ __align__(16) double sbuf[];
    const int2 tile = a.tiles[blockIdx.x];
    const int a0 = tile.x, b0 = tile.y;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int64_t N = a.n;
    double best[kSub][kSubB];
    uint32_t bstep[kSub][kSubB];
#pragma unroll
    for (int i = 0; i < kSub; ++i) {
        const int ai = a0 + ty * kSub + i;
        const int bound = ai < N ? a.bound[ai] : (int)N;
        const int64_t base = ai < N ? a.base[ai] : 0;
#pragma unroll
        for (int j = 0; j < kSubB; ++j) {
            const int bj = b0 + tx + 16 * j;
            best[i][j] = DBL_MAX;
            bstep[i][j] = 0xFFFFFFFFu;
            if (ai < N && bj < N && bj >= bound && a.init == 0) {
                best[i][j] = a.min_d2[base + bj];
                bstep[i][j] = a.min_step[base + bj];
            }
        }
    }
    const int nchunks = (a.step_hi - a.step_lo + kStepChunk - 1) / kStepChunk;
    if (nchunks > 0)
        stage_chunk(sbuf, a.traj_r, N, a0, b0, a.step_lo, min(kStepChunk, a.step_hi - a.step_lo));
    for (int ch = 0; ch < nchunks; ++ch) {
        const int k0 = a.step_lo + ch * kStepChunk;
        const int kc = min(kStepChunk, a.step_hi - k0);
        if (ch + 1 < nchunks) { // the next chunk's copies fly while this chunk is screened
            const int k1 = k0 + kStepChunk;
            stage_chunk(sbuf + ((ch + 1) & 1) * kChunkDoubles, a.traj_r, N, a0, b0, k1,
                min(kStepChunk, a.step_hi - k1));
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        const double* buf = sbuf + (ch & 1) * kChunkDoubles;
        for (int k = 0; k < kc; ++k) {
            const double* row = buf + k * 3 * kRow; // [axis][a tile | b tile]
            double ax[kSub], ay[kSub], az[kSub], bx[kSubB], by[kSubB], bz[kSubB];
#pragma unroll
            for (int i = 0; i < kSub; i += 2) {
                const double2 x = *reinterpret_cast<const double2*>(row + 0 * kRow + ty * kSub + i);
                const double2 y = *reinterpret_cast<const double2*>(row + 1 * kRow + ty * kSub + i);
                const double2 z = *reinterpret_cast<const double2*>(row + 2 * kRow + ty * kSub + i);
                ax[i] = x.x;
                ax[i + 1] = x.y;
                ay[i] = y.x;
                ay[i + 1] = y.y;
                az[i] = z.x;
                az[i + 1] = z.y;
            }
#pragma unroll
            for (int j = 0; j < kSubB; ++j) {
                bx[j] = row[0 * kRow + kTileA + tx + 16 * j];
                by[j] = row[1 * kRow + kTileA + tx + 16 * j];
                bz[j] = row[2 * kRow + kTileA + tx + 16 * j];
            }
            const uint32_t step = (uint32_t)(a.step_offset + k0 + k);
#pragma unroll
            for (int i = 0; i < kSub; ++i)
#pragma unroll
                for (int j = 0; j < kSubB; ++j) {
                    const double dx = ax[i] - bx[j];
                    const double dy = ay[i] - by[j];
                    const double dz = az[i] - bz[j];
                    const double d2 = dx * dx + dy * dy + dz * dz;
                    if (d2 < best[i][j]) {
                        best[i][j] = d2;
                        bstep[i][j] = step;
                    }
                }
        }
        __syncthreads(); // the buffer is staged again two chunks on
    }
#pragma unroll
    for (int i = 0; i < kSub; ++i) {
        const int ai = a0 + ty * kSub + i;
        if (ai >= N)
            continue;
        const int bound = a.bound[ai];
        const int64_t base = a.base[ai];
#pragma unroll
        for (int j = 0; j < kSubB; ++j) {
            const int bj = b0 + tx + 16 * j;
            if (bj < N && bj >= bound) {
                a.min_d2[base + bj] = best[i][j];
                a.min_step[base + bj] = bstep[i][j];
            }
        }
    }
}

__global__ void __launch_bounds__(128) refine_kernel(RefineArgs a)
{
    const int64_t idx = a.pair_lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= a.pair_hi)
        return;
    // pair index -> (a, b): binary search of the set whose map range holds idx
    // (inverse of PartitionParameters::GetPartitionMapIdx, partition_parameters.cuh:50-91)
    int lo = 0, hi = a.num_sets - 2;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (a.map_offsets[mid] <= (uint64_t)idx)
            lo = mid;
        else
            hi = mid - 1;
    }
    const uint64_t rel = (uint64_t)idx - a.map_offsets[lo];
    const int64_t oa = (int64_t)(rel / a.num_higher[lo]) + a.set_offsets[lo];
    const int64_t ob = (int64_t)(rel % a.num_higher[lo]) + a.set_offsets[lo + 1];
    const uint32_t cs = a.min_step[idx];
    const int64_t N = a.n;
    const double h = a.h;
    double dist = sqrt(a.min_d2[idx]);
    double tca;
    double pa[3], pb[3];
    // CalculateClosestApproachesKernel (device.cu:100-110): minimum on the first or last screened
    // step is not refined; the sampled positions of that step are reported.
    if (cs == 0 || cs == a.total_steps - 1 || cs == 0xFFFFFFFFu) {
        tca = (cs == 0 || cs == 0xFFFFFFFFu) ? 0.0 : (double)a.total_steps * h;
        const int64_t k = (cs == 0xFFFFFFFFu) ? 0 : cs;
        for (int c = 0; c < 3; ++c) {
            pa[c] = a.traj_r[(k * 3 + c) * N + oa];
            pb[c] = a.traj_r[(k * 3 + c) * N + ob];
        }
    } else {
        Pair6 P;
        P.dt = h;
        for (int c = 0; c < 3; ++c) {
            double q[2][9];
            for (int node = 0; node < 3; ++node) {
                const int64_t k = (int64_t)cs - 1 + node;
                const int64_t ra = (k * 3 + c) * N;
                q[0][node * 3 + 0] = a.traj_r[ra + oa];
                q[0][node * 3 + 1] = a.traj_v[ra + oa];
                q[0][node * 3 + 2] = a.traj_a[ra + oa];
                q[1][node * 3 + 0] = a.traj_r[ra + ob];
                q[1][node * 3 + 1] = a.traj_v[ra + ob];
                q[1][node * 3 + 2] = a.traj_a[ra + ob];
            }
            herm_build(P.A[c], q[0][0], q[0][1], q[0][2], q[0][3], q[0][4], q[0][5], q[0][6],
                q[0][7], q[0][8], h);
            herm_build(P.B[c], q[1][0], q[1][1], q[1][2], q[1][3], q[1][4], q[1][5], q[1][6],
                q[1][7], q[1][8], h);
        }
        const double t = find_root(P, 0.0, h);
        tca = t + (double)cs * h;
        double d2 = 0.0;
        for (int c = 0; c < 3; ++c) {
            pa[c] = herm_eval(P.A[c], h, t);
            pb[c] = herm_eval(P.B[c], h, t);
            const double d = pa[c] - pb[c];
            d2 += d * d;
        }
        dist = sqrt(d2);
    }
    a.dist[idx] = dist;
    a.time[idx] = tca;
    for (int c = 0; c < 3; ++c) {
        a.pos_a[idx * 3 + c] = pa[c];
        a.pos_b[idx * 3 + c] = pb[c];
    }
}

// Pairs whose refined distance is below the threshold, appended in any order.
__global__ void select_kernel(const double* dist, int64_t num_pairs, double threshold,
    unsigned long long* count, int64_t* out, int64_t capacity)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= num_pairs)
        return;
    if (dist[idx] < threshold) {
        const unsigned long long slot = atomicAdd(count, 1ull);
        if ((int64_t)slot < capacity)
            out[slot] = idx;
    }
}

cudaError_t launch_screen(const ScreenArgs& a, int num_tiles, cudaStream_t s)
{
    if (num_tiles <= 0 || a.step_hi <= a.step_lo)
        return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(screen_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)kScreenSmem);
    if (e != cudaSuccess)
        return e;
    screen_kernel<<<num_tiles, 256, kScreenSmem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_refine(const RefineArgs& a, cudaStream_t s)
{
    if (a.pair_lo < 0 || a.pair_hi > a.num_pairs || a.pair_hi <= a.pair_lo)
        return cudaSuccess;
    const int64_t blocks = (a.pair_hi - a.pair_lo + 127) / 128;
    refine_kernel<<<(unsigned)blocks, 128, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_select(const double* dist, int64_t num_pairs, double threshold,
    unsigned long long* count, int64_t* out, int64_t capacity, cudaStream_t s)
{
    if (num_pairs <= 0)
        return cudaSuccess;
    select_kernel<<<(unsigned)((num_pairs + 255) / 256), 256, 0, s>>>(dist, num_pairs, threshold,
        count, out, capacity);
    return cudaGetLastError();
}

} // namespace gpop
