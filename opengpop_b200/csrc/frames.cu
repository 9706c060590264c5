// frames.cu -- per-epoch ITRS->GCRS matrix table on the device (replaces TimePointParamsKernel and
// the seven batched 3x3 GEMMs of lib/force_model/src/time_points.cu:26-71,146-201).
//
// One warp per epoch: the 2,414 nutation terms (IERS 2010 Tables 5.3a/b, both j = 0 and j = 1
// series for longitude and obliquity) are split across the 32 lanes and combined by a fixed-order
// shuffle reduction; lane 0 then evaluates EOP, leap seconds, precession, GAST and the matrix chain.
#include "frames.cuh"
#include "kernels.h"

namespace gpop {

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ double series_sum(const NutTerm* terms, int count, const double* F, int lane)
{
    double acc = 0.0;
    for (int i = lane; i < count; i += 32)
        acc += frames::nutation_term(terms[i], F);
    return warp_sum(acc);
}

__global__ void __launch_bounds__(256) frames_kernel(FrameData fd, int y, int mo, int d, int hh,
    int mi, const double* __restrict__ sec_args, int count, double* __restrict__ m_out,
    double* __restrict__ mjd_out)
{
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= count)
        return;
    // TimePointParamsKernel (time_points.cu:44-52): UTC MJD, EOP, UT1 and TT of this epoch
    const double mjd_utc = frames::calendar_to_mjd(y, mo, d, hh, mi, sec_args[warp]);
    const EopRec eop = frames::eop_at(fd.eop, fd.n_eop, mjd_utc);
    const double mjd_ut1 = mjd_utc + eop.ut1 / 86400.0;
    const double mjd_tt
        = mjd_utc + (frames::leap_at(fd.leap_mjd, fd.leap_val, fd.n_leap, mjd_utc) + frames::kTtTai) / 86400.0;
    const double t = (mjd_tt - frames::kMjdJ2000) / 36525.0;
    double F[14];
    frames::fundamental_args(t, F);
    const NutTerm* lon1 = fd.nut + fd.n_lon0;
    const NutTerm* obl0 = lon1 + fd.n_lon1;
    const NutTerm* obl1 = obl0 + fd.n_obl0;
    const double dpsi = series_sum(fd.nut, fd.n_lon0, F, lane) + series_sum(lon1, fd.n_lon1, F, lane) * t;
    const double deps = series_sum(obl0, fd.n_obl0, F, lane) + series_sum(obl1, fd.n_obl1, F, lane) * t;
    if (lane == 0) {
        double M[9];
        frames::assemble(t, F, dpsi, deps, mjd_ut1, mjd_tt, eop, M);
        for (int k = 0; k < 9; ++k)
            m_out[(size_t)warp * 9 + k] = M[k];
        if (mjd_out)
            mjd_out[warp] = mjd_utc;
    }
}

cudaError_t launch_frames(const FrameData& fd, int y, int mo, int d, int hh, int mi,
    const double* sec_args, int count, double* m_out, double* mjd_out, cudaStream_t s)
{
    if (count <= 0)
        return cudaSuccess;
    const int threads = 256;
    const int blocks = (int)(((int64_t)count * 32 + threads - 1) / threads);
    frames_kernel<<<blocks, threads, 0, s>>>(fd, y, mo, d, hh, mi, sec_args, count, m_out, mjd_out);
    return cudaGetLastError();
}

} // namespace gpop
