// model.h -- host-side model data: loaders for the gravity field, nutation series, EOP and leap
// seconds, and the builder of the device gravity tables.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace gpop {

// One nutation term: amplitudes in micro-arcseconds and the 14 integer argument multipliers
// (IERS 2010 Tables 5.3a/b; loader behaviour of dataset_loaders.cu:30-91).
struct NutTerm {
    double sin_uas;
    double cos_uas;
    int8_t args[14];
    int8_t pad[2];
};
static_assert(sizeof(NutTerm) == 32, "NutTerm is the device layout");

// Earth-orientation record (force_model/include/force_model/types.cuh:66-71): UTC MJD, polar
// motion x_p, y_p in radians, UT1-UTC in seconds.
struct EopRec {
    double mjd, xp, yp, ut1;
};

struct ModelData {
    // gravity field (ICGEM gfc), truncated to `degree`
    int degree = 0;
    double gm = 0, radius = 0;
    std::vector<double> C, S; // triangular, index n(n+1)/2 + m
    // frames
    std::vector<NutTerm> lon0, lon1, obl0, obl1;
    std::vector<EopRec> eop;
    std::vector<double> leap_mjd, leap_val;
};

// Loads every data set from `dir`. degree <= 0 keeps the gfc header's max_degree. Returns false and
// fills `err` on failure (missing file, malformed header, non-static model).
bool load_model(const std::string& dir, int degree, ModelData& out, std::string& err);

// Gravity table entry, one per (n, m) with n >= m, stored column by column (m outer, n = m..L).
// With the rescaled derived-Legendre recursion
//   Q(m,m) = q^m, Q(m+1,m) = u Q(m,m), Q(n,m) = u Q(n-1,m) - c(n,m) w Q(n-2,m)
// (q = R/r, u = q z/r, w = q^2, c = ((n-1)^2 - m^2)/((2n-1)(2n-3))), the reference's P-bar times
// (R/r)^n equals sigma(n,m) Q(n,m). sigma is folded into the six coefficients:
//   g = sigma (1+n+m) (C, S)(n,m)          -> G sum, paired with (C_m, S_m)
//   j = sigma (C, S)(n,m)                  -> J and K sums, paired with m (C_m-1, S_m-1)
//   h = sigma zeta(n,m-1) (C, S)(n,m-1)    -> H sum, paired with (C_m-1, S_m-1)
// Terms of degree n < 2 carry zero coefficients, as in gravity_source_device.cu:147-153.
struct alignas(16) GravEntry64 {
    double c, pad, g1, g2, j1, j2, h1, h2;
};
// FP32 entry: the recursion constant is stored negated, twice ((-c, -c) is the packed operand of
// the two-object recursion).
struct alignas(16) GravEntry32 {
    float c, pad, g1, g2, j1, j2, h1, h2;
};
static_assert(sizeof(GravEntry64) == 64, "layout");
static_assert(sizeof(GravEntry32) == 32, "layout");

#ifdef __CUDACC__
#define GPOP_HOST_DEVICE __host__ __device__
#else
#define GPOP_HOST_DEVICE
#endif
GPOP_HOST_DEVICE inline int grav_entries(int L) { return (L + 1) * (L + 2) / 2; }
// First entry of column m in the column-major triangle with rows n = m..L.
GPOP_HOST_DEVICE inline int grav_col_offset(int m, int L) { return m * (L + 1) - (m * (m - 1)) / 2; }

// Builds the FP64 and FP32 tables for degree L (= model degree).
void build_gravity_tables(const ModelData& md, std::vector<GravEntry64>& t64, std::vector<GravEntry32>& t32);

// Lane layout of the tables, for kernels whose lanes walk different columns at once (P lanes per
// object, lane l on columns l, l + P, ...). Each column starts on the 16-byte slot m mod 8 of a
// 128-byte shared-memory row, so eight lanes that read entry i of eight consecutive columns hit
// eight different bank groups. Blob: int column bases (in 16-byte units from their table) at
// byte 0 (FP64, up to 128 columns) and byte 512 (FP32), the FP64 table at kLaneOff64 and the
// FP32 table (if any) at off32, a multiple of 128 bytes.
constexpr uint32_t kLaneOff64 = 1024;
constexpr int kLaneMaxDegree = 126;
// t64 has degree L64 (column-major as grav_col_offset); t32 (may be NULL) degree L32.
void build_lane_blob(const GravEntry64* t64, int L64, const GravEntry32* t32, int L32,
    std::vector<uint8_t>& blob, uint32_t& off32);

} // namespace gpop
