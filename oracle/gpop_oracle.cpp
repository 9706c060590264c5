/*
 * gpop_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * CPU FP64 restatement of the OpenGPOP propagation and closest-approach path. Each function states
 * the reference file:line it follows (paths relative to the reference project root). Operation
 * order follows the reference wherever the reference fixes it; where the reference hands a sum to
 * cuBLAS (gemv/gemm/axpy) or Thrust (reduce_by_key), whose internal order is not specified, the
 * sum here runs left to right.
 *
 * Built by oracle/Makefile into oracle/liboracle.so (g++ -O2 -fopenmp). Loaded with ctypes.
 */
#include "gpop_oracle.h"

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// lib/force_model/include/force_model/constants.cuh:21-33
constexpr double kPi = 3.14159265358979324;
constexpr double kArcsPerRad = 3600.0 * 180.0 / kPi;
constexpr double kMjdJ2000 = 51544.5;
constexpr double kMjd1900 = 15020.0;
constexpr double kTtTai = 32.184;
constexpr int kRkStages = 10;
const double kRkNodes[kRkStages]
    = { 0.0, 4.0 / 27.0, 2.0 / 9.0, 1.0 / 3.0, 1.0 / 2.0, 2.0 / 3.0, 1.0 / 6.0, 1.0, 5.0 / 6.0, 1.0 };

// 10-stage RK8 Butcher table (lib/common/gpu_constants/gpu_constants/gpu_constants.cuh:22-35).
const double kRkB[10] = { 41.0 / 840.0, 0.0, 0.0, 27.0 / 840.0, 272.0 / 840.0, 27.0 / 840.0,
    216.0 / 840.0, 0.0, 216.0 / 840.0, 41.0 / 840.0 };
const double kRkA[9][9] = {
    { 4.0 / 27, 0, 0, 0, 0, 0, 0, 0, 0 },
    { 1.0 / 18, 3.0 / 18, 0, 0, 0, 0, 0, 0, 0 },
    { 1.0 / 12, 0.0, 3.0 / 12, 0, 0, 0, 0, 0, 0 },
    { 1.0 / 8, 0, 0, 3.0 / 8, 0, 0, 0, 0, 0 },
    { 13.0 / 54, 0.0, -27.0 / 54, 42.0 / 54, 8.0 / 54, 0, 0, 0, 0 },
    { 389.0 / 4320, 0.0, -54.0 / 4320, 966.0 / 4320, -824.0 / 4320.0, 243.0 / 4320, 0, 0, 0 },
    { -234.0 / 20, 0, 81.0 / 20, -1164.0 / 20, 656.0 / 20, -122.0 / 20, 800.0 / 20, 0, 0 },
    { -127.0 / 288, 0.0, 18.0 / 288, -678.0 / 288, 456.0 / 288, -9.0 / 288, 576.0 / 288, 4.0 / 288,
        0 },
    { 1481.0 / 820, 0.0, -81.0 / 820, 7104.0 / 820, -3376.0 / 820, 72.0 / 820, -5040.0 / 820,
        -60.0 / 820, 720.0 / 820 },
};

// Eighth-order Gauss-Jackson (GJ) and summed-Adams (SA) ordinate-form coefficients,
// rows 0..8 = mid-corrector at points -4..+4, row 9 = predictor (Berry & Healy 2004, tables 5-6;
// gpu_constants.cuh:37-98).
const double kGJ[10][9] = {
    { 3250433.0 / 53222400.0, 572741.0 / 5702400.0, -8701681.0 / 39916800.0,
        4026311.0 / 13305600.0, -917039.0 / 3193344.0, 7370669.0 / 39916800.0,
        -1025779.0 / 13305600.0, 754331.0 / 39916800.0, -330157.0 / 159667200.0 },
    { -330157.0 / 159667200.0, 530113.0 / 6652800.0, 518887.0 / 19958400.0, -27631.0 / 623700.0,
        44773.0 / 1064448.0, -531521.0 / 19958400.0, 109343.0 / 9979200.0, -1261.0 / 475200.0,
        45911.0 / 159667200.0 },
    { 45911.0 / 159667200.0, -185839.0 / 39916800.0, 171137.0 / 1900800.0, 73643.0 / 39916800.0,
        -25775.0 / 3193344.0, 77597.0 / 13305600.0, -98911.0 / 39916800.0, 24173.0 / 39916800.0,
        -3499.0 / 53222400.0 },
    { -3499.0 / 53222400.0, 4387.0 / 4989600.0, -35039.0 / 4989600.0, 90817.0 / 950400.0,
        -20561.0 / 3193344.0, 2117.0 / 9979200.0, 2059.0 / 6652800.0, -317.0 / 2851200.0,
        317.0 / 22809600.0 },
    { 317.0 / 22809600.0, -2539.0 / 13305600.0, 55067.0 / 39916800.0, -326911.0 / 39916800.0,
        14797.0 / 152064.0, -326911.0 / 39916800.0, 55067.0 / 39916800.0, -2539.0 / 13305600.0,
        317.0 / 22809600.0 },
    { 317.0 / 22809600.0, -317.0 / 2851200.0, 2059.0 / 6652800.0, 2117.0 / 9979200.0,
        -20561.0 / 3193344.0, 90817.0 / 950400.0, -35039.0 / 4989600.0, 4387.0 / 4989600.0,
        -3499.0 / 53222400.0 },
    { -3499.0 / 53222400.0, 24173.0 / 39916800.0, -98911.0 / 39916800.0, 77597.0 / 13305600.0,
        -25775.0 / 3193344.0, 73643.0 / 39916800.0, 171137.0 / 1900800.0, -185839.0 / 39916800.0,
        45911.0 / 159667200.0 },
    { 45911.0 / 159667200.0, -1261.0 / 475200.0, 109343.0 / 9979200.0, -531521.0 / 19958400.0,
        44773.0 / 1064448.0, -27631.0 / 623700.0, 518887.0 / 19958400.0, 530113.0 / 6652800.0,
        -330157.0 / 159667200.0 },
    { -330157.0 / 159667200.0, 754331.0 / 39916800.0, -1025779.0 / 13305600.0,
        7370669.0 / 39916800.0, -917039.0 / 3193344.0, 4026311.0 / 13305600.0,
        -8701681.0 / 39916800.0, 572741.0 / 5702400.0, 3250433.0 / 53222400.0 },
    { 3250433.0 / 53222400.0, -11011481.0 / 19958400.0, 6322573.0 / 2851200.0,
        -8660609.0 / 1663200.0, 25162927.0 / 3193344.0, -159314453.0 / 19958400.0,
        18071351.0 / 3326400.0, -24115843.0 / 9979200.0, 103798439.0 / 159667200.0 },
};
const double kSA[10][9] = {
    { 19087.0 / 89600.0, -427487.0 / 725760.0, 3498217.0 / 3628800.0, -500327.0 / 403200.0,
        6467.0 / 5670.0, -2616161.0 / 3628800.0, 24019.0 / 80640.0, -263077.0 / 3628800.0,
        8183.0 / 1036800.0 },
    { 8183.0 / 1036800.0, 57251.0 / 403200.0, -1106377.0 / 3628800.0, 218483.0 / 725760.0,
        -69.0 / 280.0, 530177.0 / 3628800.0, -210359.0 / 3628800.0, 5533.0 / 403200.0,
        -425.0 / 290304.0 },
    { -425.0 / 290304.0, 76453.0 / 3628800.0, 5143.0 / 57600.0, -660127.0 / 3628800.0,
        661.0 / 5670.0, -4997.0 / 80640.0, 83927.0 / 3628800.0, -19109.0 / 3628800.0,
        7.0 / 12800.0 },
    { 7.0 / 12800.0, -23173.0 / 3628800.0, 29579.0 / 725760.0, 2497.0 / 57600.0,
        -2563.0 / 22680.0, 172993.0 / 3628800.0, -6463.0 / 403200.0, 2497.0 / 725760.0,
        -2497.0 / 7257600.0 },
    { -2497.0 / 7257600.0, 1469.0 / 403200.0, -68119.0 / 3628800.0, 252769.0 / 3628800.0, 0.0,
        -252769.0 / 3628800.0, 68119.0 / 3628800.0, -1469.0 / 403200.0, 2497.0 / 7257600.0 },
    { 2497.0 / 7257600.0, -2497.0 / 725760.0, 6463.0 / 403200.0, -172993.0 / 3628800.0,
        2563.0 / 22680.0, -2497.0 / 57600.0, -29579.0 / 725760.0, 23173.0 / 3628800.0,
        -7.0 / 12800.0 },
    { -7.0 / 12800.0, 19109.0 / 3628800.0, -83927.0 / 3628800.0, 4997.0 / 80640.0,
        -661.0 / 5670.0, 660127.0 / 3628800.0, -5143.0 / 57600.0, -76453.0 / 3628800.0,
        425.0 / 290304.0 },
    { 425.0 / 290304.0, -5533.0 / 403200.0, 210359.0 / 3628800.0, -530177.0 / 3628800.0,
        69.0 / 280.0, -218483.0 / 725760.0, 1106377.0 / 3628800.0, -57251.0 / 403200.0,
        -8183.0 / 1036800.0 },
    { -8183.0 / 1036800.0, 263077.0 / 3628800.0, -24019.0 / 80640.0, 2616161.0 / 3628800.0,
        -6467.0 / 5670.0, 500327.0 / 403200.0, -3498217.0 / 3628800.0, 427487.0 / 725760.0,
        -19087.0 / 89600.0 },
    { 25713.0 / 89600.0, -9401029.0 / 3628800.0, 5393233.0 / 518400.0, -9839609.0 / 403200.0,
        167287.0 / 4536.0, -135352319.0 / 3628800.0, 10219841.0 / 403200.0,
        -40987771.0 / 3628800.0, 3288521.0 / 1036800.0 },
};

inline size_t tri(size_t n, size_t m) { return n * (n + 1) / 2 + m; } // gpu_utils.cuh:64
inline size_t tri_size(size_t N) { return N * (N + 1) / 2; } // gpu_utils.cuh:67

struct NutTerm {
    double sin_uas, cos_uas;
    int args[14];
};

struct EopRec {
    double mjd, xp, yp, ut1;
};

struct Data {
    // gravity
    unsigned N = 0; // degree + 1
    double GM = 0, R = 0;
    std::vector<double> C, S; // triangular
    std::vector<double> xi, eta, zeta, delta, pdiag; // auxiliary tables
    // frames
    std::vector<NutTerm> lon0, lon1, obl0, obl1;
    std::vector<EopRec> eop;
    std::vector<double> leap_mjd, leap_val;
};

// lib/force_model/src/utility/dataset_loaders.cu:30-91
void load_nutation(const std::string& path, std::vector<NutTerm>& j0, std::vector<NutTerm>& j1)
{
    std::ifstream f(path);
    if (!f.is_open())
        throw std::runtime_error("cannot open " + path);
    std::string line;
    int section = 0;
    while (std::getline(f, line)) {
        if (line.find("j = 0") != std::string::npos) {
            section = 0;
            continue;
        }
        if (line.find("j = 1") != std::string::npos) {
            section = 1;
            continue;
        }
        std::istringstream is(line);
        int idx;
        if (!(is >> idx))
            continue;
        NutTerm t;
        if (!(is >> t.sin_uas >> t.cos_uas))
            continue;
        bool ok = true;
        for (int k = 0; k < 14; ++k)
            if (!(is >> t.args[k])) {
                ok = false;
                break;
            }
        if (!ok)
            continue;
        (section == 0 ? j0 : j1).push_back(t);
    }
}

// dataset_loaders.cu:93-158 (fixed-width finals2000A columns)
void load_eop(const std::string& path, std::vector<EopRec>& out)
{
    std::ifstream f(path);
    if (!f.is_open())
        throw std::runtime_error("cannot open " + path);
    std::string line;
    const char* ws = " \t\n\r\f\v";
    while (std::getline(f, line)) {
        size_t e = line.find_last_not_of(ws);
        if (e == std::string::npos)
            line.clear();
        else
            line.erase(e + 1);
        if (line.empty() || line[0] == '#' || line.length() < 68)
            continue;
        try {
            EopRec r;
            r.mjd = std::stod(line.substr(7, 8));
            r.xp = std::stod(line.substr(18, 9)) / kArcsPerRad;
            r.yp = std::stod(line.substr(37, 9)) / kArcsPerRad;
            r.ut1 = std::stod(line.substr(58, 10));
            out.push_back(r);
        } catch (const std::exception&) {
            continue;
        }
    }
}

double ntp_to_mjd(long long ntp) { return kMjd1900 + (static_cast<double>(ntp) / 86400.0); } // ref_sys_trans.cu:373-376

// dataset_loaders.cu:160-217
void load_leap(const std::string& path, std::vector<double>& mjd, std::vector<double>& val)
{
    std::ifstream f(path);
    if (!f.is_open())
        throw std::runtime_error("cannot open " + path);
    std::string line;
    while (std::getline(f, line)) {
        size_t first = line.find_first_not_of(" \t");
        if (line.empty() || first == std::string::npos || line[first] == '#')
            continue;
        std::stringstream ss(line);
        long long ntp;
        double dtai;
        if (ss >> ntp >> dtai) {
            mjd.push_back(ntp_to_mjd(ntp));
            val.push_back(dtai);
        }
    }
}

// dataset_loaders.cu:219-299, then the truncation to a requested degree (equivalent to a gfc copy
// with a smaller max_degree in its header).
void load_gravity(const std::string& path, int degree, Data& d)
{
    std::ifstream f(path);
    if (!f.is_open())
        throw std::runtime_error("cannot open " + path);
    std::string line;
    bool head_end = false;
    unsigned N = 0;
    while (std::getline(f, line)) {
        if (line.find("end_of_head") != std::string::npos) {
            head_end = true;
            break;
        }
        std::istringstream is(line);
        std::string tok;
        is >> tok;
        if (tok == "earth_gravity_constant")
            is >> d.GM;
        else if (tok == "radius")
            is >> d.R;
        else if (tok == "max_degree") {
            unsigned md;
            is >> md;
            N = md + 1;
        }
    }
    if (!head_end)
        throw std::runtime_error("gfc: end_of_head not found");
    if (degree > 0 && (unsigned)degree + 1 < N)
        N = degree + 1;
    d.N = N;
    d.C.assign(tri_size(N), 0.0);
    d.S.assign(tri_size(N), 0.0);
    bool first = true;
    while (std::getline(f, line)) {
        if (line.empty())
            continue;
        std::istringstream is(line);
        std::string key;
        is >> key;
        if (first) {
            if (key != "gfc")
                throw std::runtime_error("gfc: only static models accepted");
            first = false;
        }
        if (key == "gfc") {
            unsigned L, M;
            double c, s;
            if (is >> L >> M >> c >> s) {
                if (L < N && M <= L) {
                    d.C[tri(L, M)] = c;
                    d.S[tri(L, M)] = s;
                }
            }
        }
    }
    // gravity_source.cu:76-89 (delta, Pbar diagonal) and gravity_source_device.cu:20-46 (xi, eta, zeta)
    size_t T = tri_size(N);
    d.delta.assign(N, 0.0);
    d.pdiag.assign(N, 0.0);
    d.pdiag[0] = 1.0;
    if (N > 1) {
        d.pdiag[1] = std::sqrt(3.0);
        d.delta[1] = std::sqrt(3.0);
    }
    for (unsigned i = 2; i < N; ++i) {
        double prev = d.pdiag[i - 1];
        double tmp = 2.0 * (double)i + 1.0;
        d.pdiag[i] = prev * std::sqrt(tmp / (2.0 * (double)i));
        d.delta[i] = prev * std::sqrt(tmp);
    }
    d.xi.assign(T, 0.0);
    d.eta.assign(T, 0.0);
    d.zeta.assign(T, 0.0);
    for (unsigned nn = 0; nn < N; ++nn)
        for (unsigned mm = 0; mm < nn; ++mm) {
            double n = nn, m = mm;
            size_t k = tri(nn, mm);
            d.xi[k] = std::sqrt((2.0 * n - 1.0) * (2.0 * n + 1.0) / ((n - m) * (n + m)));
            d.eta[k] = std::sqrt((n + m - 1.0) * (2.0 * n + 1.0) * (n - m - 1.0)
                / ((n + m) * (n - m) * (2.0 * n - 3.0)));
            d.zeta[k] = (mm == 0) ? std::sqrt(n * (n + 1.0) / 2.0) : std::sqrt((n - m) * (n + m + 1.0));
        }
}

// ---------------- reference-system transforms (ref_sys_trans.cu) ----------------
inline size_t sq(size_t row, size_t col) { return col * 3 + row; } // gpu_utils.cuh:60

void rot_x(double a, double* p) // ref_sys_trans.cu:24-37
{
    double c = std::cos(a), s = std::sin(a);
    p[sq(0, 0)] = 1.0; p[sq(0, 1)] = 0.0; p[sq(0, 2)] = 0.0;
    p[sq(1, 0)] = 0.0; p[sq(1, 1)] = c;   p[sq(1, 2)] = s;
    p[sq(2, 0)] = 0.0; p[sq(2, 1)] = -s;  p[sq(2, 2)] = c;
}
void rot_y(double a, double* p) // ref_sys_trans.cu:39-52
{
    double c = std::cos(a), s = std::sin(a);
    p[sq(0, 0)] = c;   p[sq(0, 1)] = 0.0; p[sq(0, 2)] = -s;
    p[sq(1, 0)] = 0.0; p[sq(1, 1)] = 1.0; p[sq(1, 2)] = 0.0;
    p[sq(2, 0)] = s;   p[sq(2, 1)] = 0.0; p[sq(2, 2)] = c;
}
void rot_z(double a, double* p) // ref_sys_trans.cu:54-67
{
    double c = std::cos(a), s = std::sin(a);
    p[sq(0, 0)] = c;   p[sq(0, 1)] = s;   p[sq(0, 2)] = 0.0;
    p[sq(1, 0)] = -s;  p[sq(1, 1)] = c;   p[sq(1, 2)] = 0.0;
    p[sq(2, 0)] = 0.0; p[sq(2, 1)] = 0.0; p[sq(2, 2)] = 1.0;
}

// C = A * B, column-major 3x3 (the cuBLAS DgemmStridedBatched calls of time_points.cu:146-152)
void matmul3(const double* A, const double* B, double* C)
{
    double t[9];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k)
                s += A[sq(i, k)] * B[sq(k, j)];
            t[sq(i, j)] = s;
        }
    std::memcpy(C, t, sizeof(t));
}

double calendar_to_mjd(int year, int mon, int day, int h, int min, double sec) // ref_sys_trans.cu:122-144
{
    if (mon <= 2) {
        --year;
        mon += 12;
    }
    int B;
    if ((10000L * year + 100L * mon + day) <= 15821004L)
        B = -2 + ((year + 4716) / 4) - 1179;
    else if ((10000L * year + 100L * mon + day) >= 15821015L)
        B = (year / 400) - (year / 100) + (year / 4);
    else
        return -1.0;
    long mjd = 365L * year - 679004L + B + int(30.6001 * (mon + 1)) + day;
    double frac = (h + min / 60.0 + sec / 3600.0) / 24.0;
    return mjd + frac;
}

void ftable(double t, double* F) // ref_sys_trans.cu:164-233 (IERS 2010 eqs. 5.43, 5.44)
{
    const double l[] = { 134.96340251 * 3600.0, 1717915923.2178, 31.8792, 0.051635, -0.00024470 };
    const double lp[] = { 357.52910918 * 3600.0, 129596581.0481, -0.5532, 0.000136, -0.00001149 };
    const double fa[] = { 93.27209062 * 3600.0, 1739527262.8478, -12.7512, -0.001037, 0.00000417 };
    const double dd[] = { 297.85019547 * 3600.0, 1602961601.2090, -6.3706, 0.006593, -0.00003169 };
    const double om[] = { 125.04455501 * 3600.0, -6962890.5431, 7.4722, 0.007702, -0.00005939 };
    const double* lun[5] = { l, lp, fa, dd, om };
    for (int a = 0; a < 5; ++a) {
        double v = lun[a][4];
        for (int i = 3; i >= 0; --i)
            v = v * t + lun[a][i];
        F[a] = v;
    }
    for (int i = 0; i < 5; ++i)
        F[i] /= kArcsPerRad;
    const double pl[9][3] = {
        { 4.402608842, 2608.7903141574, 0.0 },
        { 3.176146697, 1021.3285546211, 0.0 },
        { 1.753470314, 628.3075849991, 0.0 },
        { 6.203480913, 334.0612426700, 0.0 },
        { 0.599546497, 52.9690962641, 0.0 },
        { 0.874016757, 21.3299104960, 0.0 },
        { 5.481293872, 7.4781598567, 0.0 },
        { 5.311886287, 3.8133035638, 0.0 },
        { 0.0, 0.02438175, 0.00000538691 },
    };
    for (int a = 0; a < 9; ++a) {
        double v = pl[a][2];
        for (int i = 1; i >= 0; --i)
            v = v * t + pl[a][i];
        F[5 + a] = v;
    }
    for (int i = 0; i < 14; ++i)
        F[i] = std::fmod(F[i], 2.0 * M_PI);
}

double nut_delta(const double* F, const std::vector<NutTerm>& terms) // ref_sys_trans.cu:241-254
{
    double result = 0;
    for (int i = (int)terms.size() - 1; i >= 0; --i) {
        double arg = 0;
        for (int k = 13; k >= 0; --k)
            arg += F[k] * terms[i].args[k];
        result += terms[i].sin_uas / (kArcsPerRad * 1e6) * std::sin(arg);
        result += terms[i].cos_uas / (kArcsPerRad * 1e6) * std::cos(arg);
    }
    return result;
}

void precession(double t, double& epsA, double& gam, double& phi, double& psi) // ref_sys_trans.cu:262-291
{
    const double e[] = { 84381.406, -46.836769, -0.0001831, 0.00200340, -0.000000576, -0.0000000434 };
    const double g[] = { -0.052928, 10.556378, 0.4932044, -0.00031238, -0.000002788, 0.0000000260 };
    const double p[] = { 84381.412819, -46.811016, 0.0511268, 0.00053289, -0.000000440, -0.0000000176 };
    const double s[] = { -0.041775, 5038.481484, 1.5584175, -0.00018522, -0.000026452, -0.0000000148 };
    epsA = e[5];
    gam = g[5];
    phi = p[5];
    psi = s[5];
    for (int i = 4; i >= 0; --i) {
        epsA = epsA * t + e[i];
        gam = gam * t + g[i];
        phi = phi * t + p[i];
        psi = psi * t + s[i];
    }
    epsA /= kArcsPerRad;
    gam /= kArcsPerRad;
    phi /= kArcsPerRad;
    psi /= kArcsPerRad;
}

double gast(double mjd_ut1, double mjd_tt, double dpsi, double epsA, const double* F) // ref_sys_trans.cu:75-119
{
    double T = (mjd_tt - kMjdJ2000) / 36525.0;
    double Du = mjd_ut1 - kMjdJ2000;
    double Du_mod_1 = Du - std::floor(Du);
    double gmst = 86400.0 * (0.7790572732640 + 0.00273781191135448 * Du + Du_mod_1);
    const double c[6] = { 0.00096707, 307.47710227, 0.092772113, -0.0000000293, -0.00000199707, -2.453e-9 };
    double poly = c[5];
    for (int i = 4; i >= 0; --i)
        poly = poly * T + c[i];
    gmst += poly;
    gmst *= (M_PI / 43200.0);
    double l = F[0], lp = F[1], f = F[2], D = F[3], Om = F[4];
    double ee = 0.0;
    ee -= 0.00000087 * T * std::sin(Om);
    ee -= 0.00000063 * std::sin(l - Om);
    ee -= 0.00000063 * std::sin(l + Om);
    ee -= 0.00000126 * std::sin(lp - Om);
    ee -= 0.00000141 * std::sin(lp + Om);
    ee -= 0.00000172 * std::sin(3.0 * Om);
    ee += 0.00000198 * std::sin(2.0 * f + Om);
    ee += 0.00000202 * std::sin(2.0 * f + 3.0 * Om);
    ee -= 0.00000455 * std::sin(2.0 * f - 2.0 * D + 2.0 * Om);
    ee += 0.00001121 * std::sin(2.0 * f - 2.0 * D + Om);
    ee += 0.00001175 * std::sin(2.0 * f - 2.0 * D + 3.0 * Om);
    ee += 0.00006352 * std::sin(2.0 * Om);
    ee += 0.00264096 * std::sin(Om);
    ee *= (M_PI / 43200.0) / 15.0;
    ee += dpsi * std::cos(epsA);
    return std::fmod(gmst + ee, 2 * M_PI);
}

EopRec eop_record(const Data& d, double mjd) // force_model/include/force_model/types.cuh:79-130
{
    const auto& r = d.eop;
    if (r.empty())
        return { -1.0, 0.0, 0.0, 0.0 };
    if (mjd <= r[0].mjd)
        return r[0];
    if (mjd >= r.back().mjd)
        return r.back();
    int left = 0, right = (int)r.size() - 1;
    while (left <= right) {
        int mid = left + (right - left) / 2;
        double cur = r[mid].mjd;
        if (cur == mjd)
            return r[mid];
        else if (cur < mjd)
            left = mid + 1;
        else
            right = mid - 1;
    }
    const EopRec& r0 = r[right];
    const EopRec& r1 = r[left];
    double fr = (mjd - r0.mjd) / (r1.mjd - r0.mjd);
    EopRec o;
    o.mjd = mjd;
    o.xp = r0.xp + fr * (r1.xp - r0.xp);
    o.yp = r0.yp + fr * (r1.yp - r0.yp);
    o.ut1 = r0.ut1 + fr * (r1.ut1 - r0.ut1);
    return o;
}

double leap_seconds(const Data& d, double mjd) // types.cuh:140-152
{
    if (d.leap_mjd.empty())
        return 0.0;
    for (size_t i = d.leap_mjd.size(); i-- > 0;)
        if (mjd >= d.leap_mjd[i])
            return d.leap_val[i];
    return d.leap_val[0];
}

// time_points.cu:26-71 (one epoch) followed by the matrix chain of time_points.cu:160-201
void frame_matrix(const Data& d, const or_time& st, double sec_arg, double* M, double* mjd_out)
{
    double mjd_utc = calendar_to_mjd(st.year, st.month, st.day, st.hour, st.min, sec_arg);
    if (mjd_out)
        *mjd_out = mjd_utc;
    EopRec eop = eop_record(d, mjd_utc);
    double mjd_ut1 = mjd_utc + eop.ut1 / 86400.0; // ref_sys_trans.cu:153-156
    double mjd_tt = mjd_utc + (leap_seconds(d, mjd_utc) + kTtTai) / 86400.0; // :147-150
    // CreateQMatrixComponents (ref_sys_trans.cu:305-337)
    double t = (mjd_tt - kMjdJ2000) / 36525.0;
    double F[14];
    ftable(t, F);
    double dpsi = 0, deps = 0;
    dpsi += nut_delta(F, d.lon0);
    dpsi += nut_delta(F, d.lon1) * t;
    deps += nut_delta(F, d.obl0);
    deps += nut_delta(F, d.obl1) * t;
    double epsA, gam, phi, psib;
    precession(t, epsA, gam, phi, psib);
    double psi = psib + dpsi;
    double eps = epsA + deps;
    double Q1[9], Q2[9], Q3[9], Q4[9], W1[9], W2[9], W3[9], R[9];
    rot_z(-gam, Q1);
    rot_x(-phi, Q2);
    rot_z(psi, Q3);
    rot_x(eps, Q4);
    // CreateWMatrixComponents (:348-358)
    double sp = -47e-6 * t / kArcsPerRad;
    rot_z(-sp, W1);
    rot_y(eop.xp, W2);
    rot_x(eop.yp, W3);
    // CreateRMatrix (:366-370)
    rot_z(-gast(mjd_ut1, mjd_tt, dpsi, epsA, F), R);
    // ComputeITRStoGCRS association order (time_points.cu:160-201)
    double A[9], B[9], Q[9], W[9], QR[9];
    matmul3(Q1, Q2, A);
    matmul3(Q3, Q4, B);
    matmul3(A, B, Q);
    matmul3(W1, W2, A);
    matmul3(A, W3, W);
    matmul3(Q, R, QR);
    matmul3(QR, W, M);
}

// time_points.cu:34-46: seconds argument of table entry idx, (sec - before h) + time from start
double table_sec(const or_time& st, double h, int idx, bool midpoints, int before)
{
    double from_start;
    if (midpoints)
        from_start = ((double)(idx / kRkStages) + kRkNodes[idx % kRkStages]) * h;
    else
        from_start = idx * h;
    return (st.sec - (double)before * h) + from_start;
}

// ---------------- gravity (gravity_source.cu:168-262 + gravity_source_device.cu:63-239) ----------------
// R = double is the oracle; R = long double (x87 extended) serves the finite differences of the
// adjoint checks, which need less rounding noise than double gives.
template <typename R>
void gravity_itrs(const Data& d, const R* p, R* a, std::vector<R>& P, std::vector<R>& Cm,
    std::vector<R>& Sm, std::vector<R>& sums)
{
    const unsigned N = d.N;
    R x = p[0], y = p[1], z = p[2];
    R r = std::sqrt(x * x + y * y + z * z);
    R eps = z / r;
    // ComputePbarKernel: per column m, subdiagonal then column recursion (eq. 7-12, 7-16)
    for (unsigned m = 0; m < N; ++m)
        P[tri(m, m)] = d.pdiag[m];
    for (unsigned m = 0; m + 1 < N; ++m) {
        unsigned n = m + 1;
        P[tri(n, n - 1)] = eps * d.delta[n];
        while (n != N - 1) {
            ++n;
            size_t nm = tri(n, m);
            P[nm] = d.xi[nm] * eps * P[tri(n - 1, m)] - d.eta[nm] * P[tri(n - 2, m)];
        }
    }
    // ComputeCmSmKernel (eq. 3-18)
    Cm[0] = 1;
    Sm[0] = 0;
    if (N > 1) {
        Cm[1] = x / r;
        Sm[1] = y / r;
    }
    for (unsigned i = 2; i < N; ++i) {
        Cm[i] = Cm[1] * Cm[i - 1] - Sm[1] * Sm[i - 1];
        Sm[i] = Sm[1] * Cm[i - 1] + Cm[1] * Sm[i - 1];
    }
    // PrepareMSumKernel + SumM (eq. 4-11), per-n sums over m
    R* Gn = sums.data();
    R* Hn = Gn + N;
    R* Jn = Hn + N;
    R* Kn = Jn + N;
    for (unsigned n = 0; n < N; ++n) {
        R g = 0, h = 0, j = 0, k = 0;
        for (unsigned m = 0; m <= n; ++m) {
            R tg, th, tj, tk;
            size_t nm = tri(n, m);
            R Pnm = P[nm];
            R Pnm1 = (n > m) ? P[tri(n, m + 1)] : R(0);
            R Cnm = d.C[nm], Snm = d.S[nm];
            if (n < 2) {
                tg = th = tj = tk = 0;
            } else if (m == 0) {
                R Pn0 = P[tri(n, 0)];
                R Pn1 = P[tri(n, 1)];
                R Cn0 = d.C[tri(n, 0)];
                tj = 0;
                tk = 0;
                tg = Cn0 * R(n + 1) * Pn0;
                th = d.zeta[tri(n, 0)] * Cn0 * Pn1;
            } else {
                R c = Cm[m], s = Sm[m], c1 = Cm[m - 1], s1 = Sm[m - 1];
                tj = (R)m * Pnm * (Cnm * c1 + Snm * s1);
                tk = -(R)m * Pnm * (Cnm * s1 - Snm * c1);
                tg = (R)(1 + n + m) * Pnm * (Cnm * c + Snm * s);
                th = d.zeta[nm] * Pnm1 * (Cnm * c + Snm * s);
            }
            g += tg;
            h += th;
            j += tj;
            k += tk;
        }
        Gn[n] = g;
        Hn[n] = h;
        Jn[n] = j;
        Kn[n] = k;
    }
    // PrepareNSumKernel + SumN (eq. 4-12)
    R base = d.R / r;
    R coeff = base * base;
    for (unsigned n = 2; n < N; ++n) {
        Gn[n] *= coeff;
        Hn[n] *= coeff;
        Kn[n] *= coeff;
        Jn[n] *= coeff;
        coeff *= base;
    }
    R G = 0, H = 0, J = 0, K = 0;
    for (unsigned n = 0; n < N; ++n) {
        G += Gn[n];
        H += Hn[n];
        J += Jn[n];
        K += Kn[n];
    }
    // CalculateAcceleration (eq. 4-13)
    G = G + 1;
    R Lambda = G + z * H / r;
    R ax = Lambda * x / r - J;
    R ay = Lambda * y / r - K;
    R az = Lambda * z / r - H;
    R c = -d.GM / (r * r);
    a[0] = c * ax;
    a[1] = c * ay;
    a[2] = c * az;
}

template <typename R> struct GravScratchT {
    std::vector<R> P, Cm, Sm, sums;
    explicit GravScratchT(const Data& d)
        : P(tri_size(d.N))
        , Cm(d.N)
        , Sm(d.N)
        , sums(4 * d.N)
    {
    }
};
using GravScratch = GravScratchT<double>;

// GravitySource::ComputeAcceleration frame handling: r_itrs = M^T r_gcrs, a_gcrs = M a_itrs
template <typename R>
void gravity_gcrs(const Data& d, const double* M, const R* r, R* a, GravScratchT<R>& s)
{
    R p[3], ai[3];
    if (M) {
        for (int j = 0; j < 3; ++j) {
            R v = 0.0;
            for (int i = 0; i < 3; ++i)
                v += M[sq(i, j)] * r[i];
            p[j] = v;
        }
    } else {
        p[0] = r[0];
        p[1] = r[1];
        p[2] = r[2];
    }
    gravity_itrs(d, p, ai, s.P, s.Cm, s.Sm, s.sums);
    if (M) {
        for (int i = 0; i < 3; ++i) {
            R v = 0.0;
            for (int j = 0; j < 3; ++j)
                v += M[sq(i, j)] * ai[j];
            a[i] = v;
        }
    } else {
        a[0] = ai[0];
        a[1] = ai[1];
        a[2] = ai[2];
    }
}

// ---------------- analytic force models (unit_tests/include/gpu_test_helpers.cuh:19-145) ----------------
template <typename R> void analytic(int kind, const R* pos, const R* vel, R t, R* out)
{
    switch (kind) {
    case OR_FORCE_ZERO:
        out[0] = out[1] = out[2] = 0;
        return;
    case OR_FORCE_CONST:
        out[0] = 1;
        out[1] = 2;
        out[2] = 3;
        return;
    case OR_FORCE_POLY7: {
        R v = -3 * 2 * t + 7 * 6 * t * t * t * t * t;
        out[0] = out[1] = out[2] = v;
        return;
    }
    case OR_FORCE_POLY8: {
        R v = 56 * std::pow(t, 6) - 42 * std::pow(t, 5) + 60 * std::pow(t, 4)
            - 100 * std::pow(t, 3) - 120 * std::pow(t, 2) + 6 * t - 2;
        out[0] = out[1] = out[2] = v;
        return;
    }
    case OR_FORCE_POLY9: {
        R v = 72 * std::pow(t, 7) + 56 * std::pow(t, 6) - 42 * std::pow(t, 5)
            + 60 * std::pow(t, 4) - 100 * std::pow(t, 3) - 120 * std::pow(t, 2) + 6 * t - 2;
        out[0] = out[1] = out[2] = v;
        return;
    }
    case OR_FORCE_EXP: {
        R v = std::exp(-t);
        out[0] = out[1] = out[2] = v;
        return;
    }
    case OR_FORCE_DAMPED:
        for (int i = 0; i < 3; ++i)
            out[i] = -2 * pos[i] - 2 * vel[i];
        return;
    default:
        out[0] = out[1] = out[2] = 0;
    }
}

// Force model seen by the integrator: IForceModel's generation/propagation methods
// (lib/force_model/include/force_model/iforce_model.cuh:19-33).
struct Force {
    const Data* d = nullptr;
    int kind = OR_FORCE_GRAVITY;
    double h = 0;
    uint32_t flags = 0;
    std::vector<double> gen_m; // 80 x 9 (generation epochs)
    std::vector<double> prop_m; // (steps + 5) x 9 (propagation epochs, index i <-> (i-4) h)

    // ForceModel::ComputeGenerationAcceleration (force_model.cu:59-89) / mock (mock_force_model.cuh:65-82)
    template <typename R>
    void gen(const R* r, const R* v, int step, int k, R* a, GravScratchT<R>* gs) const
    {
        if (kind == OR_FORCE_GRAVITY) {
            int s = step > 0 ? step - 1 : step;
            gravity_gcrs(*d, &gen_m[((s + 4) * kRkStages + k) * 9], r, a, *gs);
        } else {
            int dir = step > 0 ? -1 : 1;
            double t = static_cast<double>(step + dir) * h + (-dir) * kRkNodes[k] * h;
            analytic<R>(kind, r, v, (R)t, a);
        }
    }
    // ForceModel::ComputePropagationAcceleration (force_model.cu:91-109) / mock (:94-106)
    template <typename R>
    void prop(const R* r, const R* v, int idx, R* a, GravScratchT<R>* gs) const
    {
        if (kind == OR_FORCE_GRAVITY) {
            gravity_gcrs(*d, &prop_m[idx * 9], r, a, *gs);
        } else {
            double t = (double)(idx - 4) * h;
            analytic<R>(kind, r, v, (R)t, a);
        }
    }
};

// Generation epochs. Reference rule (force_model.cu:69-71): entry (s', k) = (s' + c_k) h with
// s' = step-1 for forward and s' = step for backward steps (quirk Q1 for the backward ones).
// With OR_FLAG_FIX_Q1 the backward entries use the true stage time -(i-1) h - c_k h.
void build_tables(Force& f, const or_time& st, int steps)
{
    if (f.kind != OR_FORCE_GRAVITY)
        return;
    f.gen_m.assign(80 * 9, 0.0);
    for (int idx = 0; idx < 80; ++idx) {
        double sec = table_sec(st, f.h, idx, true, 4);
        if (f.flags & OR_FLAG_FIX_Q1) {
            int sp = idx / kRkStages - 4; // s'
            int k = idx % kRkStages;
            if (sp < 0) // backward step -i with i = -sp: true stage time -(i-1) h - c_k h
                sec = (st.sec - 4.0 * f.h) + (((double)(sp + 1) - kRkNodes[k]) * f.h + 4.0 * f.h);
        }
        frame_matrix(*f.d, st, sec, &f.gen_m[idx * 9], nullptr);
    }
    int len = 4 + std::max(steps, 4) + 1;
    f.prop_m.assign((size_t)len * 9, 0.0);
    for (int idx = 0; idx < len; ++idx)
        frame_matrix(*f.d, st, table_sec(st, f.h, idx, false, 4), &f.prop_m[idx * 9], nullptr);
}

template <typename R> struct StartupT {
    R r[9][3], v[9][3], a[9][3], s[9][3], S[9][3];
};
using Startup = StartupT<double>;

// RK8::step (lib/gpu_startup/src/gpu_startup.cu:108-144) for one object
template <typename R> void rk8_step(const Force& f, int step, StartupT<R>& sd, GravScratchT<R>* gs)
{
    R hh = step > 0 ? (R)f.h : -(R)f.h;
    int dir = step > 0 ? -1 : 1;
    int base = 4 + step + dir;
    R Kx[10][3] = {}, Kv[10][3] = {};
    R tx[3], tv[3];
    for (int j = 0; j < 3; ++j) {
        tx[j] = sd.r[base][j];
        tv[j] = sd.v[base][j];
        Kx[0][j] = tv[j];
    }
    f.gen(tx, tv, step, 0, Kv[0], gs);
    for (int k = 1; k <= 9; ++k) {
        for (int j = 0; j < 3; ++j) {
            R sx = 0, sv = 0;
            for (int i = 0; i < 9; ++i) {
                sx += kRkA[k - 1][i] * Kx[i][j];
                sv += kRkA[k - 1][i] * Kv[i][j];
            }
            tx[j] = hh * sx + sd.r[base][j];
            tv[j] = hh * sv + sd.v[base][j];
        }
        f.gen(tx, tv, step, k, Kv[k], gs);
        for (int j = 0; j < 3; ++j)
            Kx[k][j] = tv[j];
    }
    int col = 4 + step;
    for (int j = 0; j < 3; ++j) {
        R sx = 0, sv = 0;
        for (int k = 0; k < 10; ++k) {
            sx += Kx[k][j] * kRkB[k];
            sv += Kv[k][j] * kRkB[k];
        }
        sd.v[col][j] = hh * sv + sd.v[base][j];
        sd.r[col][j] = hh * sx + sd.r[base][j];
    }
}

// StartupPredictor::Predict (gpu_startup.cu:146-168)
template <typename R> void rk8_all(const Force& f, const R* r0, const R* v0, StartupT<R>& sd, GravScratchT<R>* gs)
{
    std::memset(&sd, 0, sizeof(sd));
    for (int j = 0; j < 3; ++j) {
        sd.r[4][j] = r0[j];
        sd.v[4][j] = v0[j];
    }
    for (int i = 1; i <= 4; ++i) {
        rk8_step(f, i, sd, gs);
        rk8_step(f, -i, sd, gs);
    }
}

// StartupCorrector::CalculateAccelerationMatrix (gpu_startup.cu:196-224)
template <typename R> void corr_accel(const Force& f, StartupT<R>& sd, bool epoch, GravScratchT<R>* gs)
{
    for (int i = 0; i < 9; ++i) {
        if (i == 4 && !epoch)
            continue;
        f.prop(sd.r[i], sd.v[i], i, sd.a[i], gs);
    }
}

// StartupCorrector::CalculateS0 (gpu_startup.cu:170-195): column 4 of s and S
template <typename R> void corr_s0(const Force& f, StartupT<R>& sd)
{
    R hinv = 1 / (R)f.h;
    R h2inv = 1 / ((R)f.h * (R)f.h);
    for (int j = 0; j < 3; ++j) {
        R sb = 0, sa = 0;
        for (int k = 0; k < 9; ++k) {
            sb += kSA[4][k] * sd.a[k][j];
            sa += kGJ[4][k] * sd.a[k][j];
        }
        sd.s[4][j] = hinv * sd.v[4][j] + (-sb);
        sd.S[4][j] = h2inv * sd.r[4][j] + (-sa);
    }
}

// CalculateAllSKernel (lib/gpu_startup/src/device/calculate_all_s.cu:19-47)
template <typename R> void corr_all_s(StartupT<R>& sd)
{
    for (int i = 1; i <= 4; ++i)
        for (int j = 0; j < 3; ++j) {
            sd.s[4 + i][j] = sd.s[4 + i - 1][j] + (sd.a[4 + i - 1][j] + sd.a[4 + i][j]) / 2;
            sd.s[4 - i][j] = sd.s[4 - i + 1][j] - (sd.a[4 - i + 1][j] + sd.a[4 - i][j]) / 2;
            sd.S[4 + i][j] = sd.s[4 + i - 1][j] + sd.S[4 + i - 1][j] + sd.a[4 + i - 1][j] / 2;
            sd.S[4 - i][j] = -sd.s[4 - i + 1][j] + sd.S[4 - i + 1][j] + sd.a[4 - i + 1][j] / 2;
        }
}

// StartupCorrector::Correct (gpu_startup.cu:247-294)
template <typename R> void corr_correct(const Force& f, StartupT<R>& sd, GravScratchT<R>* gs)
{
    corr_s0(f, sd);
    corr_all_s(sd);
    R h2 = (R)f.h * (R)f.h;
    for (int c = 0; c < 9; ++c) {
        if (c == 4)
            continue; // epoch column restored (MoveStateToTemp / MoveStateToMatrix)
        for (int j = 0; j < 3; ++j) {
            R sv = 0, sr = 0;
            for (int k = 0; k < 9; ++k) {
                sv += sd.a[k][j] * kSA[c][k];
                sr += sd.a[k][j] * kGJ[c][k];
            }
            sd.v[c][j] = (R)f.h * (sv + sd.s[c][j]);
            sd.r[c][j] = h2 * (sr + sd.S[c][j]);
        }
    }
    corr_accel(f, sd, false, gs);
}

template <typename R>
void startup_all(const Force& f, int ncorr, const R* r0, const R* v0, StartupT<R>& sd, GravScratchT<R>* gs)
{
    rk8_all(f, r0, v0, sd, gs); // GpuStartup::Startup (gpu_startup.cu:55-68)
    corr_accel(f, sd, true, gs);
    for (int i = 0; i < ncorr; ++i)
        corr_correct(f, sd, gs);
}

// Predictor::Predict (lib/gpu_integrator/src/prediction.cu:49-74) +
// FinalizePredictionKernel / MoveAccelerationsKernel (gpu_integrator/src/device/dev_functions.cu:20-50)
template <typename R>
void predict(const Force& f, int step, R* r, R* v, R (*acc)[3], R* s, R* S, GravScratchT<R>* gs)
{
    R vt[3], rt[3];
    for (int j = 0; j < 3; ++j) {
        R sv = 0, sr = 0;
        for (int k = 0; k < 9; ++k) {
            sv += acc[k][j] * kSA[9][k];
            sr += acc[k][j] * kGJ[9][k];
        }
        vt[j] = sv;
        rt[j] = sr;
    }
    for (int j = 0; j < 3; ++j) {
        S[j] += s[j] + acc[8][j] / 2;
        v[j] = (vt[j] + s[j] + acc[8][j] / 2) * (R)f.h;
        r[j] = (rt[j] + S[j]) * (R)f.h * (R)f.h;
    }
    for (int k = 0; k < 8; ++k)
        for (int j = 0; j < 3; ++j)
            acc[k][j] = acc[k + 1][j];
    f.prop(r, v, step + 4, acc[8], gs);
}

// GpuPropagator::Correct (lib/gpu_propagator/src/gpu_propagator.cu:86-119) + UpdateSmallSKernel and
// FinalizeCorrectionKernel (gpu_propagator/src/device/dev_functions.cu:36-69)
template <typename R>
void correct(const Force& f, int step, int ncorr, R* r, R* v, R (*acc)[3], R* s, const R* S,
    GravScratchT<R>* gs)
{
    R prev[3], s1[3], s2[3];
    for (int j = 0; j < 3; ++j) {
        prev[j] = s[j];
        R a1 = 0, a2 = 0;
        for (int k = 0; k < 8; ++k) {
            a1 += acc[k][j] * kSA[8][k];
            a2 += acc[k][j] * kGJ[8][k];
        }
        s1[j] = a1;
        s2[j] = a2;
    }
    for (int it = 0; it < ncorr; ++it) {
        f.prop(r, v, step + 4, acc[8], gs);
        for (int j = 0; j < 3; ++j)
            s[j] = prev[j] + (acc[8][j] + acc[7][j]) / 2;
        for (int j = 0; j < 3; ++j) {
            v[j] = (R)f.h * (s1[j] + acc[8][j] * kSA[8][8] + s[j]);
            r[j] = (R)f.h * (R)f.h * (s2[j] + acc[8][j] * kGJ[8][8] + S[j]);
        }
    }
}

template <typename R>
void propagate_one(const Force& f, int steps, int ncorr, const R* r0, const R* v0, int64_t n, int64_t obj,
    R* r_steps, R* v_steps, R* a_steps, R* rf, R* vf)
{
    GravScratchT<R> gs(*f.d);
    StartupT<R> sd;
    startup_all(f, ncorr, r0, v0, sd, &gs);
    R s[3], S[3], acc[9][3], r[3], v[3];
    for (int j = 0; j < 3; ++j) {
        s[j] = sd.s[8][j];
        S[j] = sd.S[8][j];
        r[j] = sd.r[8][j]; // the caller's buffer holds column 8 after startup
        v[j] = sd.v[8][j];
    }
    std::memcpy(acc, sd.a, sizeof(acc));
    for (int step = 1; step <= steps; ++step) {
        if (step <= 4) { // CopyStartupStateKernel (dev_functions.cu:22-34)
            for (int j = 0; j < 3; ++j) {
                r[j] = sd.r[step + 4][j];
                v[j] = sd.v[step + 4][j];
            }
        } else {
            predict(f, step, r, v, acc, s, S, &gs);
            correct(f, step, ncorr, r, v, acc, s, S, &gs);
        }
        size_t o = ((size_t)(step - 1) * n + obj) * 3;
        // Exported acceleration (MoveColumnToVectorKernel, column 8). Quirk Q3: for steps 1..4 the
        // reference exports the startup column 8 (t = 4h); OR_FLAG_FIX_Q3 exports column step+4.
        const R* ea = acc[8];
        if (step <= 4 && (f.flags & OR_FLAG_FIX_Q3))
            ea = sd.a[step + 4];
        for (int j = 0; j < 3; ++j) {
            if (r_steps)
                r_steps[o + j] = r[j];
            if (v_steps)
                v_steps[o + j] = v[j];
            if (a_steps)
                a_steps[o + j] = ea[j];
        }
    }
    if (steps == 0) {
        for (int j = 0; j < 3; ++j) {
            r[j] = r0[j];
            v[j] = v0[j];
        }
    }
    for (int j = 0; j < 3; ++j) {
        rf[j] = r[j];
        vf[j] = v[j];
    }
}

// ---------------- closest approach ----------------
struct Part {
    uint32_t num_sets;
    const uint32_t* set_ids;
    const uint32_t* set_offsets;
    const uint32_t* num_higher;
    const uint64_t* map_offsets;
};

// PartitionParameters::GetPartitionMapIdx (partition_parameters.cuh:50-69)
int64_t part_idx(const Part& p, uint32_t a, uint32_t b)
{
    if (a > b)
        std::swap(a, b);
    uint32_t sa = p.set_ids[a];
    if (sa == p.num_sets - 1)
        return -1;
    int64_t off1 = (int64_t)b - (int64_t)p.set_offsets[sa + 1];
    if (off1 < 0)
        return -1;
    return off1 + (int64_t)p.map_offsets[sa] + (int64_t)(a - p.set_offsets[sa]) * p.num_higher[sa];
}

// PartitionParameters::GetPartitionMapPair (partition_parameters.cuh:71-91)
bool part_pair(const Part& p, uint64_t idx, uint32_t& a, uint32_t& b)
{
    uint32_t sa = 0;
    while (sa < p.num_sets - 1 && p.map_offsets[sa + 1] <= idx)
        sa++;
    if (sa >= p.num_sets - 1)
        return false;
    uint64_t mo = p.map_offsets[sa];
    uint64_t hi = p.num_higher[sa];
    a = (uint32_t)((idx - mo) / hi) + p.set_offsets[sa];
    b = (uint32_t)((idx - mo) % hi) + p.set_offsets[sa + 1];
    return true;
}

// HermitePolynomial (lib/closest_approach/include/closest_approach/utility/interpolation.cuh:27-98)
template <typename R> struct HermiteT {
    R c[9];
    R dt;
    HermiteT() { }
    HermiteT(R p0, R v0, R a0, R p1, R v1, R a1, R p2, R v2, R a2, R dt_)
        : dt(dt_)
    {
        R t[9] = { 0.0, 0.0, 0.0, dt, dt, dt, 2.0 * dt, 2.0 * dt, 2.0 * dt };
        c[0] = c[1] = c[2] = p0;
        c[3] = c[4] = c[5] = p1;
        c[6] = c[7] = c[8] = p2;
        for (int j = 1; j < 9; j++)
            for (int i = 8; i >= j; i--) {
                if (t[i] == t[i - j]) {
                    if (j == 1)
                        c[i] = (i < 3) ? v0 : (i < 6) ? v1 : v2;
                    else if (j == 2)
                        c[i] = ((i < 3) ? a0 : (i < 6) ? a1 : a2) / 2.0;
                } else {
                    c[i] = (c[i] - c[i - 1]) / (t[i] - t[i - j]);
                }
            }
    }
    R operator()(R t) const
    {
        R z[9] = { 0.0, 0.0, 0.0, dt, dt, dt, 2.0 * dt, 2.0 * dt, 2.0 * dt };
        R res = c[0], term = 1.0;
        for (int i = 1; i < 9; ++i) {
            term *= (t - z[i - 1]);
            res += c[i] * term;
        }
        return res;
    }
    R deriv(R te) const
    {
        R z[9] = { 0.0, 0.0, 0.0, dt, dt, dt, 2.0 * dt, 2.0 * dt, 2.0 * dt };
        R res = 0.0, Nn = 1.0, dN = 0.0;
        for (int i = 0; i < 9; ++i) {
            res += c[i] * dN;
            if (i < 8) {
                dN = dN * (te - z[i]) + Nn;
                Nn *= (te - z[i]);
            }
        }
        return res;
    }
};
using Hermite = HermiteT<double>;

template <typename R> struct InterpT {
    HermiteT<R> x, y, z;
};
using Interp = InterpT<double>;

// ApproachFunc (interpolation.cuh:106-123)
template <typename R> R approach(const InterpT<R>& A, const InterpT<R>& B, R t)
{
    R dx = A.x(t) - B.x(t);
    R dy = A.y(t) - B.y(t);
    R dz = A.z(t) - B.z(t);
    R ddx = A.x.deriv(t) - B.x.deriv(t);
    R ddy = A.y.deriv(t) - B.y.deriv(t);
    R ddz = A.z.deriv(t) - B.z.deriv(t);
    return (dx * ddx) + (dy * ddy) + (dz * ddz);
}

// FindRoot (interpolation.cuh:126-152), secant
template <typename R, typename F> R find_root(F f, R x0, R x1, R tol = 1e-7, int max_iter = 100)
{
    R f0 = f(x0);
    R f1 = f(x1);
    for (int i = 0; i < max_iter; ++i) {
        if (std::fabs(f1 - f0) < R(1e-14))
            return x1;
        R xn = x1 - f1 * (x1 - x0) / (f1 - f0);
        R fn = f(xn);
        if (std::fabs(xn - x1) < tol || std::fabs(fn) < tol)
            return xn;
        x0 = x1;
        f0 = f1;
        x1 = xn;
        f1 = fn;
    }
    return x1;
}

// nodes27 layout: axis (x,y,z) x [before p,v,a; closest p,v,a; after p,v,a]
template <typename R> InterpT<R> make_interp(const R* n27, R dt)
{
    InterpT<R> I;
    HermiteT<R>* hs[3] = { &I.x, &I.y, &I.z };
    for (int ax = 0; ax < 3; ++ax) {
        const R* q = n27 + ax * 9;
        *hs[ax] = HermiteT<R>(q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8], dt);
    }
    return I;
}

// One pair's closest approach over stored trajectories [steps][3] of A and B (positions, velocities,
// exported accelerations): the running minimum and node capture of or_ca_screen for a single pair,
// then or_ca_refine's refinement. Templated so that the long double finite differences use it.
template <typename R>
void pair_closest(const R* rA, const R* vA, const R* aA, const R* rB, const R* vB, const R* aB, int steps,
    R h, R& miss, R& tca)
{
    R mind = std::numeric_limits<R>::max();
    uint32_t cs = 0xFFFFFFFFu;
    R nodes[54] = {};
    R last[18] = {}; // A then B: p, v, a (zero before the first step)
    auto put = [&](int o, int node, const R* p, const R* v, const R* a) {
        for (int ax = 0; ax < 3; ++ax) {
            nodes[o * 27 + ax * 9 + node * 3 + 0] = p[ax];
            nodes[o * 27 + ax * 9 + node * 3 + 1] = v[ax];
            nodes[o * 27 + ax * 9 + node * 3 + 2] = a[ax];
        }
    };
    for (int k = 0; k < steps; ++k) {
        const R *pa = rA + 3 * k, *va = vA + 3 * k, *xa = aA + 3 * k;
        const R *pb = rB + 3 * k, *vb = vB + 3 * k, *xb = aB + 3 * k;
        R dx = pa[0] - pb[0], dy = pa[1] - pb[1], dz = pa[2] - pb[2];
        R dist = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (dist < mind) {
            mind = dist;
            cs = (uint32_t)k;
            put(0, 1, pa, va, xa);
            put(1, 1, pb, vb, xb);
            put(0, 0, last, last + 3, last + 6);
            put(1, 0, last + 9, last + 12, last + 15);
        } else if (cs == (uint32_t)k - 1) {
            put(0, 2, pa, va, xa);
            put(1, 2, pb, vb, xb);
        }
        for (int j = 0; j < 3; ++j) {
            last[j] = pa[j];
            last[3 + j] = va[j];
            last[6 + j] = xa[j];
            last[9 + j] = pb[j];
            last[12 + j] = vb[j];
            last[15 + j] = xb[j];
        }
    }
    miss = mind;
    if (cs == 0) {
        tca = 0;
        return;
    }
    if (cs == (uint32_t)steps - 1) {
        tca = (R)steps * h;
        return;
    }
    InterpT<R> A = make_interp<R>(nodes, h), B = make_interp<R>(nodes + 27, h);
    R t = find_root<R>([&](R tt) { return approach<R>(A, B, tt); }, R(0), h);
    tca = t + (R)cs * h;
    R dx = A.x(t) - B.x(t), dy = A.y(t) - B.y(t), dz = A.z(t) - B.z(t);
    miss = std::sqrt(dx * dx + dy * dy + dz * dz);
}

int nthreads(int t)
{
#ifdef _OPENMP
    return t > 0 ? t : omp_get_max_threads();
#else
    (void)t;
    return 1;
#endif
}

} // namespace

// =====================================================================================
extern "C" {

void* or_data_load(const char* dir, int32_t degree)
{
    try {
        Data* d = new Data();
        std::string base(dir);
        if (!base.empty() && base.back() != '/')
            base += '/';
        load_gravity(base + "JGM3.gfc", degree, *d);
        load_nutation(base + "IAU2000_R06_NutLon.txt", d->lon0, d->lon1);
        load_nutation(base + "IAU2000_R06_NutObl.txt", d->obl0, d->obl1);
        load_eop(base + "IAU2000A_EOP.txt", d->eop);
        load_leap(base + "leap-seconds.list", d->leap_mjd, d->leap_val);
        return d;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return nullptr;
    }
}
void or_data_free(void* d) { delete static_cast<Data*>(d); }
int32_t or_data_degree(const void* d) { return (int32_t) static_cast<const Data*>(d)->N - 1; }
double or_data_gm(const void* d) { return static_cast<const Data*>(d)->GM; }
double or_data_radius(const void* d) { return static_cast<const Data*>(d)->R; }
int64_t or_data_eop_count(const void* d) { return (int64_t) static_cast<const Data*>(d)->eop.size(); }
int64_t or_data_leap_count(const void* d) { return (int64_t) static_cast<const Data*>(d)->leap_mjd.size(); }
int64_t or_data_nut_count(const void* dv, int32_t which)
{
    const Data* d = static_cast<const Data*>(dv);
    const std::vector<NutTerm>* t[4] = { &d->lon0, &d->lon1, &d->obl0, &d->obl1 };
    return (which >= 0 && which < 4) ? (int64_t)t[which]->size() : -1;
}
void or_data_eop_record(const void* d, double mjd, double out[4])
{
    EopRec r = eop_record(*static_cast<const Data*>(d), mjd);
    out[0] = r.mjd;
    out[1] = r.xp;
    out[2] = r.yp;
    out[3] = r.ut1;
}
double or_data_leap_seconds(const void* d, double mjd) { return leap_seconds(*static_cast<const Data*>(d), mjd); }
void or_data_coef(const void* dv, int32_t n, int32_t m, double* c, double* s)
{
    const Data* d = static_cast<const Data*>(dv);
    *c = d->C[tri(n, m)];
    *s = d->S[tri(n, m)];
}

double or_calendar_to_mjd(int32_t y, int32_t mon, int32_t day, int32_t h, int32_t min, double sec)
{
    return calendar_to_mjd(y, mon, day, h, min, sec);
}
void or_ftable(double t, double F[14]) { ftable(t, F); }
void or_precession(double t, double o[4]) { precession(t, o[0], o[1], o[2], o[3]); }
void or_nutation(const void* dv, double mjd_tt, double o[2])
{
    const Data* d = static_cast<const Data*>(dv);
    double t = (mjd_tt - kMjdJ2000) / 36525.0;
    double F[14];
    ftable(t, F);
    o[0] = nut_delta(F, d->lon0) + nut_delta(F, d->lon1) * t;
    o[1] = nut_delta(F, d->obl0) + nut_delta(F, d->obl1) * t;
}
double or_gast(double ut1, double tt, double dpsi, double epsA, const double F[14]) { return gast(ut1, tt, dpsi, epsA, F); }
double or_ntp_to_mjd(int64_t ntp) { return ntp_to_mjd(ntp); }
void or_rot(int32_t axis, double angle, double out[9])
{
    if (axis == 0)
        rot_x(angle, out);
    else if (axis == 1)
        rot_y(angle, out);
    else
        rot_z(angle, out);
}

void or_frame_matrices(const void* dv, const or_time* st, double h, int32_t count, int32_t mid,
    int32_t before, double* m_out, double* mjd_out)
{
    const Data* d = static_cast<const Data*>(dv);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < count; ++i)
        frame_matrix(*d, *st, table_sec(*st, h, i, mid != 0, before), m_out + (size_t)i * 9,
            mjd_out ? mjd_out + i : nullptr);
}

void or_gravity(const void* dv, int64_t n, const double* r, const double* m9, double* a)
{
    const Data* d = static_cast<const Data*>(dv);
#pragma omp parallel
    {
        GravScratch gs(*d);
#pragma omp for schedule(static)
        for (int64_t i = 0; i < n; ++i)
            gravity_gcrs(*d, m9, r + 3 * i, a + 3 * i, gs);
    }
}

static Force make_force(const void* dv, int32_t kind, const or_time* st, double h, int steps, uint32_t flags)
{
    Force f;
    f.d = static_cast<const Data*>(dv);
    f.kind = kind;
    f.h = h;
    f.flags = flags;
    if (kind == OR_FORCE_GRAVITY)
        build_tables(f, *st, steps);
    return f;
}

static void unpack27(const Startup& sd, double* r, double* v, double* a, double* s, double* S)
{
    if (r) std::memcpy(r, sd.r, 27 * sizeof(double));
    if (v) std::memcpy(v, sd.v, 27 * sizeof(double));
    if (a) std::memcpy(a, sd.a, 27 * sizeof(double));
    if (s) std::memcpy(s, sd.s, 27 * sizeof(double));
    if (S) std::memcpy(S, sd.S, 27 * sizeof(double));
}

void or_rk8(const void* dv, int32_t kind, const or_time* st, double h, const double r0[3],
    const double v0[3], uint32_t flags, double* r27, double* v27)
{
    Force f = make_force(dv, kind, st, h, 4, flags);
    std::vector<GravScratch> gs;
    if (f.d)
        gs.emplace_back(*f.d);
    Startup sd;
    rk8_all(f, r0, v0, sd, gs.empty() ? nullptr : &gs[0]);
    unpack27(sd, r27, v27, nullptr, nullptr, nullptr);
}

void or_startup(const void* dv, int32_t kind, const or_time* st, double h, int32_t ncorr,
    const double r0[3], const double v0[3], uint32_t flags, double* r27, double* v27, double* a27,
    double* s27, double* S27)
{
    Force f = make_force(dv, kind, st, h, 4, flags);
    std::vector<GravScratch> gs;
    if (f.d)
        gs.emplace_back(*f.d);
    Startup sd;
    startup_all(f, ncorr, r0, v0, sd, gs.empty() ? nullptr : &gs[0]);
    unpack27(sd, r27, v27, a27, s27, S27);
}

void or_corrector_unit(int32_t kind, double h, int32_t op, double* r27, double* v27, double* a27,
    double* s27, double* S27)
{
    Force f;
    f.kind = kind;
    f.h = h;
    Startup sd;
    std::memset(&sd, 0, sizeof(sd));
    std::memcpy(sd.r, r27, sizeof(sd.r));
    std::memcpy(sd.v, v27, sizeof(sd.v));
    corr_accel<double>(f, sd, true, nullptr);
    if (op == 1) {
        corr_s0(f, sd);
    } else if (op == 2) {
        corr_correct<double>(f, sd, nullptr);
    }
    unpack27(sd, r27, v27, a27, s27, S27);
}

void or_predict_unit(int32_t kind, double h, int32_t step, double* r, double* v, double* a27,
    double* s, double* S)
{
    Force f;
    f.kind = kind;
    f.h = h;
    predict<double>(f, step, r, v, reinterpret_cast<double(*)[3]>(a27), s, S, nullptr);
}

void or_finalize_correction_unit(double h, double* r, double* v, const double* a27, const double* s,
    const double* S)
{
    const double(*acc)[3] = reinterpret_cast<const double(*)[3]>(a27);
    for (int j = 0; j < 3; ++j) {
        v[j] = h * (v[j] + acc[8][j] * kSA[8][8] + s[j]);
        r[j] = h * h * (r[j] + acc[8][j] * kGJ[8][8] + S[j]);
    }
}

int32_t or_propagate(const void* dv, int32_t kind, const or_time* st, double h, int32_t steps,
    int32_t ncorr, int64_t n, const double* r0, const double* v0, uint32_t flags, double* r_steps,
    double* v_steps, double* a_steps, double* r_final, double* v_final, int32_t threads)
{
    if (n <= 0 || h == 0.0 || steps < 0)
        return 1;
    if (kind == OR_FORCE_GRAVITY && !dv)
        return 1;
    Force f = make_force(dv, kind, st, h, steps, flags);
    Data dummy;
    if (!f.d) {
        dummy.N = 1;
        f.d = &dummy;
    }
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads(threads))
    for (int64_t i = 0; i < n; ++i)
        propagate_one(f, steps, ncorr, r0 + 3 * i, v0 + 3 * i, n, i, r_steps, v_steps, a_steps,
            r_final + 3 * i, v_final + 3 * i);
    return 0;
}

int32_t or_partition(const uint32_t* ids, int64_t n, uint32_t* num_sets, uint64_t* num_pairs,
    uint32_t* set_offsets, uint32_t* num_higher, uint64_t* map_offsets)
{
    // PartitionParameters::Calculate (partition_parameters.cuh:94-135)
    std::vector<uint32_t> offs { 0 }, sizes, higher;
    std::vector<uint64_t> maps { 0 };
    uint32_t prev = ids[0], prev_change = 0;
    for (int64_t i = 1; i < n; ++i) {
        if (ids[i] < prev || ids[i] > prev + 1)
            return 0;
        if (ids[i] > prev) {
            offs.push_back((uint32_t)i);
            sizes.push_back((uint32_t)i - prev_change);
            higher.push_back((uint32_t)(n - i));
            maps.push_back(maps.back() + (uint64_t)sizes.back() * higher.back());
            prev_change = (uint32_t)i;
        }
        prev = ids[i];
    }
    sizes.push_back((uint32_t)n - prev_change);
    higher.push_back(0);
    *num_sets = (uint32_t)offs.size();
    *num_pairs = maps.back();
    std::copy(offs.begin(), offs.end(), set_offsets);
    std::copy(higher.begin(), higher.end(), num_higher);
    std::copy(maps.begin(), maps.end(), map_offsets);
    return 1;
}

int64_t or_partition_map_idx(const uint32_t* ids, uint32_t ns, const uint32_t* so, const uint32_t* nh,
    const uint64_t* mo, uint32_t a, uint32_t b)
{
    Part p { ns, ids, so, nh, mo };
    return part_idx(p, a, b);
}

int32_t or_partition_map_pair(uint32_t ns, const uint32_t* so, const uint32_t* nh, const uint64_t* mo,
    uint64_t idx, uint32_t* a, uint32_t* b)
{
    Part p { ns, nullptr, so, nh, mo };
    return part_pair(p, idx, *a, *b) ? 1 : 0;
}

void or_hermite_coeffs(const double q[9], double dt, double c[9])
{
    Hermite H(q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8], dt);
    std::memcpy(c, H.c, sizeof(H.c));
}
double or_hermite_eval(const double c[9], double dt, double t)
{
    Hermite H;
    std::memcpy(H.c, c, sizeof(H.c));
    H.dt = dt;
    return H(t);
}
double or_hermite_deriv(const double c[9], double dt, double t)
{
    Hermite H;
    std::memcpy(H.c, c, sizeof(H.c));
    H.dt = dt;
    return H.deriv(t);
}
double or_approach_func(const double* A27, const double* B27, double dt, double t)
{
    Interp A = make_interp(A27, dt), B = make_interp(B27, dt);
    return approach(A, B, t);
}
double or_find_root_approach(const double* A27, const double* B27, double dt, double x0, double x1,
    double tol, int32_t max_iter)
{
    Interp A = make_interp(A27, dt), B = make_interp(B27, dt);
    return find_root([&](double t) { return approach(A, B, t); }, x0, x1, tol, max_iter);
}
double or_find_root_test(int32_t fn, double x0, double x1, double tol, int32_t max_iter)
{
    auto f = [fn](double x) { return fn == 0 ? 3.0 * x - 6.0 : fn == 1 ? x * x - 9.0 : x * x; };
    return find_root(f, x0, x1, tol, max_iter);
}

// UpdateClosestApproachKernel (lib/closest_approach/src/device.cu:56-91) over a block of steps,
// race-free: "last" is the previous step's state of each object.
void or_ca_screen(int64_t n, int32_t steps, const double* r, const double* v, const double* a,
    const uint32_t* ids, uint32_t step_offset, int32_t init, or_ca_state* st, int32_t threads)
{
    std::vector<uint32_t> so(n), nh(n);
    std::vector<uint64_t> mo(n);
    uint32_t ns;
    uint64_t P;
    if (!or_partition(ids, n, &ns, &P, so.data(), nh.data(), mo.data()))
        return;
    Part p { ns, ids, so.data(), nh.data(), mo.data() };
    if (init) {
        for (uint64_t i = 0; i < P; ++i) {
            st->min_dist[i] = std::numeric_limits<double>::max();
            st->closest_step[i] = 0xFFFFFFFFu;
        }
        std::fill(st->nodes, st->nodes + P * 54, 0.0);
        std::fill(st->last, st->last + n * 9, 0.0);
    }
    // node layout per pair: [object o (0=A,1=B)][axis][node (before p,v,a; closest p,v,a; after p,v,a)]
    auto put = [&](uint64_t pi, int o, int node, int64_t obj, const double* pp, const double* vv,
                   const double* aa) {
        double* q = st->nodes + pi * 54 + o * 27;
        for (int ax = 0; ax < 3; ++ax) {
            q[ax * 9 + node * 3 + 0] = pp[obj * 3 + ax];
            q[ax * 9 + node * 3 + 1] = vv[obj * 3 + ax];
            q[ax * 9 + node * 3 + 2] = aa[obj * 3 + ax];
        }
    };
    std::vector<double> lp(n * 3), lv(n * 3), la(n * 3);
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            lp[i * 3 + c] = st->last[i * 9 + c];
            lv[i * 3 + c] = st->last[i * 9 + 3 + c];
            la[i * 3 + c] = st->last[i * 9 + 6 + c];
        }
    for (int k = 0; k < steps; ++k) {
        const double* pos = r + (size_t)k * n * 3;
        const double* vel = v + (size_t)k * n * 3;
        const double* acc = a + (size_t)k * n * 3;
        uint32_t stepNum = step_offset + (uint32_t)k;
#pragma omp parallel for schedule(static) num_threads(nthreads(threads))
        for (int64_t pi = 0; pi < (int64_t)P; ++pi) {
            uint32_t A, B;
            if (!part_pair(p, (uint64_t)pi, A, B))
                continue;
            double dx = pos[A * 3] - pos[B * 3];
            double dy = pos[A * 3 + 1] - pos[B * 3 + 1];
            double dz = pos[A * 3 + 2] - pos[B * 3 + 2];
            double dist = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (dist < st->min_dist[pi]) {
                st->min_dist[pi] = dist;
                st->closest_step[pi] = stepNum;
                put(pi, 0, 1, A, pos, vel, acc);
                put(pi, 1, 1, B, pos, vel, acc);
                put(pi, 0, 0, A, lp.data(), lv.data(), la.data());
                put(pi, 1, 0, B, lp.data(), lv.data(), la.data());
            } else if (st->closest_step[pi] == stepNum - 1) {
                put(pi, 0, 2, A, pos, vel, acc);
                put(pi, 1, 2, B, pos, vel, acc);
            }
        }
        std::memcpy(lp.data(), pos, n * 3 * sizeof(double));
        std::memcpy(lv.data(), vel, n * 3 * sizeof(double));
        std::memcpy(la.data(), acc, n * 3 * sizeof(double));
    }
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            st->last[i * 9 + c] = lp[i * 3 + c];
            st->last[i * 9 + 3 + c] = lv[i * 3 + c];
            st->last[i * 9 + 6 + c] = la[i * 3 + c];
        }
}

// CalculateClosestApproachesKernel (lib/closest_approach/src/device.cu:93-173)
void or_ca_refine(int64_t n, const uint32_t* ids, double h, uint32_t total_steps,
    const or_ca_state* st, double* dist_out, double* time_out, double* pa, double* pb, int32_t threads)
{
    std::vector<uint32_t> so(n), nh(n);
    std::vector<uint64_t> mo(n);
    uint32_t ns;
    uint64_t P;
    if (!or_partition(ids, n, &ns, &P, so.data(), nh.data(), mo.data()))
        return;
#pragma omp parallel for schedule(static) num_threads(nthreads(threads))
    for (int64_t pi = 0; pi < (int64_t)P; ++pi) {
        uint32_t cs = st->closest_step[pi];
        dist_out[pi] = st->min_dist[pi];
        // The reference leaves the positions unwritten when the minimum sits on the first or last
        // screened step (quirk Q5); both sides here report the sampled positions of that step.
        for (int c = 0; c < 3; ++c) {
            pa[pi * 3 + c] = st->nodes[pi * 54 + c * 9 + 3];
            pb[pi * 3 + c] = st->nodes[pi * 54 + 27 + c * 9 + 3];
        }
        if (cs == 0) {
            time_out[pi] = 0.0;
            continue;
        }
        if (cs == total_steps - 1) {
            time_out[pi] = (double)total_steps * h;
            continue;
        }
        const double* q = st->nodes + pi * 54;
        Interp A = make_interp(q, h), B = make_interp(q + 27, h);
        double t = find_root([&](double tt) { return approach(A, B, tt); }, 0.0, h);
        time_out[pi] = t + st->closest_step[pi] * h;
        double dx = A.x(t) - B.x(t);
        double dy = A.y(t) - B.y(t);
        double dz = A.z(t) - B.z(t);
        dist_out[pi] = std::sqrt(dx * dx + dy * dy + dz * dz);
        pa[pi * 3] = A.x(t);
        pa[pi * 3 + 1] = A.y(t);
        pa[pi * 3 + 2] = A.z(t);
        pb[pi * 3] = B.x(t);
        pb[pi * 3 + 1] = B.y(t);
        pb[pi * 3 + 2] = B.z(t);
    }
}

} // extern "C"

template <typename LD>
static int32_t miss_fd(const void* dv, const or_time* st, double h, int32_t steps, int32_t ncorr,
    int64_t n_pairs, const double* rA, const double* vA, const double* rB, const double* vB, double dr,
    double dvel, double* miss, double* tca, double* grad, int32_t threads)
{
    if (!dv || n_pairs <= 0 || steps < 1 || h == 0.0)
        return 1;
    Force f = make_force(dv, OR_FORCE_GRAVITY, st, h, steps, 0);
    // run 0: the pair as given; run 1 + 2 c + s: component c (0..11: r_A, v_A, r_B, v_B) moved by
    // +step (s = 0) or -step (s = 1)
    const int runs = 25;
    std::vector<LD> out((size_t)n_pairs * runs * 2, LD(0));
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads(threads))
    for (int64_t job = 0; job < n_pairs * runs; ++job) {
        const int64_t p = job / runs;
        const int run = (int)(job % runs);
        LD x0[2][6];
        for (int j = 0; j < 3; ++j) {
            x0[0][j] = rA[3 * p + j];
            x0[0][3 + j] = vA[3 * p + j];
            x0[1][j] = rB[3 * p + j];
            x0[1][3 + j] = vB[3 * p + j];
        }
        if (run > 0) {
            const int c = (run - 1) / 2;
            const LD stepv = c % 6 < 3 ? (LD)dr : (LD)dvel;
            x0[c / 6][c % 6] += (run - 1) % 2 == 0 ? stepv : -stepv;
        }
        std::vector<LD> tr[2][3];
        LD rf[3], vf[3];
        for (int o = 0; o < 2; ++o) {
            for (int k = 0; k < 3; ++k)
                tr[o][k].assign((size_t)steps * 3, LD(0));
            propagate_one<LD>(f, steps, ncorr, x0[o], x0[o] + 3, 1, 0, tr[o][0].data(), tr[o][1].data(),
                tr[o][2].data(), rf, vf);
        }
        LD m, t;
        pair_closest<LD>(tr[0][0].data(), tr[0][1].data(), tr[0][2].data(), tr[1][0].data(), tr[1][1].data(),
            tr[1][2].data(), steps, (LD)h, m, t);
        out[(size_t)job * 2] = m;
        out[(size_t)job * 2 + 1] = t;
    }
    for (int64_t p = 0; p < n_pairs; ++p) {
        const LD* o = out.data() + (size_t)p * runs * 2;
        miss[p] = (double)o[0];
        tca[p] = (double)o[1];
        for (int c = 0; c < 12; ++c) {
            const LD stepv = c % 6 < 3 ? (LD)dr : (LD)dvel;
            grad[p * 12 + c] = (double)((o[(1 + 2 * c) * 2] - o[(2 + 2 * c) * 2]) / (2 * stepv));
        }
    }
    return 0;
}

extern "C" {

int32_t or_miss_fd_ld(const void* dv, const or_time* st, double h, int32_t steps, int32_t ncorr,
    int64_t n_pairs, const double* rA, const double* vA, const double* rB, const double* vB, double dr,
    double dvel, double* miss, double* tca, double* grad, int32_t threads)
{
    return miss_fd<long double>(dv, st, h, steps, ncorr, n_pairs, rA, vA, rB, vB, dr, dvel, miss, tca, grad,
        threads);
}

int32_t or_miss_fd(const void* dv, const or_time* st, double h, int32_t steps, int32_t ncorr,
    int64_t n_pairs, const double* rA, const double* vA, const double* rB, const double* vB, double dr,
    double dvel, double* miss, double* tca, double* grad, int32_t threads)
{
    return miss_fd<double>(dv, st, h, steps, ncorr, n_pairs, rA, vA, rB, vB, dr, dvel, miss, tca, grad,
        threads);
}

} // extern "C"
