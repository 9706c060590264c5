// model.cpp -- model data loaders and gravity-table builder (host side of the product).
#include "model.h"

#include <cstring>

#include <cmath>
#include <fstream>
#include <sstream>

namespace gpop {
namespace {

constexpr double kPi = 3.14159265358979324;
constexpr double kArcsPerRad = 3600.0 * 180.0 / kPi; // force_model/constants.cuh:22

inline size_t tri(size_t n, size_t m) { return n * (n + 1) / 2 + m; }

// Nutation series loader, same acceptance rules as dataset_loaders.cu:30-91: a "j = 0"/"j = 1" line
// selects the series; a data row is an index, two amplitudes and 14 integer multipliers.
bool load_nutation(const std::string& path, std::vector<NutTerm>& j0, std::vector<NutTerm>& j1,
    std::string& err)
{
    std::ifstream f(path);
    if (!f.is_open()) {
        err = "cannot open " + path;
        return false;
    }
    std::string line;
    int series = 0;
    while (std::getline(f, line)) {
        if (line.find("j = 0") != std::string::npos) {
            series = 0;
            continue;
        }
        if (line.find("j = 1") != std::string::npos) {
            series = 1;
            continue;
        }
        std::istringstream is(line);
        int index;
        NutTerm t {};
        if (!(is >> index) || !(is >> t.sin_uas >> t.cos_uas))
            continue;
        bool ok = true;
        for (int k = 0; k < 14 && ok; ++k) {
            int a;
            if (!(is >> a) || a < -127 || a > 127)
                ok = false;
            else
                t.args[k] = (int8_t)a;
        }
        if (ok)
            (series == 0 ? j0 : j1).push_back(t);
    }
    if (j0.empty()) {
        err = "no nutation terms in " + path;
        return false;
    }
    return true;
}

// finals2000A fixed-width columns (dataset_loaders.cu:93-158): MJD 7..14, x_p 18..26, y_p 37..45
// (arcsec), UT1-UTC 58..67 (s). Rows shorter than 68 characters or unparsable are skipped.
bool load_eop(const std::string& path, std::vector<EopRec>& out, std::string& err)
{
    std::ifstream f(path);
    if (!f.is_open()) {
        err = "cannot open " + path;
        return false;
    }
    std::string line;
    while (std::getline(f, line)) {
        size_t e = line.find_last_not_of(" \t\n\r\f\v");
        line.erase(e == std::string::npos ? 0 : e + 1);
        if (line.empty() || line[0] == '#' || line.size() < 68)
            continue;
        try {
            EopRec r;
            r.mjd = std::stod(line.substr(7, 8));
            r.xp = std::stod(line.substr(18, 9)) / kArcsPerRad;
            r.yp = std::stod(line.substr(37, 9)) / kArcsPerRad;
            r.ut1 = std::stod(line.substr(58, 10));
            out.push_back(r);
        } catch (const std::exception&) {
        }
    }
    if (out.empty()) {
        err = "no EOP records in " + path;
        return false;
    }
    return true;
}

// leap-seconds.list (dataset_loaders.cu:160-217): "<NTP seconds> <TAI-UTC>" rows.
bool load_leap(const std::string& path, std::vector<double>& mjd, std::vector<double>& val,
    std::string& err)
{
    std::ifstream f(path);
    if (!f.is_open()) {
        err = "cannot open " + path;
        return false;
    }
    std::string line;
    while (std::getline(f, line)) {
        size_t first = line.find_first_not_of(" \t");
        if (first == std::string::npos || line[first] == '#')
            continue;
        std::istringstream is(line);
        long long ntp;
        double dtai;
        if (is >> ntp >> dtai) {
            mjd.push_back(15020.0 + static_cast<double>(ntp) / 86400.0);
            val.push_back(dtai);
        }
    }
    if (mjd.empty()) {
        err = "no leap seconds in " + path;
        return false;
    }
    return true;
}

// ICGEM gfc reader (dataset_loaders.cu:219-299) with truncation to `degree`.
bool load_gfc(const std::string& path, int degree, ModelData& md, std::string& err)
{
    std::ifstream f(path);
    if (!f.is_open()) {
        err = "cannot open " + path;
        return false;
    }
    std::string line;
    bool head = false;
    int max_degree = -1;
    while (std::getline(f, line)) {
        if (line.find("end_of_head") != std::string::npos) {
            head = true;
            break;
        }
        std::istringstream is(line);
        std::string key;
        is >> key;
        if (key == "earth_gravity_constant")
            is >> md.gm;
        else if (key == "radius")
            is >> md.radius;
        else if (key == "max_degree")
            is >> max_degree;
    }
    if (!head) {
        err = "invalid ICGEM file (no end_of_head): " + path;
        return false;
    }
    if (max_degree < 2 || md.gm <= 0 || md.radius <= 0) {
        err = "invalid ICGEM header in " + path;
        return false;
    }
    int L = (degree > 0 && degree < max_degree) ? degree : max_degree;
    md.degree = L;
    md.C.assign(tri(L + 1, 0), 0.0);
    md.S.assign(tri(L + 1, 0), 0.0);
    bool first = true;
    while (std::getline(f, line)) {
        if (line.empty())
            continue;
        std::istringstream is(line);
        std::string key;
        is >> key;
        if (first) {
            if (key != "gfc") {
                err = "only static gravity models (gfc) are accepted, found: " + key;
                return false;
            }
            first = false;
        }
        if (key != "gfc")
            continue;
        unsigned n, m;
        double c, s;
        if ((is >> n >> m >> c >> s) && (int)n <= L && m <= n) {
            md.C[tri(n, m)] = c;
            md.S[tri(n, m)] = s;
        }
    }
    return true;
}

} // namespace

bool load_model(const std::string& dir, int degree, ModelData& out, std::string& err)
{
    std::string base = dir;
    if (!base.empty() && base.back() != '/')
        base += '/';
    return load_gfc(base + "JGM3.gfc", degree, out, err)
        && load_nutation(base + "IAU2000_R06_NutLon.txt", out.lon0, out.lon1, err)
        && load_nutation(base + "IAU2000_R06_NutObl.txt", out.obl0, out.obl1, err)
        && load_eop(base + "IAU2000A_EOP.txt", out.eop, err)
        && load_leap(base + "leap-seconds.list", out.leap_mjd, out.leap_val, err);
}

void build_gravity_tables(const ModelData& md, std::vector<GravEntry64>& t64, std::vector<GravEntry32>& t32)
{
    const int L = md.degree;
    t64.assign(grav_entries(L), GravEntry64 {});
    t32.assign(grav_entries(L), GravEntry32 {});
    // Diagonal of the derived Legendre functions (gravity_source.cu:76-89), in long double.
    std::vector<long double> pdiag(L + 1);
    pdiag[0] = 1.0L;
    if (L >= 1)
        pdiag[1] = std::sqrt(3.0L);
    for (int i = 2; i <= L; ++i)
        pdiag[i] = pdiag[i - 1] * std::sqrt((2.0L * i + 1.0L) / (2.0L * i));
    for (int m = 0; m <= L; ++m) {
        long double sigma = pdiag[m];
        for (int n = m; n <= L; ++n) {
            if (n > m) { // sigma(n,m) = xi(n,m) sigma(n-1,m); xi of gravity_source_device.cu:37
                long double nn = n, mm = m;
                sigma *= std::sqrt((2.0L * nn - 1.0L) * (2.0L * nn + 1.0L) / ((nn - mm) * (nn + mm)));
            }
            GravEntry64& e = t64[grav_col_offset(m, L) + (n - m)];
            long double c = 0.0L;
            if (n >= m + 2)
                c = ((long double)(n - 1) * (n - 1) - (long double)m * m)
                    / ((2.0L * n - 1.0L) * (2.0L * n - 3.0L));
            e.c = (double)c;
            if (n >= 2) {
                long double Cnm = md.C[tri(n, m)], Snm = md.S[tri(n, m)];
                e.g1 = (double)(sigma * (1 + n + m) * Cnm);
                e.g2 = (double)(sigma * (1 + n + m) * Snm);
                e.j1 = (double)(sigma * Cnm);
                e.j2 = (double)(sigma * Snm);
                if (m >= 1) {
                    int mp = m - 1; // zeta(n, m-1) of gravity_source_device.cu:40-45
                    long double zeta = (mp == 0) ? std::sqrt((long double)n * (n + 1.0L) / 2.0L)
                                                 : std::sqrt((long double)(n - mp) * (n + mp + 1.0L));
                    e.h1 = (double)(sigma * zeta * (long double)md.C[tri(n, mp)]);
                    e.h2 = (double)(sigma * zeta * (long double)md.S[tri(n, mp)]);
                }
            }
            GravEntry32& f = t32[grav_col_offset(m, L) + (n - m)];
            f.c = f.pad = (float)(-e.c); // the FP32 walk adds (-c w) Q(n-2), packed in pairs
            f.g1 = (float)e.g1;
            f.g2 = (float)e.g2;
            f.j1 = (float)e.j1;
            f.j2 = (float)e.j2;
            f.h1 = (float)e.h1;
            f.h2 = (float)e.h2;
        }
    }
}

void build_lane_blob(const GravEntry64* t64, int L64, const GravEntry32* t32, int L32,
    std::vector<uint8_t>& blob, uint32_t& off32)
{
    // column bases in 16-byte units: base(m) = m (mod 8), each column after the previous one
    auto bases = [](int L, int quads_per_entry, std::vector<int>& b) {
        b.assign(L + 2, 0);
        int q = 0;
        for (int m = 0; m <= L + 1; ++m) {
            while (q % 8 != m % 8)
                ++q;
            b[m] = q;
            if (m <= L)
                q += quads_per_entry * (L - m + 1);
        }
    };
    std::vector<int> b64, b32;
    bases(L64, 4, b64);
    const size_t bytes64 = (size_t)(b64[L64 + 1] + 4) * 16; // one zero entry past the end
    off32 = (uint32_t)(((kLaneOff64 + bytes64) + 127) / 128 * 128);
    size_t total = off32;
    if (t32) {
        bases(L32, 2, b32);
        total += (size_t)(b32[L32 + 1] + 2) * 16;
    }
    blob.assign(total, 0);
    int* cb64 = reinterpret_cast<int*>(blob.data());
    int* cb32 = reinterpret_cast<int*>(blob.data() + 512);
    for (int m = 0; m <= L64; ++m) {
        cb64[m] = b64[m];
        std::memcpy(blob.data() + kLaneOff64 + (size_t)b64[m] * 16, t64 + grav_col_offset(m, L64),
            sizeof(GravEntry64) * (L64 - m + 1));
    }
    if (t32)
        for (int m = 0; m <= L32; ++m) {
            cb32[m] = b32[m];
            std::memcpy(blob.data() + off32 + (size_t)b32[m] * 16, t32 + grav_col_offset(m, L32),
                sizeof(GravEntry32) * (L32 - m + 1));
        }
}

} // namespace gpop
