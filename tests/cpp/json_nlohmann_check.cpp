// The CLI's JSON writer (opengpop_b200/csrc/json.h) against nlohmann::json 3.11.3, the library the
// reference CLI writes its output with (exec/main.cpp:87-88,100-101: jOutput.dump(4)). Compiled
// by the test with the nlohmann header found in the Python environment (it is not part of this
// repository). Checks number formatting on edge values and about a million random doubles, string
// escaping, and whole propagate / closest-approach output documents byte for byte.
// Prints one line per mismatch (at most 20) and exits 0 when everything matches.
#include "json.h"

#include <nlohmann/json.hpp>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>
#include <string>
#include <vector>

using gpop::json::Value;

static int g_bad = 0;

static void check_number(double d)
{
    const std::string ours = gpop::json::format_double(d);
    const std::string theirs = nlohmann::json(d).dump();
    if (ours != theirs && ++g_bad <= 20)
        std::printf("number %.17g (bits %016llx): ours %s, nlohmann %s\n", d,
            (unsigned long long)[&] { uint64_t u; std::memcpy(&u, &d, 8); return u; }(), ours.c_str(),
            theirs.c_str());
}

static void check_string(const std::string& s)
{
    std::string ours;
    gpop::json::escape(ours, s);
    const std::string theirs = nlohmann::json(s).dump();
    if (ours != theirs && ++g_bad <= 20)
        std::printf("string of %zu bytes: ours %s, nlohmann %s\n", s.size(), ours.c_str(), theirs.c_str());
}

static Value vec3_list(const std::vector<double>& x)
{
    Value a = Value::array();
    for (size_t i = 0; i + 2 < x.size(); i += 3) {
        Value p = Value::array();
        for (int c = 0; c < 3; ++c)
            p.arr.push_back(Value::number(x[i + c]));
        a.arr.push_back(p);
    }
    return a;
}

static nlohmann::json vec3_list_n(const std::vector<double>& x)
{
    nlohmann::json a = nlohmann::json::array();
    for (size_t i = 0; i + 2 < x.size(); i += 3)
        a.push_back(nlohmann::json::array({ x[i], x[i + 1], x[i + 2] }));
    return a;
}

static void check_documents(std::mt19937_64& rng)
{
    std::uniform_real_distribution<double> pos(-4.2e7, 4.2e7), vel(-8000.0, 8000.0), dist(0.0, 5000.0),
        tim(0.0, 259200.0);
    for (int doc = 0; doc < 20; ++doc) {
        const int n = doc == 0 ? 0 : 1 + doc * 3;
        std::vector<double> r(3 * n), v(3 * n), r2(3 * n), v2(3 * n);
        for (int i = 0; i < 3 * n; ++i) {
            r[i] = doc == 1 ? 7.0e6 : pos(rng);
            v[i] = doc == 1 ? 0.0 : vel(rng);
            r2[i] = pos(rng);
            v2[i] = vel(rng);
        }
        const double sec = doc % 2 ? 42.0 : 0.125 * doc;
        // propagate output (PropagationOutput of exec/runner.cuh)
        Value start = Value::object();
        start.obj["Year"] = Value::integer(2023);
        start.obj["Month"] = Value::integer(4);
        start.obj["Day"] = Value::integer(29);
        start.obj["Hour"] = Value::integer(22);
        start.obj["Min"] = Value::integer(59);
        start.obj["Sec"] = Value::number(sec);
        Value top = Value::object();
        top.obj["propagationStart"] = start;
        top.obj["propagationSeconds"] = Value::integer(86400 + doc);
        top.obj["positionsStart"] = vec3_list(r);
        top.obj["velocitiesStart"] = vec3_list(v);
        top.obj["positionsEnd"] = vec3_list(r2);
        top.obj["velocitiesEnd"] = vec3_list(v2);
        nlohmann::json jt = { { "Year", 2023 }, { "Month", 4 }, { "Day", 29 }, { "Hour", 22 },
            { "Min", 59 }, { "Sec", sec } };
        nlohmann::json j;
        j["propagationStart"] = jt;
        j["propagationSeconds"] = 86400 + doc;
        j["positionsStart"] = vec3_list_n(r);
        j["velocitiesStart"] = vec3_list_n(v);
        j["positionsEnd"] = vec3_list_n(r2);
        j["velocitiesEnd"] = vec3_list_n(v2);
        if (gpop::json::dump(top, 4) != j.dump(4) && ++g_bad <= 20)
            std::printf("propagate document %d differs\n", doc);
        // closest-approach output (ClosestApproachOutput), whole-document and streaming writers
        Value ca = Value::object();
        ca.obj["propagationStart"] = start;
        ca.obj["propagationSeconds"] = Value::integer(259200);
        ca.obj["positionsStart"] = vec3_list(r);
        ca.obj["velocitiesStart"] = vec3_list(v);
        nlohmann::json jc;
        jc["propagationStart"] = jt;
        jc["propagationSeconds"] = 259200;
        jc["positionsStart"] = vec3_list_n(r);
        jc["velocitiesStart"] = vec3_list_n(v);
        jc["closestApproaches"] = nlohmann::json::array();
        std::vector<Value> recs;
        for (int k = 0; k < n * 2; ++k) {
            const double d = k == 0 ? 0.0 : dist(rng), t = k == 1 ? 0.0 : tim(rng);
            Value x = Value::object();
            x.obj["objectIndex1"] = Value::integer(k / 2);
            x.obj["objectIndex2"] = Value::integer(k + 1);
            x.obj["distance"] = Value::number(d);
            x.obj["time"] = Value::number(t);
            const char* keys[6] = { "positionAx", "positionAy", "positionAz", "positionBx", "positionBy",
                "positionBz" };
            nlohmann::json jx = { { "objectIndex1", k / 2 }, { "objectIndex2", k + 1 }, { "distance", d },
                { "time", t } };
            for (int c = 0; c < 6; ++c) {
                const double p = pos(rng);
                x.obj[keys[c]] = Value::number(p);
                jx[keys[c]] = p;
            }
            recs.push_back(x);
            jc["closestApproaches"].push_back(jx);
        }
        Value whole = ca;
        whole.obj["closestApproaches"] = Value::array();
        whole.obj["closestApproaches"].arr = recs;
        const std::string expect = jc.dump(4);
        if (gpop::json::dump(whole, 4) != expect && ++g_bad <= 20)
            std::printf("closest-approach document %d differs\n", doc);
        std::ostringstream os;
        gpop::json::dump_streaming(os, ca, "closestApproaches", recs.size(),
            [&](size_t e) -> const Value& { return recs[e]; });
        if (os.str() != expect && ++g_bad <= 20)
            std::printf("streamed closest-approach document %d differs\n", doc);
    }
}

int main()
{
    const double edge[] = { 0.0, -0.0, 1.0, -1.0, 0.5, 7.0e6, -7.0e6, 6878136.3, 7612.6081732238688,
        1e15, 1e16, 9.99e14, 999999999999999.0, 1234567890123456.0, 1e-4, 1e-5, 1.5e-5, 0.00012345,
        -0.0001, 1e-300, 1e300, 1.7976931348623157e308, 4.9406564584124654e-324,
        2.2250738585072014e-308, 2.2250738585072009e-308, 0.1, 0.2, 0.3, 1.0 / 3.0, 2.0 / 3.0,
        123456789012345.0, 12345678901234567.0, 100.0, 1e21, 1e22, 1e23, 5e-324, 9007199254740993.0,
        3.14159265358979, 86400.0, 259200.0, 42.0, 0.001, 29.999999999999996, 1e7, 1e-7 };
    for (double d : edge)
        check_number(d);
    std::mt19937_64 rng(20240101);
    std::uniform_real_distribution<double> u01(0.0, 1.0);
    std::uniform_int_distribution<int> expo(-330, 310);
    for (int i = 0; i < 300000; ++i) {
        // random bit patterns (finite ones)
        uint64_t bits = rng();
        double d;
        std::memcpy(&d, &bits, 8);
        if (std::isfinite(d))
            check_number(d);
        // magnitudes spread over the whole exponent range
        check_number((u01(rng) - 0.5) * std::pow(10.0, expo(rng)));
        // the ranges this CLI writes: positions, velocities, distances, times
        check_number((u01(rng) - 0.5) * 8.4e7);
        check_number((u01(rng) - 0.5) * 1.6e4);
    }
    for (int i = 0; i < 100000; ++i) {
        // short decimals and integral values, where the fixed/exponent choice matters
        const int digits = 1 + (int)(rng() % 17);
        const double m = (double)(rng() % (uint64_t)std::pow(10.0, std::min(digits, 15)));
        check_number(m * std::pow(10.0, (int)(rng() % 40) - 20));
        check_number((double)(int64_t)(rng() >> (rng() % 64)));
    }
    check_string("");
    check_string("propagationStart");
    check_string(std::string("a\"b\\c\b\f\n\r\t\x01\x1f\x7f end", 17));
    check_string("caf\xc3\xa9 \xe2\x82\xac");
    check_documents(rng);
    if (g_bad)
        std::printf("%d mismatches\n", g_bad);
    else
        std::printf("ok\n");
    return g_bad ? 1 : 0;
}
