// exec_main.cpp -- the `exec` command line of the reference (exec/main.cpp:52-107,
// exec/runner.cu:11-119) over libgpop.so.
//
//   gpop_exec propagate        -i in.json [-o propagation_out.json]
//   gpop_exec closest-approach -i in.json [-o closest_approach_out.json]
//
// Same subcommands, options, defaults, input keys and output keys as the reference. Added options
// (defaults keep the reference behaviour): --step S (the reference fixes the step near 30 s),
// --degree L, --precision fp64|mixed, --threshold M (closest approach: only pairs with distance
// below M metres; default: every cross-set pair), --data DIR, --device D.
#include "gpop.h"
#include "json.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

using gpop::json::Value;

namespace {

constexpr double kIdealStepSize = 30.0; // exec/runner.cuh:6

struct Options {
    std::string cmd, input, output, data_dir;
    double step = 0.0, threshold = -1.0;
    int degree = 0, device = 0;
    std::string precision = "fp64";
};

int usage(const char* prog, const std::string& msg)
{
    if (!msg.empty())
        std::cerr << msg << "\n";
    std::cerr << "Open GPU-Parallelised Orbit Propagator (B200)\n"
              << "Usage: " << prog << " {propagate|closest-approach} -i,--input FILE [-o,--output FILE]\n"
              << "       [--step S] [--degree L] [--precision fp64|mixed] [--threshold M] [--data DIR]"
                 " [--device D]\n";
    return 109; // the exit code CLI11 uses for a parse error
}

std::string default_data_dir(const char* argv0)
{
    // <pkg>/bin/gpop_exec -> <pkg>/data
    std::string p(argv0);
    const size_t slash = p.rfind('/');
    std::string dir = slash == std::string::npos ? std::string(".") : p.substr(0, slash);
    return dir + "/../data";
}

gpop_time read_time(const Value& t)
{
    gpop_time out;
    out.year = (int32_t)t.at("Year").as_int();
    out.month = (int32_t)t.at("Month").as_int();
    out.day = (int32_t)t.at("Day").as_int();
    out.hour = (int32_t)t.at("Hour").as_int();
    out.min = (int32_t)t.at("Min").as_int();
    out.sec = t.at("Sec").as_double();
    return out;
}

Value write_time(const gpop_time& t)
{
    Value o = Value::object();
    o.obj["Year"] = Value::integer(t.year);
    o.obj["Month"] = Value::integer(t.month);
    o.obj["Day"] = Value::integer(t.day);
    o.obj["Hour"] = Value::integer(t.hour);
    o.obj["Min"] = Value::integer(t.min);
    o.obj["Sec"] = Value::number(t.sec);
    return o;
}

std::vector<double> read_vec3s(const Value& a, const char* name)
{
    if (a.kind != Value::Array)
        throw std::runtime_error(std::string(name) + " must be an array");
    std::vector<double> out;
    out.reserve(a.arr.size() * 3);
    for (const Value& e : a.arr) {
        if (e.kind != Value::Array || e.arr.size() != 3)
            throw std::runtime_error(std::string(name) + " must hold [x, y, z] triples");
        for (const Value& c : e.arr)
            out.push_back(c.as_double());
    }
    return out;
}

Value write_vec3s(const double* v, size_t n)
{
    Value a = Value::array();
    a.arr.reserve(n);
    for (size_t i = 0; i < n; ++i) {
        Value t = Value::array();
        for (int c = 0; c < 3; ++c)
            t.arr.push_back(Value::number(v[i * 3 + c]));
        a.arr.push_back(std::move(t));
    }
    return a;
}

int fail_ctx(gpop_ctx* ctx, gpop_status st, const char* what)
{
    std::cerr << "Error: " << what << ": " << gpop_status_string(st) << ": "
              << (ctx ? gpop_last_error(ctx) : "") << "\n";
    return 1;
}

int run(const Options& o)
{
    std::ifstream ifs(o.input);
    if (!ifs.is_open()) {
        std::cerr << "--input: File does not exist: " << o.input << "\n";
        return 105;
    }
    std::stringstream ss;
    ss << ifs.rdbuf();
    Value in = gpop::json::parse(ss.str());
    const gpop_time start = read_time(in.at("propagationStart"));
    const int64_t seconds = in.at("propagationSeconds").as_int();
    std::vector<double> r = read_vec3s(in.at("positions"), "positions");
    std::vector<double> v = read_vec3s(in.at("velocities"), "velocities");
    const int64_t n = (int64_t)r.size() / 3;
    if ((int64_t)v.size() != 3 * n)
        throw std::runtime_error("positions and velocities differ in size");
    // step rule of exec/runner.cu:13-15: floor(seconds / 30) steps of seconds / steps
    int64_t steps;
    double h;
    if (o.step > 0) {
        steps = (int64_t)std::floor((double)seconds / o.step);
        h = steps > 0 ? (double)seconds / (double)steps : o.step;
    } else {
        steps = (int64_t)((double)seconds / kIdealStepSize);
        h = steps > 0 ? (double)seconds / (double)steps : kIdealStepSize;
    }
    if (steps <= 0)
        throw std::runtime_error("propagationSeconds too short for one step");

    gpop_config cfg;
    gpop_config_default(&cfg);
    cfg.data_dir = o.data_dir.c_str();
    cfg.device = o.device;
    cfg.gravity_degree = o.degree;
    cfg.precision = o.precision == "mixed" ? GPOP_MIXED : GPOP_FP64;
    gpop_ctx* ctx = nullptr;
    gpop_status st = gpop_create(&cfg, &ctx);
    if (st != GPOP_OK) {
        int rc = fail_ctx(ctx, st, "initialising the force model");
        gpop_destroy(ctx);
        return rc;
    }
    Value out = Value::object();
    std::vector<gpop_ca_record> ca_records;
    bool streamed = false; // closestApproaches written record by record
    out.obj["propagationStart"] = write_time(start);
    out.obj["propagationSeconds"] = Value::integer(seconds);
    out.obj["positionsStart"] = write_vec3s(r.data(), n);
    out.obj["velocitiesStart"] = write_vec3s(v.data(), n);
    const auto t0 = std::chrono::steady_clock::now();
    if (o.cmd == "propagate") {
        std::vector<double> re(r.size()), ve(v.size());
        st = gpop_propagate(ctx, &start, h, (int32_t)steps, n, r.data(), v.data(), re.data(), ve.data());
        if (st != GPOP_OK) {
            int rc = fail_ctx(ctx, st, "propagation");
            gpop_destroy(ctx);
            return rc;
        }
        out.obj["positionsEnd"] = write_vec3s(re.data(), n);
        out.obj["velocitiesEnd"] = write_vec3s(ve.data(), n);
    } else {
        const Value& sets = in.at("setIndices");
        std::vector<uint32_t> ids;
        for (const Value& e : sets.arr)
            ids.push_back((uint32_t)e.as_int());
        if ((int64_t)ids.size() != n) {
            std::cerr << "Error: Size mismatch. Positions: " << n << ", setIndices: " << ids.size() << "\n";
            gpop_destroy(ctx);
            return 1;
        }
        gpop_ca* ca = nullptr;
        st = gpop_ca_create(ctx, &start, h, n, r.data(), v.data(), ids.data(), &ca);
        if (st == GPOP_OK)
            st = gpop_ca_propagate(ca, (int32_t)steps);
        int64_t count = 0;
        if (st == GPOP_OK)
            st = gpop_ca_find(ca, o.threshold, nullptr, 0, &count);
        std::vector<gpop_ca_record> recs(count > 0 ? count : 0);
        if (st == GPOP_OK && count > 0)
            st = gpop_ca_find(ca, o.threshold, recs.data(), count, &count);
        if (st != GPOP_OK) {
            int rc = fail_ctx(ctx, st, "closest approach");
            gpop_ca_destroy(ca);
            gpop_destroy(ctx);
            return rc;
        }
        ca_records = std::move(recs);
        gpop_ca_destroy(ca);
        streamed = true;
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cerr << "Computed " << n << " objects x " << steps << " steps of " << h << " s in " << secs << " s\n";
    gpop_destroy(ctx);
    std::ofstream ofs(o.output);
    if (!ofs.is_open()) {
        std::cerr << "Error: cannot write " << o.output << "\n";
        return 1;
    }
    if (streamed) {
        gpop::json::dump_streaming(ofs, out, "closestApproaches", ca_records.size(), [&](size_t k) {
            const gpop_ca_record& rc = ca_records[k]; // exec/runner.cu:96-106, main.cpp:35-36 keys
            Value x = Value::object();
            x.obj["objectIndex1"] = Value::integer(rc.object_index1);
            x.obj["objectIndex2"] = Value::integer(rc.object_index2);
            x.obj["distance"] = Value::number(rc.distance);
            x.obj["time"] = Value::number(rc.time);
            x.obj["positionAx"] = Value::number(rc.position_a[0]);
            x.obj["positionAy"] = Value::number(rc.position_a[1]);
            x.obj["positionAz"] = Value::number(rc.position_a[2]);
            x.obj["positionBx"] = Value::number(rc.position_b[0]);
            x.obj["positionBy"] = Value::number(rc.position_b[1]);
            x.obj["positionBz"] = Value::number(rc.position_b[2]);
            return x;
        });
    } else {
        ofs << gpop::json::dump(out, 4);
    }
    std::cout << "Saved to: " << o.output << "\n";
    return 0;
}

} // namespace

int main(int argc, char** argv)
{
    Options o;
    o.data_dir = default_data_dir(argv[0]);
    if (argc < 2)
        return usage(argv[0], "A subcommand is required");
    o.cmd = argv[1];
    if (o.cmd == "-h" || o.cmd == "--help")
        return usage(argv[0], "") == 109 ? 0 : 0;
    if (o.cmd != "propagate" && o.cmd != "closest-approach")
        return usage(argv[0], "The following argument was not expected: " + o.cmd);
    o.output = o.cmd == "propagate" ? "propagation_out.json" : "closest_approach_out.json";
    for (int i = 2; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&](const char* name) -> std::string {
            if (i + 1 >= argc)
                throw std::runtime_error(std::string(name) + " requires an argument");
            return argv[++i];
        };
        try {
            if (a == "-i" || a == "--input")
                o.input = next("--input");
            else if (a == "-o" || a == "--output")
                o.output = next("--output");
            else if (a == "--step")
                o.step = std::stod(next("--step"));
            else if (a == "--degree")
                o.degree = std::stoi(next("--degree"));
            else if (a == "--precision")
                o.precision = next("--precision");
            else if (a == "--threshold")
                o.threshold = std::stod(next("--threshold"));
            else if (a == "--data")
                o.data_dir = next("--data");
            else if (a == "--device")
                o.device = std::stoi(next("--device"));
            else
                return usage(argv[0], "The following argument was not expected: " + a);
        } catch (const std::exception& e) {
            return usage(argv[0], e.what());
        }
    }
    if (o.input.empty())
        return usage(argv[0], "--input is required");
    if (o.precision != "fp64" && o.precision != "mixed")
        return usage(argv[0], "--precision must be fp64 or mixed");
    std::cout << (o.cmd == "propagate" ? "Running Propagation...\n" : "Running Closest Approach Calculation...\n");
    try {
        return run(o);
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << "\n";
        return 1;
    }
}
