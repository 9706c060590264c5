// The streaming JSON writer of the CLI against the whole-document writer: same bytes for the
// closest-approach layout with 0, 1 and many records. Exit status 0 when all match.
#include "json.h"

#include <cstdio>
#include <sstream>

using gpop::json::Value;

static Value record(size_t k)
{
    Value x = Value::object();
    x.obj["objectIndex1"] = Value::integer((int64_t)k);
    x.obj["objectIndex2"] = Value::integer((int64_t)(k * 7 + 3));
    x.obj["distance"] = Value::number(1234.5 + 0.1 * (double)k);
    x.obj["time"] = Value::number(1e-3 * (double)k);
    x.obj["positionAx"] = Value::number(-7.0e6 + (double)k);
    x.obj["positionAy"] = Value::number(1.0 / 3.0);
    x.obj["positionAz"] = Value::number(0.0);
    x.obj["positionBx"] = Value::number(6.5e6);
    x.obj["positionBy"] = Value::number(-2.5e-7 * (double)k);
    x.obj["positionBz"] = Value::number(1e300);
    return x;
}

int main()
{
    int bad = 0;
    for (size_t count : { (size_t)0, (size_t)1, (size_t)2, (size_t)5000 }) {
        Value top = Value::object();
        Value t = Value::object();
        t.obj["Year"] = Value::integer(2024);
        t.obj["Sec"] = Value::number(0.5);
        top.obj["propagationStart"] = t;
        top.obj["propagationSeconds"] = Value::integer(86400);
        Value pos = Value::array();
        for (int i = 0; i < 3; ++i) {
            Value p = Value::array();
            for (int c = 0; c < 3; ++c)
                p.arr.push_back(Value::number(1.5 * i + c));
            pos.arr.push_back(p);
        }
        top.obj["positionsStart"] = pos;
        top.obj["velocitiesStart"] = pos;
        Value full = top;
        Value arr = Value::array();
        for (size_t k = 0; k < count; ++k)
            arr.arr.push_back(record(k));
        full.obj["closestApproaches"] = arr;
        std::ostringstream os;
        gpop::json::dump_streaming(os, top, "closestApproaches", count, record);
        if (os.str() != gpop::json::dump(full, 4)) {
            std::printf("mismatch at %zu records\n", count);
            bad = 1;
        }
    }
    return bad;
}
