// json.h -- minimal JSON value, parser and writer for the exec CLI's input/output files.
//
// Output follows the layout of nlohmann::json::dump(4), which the reference CLI uses
// (exec/main.cpp:87-90,100-102): objects with keys in sorted order, 4-space indentation, one array
// element per line, integers without a fraction, floating-point numbers in nlohmann's form
// (format_double).
#pragma once
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <ostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace gpop {
namespace json {

struct Value {
    enum Kind { Null, Bool, Int, Float, String, Array, Object } kind = Null;
    bool b = false;
    int64_t i = 0;
    double f = 0.0;
    std::string s;
    std::vector<Value> arr;
    std::map<std::string, Value> obj; // sorted keys, as nlohmann's default object

    Value() = default;
    static Value integer(int64_t v)
    {
        Value x;
        x.kind = Int;
        x.i = v;
        return x;
    }
    static Value number(double v)
    {
        Value x;
        x.kind = Float;
        x.f = v;
        return x;
    }
    static Value array()
    {
        Value x;
        x.kind = Array;
        return x;
    }
    static Value object()
    {
        Value x;
        x.kind = Object;
        return x;
    }
    double as_double() const
    {
        if (kind == Int)
            return (double)i;
        if (kind == Float)
            return f;
        throw std::runtime_error("expected a number");
    }
    int64_t as_int() const
    {
        if (kind == Int)
            return i;
        if (kind == Float && std::floor(f) == f)
            return (int64_t)f;
        throw std::runtime_error("expected an integer");
    }
    const Value& at(const std::string& k) const
    {
        auto it = obj.find(k);
        if (kind != Object || it == obj.end())
            throw std::runtime_error("missing key \"" + k + "\"");
        return it->second;
    }
    bool has(const std::string& k) const { return kind == Object && obj.count(k); }
};

class Parser {
public:
    explicit Parser(const std::string& t)
        : t_(t)
    {
    }
    Value parse()
    {
        Value v = value();
        ws();
        if (p_ != t_.size())
            fail("trailing characters");
        return v;
    }

private:
    const std::string& t_;
    size_t p_ = 0;
    [[noreturn]] void fail(const char* what) const
    {
        throw std::runtime_error(std::string("JSON parse error at offset ") + std::to_string(p_) + ": " + what);
    }
    void ws()
    {
        while (p_ < t_.size() && (t_[p_] == ' ' || t_[p_] == '\n' || t_[p_] == '\r' || t_[p_] == '\t'))
            ++p_;
    }
    bool eat(char c)
    {
        ws();
        if (p_ < t_.size() && t_[p_] == c) {
            ++p_;
            return true;
        }
        return false;
    }
    Value value()
    {
        ws();
        if (p_ >= t_.size())
            fail("unexpected end");
        const char c = t_[p_];
        if (c == '{')
            return object();
        if (c == '[')
            return array();
        if (c == '"') {
            Value v;
            v.kind = Value::String;
            v.s = string();
            return v;
        }
        if (t_.compare(p_, 4, "true") == 0) {
            p_ += 4;
            Value v;
            v.kind = Value::Bool;
            v.b = true;
            return v;
        }
        if (t_.compare(p_, 5, "false") == 0) {
            p_ += 5;
            Value v;
            v.kind = Value::Bool;
            return v;
        }
        if (t_.compare(p_, 4, "null") == 0) {
            p_ += 4;
            return Value();
        }
        return number();
    }
    Value number()
    {
        const size_t b = p_;
        bool is_float = false;
        if (p_ < t_.size() && (t_[p_] == '-' || t_[p_] == '+'))
            ++p_;
        while (p_ < t_.size()) {
            const char c = t_[p_];
            if (c >= '0' && c <= '9') {
                ++p_;
            } else if (c == '.' || c == 'e' || c == 'E' || ((c == '-' || c == '+') && (t_[p_ - 1] == 'e' || t_[p_ - 1] == 'E'))) {
                is_float = true;
                ++p_;
            } else {
                break;
            }
        }
        if (p_ == b)
            fail("expected a value");
        const char* s = t_.data() + b;
        const char* e = t_.data() + p_;
        if (*s == '+')
            ++s;
        if (!is_float) {
            int64_t v = 0;
            auto r = std::from_chars(s, e, v);
            if (r.ec == std::errc() && r.ptr == e)
                return Value::integer(v);
        }
        double d = 0.0;
        auto r = std::from_chars(s, e, d);
        if (r.ec != std::errc() || r.ptr != e)
            fail("bad number");
        return Value::number(d);
    }
    std::string string()
    {
        if (!eat('"'))
            fail("expected a string");
        std::string out;
        while (p_ < t_.size() && t_[p_] != '"') {
            char c = t_[p_++];
            if (c == '\\' && p_ < t_.size()) {
                const char e = t_[p_++];
                switch (e) {
                case 'n': c = '\n'; break;
                case 't': c = '\t'; break;
                case 'r': c = '\r'; break;
                case 'b': c = '\b'; break;
                case 'f': c = '\f'; break;
                default: c = e;
                }
            }
            out += c;
        }
        if (p_ >= t_.size())
            fail("unterminated string");
        ++p_;
        return out;
    }
    Value array()
    {
        Value v = Value::array();
        eat('[');
        if (eat(']'))
            return v;
        do {
            v.arr.push_back(value());
        } while (eat(','));
        if (!eat(']'))
            fail("expected ']'");
        return v;
    }
    Value object()
    {
        Value v = Value::object();
        eat('{');
        if (eat('}'))
            return v;
        do {
            ws();
            std::string k = string();
            if (!eat(':'))
                fail("expected ':'");
            v.obj[k] = value();
        } while (eat(','));
        if (!eat('}'))
            fail("expected '}'");
        return v;
    }
};

inline Value parse(const std::string& text) { return Parser(text).parse(); }

// Shortest-digit generation by Grisu2 (F. Loitsch, "Printing floating-point numbers quickly and
// accurately with integers", PLDI 2010), with the parameters of nlohmann::json 3.11.3, whose
// digits the reference CLI's output carries (exec/main.cpp:87-88,100-101: jOutput.dump(4)):
// scaled exponents in [-60, -32], cached powers 10^k for k = -300, -292, ..., 324, the boundary
// interval narrowed by one unit on each side, digits of the upper boundary cut as soon as the
// remainder lies inside the interval, then the last digit lowered while that brings the digits
// closer to the value (Grisu2's rounding step). Grisu2 always gives digits that read back to the
// same double, but not always the shortest or the closest such digits, so the bytes depend on
// these choices.
namespace grisu {

struct Fp {
    uint64_t f; // significand
    int e; // binary exponent: value = f * 2^e
};

// Upper 64 bits of the 128-bit product, rounded to nearest (ties up).
inline Fp mul(Fp a, Fp b)
{
    const unsigned __int128 p = (unsigned __int128)a.f * b.f;
    const uint64_t hi = (uint64_t)(p >> 64), lo = (uint64_t)p;
    return { hi + (lo >> 63), a.e + b.e + 64 };
}

inline Fp normalize(Fp x)
{
    while (!(x.f >> 63)) {
        x.f <<= 1;
        x.e -= 1;
    }
    return x;
}

// 10^k rounded to nearest as f * 2^e with bit 63 of f set, for k = -300 + 8 i.
struct Pow10 {
    uint64_t f;
    int e;
    int k;
};
inline const Pow10& cached_pow10(int i)
{
    static const Pow10 table[79] = {
    { 0xAB70FE17C79AC6CAULL, -1060, -300 },
    { 0xFF77B1FCBEBCDC4FULL, -1034, -292 },
    { 0xBE5691EF416BD60CULL, -1007, -284 },
    { 0x8DD01FAD907FFC3CULL, -980, -276 },
    { 0xD3515C2831559A83ULL, -954, -268 },
    { 0x9D71AC8FADA6C9B5ULL, -927, -260 },
    { 0xEA9C227723EE8BCBULL, -901, -252 },
    { 0xAECC49914078536DULL, -874, -244 },
    { 0x823C12795DB6CE57ULL, -847, -236 },
    { 0xC21094364DFB5637ULL, -821, -228 },
    { 0x9096EA6F3848984FULL, -794, -220 },
    { 0xD77485CB25823AC7ULL, -768, -212 },
    { 0xA086CFCD97BF97F4ULL, -741, -204 },
    { 0xEF340A98172AACE5ULL, -715, -196 },
    { 0xB23867FB2A35B28EULL, -688, -188 },
    { 0x84C8D4DFD2C63F3BULL, -661, -180 },
    { 0xC5DD44271AD3CDBAULL, -635, -172 },
    { 0x936B9FCEBB25C996ULL, -608, -164 },
    { 0xDBAC6C247D62A584ULL, -582, -156 },
    { 0xA3AB66580D5FDAF6ULL, -555, -148 },
    { 0xF3E2F893DEC3F126ULL, -529, -140 },
    { 0xB5B5ADA8AAFF80B8ULL, -502, -132 },
    { 0x87625F056C7C4A8BULL, -475, -124 },
    { 0xC9BCFF6034C13053ULL, -449, -116 },
    { 0x964E858C91BA2655ULL, -422, -108 },
    { 0xDFF9772470297EBDULL, -396, -100 },
    { 0xA6DFBD9FB8E5B88FULL, -369, -92 },
    { 0xF8A95FCF88747D94ULL, -343, -84 },
    { 0xB94470938FA89BCFULL, -316, -76 },
    { 0x8A08F0F8BF0F156BULL, -289, -68 },
    { 0xCDB02555653131B6ULL, -263, -60 },
    { 0x993FE2C6D07B7FACULL, -236, -52 },
    { 0xE45C10C42A2B3B06ULL, -210, -44 },
    { 0xAA242499697392D3ULL, -183, -36 },
    { 0xFD87B5F28300CA0EULL, -157, -28 },
    { 0xBCE5086492111AEBULL, -130, -20 },
    { 0x8CBCCC096F5088CCULL, -103, -12 },
    { 0xD1B71758E219652CULL, -77, -4 },
    { 0x9C40000000000000ULL, -50, 4 },
    { 0xE8D4A51000000000ULL, -24, 12 },
    { 0xAD78EBC5AC620000ULL, 3, 20 },
    { 0x813F3978F8940984ULL, 30, 28 },
    { 0xC097CE7BC90715B3ULL, 56, 36 },
    { 0x8F7E32CE7BEA5C70ULL, 83, 44 },
    { 0xD5D238A4ABE98068ULL, 109, 52 },
    { 0x9F4F2726179A2245ULL, 136, 60 },
    { 0xED63A231D4C4FB27ULL, 162, 68 },
    { 0xB0DE65388CC8ADA8ULL, 189, 76 },
    { 0x83C7088E1AAB65DBULL, 216, 84 },
    { 0xC45D1DF942711D9AULL, 242, 92 },
    { 0x924D692CA61BE758ULL, 269, 100 },
    { 0xDA01EE641A708DEAULL, 295, 108 },
    { 0xA26DA3999AEF774AULL, 322, 116 },
    { 0xF209787BB47D6B85ULL, 348, 124 },
    { 0xB454E4A179DD1877ULL, 375, 132 },
    { 0x865B86925B9BC5C2ULL, 402, 140 },
    { 0xC83553C5C8965D3DULL, 428, 148 },
    { 0x952AB45CFA97A0B3ULL, 455, 156 },
    { 0xDE469FBD99A05FE3ULL, 481, 164 },
    { 0xA59BC234DB398C25ULL, 508, 172 },
    { 0xF6C69A72A3989F5CULL, 534, 180 },
    { 0xB7DCBF5354E9BECEULL, 561, 188 },
    { 0x88FCF317F22241E2ULL, 588, 196 },
    { 0xCC20CE9BD35C78A5ULL, 614, 204 },
    { 0x98165AF37B2153DFULL, 641, 212 },
    { 0xE2A0B5DC971F303AULL, 667, 220 },
    { 0xA8D9D1535CE3B396ULL, 694, 228 },
    { 0xFB9B7CD9A4A7443CULL, 720, 236 },
    { 0xBB764C4CA7A44410ULL, 747, 244 },
    { 0x8BAB8EEFB6409C1AULL, 774, 252 },
    { 0xD01FEF10A657842CULL, 800, 260 },
    { 0x9B10A4E5E9913129ULL, 827, 268 },
    { 0xE7109BFBA19C0C9DULL, 853, 276 },
    { 0xAC2820D9623BF429ULL, 880, 284 },
    { 0x80444B5E7AA7CF85ULL, 907, 292 },
    { 0xBF21E44003ACDD2DULL, 933, 300 },
    { 0x8E679C2F5E44FF8FULL, 960, 308 },
    { 0xD433179D9C8CB841ULL, 986, 316 },
    { 0x9E19DB92B4E31BA9ULL, 1013, 324 },
    };
    return table[i];
}

// Largest power of ten not above n (n > 0), and the number of decimal digits of n.
inline int digits_of(uint32_t n, uint32_t& pow10)
{
    int k = 1;
    pow10 = 1;
    while (n / pow10 >= 10) {
        pow10 *= 10;
        ++k;
    }
    return k;
}

// Lowers the last digit while the digits stay inside the interval and come closer to the value.
// rest: upper boundary minus the digits; dist: upper boundary minus the value; delta: interval
// width; unit: one unit of the last digit (all in the same scaled fixed point).
inline void round_last(char* buf, int len, uint64_t dist, uint64_t delta, uint64_t rest, uint64_t unit)
{
    while (rest < dist && delta - rest >= unit
        && (rest + unit < dist || dist - rest > rest + unit - dist)) {
        buf[len - 1]--;
        rest += unit;
    }
}

// Digits of a finite v > 0 into buf (no sign, no point); returns their count, and dec_exp with
// v ~ digits x 10^dec_exp.
inline int digits(double v, char* buf, int& dec_exp)
{
    uint64_t bits;
    std::memcpy(&bits, &v, 8);
    const uint64_t frac = bits & ((1ull << 52) - 1);
    const int bexp = (int)(bits >> 52);
    const Fp x = bexp == 0 ? Fp { frac, -1074 } : Fp { frac | (1ull << 52), bexp - 1075 };
    // boundaries: halfway to the neighbouring doubles (the lower one is closer at a power of two)
    const bool lower_closer = frac == 0 && bexp > 1;
    const Fp hi = normalize(Fp { 2 * x.f + 1, x.e - 1 });
    Fp lo = lower_closer ? Fp { 4 * x.f - 1, x.e - 2 } : Fp { 2 * x.f - 1, x.e - 1 };
    lo = Fp { lo.f << (lo.e - hi.e), hi.e };
    const Fp w0 = normalize(x);
    // the cached power that brings the upper boundary's exponent into [-60, -32]
    const int t = -60 - hi.e - 1;
    const int kmin = (t * 78913) / (1 << 18) + (t > 0 ? 1 : 0); // ceil(t log10 2)
    const Pow10& c = cached_pow10((300 + kmin + 7) / 8);
    const Fp w = mul(w0, Fp { c.f, c.e });
    const Fp mlo = mul(lo, Fp { c.f, c.e });
    const Fp mhi = mul(hi, Fp { c.f, c.e });
    const uint64_t upper = mhi.f - 1, lower = mlo.f + 1; // narrowed interval
    const int shift = -mhi.e;
    const uint64_t one = 1ull << shift;
    uint64_t delta = upper - lower;
    uint64_t dist = upper - w.f;
    uint32_t p1 = (uint32_t)(upper >> shift);
    uint64_t p2 = upper & (one - 1);
    dec_exp = -c.k;
    int len = 0;
    uint32_t pow10;
    int n = digits_of(p1, pow10);
    while (n > 0) {
        buf[len++] = (char)('0' + p1 / pow10);
        p1 %= pow10;
        --n;
        const uint64_t rest = ((uint64_t)p1 << shift) + p2;
        if (rest <= delta) {
            dec_exp += n;
            round_last(buf, len, dist, delta, rest, (uint64_t)pow10 << shift);
            return len;
        }
        pow10 /= 10;
    }
    int m = 0;
    for (;;) {
        p2 *= 10;
        delta *= 10;
        dist *= 10;
        buf[len++] = (char)('0' + (p2 >> shift));
        p2 &= one - 1;
        ++m;
        if (p2 <= delta)
            break;
    }
    dec_exp -= m;
    round_last(buf, len, dist, delta, p2, one);
    return len;
}

} // namespace grisu

// The number form of nlohmann::json's dump(): Grisu2 digits d1..dk of |d| and the position n of
// the decimal point (|d| = 0.d1..dk x 10^n). Then
//   k <= n <= 15      d1..dk, n - k zeros, ".0"        (7000000.0)
//   0 < n <= 15       d1..dn "." dn+1..dk              (7612.608173223869)
//   -4 < n <= 0       "0." -n zeros d1..dk             (0.0001)
//   otherwise         d1 ["." d2..dk] "e" sign, at least two exponent digits (1e+15, 1.5e-05)
// with a leading '-' for negative values (negative zero included: -0.0); non-finite values are
// written as null.
inline std::string format_double(double d)
{
    if (!std::isfinite(d))
        return "null";
    std::string out = std::signbit(d) ? "-" : "";
    d = std::fabs(d);
    if (d == 0.0)
        return out + "0.0";
    char buf[32];
    int dec_exp = 0;
    const int k = grisu::digits(d, buf, dec_exp);
    const std::string digits(buf, (size_t)k);
    const int n = k + dec_exp;
    if (k <= n && n <= 15)
        return out + digits + std::string((size_t)(n - k), '0') + ".0";
    if (0 < n && n <= 15)
        return out + digits.substr(0, (size_t)n) + "." + digits.substr((size_t)n);
    if (-4 < n && n <= 0)
        return out + "0." + std::string((size_t)(-n), '0') + digits;
    out += digits.substr(0, 1);
    if (k > 1)
        out += "." + digits.substr(1);
    const int e = n - 1;
    out += e < 0 ? "e-" : "e+";
    const std::string ed = std::to_string(e < 0 ? -e : e);
    return out + (ed.size() < 2 ? "0" + ed : ed);
}

inline void escape(std::string& out, const std::string& s)
{
    out += '"';
    // JSON's short escapes, \u00xx (lower-case hex) for the other control characters; every other
    // byte, UTF-8 included, is written as it is
    for (char c : s) {
        const unsigned char u = (unsigned char)c;
        switch (c) {
        case '"':
            out += "\\\"";
            break;
        case '\\':
            out += "\\\\";
            break;
        case '\b':
            out += "\\b";
            break;
        case '\f':
            out += "\\f";
            break;
        case '\n':
            out += "\\n";
            break;
        case '\r':
            out += "\\r";
            break;
        case '\t':
            out += "\\t";
            break;
        default:
            if (u < 0x20) {
                static const char hex[] = "0123456789abcdef";
                out += "\\u00";
                out += hex[u >> 4];
                out += hex[u & 15];
            } else {
                out += c;
            }
        }
    }
    out += '"';
}

inline void dump(const Value& v, std::string& out, int indent, int level)
{
    const std::string pad((size_t)indent * (level + 1), ' ');
    const std::string pad0((size_t)indent * level, ' ');
    switch (v.kind) {
    case Value::Null:
        out += "null";
        break;
    case Value::Bool:
        out += v.b ? "true" : "false";
        break;
    case Value::Int:
        out += std::to_string(v.i);
        break;
    case Value::Float:
        out += format_double(v.f);
        break;
    case Value::String:
        escape(out, v.s);
        break;
    case Value::Array:
        if (v.arr.empty()) {
            out += "[]";
            break;
        }
        out += "[\n";
        for (size_t k = 0; k < v.arr.size(); ++k) {
            out += pad;
            dump(v.arr[k], out, indent, level + 1);
            out += k + 1 < v.arr.size() ? ",\n" : "\n";
        }
        out += pad0 + "]";
        break;
    case Value::Object: {
        if (v.obj.empty()) {
            out += "{}";
            break;
        }
        out += "{\n";
        size_t k = 0;
        for (const auto& kv : v.obj) {
            out += pad;
            escape(out, kv.first);
            out += ": ";
            dump(kv.second, out, indent, level + 1);
            out += ++k < v.obj.size() ? ",\n" : "\n";
        }
        out += pad0 + "}";
        break;
    }
    }
}

inline std::string dump(const Value& v, int indent = 4)
{
    std::string out;
    dump(v, out, indent, 0);
    return out;
}

// Writes `top` as dump(top, indent) would after setting top[key] to an array of `count` elements,
// element k given by element(k), without holding the array: the elements are formatted and
// written one at a time (closest-approach outputs run to tens of millions of records).
template <class Element>
void dump_streaming(std::ostream& os, const Value& top, const std::string& key, size_t count,
    const Element& element, int indent = 4)
{
    std::map<std::string, const Value*> keys;
    for (const auto& kv : top.obj)
        keys[kv.first] = &kv.second;
    keys[key] = nullptr;
    const std::string pad((size_t)indent, ' '), pad2((size_t)indent * 2, ' ');
    std::string buf = "{\n";
    size_t k = 0;
    for (const auto& kv : keys) {
        buf += pad;
        escape(buf, kv.first);
        buf += ": ";
        if (kv.second) {
            dump(*kv.second, buf, indent, 1);
        } else if (count == 0) {
            buf += "[]";
        } else {
            buf += "[\n";
            for (size_t e = 0; e < count; ++e) {
                buf += pad2;
                dump(element(e), buf, indent, 2);
                buf += e + 1 < count ? ",\n" : "\n";
                if (buf.size() > (1u << 20)) {
                    os << buf;
                    buf.clear();
                }
            }
            buf += pad + "]";
        }
        buf += ++k < keys.size() ? ",\n" : "\n";
    }
    buf += "}";
    os << buf;
}

} // namespace json
} // namespace gpop
