// json.h -- minimal JSON value, parser and writer for the exec CLI's input/output files.
//
// Output follows the layout of nlohmann::json::dump(4), which the reference CLI uses
// (exec/main.cpp:87-90,100-102): objects with keys in sorted order, 4-space indentation, one array
// element per line, integers without a fraction, floating-point numbers in their shortest
// round-trip form with ".0" appended to integral values.
#pragma once
#include <charconv>
#include <cmath>
#include <cstdint>
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

// Shortest round-trip decimal form; integral finite values keep a ".0"; exponents as e+NN.
inline std::string format_double(double d)
{
    if (!std::isfinite(d))
        return "null";
    char buf[64];
    auto r = std::to_chars(buf, buf + sizeof(buf), d);
    std::string s(buf, r.ptr);
    const size_t e = s.find('e');
    std::string mant = e == std::string::npos ? s : s.substr(0, e);
    std::string expo = e == std::string::npos ? "" : s.substr(e + 1);
    if (mant.find('.') == std::string::npos)
        mant += ".0";
    if (!expo.empty()) {
        const char sign = expo[0] == '-' ? '-' : '+';
        std::string digits = expo[0] == '-' || expo[0] == '+' ? expo.substr(1) : expo;
        if (digits.size() < 2)
            digits = "0" + digits;
        return mant + "e" + sign + digits;
    }
    return mant;
}

inline void escape(std::string& out, const std::string& s)
{
    out += '"';
    for (char c : s) {
        if (c == '"' || c == '\\') {
            out += '\\';
            out += c;
        } else if (c == '\n') {
            out += "\\n";
        } else {
            out += c;
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
