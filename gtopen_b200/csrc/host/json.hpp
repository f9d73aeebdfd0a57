// Minimal JSON value, parser and compact writer for the SpotConfig schema and
// the .gto save header.  Numbers keep their double value; the writer prints
// the shortest round-trip form with a ".0" suffix on integral values, the way
// serde_json prints f64 fields (so headers read back identically).
#pragma once
#include <charconv>
#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace gtob {
namespace json {

struct Value {
    enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
    bool b = false;
    bool is_int = false;  // written without a fraction (serde integer fields)
    bool is_f32 = false;  // written as the shortest f32 repr (serde f32 fields)
    double num = 0;
    std::string str;
    std::vector<Value> arr;
    std::vector<std::pair<std::string, Value>> obj;  // insertion order kept

    const Value* get(const std::string& k) const {
        for (auto& kv : obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
    static Value number(double d) { Value v; v.kind = NUM; v.num = d; return v; }
    static Value integer(long long d) { Value v; v.kind = NUM; v.num = (double)d; v.is_int = true; return v; }
    static Value f32(float d) { Value v; v.kind = NUM; v.num = d; v.is_f32 = true; return v; }
    static Value string(const std::string& s) { Value v; v.kind = STR; v.str = s; return v; }
    static Value boolean(bool x) { Value v; v.kind = BOOL; v.b = x; return v; }
    static Value array() { Value v; v.kind = ARR; return v; }
    static Value object() { Value v; v.kind = OBJ; return v; }
    Value& set(const std::string& k, Value v) { obj.emplace_back(k, std::move(v)); return *this; }
};

struct Parser {
    const std::string& s;
    size_t i = 0;
    explicit Parser(const std::string& src) : s(src) {}
    [[noreturn]] void err(const char* what) {
        throw std::runtime_error(std::string("json: ") + what + " at byte " + std::to_string(i));
    }
    void ws() { while (i < s.size() && (s[i] == ' ' || s[i] == '\n' || s[i] == '\t' || s[i] == '\r')) i++; }
    Value parse() {
        ws();
        Value v = value();
        ws();
        if (i != s.size()) err("trailing characters");
        return v;
    }
    Value value() {
        ws();
        if (i >= s.size()) err("unexpected end");
        char c = s[i];
        if (c == '{') return object();
        if (c == '[') return array();
        if (c == '"') return Value::string(string());
        if (c == 't' && s.compare(i, 4, "true") == 0) { i += 4; return Value::boolean(true); }
        if (c == 'f' && s.compare(i, 5, "false") == 0) { i += 5; return Value::boolean(false); }
        if (c == 'n' && s.compare(i, 4, "null") == 0) { i += 4; return Value(); }
        return number();
    }
    Value number() {
        size_t st = i;
        if (i < s.size() && (s[i] == '-' || s[i] == '+')) i++;
        while (i < s.size() && (isdigit((unsigned char)s[i]) || s[i] == '.' || s[i] == 'e' || s[i] == 'E' ||
                                s[i] == '-' || s[i] == '+'))
            i++;
        if (st == i) err("bad value");
        std::string tok = s.substr(st, i - st);
        char* end = nullptr;
        double d = strtod(tok.c_str(), &end);
        if (*end) err("bad number");
        return Value::number(d);
    }
    std::string string() {
        if (s[i] != '"') err("expected string");
        i++;
        std::string out;
        while (i < s.size() && s[i] != '"') {
            char c = s[i++];
            if (c == '\\') {
                if (i >= s.size()) err("bad escape");
                char e = s[i++];
                switch (e) {
                    case '"': out.push_back('"'); break;
                    case '\\': out.push_back('\\'); break;
                    case '/': out.push_back('/'); break;
                    case 'b': out.push_back('\b'); break;
                    case 'f': out.push_back('\f'); break;
                    case 'n': out.push_back('\n'); break;
                    case 'r': out.push_back('\r'); break;
                    case 't': out.push_back('\t'); break;
                    case 'u': {
                        if (i + 4 > s.size()) err("bad unicode escape");
                        unsigned cp = (unsigned)std::stoul(s.substr(i, 4), nullptr, 16);
                        i += 4;
                        if (cp < 0x80) out.push_back((char)cp);
                        else if (cp < 0x800) { out.push_back((char)(0xC0 | (cp >> 6))); out.push_back((char)(0x80 | (cp & 0x3F))); }
                        else { out.push_back((char)(0xE0 | (cp >> 12))); out.push_back((char)(0x80 | ((cp >> 6) & 0x3F))); out.push_back((char)(0x80 | (cp & 0x3F))); }
                        break;
                    }
                    default: err("bad escape");
                }
            } else {
                out.push_back(c);
            }
        }
        if (i >= s.size()) err("unterminated string");
        i++;
        return out;
    }
    Value array() {
        Value v = Value::array();
        i++;
        ws();
        if (i < s.size() && s[i] == ']') { i++; return v; }
        for (;;) {
            v.arr.push_back(value());
            ws();
            if (i < s.size() && s[i] == ',') { i++; continue; }
            if (i < s.size() && s[i] == ']') { i++; return v; }
            err("expected , or ]");
        }
    }
    Value object() {
        Value v = Value::object();
        i++;
        ws();
        if (i < s.size() && s[i] == '}') { i++; return v; }
        for (;;) {
            ws();
            std::string k = string();
            ws();
            if (i >= s.size() || s[i] != ':') err("expected :");
            i++;
            v.obj.emplace_back(k, value());
            ws();
            if (i < s.size() && s[i] == ',') { i++; continue; }
            if (i < s.size() && s[i] == '}') { i++; return v; }
            err("expected , or }");
        }
    }
};

inline Value parse(const std::string& s) { return Parser(s).parse(); }

inline std::string fmt_double(double d) {
    if (!std::isfinite(d)) return "null";
    char buf[64];
    auto r = std::to_chars(buf, buf + sizeof(buf), d);
    std::string s(buf, r.ptr);
    if (s.find_first_of(".eEn") == std::string::npos) s += ".0";
    return s;
}
inline std::string fmt_float(float f) {
    if (!std::isfinite(f)) return "null";
    char buf[64];
    auto r = std::to_chars(buf, buf + sizeof(buf), f);
    std::string s(buf, r.ptr);
    if (s.find_first_of(".eEn") == std::string::npos) s += ".0";
    return s;
}
inline void escape(const std::string& in, std::string& out) {
    out.push_back('"');
    for (char c : in) {
        switch (c) {
            case '"': out += "\\\""; break;
            case '\\': out += "\\\\"; break;
            case '\n': out += "\\n"; break;
            case '\r': out += "\\r"; break;
            case '\t': out += "\\t"; break;
            default:
                if ((unsigned char)c < 0x20) {
                    char b[8];
                    snprintf(b, sizeof(b), "\\u%04x", c);
                    out += b;
                } else {
                    out.push_back(c);
                }
        }
    }
    out.push_back('"');
}
inline void write(const Value& v, std::string& out) {
    switch (v.kind) {
        case Value::NUL: out += "null"; break;
        case Value::BOOL: out += v.b ? "true" : "false"; break;
        case Value::NUM:
            if (v.is_int) out += std::to_string((long long)v.num);
            else if (v.is_f32) out += fmt_float((float)v.num);
            else out += fmt_double(v.num);
            break;
        case Value::STR: escape(v.str, out); break;
        case Value::ARR:
            out.push_back('[');
            for (size_t k = 0; k < v.arr.size(); k++) { if (k) out.push_back(','); write(v.arr[k], out); }
            out.push_back(']');
            break;
        case Value::OBJ:
            out.push_back('{');
            for (size_t k = 0; k < v.obj.size(); k++) {
                if (k) out.push_back(',');
                escape(v.obj[k].first, out);
                out.push_back(':');
                write(v.obj[k].second, out);
            }
            out.push_back('}');
            break;
    }
}
inline std::string dump(const Value& v) { std::string s; write(v, s); return s; }

}  // namespace json
}  // namespace gtob
