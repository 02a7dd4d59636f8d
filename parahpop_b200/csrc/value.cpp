#include "value.hpp"

#include <algorithm>
#include <cerrno>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace phop {

bool Value::asBool() const {
    if (kind_ == Bool) return b_;
    throw std::runtime_error("JSON value is not a boolean");
}
double Value::asDouble() const {
    if (kind_ == Real) return d_;
    if (kind_ == Int) return (double)i_;
    throw std::runtime_error("JSON value is not a number");
}
int64_t Value::asInt() const {
    if (kind_ == Int) return i_;
    if (kind_ == Real && std::floor(d_) == d_) return (int64_t)d_;
    throw std::runtime_error("JSON value is not an integer");
}
const std::string& Value::asString() const {
    if (kind_ == String) return s_;
    throw std::runtime_error("JSON value is not a string");
}
const Value& Value::operator[](size_t i) const {
    if (kind_ != Array || i >= size()) throw std::runtime_error("JSON array index out of range");
    unpack();
    return arr_[i];
}
void Value::unpack() const {
    if (!packed_) return;
    arr_.reserve(reals_.size());
    for (double d : reals_) arr_.push_back(Value::real(d));
    reals_.clear();
    reals_.shrink_to_fit();
    packed_ = false;
}
void Value::copyReals(size_t off, size_t n, double* out) const {
    if (n == 0) return;
    if (kind_ != Array || off > size() || n > size() - off) throw std::runtime_error("JSON array index out of range");
    if (packed_) {
        std::copy(reals_.begin() + (std::ptrdiff_t)off, reals_.begin() + (std::ptrdiff_t)(off + n), out);
        return;
    }
    for (size_t k = 0; k < n; ++k) out[k] = arr_[off + k].asDouble();
}
bool Value::has(const std::string& k) const { return find(k) != nullptr; }
const Value* Value::find(const std::string& k) const {
    if (kind_ != Object) return nullptr;
    for (auto& kv : obj_)
        if (kv.first == k) return &kv.second;
    return nullptr;
}
Value* Value::find(const std::string& k) {
    if (kind_ != Object) return nullptr;
    for (auto& kv : obj_)
        if (kv.first == k) return &kv.second;
    return nullptr;
}
const Value& Value::at(const std::string& k) const {
    const Value* v = find(k);
    if (!v) throw std::runtime_error("[json.exception.out_of_range.403] key '" + k + "' not found");
    return *v;
}
Value& Value::set(const std::string& k, Value v) {
    if (kind_ == Null) kind_ = Object;
    if (Value* e = find(k)) {
        *e = std::move(v);
        return *e;
    }
    obj_.emplace_back(k, std::move(v));
    return obj_.back().second;
}
void Value::erase(const std::string& k) {
    for (size_t i = 0; i < obj_.size(); ++i)
        if (obj_[i].first == k) {
            obj_.erase(obj_.begin() + i);
            return;
        }
}
double Value::numberOr(const std::string& k, double dflt) const {
    const Value* v = find(k);
    return v ? v->asDouble() : dflt;
}

static void escape(std::string& out, const std::string& s) {
    out += '"';
    for (char c : s) {
        switch (c) {
            case '"': out += "\\\""; break;
            case '\\': out += "\\\\"; break;
            case '\n': out += "\\n"; break;
            case '\t': out += "\\t"; break;
            case '\r': out += "\\r"; break;
            default:
                if ((unsigned char)c < 0x20) {
                    char b[8];
                    std::snprintf(b, sizeof b, "\\u%04x", c);
                    out += b;
                } else {
                    out += c;
                }
        }
    }
    out += '"';
}

static void fmtDouble(std::string& out, double d) {
    if (!std::isfinite(d)) {
        out += "null";
        return;
    }
    char b[40];
    // shortest representation that round-trips
    for (int prec = 15; prec <= 17; ++prec) {
        std::snprintf(b, sizeof b, "%.*g", prec, d);
        if (std::strtod(b, nullptr) == d) break;
    }
    out += b;
    if (!std::strpbrk(b, ".eEn")) out += ".0";
}

void Value::dumpTo(std::string& out, int indent, int level) const {
    auto nl = [&](int l) {
        if (indent >= 0) {
            out += '\n';
            out.append((size_t)(indent * l), ' ');
        }
    };
    switch (kind_) {
        case Null: out += "null"; break;
        case Bool: out += b_ ? "true" : "false"; break;
        case Int: out += std::to_string(i_); break;
        case Real: fmtDouble(out, d_); break;
        case String: escape(out, s_); break;
        case Array:
            unpack();
            if (arr_.empty()) {
                out += "[]";
                break;
            }
            out += '[';
            for (size_t i = 0; i < arr_.size(); ++i) {
                if (i) out += ',';
                nl(level + 1);
                arr_[i].dumpTo(out, indent, level + 1);
            }
            nl(level);
            out += ']';
            break;
        case Object:
            if (obj_.empty()) {
                out += "{}";
                break;
            }
            out += '{';
            for (size_t i = 0; i < obj_.size(); ++i) {
                if (i) out += ',';
                nl(level + 1);
                escape(out, obj_[i].first);
                out += indent >= 0 ? ": " : ":";
                obj_[i].second.dumpTo(out, indent, level + 1);
            }
            nl(level);
            out += '}';
            break;
    }
}

std::string Value::dump(int indent) const {
    std::string out;
    dumpTo(out, indent, 0);
    return out;
}

// ---- JSON parser -----------------------------------------------------------------------------
namespace {
struct JsonParser {
    const std::string& t;
    size_t i = 0;
    explicit JsonParser(const std::string& s) : t(s) {}
    [[noreturn]] void fail(const char* what) {
        throw std::runtime_error(std::string("[json.exception.parse_error] ") + what + " at byte " + std::to_string(i));
    }
    void ws() {
        while (i < t.size() && (t[i] == ' ' || t[i] == '\n' || t[i] == '\r' || t[i] == '\t')) ++i;
    }
    Value parse() {
        ws();
        if (i >= t.size()) fail("unexpected end of input");
        const char c = t[i];
        if (c == '{') return obj();
        if (c == '[') return arr();
        if (c == '"') return Value::string(str());
        if (c == 't' && t.compare(i, 4, "true") == 0) {
            i += 4;
            return Value::boolean(true);
        }
        if (c == 'f' && t.compare(i, 5, "false") == 0) {
            i += 5;
            return Value::boolean(false);
        }
        if (c == 'n' && t.compare(i, 4, "null") == 0) {
            i += 4;
            return Value();
        }
        return num();
    }
    Value obj() {
        Value v = Value::object();
        ++i;
        ws();
        if (i < t.size() && t[i] == '}') {
            ++i;
            return v;
        }
        for (;;) {
            ws();
            if (i >= t.size() || t[i] != '"') fail("expected object key");
            std::string k = str();
            ws();
            if (i >= t.size() || t[i] != ':') fail("expected ':'");
            ++i;
            v.set(k, parse());
            ws();
            if (i < t.size() && t[i] == ',') {
                ++i;
                continue;
            }
            if (i < t.size() && t[i] == '}') {
                ++i;
                return v;
            }
            fail("expected ',' or '}'");
        }
    }
    Value arr() {
        Value v = Value::array();
        ++i;
        ws();
        if (i < t.size() && t[i] == ']') {
            ++i;
            return v;
        }
        for (;;) {
            v.push(parse());
            ws();
            if (i < t.size() && t[i] == ',') {
                ++i;
                continue;
            }
            if (i < t.size() && t[i] == ']') {
                ++i;
                return v;
            }
            fail("expected ',' or ']'");
        }
    }
    std::string str() {
        std::string out;
        ++i;
        while (i < t.size() && t[i] != '"') {
            char c = t[i++];
            if (c == '\\') {
                if (i >= t.size()) fail("bad escape");
                const char e = t[i++];
                switch (e) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'u': {
                        if (i + 4 > t.size()) fail("bad unicode escape");
                        const unsigned cp = (unsigned)std::stoul(t.substr(i, 4), nullptr, 16);
                        i += 4;
                        if (cp < 0x80) out += (char)cp;
                        else if (cp < 0x800) {
                            out += (char)(0xC0 | (cp >> 6));
                            out += (char)(0x80 | (cp & 0x3F));
                        } else {
                            out += (char)(0xE0 | (cp >> 12));
                            out += (char)(0x80 | ((cp >> 6) & 0x3F));
                            out += (char)(0x80 | (cp & 0x3F));
                        }
                        break;
                    }
                    default: out += e;
                }
            } else {
                out += c;
            }
        }
        if (i >= t.size()) fail("unterminated string");
        ++i;
        return out;
    }
    Value num() {
        const size_t s = i;
        bool real = false;
        if (t[i] == '-') ++i;
        while (i < t.size()) {
            const char c = t[i];
            if (c >= '0' && c <= '9') ++i;
            else if (c == '.' || c == 'e' || c == 'E' || c == '+' || c == '-') {
                real = true;
                ++i;
            } else break;
        }
        if (s == i) fail("syntax error");
        const std::string tok = t.substr(s, i - s);
        char* end = nullptr;
        if (!real) {
            errno = 0;
            const long long v = std::strtoll(tok.c_str(), &end, 10);
            if (*end == 0 && errno == 0) return Value::integer(v);
        }
        const double d = std::strtod(tok.c_str(), &end);
        if (*end != 0) fail("bad number");
        return Value::real(d);
    }
};

struct CborParser {
    const std::vector<uint8_t>& b;
    size_t i = 0;
    explicit CborParser(const std::vector<uint8_t>& v) : b(v) {}
    [[noreturn]] void fail() { throw std::runtime_error("Malformed CBOR data at byte " + std::to_string(i)); }
    uint64_t arg(int info) {
        if (info < 24) return (uint64_t)info;
        int n = info == 24 ? 1 : info == 25 ? 2 : info == 26 ? 4 : info == 27 ? 8 : -1;
        if (n < 0 || i + n > b.size()) fail();
        uint64_t v = 0;
        for (int k = 0; k < n; ++k) v = (v << 8) | b[i++];
        return v;
    }
    Value parse() {
        if (i >= b.size()) fail();
        const uint8_t h = b[i++];
        const int major = h >> 5, info = h & 31;
        switch (major) {
            case 0: return Value::integer((int64_t)arg(info));
            case 1: return Value::integer(-1 - (int64_t)arg(info));
            case 2:
            case 3: {
                const uint64_t n = arg(info);
                if (i + n > b.size()) fail();
                std::string s((const char*)&b[i], (size_t)n);
                i += n;
                return Value::string(s);
            }
            case 4: {
                if (info != 31) {
                    // an array of float64 items (ephemeris and orientation data) is read packed
                    const size_t save = i;
                    const uint64_t n = arg(info);
                    if (n > 0 && n <= (b.size() - i) / 9 && b[i] == 0xFB) {
                        std::vector<double> r((size_t)n);
                        size_t j = i;
                        uint64_t k = 0;
                        for (; k < n && b[j] == 0xFB; ++k, j += 9) {
                            uint64_t u = 0;
                            for (int q = 1; q <= 8; ++q) u = (u << 8) | b[j + q];
                            std::memcpy(&r[(size_t)k], &u, 8);
                        }
                        if (k == n) {
                            i = j;
                            return Value::reals(std::move(r));
                        }
                    }
                    i = save;
                }
                Value v = Value::array();
                if (info == 31) {
                    while (i < b.size() && b[i] != 0xFF) v.push(parse());
                    ++i;
                } else {
                    const uint64_t n = arg(info);
                    v.items().reserve((size_t)n);
                    for (uint64_t k = 0; k < n; ++k) v.push(parse());
                }
                return v;
            }
            case 5: {
                Value v = Value::object();
                auto one = [&]() {
                    Value k = parse();
                    Value x = parse();
                    v.members().emplace_back(k.isString() ? k.asString() : k.dump(), std::move(x));
                };
                if (info == 31) {
                    while (i < b.size() && b[i] != 0xFF) one();
                    ++i;
                } else {
                    const uint64_t n = arg(info);
                    for (uint64_t k = 0; k < n; ++k) one();
                }
                return v;
            }
            case 6: arg(info); return parse();
            case 7: {
                if (info == 20) return Value::boolean(false);
                if (info == 21) return Value::boolean(true);
                if (info == 22 || info == 23) return Value();
                if (info == 25) {
                    const uint16_t hbits = (uint16_t)arg(info);
                    const int ex = (hbits >> 10) & 0x1F, mant = hbits & 0x3FF;
                    double val = ex == 0 ? std::ldexp((double)mant, -24)
                               : ex == 31 ? (mant ? NAN : INFINITY) : std::ldexp((double)(mant + 1024), ex - 25);
                    return Value::real((hbits & 0x8000) ? -val : val);
                }
                if (info == 26) {
                    const uint32_t u = (uint32_t)arg(info);
                    float f;
                    std::memcpy(&f, &u, 4);
                    return Value::real(f);
                }
                if (info == 27) {
                    const uint64_t u = arg(info);
                    double d;
                    std::memcpy(&d, &u, 8);
                    return Value::real(d);
                }
                fail();
            }
        }
        fail();
    }
};
}  // namespace

Value parseJson(const std::string& text) {
    JsonParser p(text);
    Value v = p.parse();
    p.ws();
    if (p.i != text.size()) p.fail("trailing characters");
    return v;
}

Value parseCbor(const std::vector<uint8_t>& bytes) {
    CborParser p(bytes);
    return p.parse();
}

std::string readTextFile(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("Cannot read file: " + path);
    std::ostringstream ss;
    ss << in.rdbuf();
    return ss.str();
}

std::vector<uint8_t> readBinaryFile(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("Cannot read file: " + path);
    return std::vector<uint8_t>((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
}

}  // namespace phop
