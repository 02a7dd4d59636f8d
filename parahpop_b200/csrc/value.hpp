// Minimal JSON / CBOR document model for the configuration, targets,
// constants and ephemeris / orientation files the drop-in boundary reads.
// Objects keep insertion order for output and are searched linearly (they
// hold a handful of keys).  Parsing errors throw std::runtime_error.
#pragma once
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace phop {

class Value {
public:
    enum Kind { Null, Bool, Int, Real, String, Array, Object };

    Value() = default;
    static Value boolean(bool b) { Value v; v.kind_ = Bool; v.b_ = b; return v; }
    static Value integer(int64_t i) { Value v; v.kind_ = Int; v.i_ = i; return v; }
    static Value real(double d) { Value v; v.kind_ = Real; v.d_ = d; return v; }
    static Value string(std::string s) { Value v; v.kind_ = String; v.s_ = std::move(s); return v; }
    static Value array() { Value v; v.kind_ = Array; return v; }
    static Value object() { Value v; v.kind_ = Object; return v; }
    // An array whose items are all reals, held packed (a CBOR array of
    // float64 items, as ephemeris data is written); it reads like any array.
    static Value reals(std::vector<double> r) { Value v; v.kind_ = Array; v.packed_ = true; v.reals_ = std::move(r); return v; }

    Kind kind() const { return kind_; }
    bool isNull() const { return kind_ == Null; }
    bool isBool() const { return kind_ == Bool; }
    bool isNumber() const { return kind_ == Int || kind_ == Real; }
    bool isInt() const { return kind_ == Int; }
    bool isString() const { return kind_ == String; }
    bool isArray() const { return kind_ == Array; }
    bool isObject() const { return kind_ == Object; }

    bool asBool() const;
    double asDouble() const;
    int64_t asInt() const;
    const std::string& asString() const;

    // arrays
    size_t size() const {
        return kind_ == Array ? (packed_ ? reals_.size() : arr_.size()) : (kind_ == Object ? obj_.size() : 0);
    }
    const Value& operator[](size_t i) const;
    Value& push(Value v) { unpack(); arr_.push_back(std::move(v)); return arr_.back(); }
    const std::vector<Value>& items() const { unpack(); return arr_; }
    std::vector<Value>& items() { unpack(); return arr_; }
    // items [off, off + n) of an array of numbers as doubles (throws if out of range or not numbers)
    void copyReals(size_t off, size_t n, double* out) const;

    // objects
    bool has(const std::string& k) const;
    const Value& at(const std::string& k) const;  // throws if missing
    const Value* find(const std::string& k) const;
    Value* find(const std::string& k);
    Value& set(const std::string& k, Value v);
    void erase(const std::string& k);
    const std::vector<std::pair<std::string, Value>>& members() const { return obj_; }
    std::vector<std::pair<std::string, Value>>& members() { return obj_; }

    double numberOr(const std::string& k, double dflt) const;
    std::string dump(int indent = -1) const;

private:
    void dumpTo(std::string& out, int indent, int level) const;
    void unpack() const;  // a packed real array turned into items, on first item access
    Kind kind_ = Null;
    bool b_ = false;
    int64_t i_ = 0;
    double d_ = 0.0;
    std::string s_;
    mutable bool packed_ = false;
    mutable std::vector<double> reals_;
    mutable std::vector<Value> arr_;
    std::vector<std::pair<std::string, Value>> obj_;
};

Value parseJson(const std::string& text);
Value parseCbor(const std::vector<uint8_t>& bytes);
std::string readTextFile(const std::string& path);
std::vector<uint8_t> readBinaryFile(const std::string& path);

}  // namespace phop
