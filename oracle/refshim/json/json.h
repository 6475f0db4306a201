// Minimal jsoncpp-compatible JSON value and parser, written for this project.
//
// Test infrastructure only: it lets the reference's own force and material
// sources (Material.cu, JsonHelper.cu, Transformation.cu, Wind.cu, Magic.cu)
// compile and run on the host as the oracle's pin.  It implements only the
// subset of the jsoncpp API those files use: Value construction, operator[]
// by key and by index, isNull/isArray/isObject, asInt/asFloat/asString, size,
// and `istream >> Value`.  `//` and `/* */` comments are accepted, as jsoncpp
// does by default for the reference's scene files.
#ifndef CLOTHSTEP_REFSHIM_JSON_H
#define CLOTHSTEP_REFSHIM_JSON_H

#include <cctype>
#include <cstdlib>
#include <istream>
#include <iterator>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace Json {

enum ValueType { nullValue = 0, intValue, realValue, stringValue, booleanValue, arrayValue, objectValue };

class Value {
public:
    Value() : type_(nullValue) {}
    Value(ValueType t) : type_(t) {}
    Value(double d) : type_(realValue), num_(d) {}
    Value(int i) : type_(intValue), num_(i) {}
    Value(const std::string& s) : type_(stringValue), str_(s) {}
    Value(const char* s) : type_(stringValue), str_(s) {}
    Value(bool b) : type_(booleanValue), num_(b ? 1.0 : 0.0) {}

    bool isNull() const { return type_ == nullValue; }
    bool isArray() const { return type_ == arrayValue; }
    bool isObject() const { return type_ == objectValue; }
    bool isString() const { return type_ == stringValue; }
    bool isNumeric() const { return type_ == intValue || type_ == realValue; }

    int asInt() const { return static_cast<int>(num_); }
    float asFloat() const { return static_cast<float>(num_); }
    double asDouble() const { return num_; }
    bool asBool() const { return num_ != 0.0; }
    std::string asString() const { return str_; }

    unsigned size() const {
        if (type_ == arrayValue) return static_cast<unsigned>(arr_.size());
        if (type_ == objectValue) return static_cast<unsigned>(obj_.size());
        return 0;
    }

    const Value& operator[](int i) const {
        if (type_ != arrayValue || i < 0 || i >= static_cast<int>(arr_.size())) return null_();
        return arr_[i];
    }
    Value& operator[](int i) {
        if (type_ == nullValue) type_ = arrayValue;
        if (static_cast<int>(arr_.size()) <= i) arr_.resize(i + 1);
        return arr_[i];
    }
    const Value& operator[](const std::string& k) const {
        if (type_ != objectValue) return null_();
        auto it = obj_.find(k);
        return it == obj_.end() ? null_() : it->second;
    }
    Value& operator[](const std::string& k) {
        if (type_ == nullValue) type_ = objectValue;
        return obj_[k];
    }
    const Value& operator[](const char* k) const { return (*this)[std::string(k)]; }
    Value& operator[](const char* k) { return (*this)[std::string(k)]; }

    void append(const Value& v) {
        if (type_ == nullValue) type_ = arrayValue;
        arr_.push_back(v);
    }

    std::vector<Value>::const_iterator begin() const { return arr_.begin(); }
    std::vector<Value>::const_iterator end() const { return arr_.end(); }

    friend std::istream& operator>>(std::istream& in, Value& v) {
        std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
        size_t pos = 0;
        v = parse_(text, pos);
        return in;
    }

private:
    ValueType type_;
    double num_ = 0.0;
    std::string str_;
    std::vector<Value> arr_;
    std::map<std::string, Value> obj_;

    static const Value& null_() {
        static const Value n;
        return n;
    }

    static void skip_(const std::string& s, size_t& p) {
        for (;;) {
            while (p < s.size() && std::isspace(static_cast<unsigned char>(s[p]))) p++;
            if (p + 1 < s.size() && s[p] == '/' && s[p + 1] == '/') {
                while (p < s.size() && s[p] != '\n') p++;
            } else if (p + 1 < s.size() && s[p] == '/' && s[p + 1] == '*') {
                p += 2;
                while (p + 1 < s.size() && !(s[p] == '*' && s[p + 1] == '/')) p++;
                p += 2;
            } else {
                return;
            }
        }
    }

    static Value parse_(const std::string& s, size_t& p) {
        skip_(s, p);
        if (p >= s.size()) throw std::runtime_error("json: unexpected end");
        char c = s[p];
        if (c == '{') {
            Value v(objectValue);
            p++;
            skip_(s, p);
            if (s[p] == '}') { p++; return v; }
            for (;;) {
                skip_(s, p);
                Value key = parse_(s, p);
                skip_(s, p);
                if (s[p] != ':') throw std::runtime_error("json: expected ':'");
                p++;
                v.obj_[key.str_] = parse_(s, p);
                skip_(s, p);
                if (s[p] == ',') { p++; continue; }
                if (s[p] == '}') { p++; return v; }
                throw std::runtime_error("json: expected ',' or '}'");
            }
        }
        if (c == '[') {
            Value v(arrayValue);
            p++;
            skip_(s, p);
            if (s[p] == ']') { p++; return v; }
            for (;;) {
                v.arr_.push_back(parse_(s, p));
                skip_(s, p);
                if (s[p] == ',') { p++; continue; }
                if (s[p] == ']') { p++; return v; }
                throw std::runtime_error("json: expected ',' or ']'");
            }
        }
        if (c == '"') {
            std::string out;
            p++;
            while (p < s.size() && s[p] != '"') {
                if (s[p] == '\\' && p + 1 < s.size()) { p++; }
                out.push_back(s[p++]);
            }
            p++;
            return Value(out);
        }
        if (s.compare(p, 4, "true") == 0) { p += 4; return Value(true); }
        if (s.compare(p, 5, "false") == 0) { p += 5; return Value(false); }
        if (s.compare(p, 4, "null") == 0) { p += 4; return Value(); }
        const char* start = s.c_str() + p;
        char* stop = nullptr;
        double d = std::strtod(start, &stop);
        if (stop == start) throw std::runtime_error("json: bad token");
        p += static_cast<size_t>(stop - start);
        return Value(d);
    }
};

}  // namespace Json

#endif
