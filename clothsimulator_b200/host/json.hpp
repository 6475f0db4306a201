// JSON values for the scene and material files, with the `//` and `/* */` comments the
// reference's scene files use (conf/*.json is read with jsoncpp's default comment support,
// Simulator.cu:11-17).  Accessors mirror the reference's JsonHelper defaults: a missing key
// reads as null and parse*(json, default) returns the default for null (JsonHelper.cu:3-31).
#ifndef CLOTHSIM_HOST_JSON_HPP
#define CLOTHSIM_HOST_JSON_HPP

#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace clothsim {

class Json {
public:
    enum Type { Null, Number, String, Bool, Array, Object };

    Json() = default;
    static Json number(double d) { Json j; j.type_ = Number; j.num_ = d; return j; }
    static Json string(const std::string& s) { Json j; j.type_ = String; j.str_ = s; return j; }
    static Json boolean(bool b) { Json j; j.type_ = Bool; j.num_ = b; return j; }
    static Json array() { Json j; j.type_ = Array; return j; }
    static Json object() { Json j; j.type_ = Object; return j; }

    Type type() const { return type_; }
    bool isNull() const { return type_ == Null; }
    bool isArray() const { return type_ == Array; }
    bool isObject() const { return type_ == Object; }
    size_t size() const { return type_ == Array ? arr_.size() : (type_ == Object ? keys_.size() : 0); }

    double asDouble() const {
        if (type_ != Number && type_ != Bool) throw std::runtime_error("JSON value is not a number");
        return num_;
    }
    float asFloat() const { return static_cast<float>(asDouble()); }
    int asInt() const { return static_cast<int>(asDouble()); }
    const std::string& asString() const {
        if (type_ != String) throw std::runtime_error("JSON value is not a string");
        return str_;
    }

    const Json& operator[](size_t i) const { return i < arr_.size() && type_ == Array ? arr_[i] : null(); }
    const Json& operator[](const std::string& k) const {
        if (type_ != Object) return null();
        auto it = obj_.find(k);
        return it == obj_.end() ? null() : it->second;
    }
    Json& set(const std::string& k, Json v) {
        if (type_ == Null) type_ = Object;
        if (!obj_.count(k)) keys_.push_back(k);
        obj_[k] = std::move(v);
        return obj_[k];
    }
    void push(Json v) {
        if (type_ == Null) type_ = Array;
        arr_.push_back(std::move(v));
    }
    Json& at(size_t i) {
        if (type_ != Array || i >= arr_.size()) throw std::runtime_error("JSON: index out of range");
        return arr_[i];
    }
    Json& at(const std::string& k) {
        if (type_ != Object || !obj_.count(k)) throw std::runtime_error("JSON: missing key " + k);
        return obj_[k];
    }
    const std::vector<Json>& items() const { return arr_; }
    const std::vector<std::string>& keys() const { return keys_; }

    static Json parse(const std::string& text) {
        size_t p = 0;
        Json j = parseValue(text, p);
        skip(text, p);
        if (p != text.size()) throw std::runtime_error("JSON: trailing characters at offset " + std::to_string(p));
        return j;
    }
    static Json parseFile(const std::string& path) {
        std::ifstream in(path);
        if (!in.is_open()) throw std::runtime_error("cannot open " + path);
        std::stringstream ss;
        ss << in.rdbuf();
        return parse(ss.str());
    }

    std::string dump(int indent = 0) const {
        std::ostringstream o;
        write(o, indent, 0);
        return o.str();
    }

private:
    Type type_ = Null;
    double num_ = 0;
    std::string str_;
    std::vector<Json> arr_;
    std::map<std::string, Json> obj_;
    std::vector<std::string> keys_;

    static const Json& null() {
        static const Json n;
        return n;
    }

    static void skip(const std::string& s, size_t& p) {
        for (;;) {
            while (p < s.size() && (s[p] == ' ' || s[p] == '\t' || s[p] == '\n' || s[p] == '\r')) p++;
            if (p + 1 < s.size() && s[p] == '/' && s[p + 1] == '/') {
                while (p < s.size() && s[p] != '\n') p++;
            } else if (p + 1 < s.size() && s[p] == '/' && s[p + 1] == '*') {
                size_t e = s.find("*/", p + 2);
                if (e == std::string::npos) throw std::runtime_error("JSON: unterminated comment");
                p = e + 2;
            } else {
                return;
            }
        }
    }

    static void expect(const std::string& s, size_t& p, char c) {
        skip(s, p);
        if (p >= s.size() || s[p] != c)
            throw std::runtime_error(std::string("JSON: expected '") + c + "' at offset " + std::to_string(p));
        p++;
    }

    static std::string parseString(const std::string& s, size_t& p) {
        expect(s, p, '"');
        std::string out;
        while (p < s.size() && s[p] != '"') {
            char c = s[p++];
            if (c == '\\' && p < s.size()) {
                char e = s[p++];
                switch (e) {
                    case 'n': out.push_back('\n'); break;
                    case 't': out.push_back('\t'); break;
                    case 'r': out.push_back('\r'); break;
                    case 'b': out.push_back('\b'); break;
                    case 'f': out.push_back('\f'); break;
                    default: out.push_back(e);
                }
            } else {
                out.push_back(c);
            }
        }
        if (p >= s.size()) throw std::runtime_error("JSON: unterminated string");
        p++;
        return out;
    }

    static Json parseValue(const std::string& s, size_t& p) {
        skip(s, p);
        if (p >= s.size()) throw std::runtime_error("JSON: unexpected end of input");
        const char c = s[p];
        if (c == '{') {
            Json j = object();
            p++;
            skip(s, p);
            if (p < s.size() && s[p] == '}') { p++; return j; }
            for (;;) {
                std::string k = parseString(s, p);
                expect(s, p, ':');
                j.set(k, parseValue(s, p));
                skip(s, p);
                if (p < s.size() && s[p] == ',') { p++; continue; }
                expect(s, p, '}');
                return j;
            }
        }
        if (c == '[') {
            Json j = array();
            p++;
            skip(s, p);
            if (p < s.size() && s[p] == ']') { p++; return j; }
            for (;;) {
                j.push(parseValue(s, p));
                skip(s, p);
                if (p < s.size() && s[p] == ',') { p++; continue; }
                expect(s, p, ']');
                return j;
            }
        }
        if (c == '"') return string(parseString(s, p));
        if (s.compare(p, 4, "true") == 0) { p += 4; return boolean(true); }
        if (s.compare(p, 5, "false") == 0) { p += 5; return boolean(false); }
        if (s.compare(p, 4, "null") == 0) { p += 4; return Json(); }
        const char* b = s.c_str() + p;
        char* e = nullptr;
        double d = std::strtod(b, &e);
        if (e == b) throw std::runtime_error("JSON: unexpected character at offset " + std::to_string(p));
        p += static_cast<size_t>(e - b);
        return number(d);
    }

    void write(std::ostringstream& o, int indent, int level) const {
        const std::string pad(indent * (level + 1), ' '), pad0(indent * level, ' ');
        const char* nl = indent ? "\n" : "";
        switch (type_) {
            case Null: o << "null"; break;
            case Bool: o << (num_ != 0 ? "true" : "false"); break;
            case Number: {
                std::ostringstream t;
                t.precision(17);
                t << num_;
                o << t.str();
                break;
            }
            case String: {
                o << '"';
                for (char c : str_) {
                    if (c == '"' || c == '\\') o << '\\';
                    o << c;
                }
                o << '"';
                break;
            }
            case Array:
                o << '[' << nl;
                for (size_t i = 0; i < arr_.size(); i++) {
                    o << pad;
                    arr_[i].write(o, indent, level + 1);
                    o << (i + 1 < arr_.size() ? "," : "") << nl;
                }
                o << pad0 << ']';
                break;
            case Object:
                o << '{' << nl;
                for (size_t i = 0; i < keys_.size(); i++) {
                    o << pad << '"' << keys_[i] << "\": ";
                    obj_.at(keys_[i]).write(o, indent, level + 1);
                    o << (i + 1 < keys_.size() ? "," : "") << nl;
                }
                o << pad0 << '}';
                break;
        }
    }
};

// JsonHelper.cu:3-31 defaults.
inline float parseFloat(const Json& j, float d = 0.0f) { return j.isNull() ? d : j.asFloat(); }
inline int parseInt(const Json& j, int d = 0) { return j.isNull() ? d : j.asInt(); }
inline std::string parseString(const Json& j, const std::string& d = "") { return j.isNull() ? d : j.asString(); }

}  // namespace clothsim

#endif
