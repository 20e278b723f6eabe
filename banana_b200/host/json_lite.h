// Minimal JSON reader for scene files (objects, arrays, numbers, strings, true/false/null).
// Scene files are what Banana's solvers read with nlohmann::json through JSONHelpers
// (Utils/JSONHelpers.h); only reading is needed here.
#pragma once

#include <cctype>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace bnnhost {

struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::map<std::string, Json> obj;

    bool has(const std::string& k) const { return kind == Object && obj.count(k) != 0; }
    const Json& operator[](const std::string& k) const {
        static const Json none;
        auto it = obj.find(k);
        return (kind == Object && it != obj.end()) ? it->second : none;
    }
    const Json& operator[](size_t i) const {
        static const Json none;
        return (kind == Array && i < arr.size()) ? arr[i] : none;
    }
    size_t size() const { return kind == Array ? arr.size() : (kind == Object ? obj.size() : 0); }
};

class JsonParser {
public:
    explicit JsonParser(const std::string& text) : s_(text) {}

    Json parse() {
        Json v = value();
        ws();
        if(p_ != s_.size()) fail("trailing characters");
        return v;
    }

private:
    const std::string& s_;
    size_t p_ = 0;

    [[noreturn]] void fail(const char* what) const {
        throw std::runtime_error(std::string("scene JSON: ") + what + " at offset " + std::to_string(p_));
    }
    void ws() {
        for(;;) {
            while(p_ < s_.size() && std::isspace((unsigned char)s_[p_])) ++p_;
            // tolerate // line comments, which some hand-written scene files carry
            if(p_ + 1 < s_.size() && s_[p_] == '/' && s_[p_ + 1] == '/') {
                while(p_ < s_.size() && s_[p_] != '\n') ++p_;
                continue;
            }
            break;
        }
    }
    char peek() {
        ws();
        if(p_ >= s_.size()) fail("unexpected end");
        return s_[p_];
    }
    void expect(char c) {
        if(peek() != c) fail("unexpected character");
        ++p_;
    }
    Json value() {
        const char c = peek();
        if(c == '{') return object();
        if(c == '[') return array();
        if(c == '"') {
            Json v;
            v.kind = Json::String;
            v.str = string();
            return v;
        }
        if(c == 't' || c == 'f' || c == 'n') return literal();
        return number();
    }
    Json object() {
        Json v;
        v.kind = Json::Object;
        expect('{');
        if(peek() == '}') { ++p_; return v; }
        for(;;) {
            if(peek() != '"') fail("expected a key");
            std::string k = string();
            expect(':');
            v.obj[k] = value();
            const char c = peek();
            ++p_;
            if(c == '}') return v;
            if(c != ',') fail("expected , or }");
        }
    }
    Json array() {
        Json v;
        v.kind = Json::Array;
        expect('[');
        if(peek() == ']') { ++p_; return v; }
        for(;;) {
            v.arr.push_back(value());
            const char c = peek();
            ++p_;
            if(c == ']') return v;
            if(c != ',') fail("expected , or ]");
        }
    }
    std::string string() {
        expect('"');
        std::string out;
        while(p_ < s_.size() && s_[p_] != '"') {
            char c = s_[p_++];
            if(c == '\\' && p_ < s_.size()) {
                const char e = s_[p_++];
                switch(e) {
                    case 'n': c = '\n'; break;
                    case 't': c = '\t'; break;
                    case 'r': c = '\r'; break;
                    case 'b': c = '\b'; break;
                    case 'f': c = '\f'; break;
                    case 'u': p_ += 4; c = '?'; break;  // no non-ASCII in scene files
                    default: c = e;
                }
            }
            out.push_back(c);
        }
        if(p_ >= s_.size()) fail("unterminated string");
        ++p_;
        return out;
    }
    Json literal() {
        Json v;
        if(s_.compare(p_, 4, "true") == 0) { v.kind = Json::Bool; v.b = true; p_ += 4; }
        else if(s_.compare(p_, 5, "false") == 0) { v.kind = Json::Bool; v.b = false; p_ += 5; }
        else if(s_.compare(p_, 4, "null") == 0) { p_ += 4; }
        else fail("bad literal");
        return v;
    }
    Json number() {
        const char* b = s_.c_str() + p_;
        char* e = nullptr;
        const double d = std::strtod(b, &e);
        if(e == b) fail("bad number");
        p_ += (size_t)(e - b);
        Json v;
        v.kind = Json::Number;
        v.num = d;
        return v;
    }
};

// JSONHelpers::readValue / readBool / readVector: leave `out` unchanged when the key is absent
inline bool read_number(const Json& j, const char* key, double& out) {
    const Json& v = j[key];
    if(v.kind != Json::Number) return false;
    out = v.num;
    return true;
}
template<class T>
inline bool read_value(const Json& j, const char* key, T& out) {
    double d;
    if(!read_number(j, key, d)) return false;
    out = (T)d;
    return true;
}
inline bool read_bool(const Json& j, const char* key, bool& out) {
    const Json& v = j[key];
    if(v.kind != Json::Bool) return false;
    out = v.b;
    return true;
}
inline bool read_string(const Json& j, const char* key, std::string& out) {
    const Json& v = j[key];
    if(v.kind != Json::String) return false;
    out = v.str;
    return true;
}
template<class T>
inline bool read_vec3(const Json& j, const char* key, T out[3]) {
    const Json& v = j[key];
    if(v.kind != Json::Array || v.size() != 3) return false;
    for(int d = 0; d < 3; ++d) out[d] = (T)v[d].num;
    return true;
}

} // namespace bnnhost
