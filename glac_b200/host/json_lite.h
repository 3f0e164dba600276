// Minimal JSON reader for the run-configuration files that GLAC's job driver
// writes (objects, arrays, strings, numbers, booleans, null).  Written for this
// project; it implements the JSON grammar of RFC 8259 without extensions.
#pragma once

#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace glac_host {

class Json {
public:
    enum Type { Null, Bool, Number, String, Array, Object };

    Json() : type_(Null) {}
    static Json parse(const std::string &text) {
        size_t i = 0;
        Json v = parse_value(text, i);
        skip_ws(text, i);
        if (i != text.size()) throw std::runtime_error("json: trailing characters at offset " + std::to_string(i));
        return v;
    }

    Type type() const { return type_; }
    bool is_null() const { return type_ == Null; }
    bool has(const std::string &k) const { return type_ == Object && obj_.count(k) > 0; }
    const Json &operator[](const std::string &k) const {
        static const Json null_value;
        if (type_ != Object) throw std::runtime_error("json: not an object (looking up '" + k + "')");
        auto it = obj_.find(k);
        return it == obj_.end() ? null_value : it->second;
    }
    const Json &operator[](size_t i) const {
        if (type_ != Array || i >= arr_.size()) throw std::runtime_error("json: array index out of range");
        return arr_[i];
    }
    size_t size() const { return type_ == Array ? arr_.size() : type_ == Object ? obj_.size() : 0; }
    bool empty() const { return size() == 0 && type_ != Bool && type_ != Number && type_ != String; }

    double number() const {
        if (type_ == Number) return num_;
        if (type_ == Bool) return b_ ? 1.0 : 0.0;
        throw std::runtime_error("json: value is not a number");
    }
    bool boolean() const {
        if (type_ == Bool) return b_;
        if (type_ == Number) return num_ != 0.0;
        throw std::runtime_error("json: value is not a boolean");
    }
    const std::string &string() const {
        if (type_ != String) throw std::runtime_error("json: value is not a string");
        return str_;
    }
    std::vector<std::string> strings() const {
        std::vector<std::string> out;
        if (type_ == Null) return out;
        if (type_ != Array) throw std::runtime_error("json: value is not an array");
        for (const Json &v : arr_) out.push_back(v.string());
        return out;
    }

private:
    Type type_;
    bool b_ = false;
    double num_ = 0.0;
    std::string str_;
    std::vector<Json> arr_;
    std::map<std::string, Json> obj_;

    static void skip_ws(const std::string &s, size_t &i) {
        while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) i++;
    }
    static void expect(const std::string &s, size_t &i, char c) {
        skip_ws(s, i);
        if (i >= s.size() || s[i] != c)
            throw std::runtime_error(std::string("json: expected '") + c + "' at offset " + std::to_string(i));
        i++;
    }
    static std::string parse_string(const std::string &s, size_t &i) {
        expect(s, i, '"');
        std::string out;
        while (i < s.size() && s[i] != '"') {
            char c = s[i++];
            if (c == '\\') {
                if (i >= s.size()) break;
                char e = s[i++];
                switch (e) {
                case '"': out += '"'; break;
                case '\\': out += '\\'; break;
                case '/': out += '/'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'n': out += '\n'; break;
                case 'r': out += '\r'; break;
                case 't': out += '\t'; break;
                case 'u': {
                    if (i + 4 > s.size()) throw std::runtime_error("json: bad \\u escape");
                    unsigned cp = (unsigned)std::strtoul(s.substr(i, 4).c_str(), nullptr, 16);
                    i += 4;
                    if (cp < 0x80) out += (char)cp;
                    else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
                    else {
                        out += (char)(0xE0 | (cp >> 12));
                        out += (char)(0x80 | ((cp >> 6) & 0x3F));
                        out += (char)(0x80 | (cp & 0x3F));
                    }
                    break;
                }
                default: throw std::runtime_error("json: bad escape");
                }
            } else {
                out += c;
            }
        }
        if (i >= s.size()) throw std::runtime_error("json: unterminated string");
        i++;
        return out;
    }
    static Json parse_value(const std::string &s, size_t &i) {
        skip_ws(s, i);
        if (i >= s.size()) throw std::runtime_error("json: unexpected end of input");
        Json v;
        char c = s[i];
        if (c == '{') {
            v.type_ = Object;
            i++;
            skip_ws(s, i);
            if (i < s.size() && s[i] == '}') { i++; return v; }
            while (true) {
                std::string k = parse_string(s, i);
                expect(s, i, ':');
                v.obj_[k] = parse_value(s, i);
                skip_ws(s, i);
                if (i < s.size() && s[i] == ',') { i++; continue; }
                expect(s, i, '}');
                return v;
            }
        }
        if (c == '[') {
            v.type_ = Array;
            i++;
            skip_ws(s, i);
            if (i < s.size() && s[i] == ']') { i++; return v; }
            while (true) {
                v.arr_.push_back(parse_value(s, i));
                skip_ws(s, i);
                if (i < s.size() && s[i] == ',') { i++; continue; }
                expect(s, i, ']');
                return v;
            }
        }
        if (c == '"') {
            v.type_ = String;
            v.str_ = parse_string(s, i);
            return v;
        }
        if (s.compare(i, 4, "true") == 0) { v.type_ = Bool; v.b_ = true; i += 4; return v; }
        if (s.compare(i, 5, "false") == 0) { v.type_ = Bool; v.b_ = false; i += 5; return v; }
        if (s.compare(i, 4, "null") == 0) { i += 4; return v; }
        const char *start = s.c_str() + i;
        char *end = nullptr;
        double d = std::strtod(start, &end);
        if (end == start) throw std::runtime_error("json: bad value at offset " + std::to_string(i));
        i += (size_t)(end - start);
        v.type_ = Number;
        v.num_ = d;
        return v;
    }
};

}  // namespace glac_host
