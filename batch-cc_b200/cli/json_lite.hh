// json_lite.hh -- minimal JSON reader for the problem files of the CLI driver.
// Objects keep their keys in sorted order (std::map), so iteration follows key
// order as the reference driver's JSON library does.
#pragma once

#include <cctype>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace bcc_json {

struct Value {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Value> arr;
    std::map<std::string, Value> obj;

    const Value& operator[](const std::string& k) const {
        static const Value null_value;
        auto it = obj.find(k);
        return it == obj.end() ? null_value : it->second;
    }
    const Value& operator[](size_t i) const { return arr.at(i); }
    size_t size() const { return kind == Array ? arr.size() : kind == Object ? obj.size() : 0; }
    float f() const { return (float)num; }
};

class Parser {
  public:
    explicit Parser(const std::string& text) : s_(text) {}
    Value parse() {
        Value v = value();
        ws();
        if (i_ != s_.size()) fail("trailing characters");
        return v;
    }

  private:
    const std::string& s_;
    size_t i_ = 0;
    [[noreturn]] void fail(const char* what) { throw std::runtime_error(std::string("JSON: ") + what + " at offset " + std::to_string(i_)); }
    void ws() {
        while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) ++i_;
    }
    bool lit(const char* w) {
        size_t n = std::char_traits<char>::length(w);
        if (s_.compare(i_, n, w) == 0) {
            i_ += n;
            return true;
        }
        return false;
    }
    Value value() {
        ws();
        if (i_ >= s_.size()) fail("unexpected end");
        Value v;
        const char c = s_[i_];
        if (c == '{') {
            v.kind = Value::Object;
            ++i_;
            ws();
            if (s_[i_] == '}') {
                ++i_;
                return v;
            }
            for (;;) {
                ws();
                std::string k = string();
                ws();
                if (s_[i_++] != ':') fail("expected ':'");
                v.obj[k] = value();
                ws();
                if (s_[i_] == ',') {
                    ++i_;
                    continue;
                }
                if (s_[i_++] != '}') fail("expected '}'");
                return v;
            }
        }
        if (c == '[') {
            v.kind = Value::Array;
            ++i_;
            ws();
            if (s_[i_] == ']') {
                ++i_;
                return v;
            }
            for (;;) {
                v.arr.push_back(value());
                ws();
                if (s_[i_] == ',') {
                    ++i_;
                    continue;
                }
                if (s_[i_++] != ']') fail("expected ']'");
                return v;
            }
        }
        if (c == '"') {
            v.kind = Value::String;
            v.str = string();
            return v;
        }
        if (lit("true")) {
            v.kind = Value::Bool;
            v.b = true;
            return v;
        }
        if (lit("false")) {
            v.kind = Value::Bool;
            return v;
        }
        if (lit("null")) return v;
        char* end = nullptr;
        v.num = std::strtod(s_.c_str() + i_, &end);
        if (end == s_.c_str() + i_) fail("bad value");
        i_ = (size_t)(end - s_.c_str());
        v.kind = Value::Number;
        return v;
    }
    std::string string() {
        if (s_[i_++] != '"') fail("expected string");
        std::string out;
        while (i_ < s_.size() && s_[i_] != '"') {
            if (s_[i_] == '\\') {
                ++i_;
                const char e = s_[i_];
                out += e == 'n' ? '\n' : e == 't' ? '\t' : e;
            } else {
                out += s_[i_];
            }
            ++i_;
        }
        ++i_;
        return out;
    }
};

inline Value parse(const std::string& text) { return Parser(text).parse(); }

}  // namespace bcc_json
