// Minimal JSON reader for plan trees.
//
// Plans cross the C ABI as JSON text (the operator tree mirrors
// plan::Operator / plan::Expression).  This reader covers exactly the JSON
// subset the plan serialiser emits: objects, arrays, strings with the standard
// escapes, numbers, true/false/null.  Errors throw kdb::json::ParseError.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace kdb::json {

struct ParseError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct Value {
  enum class Kind { Null, Bool, Number, String, Array, Object };
  Kind kind = Kind::Null;
  bool b = false;
  double num = 0;
  bool is_int = false;
  int64_t i = 0;
  std::string s;
  std::vector<Value> arr;
  std::map<std::string, Value> obj;

  bool has(const std::string& k) const {
    return kind == Kind::Object && obj.count(k) > 0;
  }
  const Value& at(const std::string& k) const {
    auto it = obj.find(k);
    if (kind != Kind::Object || it == obj.end())
      throw ParseError("missing key '" + k + "'");
    return it->second;
  }
  const Value& operator[](size_t idx) const { return arr.at(idx); }
  size_t size() const { return kind == Kind::Array ? arr.size() : 0; }
  const std::string& str() const {
    if (kind != Kind::String) throw ParseError("expected string");
    return s;
  }
  int64_t as_int() const {
    if (kind == Kind::Bool) return b ? 1 : 0;
    if (kind != Kind::Number) throw ParseError("expected number");
    return is_int ? i : static_cast<int64_t>(num);
  }
  double as_double() const {
    if (kind != Kind::Number) throw ParseError("expected number");
    return is_int ? static_cast<double>(i) : num;
  }
  bool as_bool() const {
    if (kind == Kind::Bool) return b;
    if (kind == Kind::Number) return as_int() != 0;
    throw ParseError("expected bool");
  }
};

class Reader {
 public:
  explicit Reader(const std::string& text) : t_(text) {}

  Value Parse() {
    Value v = ParseValue();
    SkipWs();
    if (p_ != t_.size()) throw ParseError("trailing characters in JSON");
    return v;
  }

 private:
  const std::string& t_;
  size_t p_ = 0;

  void SkipWs() {
    while (p_ < t_.size() && (t_[p_] == ' ' || t_[p_] == '\n' || t_[p_] == '\t' ||
                              t_[p_] == '\r'))
      p_++;
  }
  char Peek() {
    SkipWs();
    if (p_ >= t_.size()) throw ParseError("unexpected end of JSON");
    return t_[p_];
  }
  void Expect(char c) {
    if (Peek() != c) throw ParseError(std::string("expected '") + c + "'");
    p_++;
  }
  bool Literal(const char* w) {
    size_t n = std::char_traits<char>::length(w);
    if (t_.compare(p_, n, w) == 0) {
      p_ += n;
      return true;
    }
    return false;
  }

  Value ParseValue() {
    char c = Peek();
    Value v;
    if (c == '{') {
      v.kind = Value::Kind::Object;
      p_++;
      if (Peek() == '}') {
        p_++;
        return v;
      }
      while (true) {
        std::string k = ParseString();
        Expect(':');
        v.obj.emplace(std::move(k), ParseValue());
        char d = Peek();
        p_++;
        if (d == '}') break;
        if (d != ',') throw ParseError("expected ',' or '}'");
      }
      return v;
    }
    if (c == '[') {
      v.kind = Value::Kind::Array;
      p_++;
      if (Peek() == ']') {
        p_++;
        return v;
      }
      while (true) {
        v.arr.push_back(ParseValue());
        char d = Peek();
        p_++;
        if (d == ']') break;
        if (d != ',') throw ParseError("expected ',' or ']'");
      }
      return v;
    }
    if (c == '"') {
      v.kind = Value::Kind::String;
      v.s = ParseString();
      return v;
    }
    if (Literal("true")) {
      v.kind = Value::Kind::Bool;
      v.b = true;
      return v;
    }
    if (Literal("false")) {
      v.kind = Value::Kind::Bool;
      v.b = false;
      return v;
    }
    if (Literal("null")) return v;
    return ParseNumber();
  }

  std::string ParseString() {
    Expect('"');
    std::string out;
    while (true) {
      if (p_ >= t_.size()) throw ParseError("unterminated string");
      char c = t_[p_++];
      if (c == '"') break;
      if (c != '\\') {
        out.push_back(c);
        continue;
      }
      if (p_ >= t_.size()) throw ParseError("bad escape");
      char e = t_[p_++];
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
          if (p_ + 4 > t_.size()) throw ParseError("bad \\u escape");
          unsigned cp = std::stoul(t_.substr(p_, 4), nullptr, 16);
          p_ += 4;
          if (cp >= 0xD800 && cp <= 0xDBFF && p_ + 6 <= t_.size() && t_[p_] == '\\' &&
              t_[p_ + 1] == 'u') {
            unsigned lo = std::stoul(t_.substr(p_ + 2, 4), nullptr, 16);
            p_ += 6;
            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
          }
          // UTF-8 encode
          if (cp < 0x80) {
            out.push_back(static_cast<char>(cp));
          } else if (cp < 0x800) {
            out.push_back(static_cast<char>(0xC0 | (cp >> 6)));
            out.push_back(static_cast<char>(0x80 | (cp & 0x3F)));
          } else if (cp < 0x10000) {
            out.push_back(static_cast<char>(0xE0 | (cp >> 12)));
            out.push_back(static_cast<char>(0x80 | ((cp >> 6) & 0x3F)));
            out.push_back(static_cast<char>(0x80 | (cp & 0x3F)));
          } else {
            out.push_back(static_cast<char>(0xF0 | (cp >> 18)));
            out.push_back(static_cast<char>(0x80 | ((cp >> 12) & 0x3F)));
            out.push_back(static_cast<char>(0x80 | ((cp >> 6) & 0x3F)));
            out.push_back(static_cast<char>(0x80 | (cp & 0x3F)));
          }
          break;
        }
        default: throw ParseError("bad escape");
      }
    }
    return out;
  }

  Value ParseNumber() {
    size_t start = p_;
    bool is_int = true;
    if (p_ < t_.size() && (t_[p_] == '-' || t_[p_] == '+')) p_++;
    while (p_ < t_.size()) {
      char c = t_[p_];
      if (c >= '0' && c <= '9') {
        p_++;
      } else if (c == '.' || c == 'e' || c == 'E' || c == '-' || c == '+') {
        is_int = false;
        p_++;
      } else if (c == 'I' || c == 'N' || c == 'n' || c == 'a' || c == 'f' || c == 'i' ||
                 c == 't' || c == 'y') {
        // Infinity / NaN as emitted by Python's json module
        is_int = false;
        p_++;
      } else {
        break;
      }
    }
    if (start == p_) throw ParseError("bad JSON value");
    std::string tok = t_.substr(start, p_ - start);
    Value v;
    v.kind = Value::Kind::Number;
    if (is_int) {
      v.is_int = true;
      v.i = std::strtoll(tok.c_str(), nullptr, 10);
      v.num = static_cast<double>(v.i);
    } else {
      v.num = std::strtod(tok.c_str(), nullptr);
    }
    return v;
  }
};

inline Value Parse(const std::string& text) { return Reader(text).Parse(); }

}  // namespace kdb::json
