// Minimal JSON reader for tapes and kernel tables (objects, arrays, strings, numbers,
// true/false/null).  Numbers keep their double value; tapes only hold integers below
// 2^53 and f64 time steps.
#pragma once
#include <cstdint>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace te {

struct JValue {
  enum Type { Null, Bool, Num, Str, Arr, Obj } type = Null;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<JValue> arr;
  std::vector<std::pair<std::string, JValue>> obj;

  const JValue* get(const char* key) const {
    if (type != Obj) return nullptr;
    for (auto& kv : obj)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
  const JValue& at(const char* key) const {
    const JValue* v = get(key);
    if (!v) throw std::runtime_error(std::string("missing key '") + key + "'");
    return *v;
  }
  int64_t i64() const {
    if (type == Bool) return b ? 1 : 0;
    if (type != Num) throw std::runtime_error("expected a number");
    return (int64_t)num;
  }
  bool truthy() const { return type == Bool ? b : (type == Num ? num != 0.0 : type != Null); }
};

class JParser {
 public:
  JParser(const char* s, size_t n) : p_(s), e_(s + n) {}
  JValue parse() {
    JValue v = value();
    ws();
    if (p_ != e_) fail("trailing characters");
    return v;
  }

 private:
  const char* p_;
  const char* e_;
  [[noreturn]] void fail(const char* m) { throw std::runtime_error(std::string("JSON: ") + m); }
  void ws() {
    while (p_ < e_ && (*p_ == ' ' || *p_ == '\n' || *p_ == '\r' || *p_ == '\t')) p_++;
  }
  bool lit(const char* s) {
    size_t n = std::char_traits<char>::length(s);
    if ((size_t)(e_ - p_) >= n && std::equal(s, s + n, p_)) {
      p_ += n;
      return true;
    }
    return false;
  }
  JValue value() {
    ws();
    if (p_ >= e_) fail("unexpected end");
    JValue v;
    char c = *p_;
    if (c == '{') {
      v.type = JValue::Obj;
      p_++;
      ws();
      if (p_ < e_ && *p_ == '}') {
        p_++;
        return v;
      }
      for (;;) {
        ws();
        if (p_ >= e_ || *p_ != '"') fail("expected a key");
        std::string k = string();
        ws();
        if (p_ >= e_ || *p_ != ':') fail("expected ':'");
        p_++;
        v.obj.emplace_back(std::move(k), value());
        ws();
        if (p_ < e_ && *p_ == ',') { p_++; continue; }
        if (p_ < e_ && *p_ == '}') { p_++; break; }
        fail("expected ',' or '}'");
      }
    } else if (c == '[') {
      v.type = JValue::Arr;
      p_++;
      ws();
      if (p_ < e_ && *p_ == ']') {
        p_++;
        return v;
      }
      for (;;) {
        v.arr.push_back(value());
        ws();
        if (p_ < e_ && *p_ == ',') { p_++; continue; }
        if (p_ < e_ && *p_ == ']') { p_++; break; }
        fail("expected ',' or ']'");
      }
    } else if (c == '"') {
      v.type = JValue::Str;
      v.str = string();
    } else if (lit("true")) {
      v.type = JValue::Bool;
      v.b = true;
    } else if (lit("false")) {
      v.type = JValue::Bool;
    } else if (lit("null")) {
      v.type = JValue::Null;
    } else {
      char* end = nullptr;
      std::string tmp(p_, (size_t)std::min<ptrdiff_t>(e_ - p_, 64));
      v.num = std::strtod(tmp.c_str(), &end);
      if (end == tmp.c_str()) fail("bad value");
      v.type = JValue::Num;
      p_ += (end - tmp.c_str());
    }
    return v;
  }
  std::string string() {
    p_++;  // opening quote
    std::string s;
    while (p_ < e_ && *p_ != '"') {
      if (*p_ == '\\') {
        p_++;
        if (p_ >= e_) fail("bad escape");
        char c = *p_++;
        switch (c) {
          case 'n': s += '\n'; break;
          case 't': s += '\t'; break;
          case 'r': s += '\r'; break;
          case 'b': s += '\b'; break;
          case 'f': s += '\f'; break;
          case 'u': {
            if (e_ - p_ < 4) fail("bad \\u escape");
            unsigned cp = (unsigned)std::strtoul(std::string(p_, 4).c_str(), nullptr, 16);
            p_ += 4;
            if (cp < 0x80) s += (char)cp;
            else if (cp < 0x800) { s += (char)(0xC0 | (cp >> 6)); s += (char)(0x80 | (cp & 0x3F)); }
            else { s += (char)(0xE0 | (cp >> 12)); s += (char)(0x80 | ((cp >> 6) & 0x3F)); s += (char)(0x80 | (cp & 0x3F)); }
            break;
          }
          default: s += c;
        }
      } else {
        s += *p_++;
      }
    }
    if (p_ >= e_) fail("unterminated string");
    p_++;
    return s;
  }
};

inline std::vector<uint8_t> base64_decode(const std::string& in) {
  static int8_t tab[256];
  static bool init = false;
  if (!init) {
    for (int i = 0; i < 256; i++) tab[i] = -1;
    const char* a = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
    for (int i = 0; i < 64; i++) tab[(uint8_t)a[i]] = (int8_t)i;
    init = true;
  }
  std::vector<uint8_t> out;
  uint32_t acc = 0;
  int bits = 0;
  for (char ch : in) {
    if (ch == '=') break;
    int v = tab[(uint8_t)ch];
    if (v < 0) continue;
    acc = (acc << 6) | (uint32_t)v;
    bits += 6;
    if (bits >= 8) {
      bits -= 8;
      out.push_back((uint8_t)((acc >> bits) & 0xFF));
    }
  }
  return out;
}

}  // namespace te
