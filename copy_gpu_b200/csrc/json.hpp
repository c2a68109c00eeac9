// json.hpp -- minimal JSON reader for RBMD configuration text.
//
// RBMD reads its configuration with jsoncpp in comment-tolerant mode (the shipped files carry
// `//` comments, e.g. rbmd/examples/H2O/rbmd.json).  This reader accepts objects, arrays,
// strings, numbers, true/false/null and both comment styles; it is all the force path needs.
#pragma once
#include <cctype>
#include <cstdlib>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace rbmdjson {

struct Value {
  enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
  bool b = false;
  double num = 0;
  std::string str;
  std::vector<Value> arr;
  std::vector<std::pair<std::string, Value>> obj;

  const Value* get(const std::string& k) const {
    if (kind != Object) return nullptr;
    for (auto& kv : obj)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
  // dotted path lookup: "hyper_parameters.neighbor.cut_off"
  const Value* path(const std::string& p) const {
    const Value* v = this;
    size_t s = 0;
    while (v && s <= p.size()) {
      size_t e = p.find('.', s);
      if (e == std::string::npos) e = p.size();
      v = v->get(p.substr(s, e - s));
      s = e + 1;
      if (e == p.size()) break;
    }
    return v;
  }
};

class Parser {
 public:
  explicit Parser(const std::string& t) : t_(t) {}
  bool parse(Value& out, std::string& err) {
    skip();
    if (!value(out, err)) return false;
    skip();
    if (i_ != t_.size()) { err = "trailing characters at offset " + std::to_string(i_); return false; }
    return true;
  }

 private:
  const std::string& t_;
  size_t i_ = 0;

  void skip() {
    for (;;) {
      while (i_ < t_.size() && (std::isspace((unsigned char)t_[i_]) || (unsigned char)t_[i_] == 0xEF ||
                                (unsigned char)t_[i_] == 0xBB || (unsigned char)t_[i_] == 0xBF))
        ++i_;
      if (i_ + 1 < t_.size() && t_[i_] == '/' && t_[i_ + 1] == '/') {
        while (i_ < t_.size() && t_[i_] != '\n') ++i_;
        continue;
      }
      if (i_ + 1 < t_.size() && t_[i_] == '/' && t_[i_ + 1] == '*') {
        size_t e = t_.find("*/", i_ + 2);
        i_ = e == std::string::npos ? t_.size() : e + 2;
        continue;
      }
      break;
    }
  }
  bool lit(const char* w) {
    size_t n = std::char_traits<char>::length(w);
    if (t_.compare(i_, n, w) == 0) { i_ += n; return true; }
    return false;
  }
  bool str(std::string& s, std::string& err) {
    if (i_ >= t_.size() || t_[i_] != '"') { err = "expected string"; return false; }
    ++i_;
    while (i_ < t_.size() && t_[i_] != '"') {
      char c = t_[i_++];
      if (c == '\\' && i_ < t_.size()) {
        char e = t_[i_++];
        switch (e) {
          case 'n': s += '\n'; break;
          case 't': s += '\t'; break;
          case 'r': s += '\r'; break;
          case 'b': s += '\b'; break;
          case 'f': s += '\f'; break;
          case 'u': i_ += 4; s += '?'; break;
          default: s += e;
        }
      } else {
        s += c;
      }
    }
    if (i_ >= t_.size()) { err = "unterminated string"; return false; }
    ++i_;
    return true;
  }
  bool value(Value& v, std::string& err) {
    skip();
    if (i_ >= t_.size()) { err = "unexpected end of text"; return false; }
    char c = t_[i_];
    if (c == '{') {
      v.kind = Value::Object;
      ++i_;
      skip();
      if (i_ < t_.size() && t_[i_] == '}') { ++i_; return true; }
      for (;;) {
        skip();
        std::string k;
        if (!str(k, err)) return false;
        skip();
        if (i_ >= t_.size() || t_[i_] != ':') { err = "expected ':' after key " + k; return false; }
        ++i_;
        Value x;
        if (!value(x, err)) return false;
        v.obj.emplace_back(k, std::move(x));
        skip();
        if (i_ < t_.size() && t_[i_] == ',') { ++i_; skip(); if (i_ < t_.size() && t_[i_] == '}') { ++i_; return true; } continue; }
        if (i_ < t_.size() && t_[i_] == '}') { ++i_; return true; }
        err = "expected ',' or '}' at offset " + std::to_string(i_);
        return false;
      }
    }
    if (c == '[') {
      v.kind = Value::Array;
      ++i_;
      skip();
      if (i_ < t_.size() && t_[i_] == ']') { ++i_; return true; }
      for (;;) {
        Value x;
        if (!value(x, err)) return false;
        v.arr.push_back(std::move(x));
        skip();
        if (i_ < t_.size() && t_[i_] == ',') { ++i_; skip(); if (i_ < t_.size() && t_[i_] == ']') { ++i_; return true; } continue; }
        if (i_ < t_.size() && t_[i_] == ']') { ++i_; return true; }
        err = "expected ',' or ']' at offset " + std::to_string(i_);
        return false;
      }
    }
    if (c == '"') { v.kind = Value::String; return str(v.str, err); }
    if (lit("true")) { v.kind = Value::Bool; v.b = true; return true; }
    if (lit("false")) { v.kind = Value::Bool; v.b = false; return true; }
    if (lit("null")) { v.kind = Value::Null; return true; }
    const char* s = t_.c_str() + i_;
    char* e = nullptr;
    double d = std::strtod(s, &e);
    if (e == s) { err = "unexpected character at offset " + std::to_string(i_); return false; }
    v.kind = Value::Number;
    v.num = d;
    i_ += (size_t)(e - s);
    return true;
  }
};

inline bool parse(const std::string& text, Value& out, std::string& err) {
  Parser p(text);
  return p.parse(out, err);
}

// typed accessors with defaults
inline double num(const Value& root, const std::string& p, double dflt, bool* found = nullptr) {
  const Value* v = root.path(p);
  if (found) *found = v && v->kind == Value::Number;
  return v && v->kind == Value::Number ? v->num : dflt;
}
inline std::string text(const Value& root, const std::string& p, const std::string& dflt,
                        bool* found = nullptr) {
  const Value* v = root.path(p);
  if (found) *found = v != nullptr;
  if (!v) return dflt;
  if (v->kind == Value::String) return v->str;
  if (v->kind == Value::Bool) return v->b ? "true" : "false";
  if (v->kind == Value::Null) return "null";
  if (v->kind == Value::Number) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.17g", v->num);
    return buf;
  }
  return dflt;
}
inline std::vector<double> nums(const Value& root, const std::string& p) {
  std::vector<double> r;
  const Value* v = root.path(p);
  if (v && v->kind == Value::Array)
    for (auto& x : v->arr)
      if (x.kind == Value::Number) r.push_back(x.num);
  return r;
}

}  // namespace rbmdjson
