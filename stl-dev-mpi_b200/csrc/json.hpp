// Minimal JSON reader for the configuration strings of the C ABI
// (objects, arrays, strings, numbers, booleans, null).
#pragma once
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace stl {

struct Json {
  enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<Json> arr;
  std::map<std::string, Json> obj;

  const Json* get(const std::string& k) const {
    if (kind != Object) return nullptr;
    auto it = obj.find(k);
    return it == obj.end() ? nullptr : &it->second;
  }
  bool has(const std::string& k) const { const Json* v = get(k); return v && v->kind != Null; }
  long long integer(const std::string& k, long long dflt) const {
    const Json* v = get(k);
    if (!v || v->kind == Null) return dflt;
    if (v->kind != Number || v->num < 0 || v->num != (double)(long long)v->num)
      throw std::runtime_error("config key '" + k + "' must be a nonnegative integer");
    return (long long)v->num;
  }
  double real(const std::string& k, double dflt) const {
    const Json* v = get(k);
    if (!v || v->kind == Null) return dflt;
    if (v->kind != Number) throw std::runtime_error("config key '" + k + "' must be a number");
    return v->num;
  }
  bool boolean(const std::string& k, bool dflt) const {
    const Json* v = get(k);
    if (!v || v->kind == Null) return dflt;
    if (v->kind != Bool) throw std::runtime_error("config key '" + k + "' must be a boolean");
    return v->b;
  }
  std::string string(const std::string& k, const std::string& dflt) const {
    const Json* v = get(k);
    if (!v || v->kind == Null) return dflt;
    if (v->kind != String) throw std::runtime_error("config key '" + k + "' must be a string");
    return v->str;
  }

  static Json parse(const char* text) {
    if (!text) throw std::runtime_error("null JSON input");
    const char* p = text;
    Json j = value(p);
    ws(p);
    if (*p) throw std::runtime_error("trailing characters after JSON value");
    return j;
  }

 private:
  static void ws(const char*& p) {
    while (*p == ' ' || *p == '\n' || *p == '\t' || *p == '\r') ++p;
  }
  static Json value(const char*& p) {
    ws(p);
    Json j;
    if (*p == '{') {
      j.kind = Object;
      ++p;
      ws(p);
      if (*p == '}') { ++p; return j; }
      for (;;) {
        ws(p);
        if (*p != '"') throw std::runtime_error("invalid JSON: expected a key");
        std::string k = strval(p);
        ws(p);
        if (*p != ':') throw std::runtime_error("invalid JSON: expected ':'");
        ++p;
        j.obj[k] = value(p);
        ws(p);
        if (*p == ',') { ++p; continue; }
        if (*p == '}') { ++p; break; }
        throw std::runtime_error("invalid JSON object");
      }
    } else if (*p == '[') {
      j.kind = Array;
      ++p;
      ws(p);
      if (*p == ']') { ++p; return j; }
      for (;;) {
        j.arr.push_back(value(p));
        ws(p);
        if (*p == ',') { ++p; continue; }
        if (*p == ']') { ++p; break; }
        throw std::runtime_error("invalid JSON array");
      }
    } else if (*p == '"') {
      j.kind = String;
      j.str = strval(p);
    } else if (!strncmp_(p, "true")) {
      j.kind = Bool; j.b = true; p += 4;
    } else if (!strncmp_(p, "false")) {
      j.kind = Bool; j.b = false; p += 5;
    } else if (!strncmp_(p, "null")) {
      j.kind = Null; p += 4;
    } else {
      char* end = nullptr;
      j.num = std::strtod(p, &end);
      if (end == p) throw std::runtime_error("invalid JSON value");
      j.kind = Number;
      p = end;
    }
    return j;
  }
  static int strncmp_(const char* p, const char* w) {
    while (*w) { if (*p != *w) return 1; ++p; ++w; }
    return 0;
  }
  static std::string strval(const char*& p) {
    std::string s;
    ++p;
    while (*p && *p != '"') {
      if (*p == '\\') {
        ++p;
        switch (*p) {
          case 'n': s += '\n'; break;
          case 't': s += '\t'; break;
          case 'r': s += '\r'; break;
          case 'b': s += '\b'; break;
          case 'f': s += '\f'; break;
          case 'u': s += '?'; p += 4; break;
          default: s += *p;
        }
        ++p;
      } else {
        s += *p++;
      }
    }
    if (*p != '"') throw std::runtime_error("invalid JSON string");
    ++p;
    return s;
  }
};

}  // namespace stl
