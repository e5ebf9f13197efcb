// Minimal JSON value + parser + writer helpers for plan trees and tune-DB rows.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace ffb {

struct Json {
  enum Type { Null, Bool, Number, String, Array, Object } type = Null;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<Json> arr;
  std::map<std::string, Json> obj;

  bool has(const std::string &k) const { return type == Object && obj.count(k) != 0; }
  const Json &at(const std::string &k) const {
    auto it = obj.find(k);
    if (type != Object || it == obj.end()) throw std::runtime_error("json: missing key " + k);
    return it->second;
  }
  int64_t i64() const {
    if (type != Number) throw std::runtime_error("json: not a number");
    return (int64_t)num;
  }
  std::vector<int64_t> ivec() const {
    if (type != Array) throw std::runtime_error("json: not an array");
    std::vector<int64_t> out;
    for (const auto &v : arr) out.push_back(v.i64());
    return out;
  }

  static Json parse(const std::string &s) {
    size_t pos = 0;
    Json v = parse_value(s, pos);
    skip(s, pos);
    if (pos != s.size()) throw std::runtime_error("json: trailing characters");
    return v;
  }

 private:
  static void skip(const std::string &s, size_t &p) {
    while (p < s.size() && (s[p] == ' ' || s[p] == '\n' || s[p] == '\t' || s[p] == '\r')) ++p;
  }
  static Json parse_value(const std::string &s, size_t &p) {
    skip(s, p);
    if (p >= s.size()) throw std::runtime_error("json: unexpected end");
    Json v;
    char c = s[p];
    if (c == '{') {
      v.type = Object;
      ++p;
      skip(s, p);
      if (p < s.size() && s[p] == '}') {
        ++p;
        return v;
      }
      while (true) {
        skip(s, p);
        Json key = parse_value(s, p);
        if (key.type != String) throw std::runtime_error("json: object key");
        skip(s, p);
        if (p >= s.size() || s[p] != ':') throw std::runtime_error("json: expected ':'");
        ++p;
        v.obj[key.str] = parse_value(s, p);
        skip(s, p);
        if (p < s.size() && s[p] == ',') {
          ++p;
          continue;
        }
        if (p < s.size() && s[p] == '}') {
          ++p;
          return v;
        }
        throw std::runtime_error("json: expected ',' or '}'");
      }
    }
    if (c == '[') {
      v.type = Array;
      ++p;
      skip(s, p);
      if (p < s.size() && s[p] == ']') {
        ++p;
        return v;
      }
      while (true) {
        v.arr.push_back(parse_value(s, p));
        skip(s, p);
        if (p < s.size() && s[p] == ',') {
          ++p;
          continue;
        }
        if (p < s.size() && s[p] == ']') {
          ++p;
          return v;
        }
        throw std::runtime_error("json: expected ',' or ']'");
      }
    }
    if (c == '"') {
      v.type = String;
      ++p;
      while (p < s.size() && s[p] != '"') {
        if (s[p] == '\\' && p + 1 < s.size()) {
          ++p;
          char e = s[p];
          v.str += e == 'n' ? '\n' : e == 't' ? '\t' : e;
        } else {
          v.str += s[p];
        }
        ++p;
      }
      if (p >= s.size()) throw std::runtime_error("json: unterminated string");
      ++p;
      return v;
    }
    if (s.compare(p, 4, "true") == 0) {
      v.type = Bool;
      v.b = true;
      p += 4;
      return v;
    }
    if (s.compare(p, 5, "false") == 0) {
      v.type = Bool;
      p += 5;
      return v;
    }
    if (s.compare(p, 4, "null") == 0) {
      p += 4;
      return v;
    }
    size_t q = p;
    while (q < s.size() && (isdigit((unsigned char)s[q]) || s[q] == '-' || s[q] == '+' || s[q] == '.' ||
                            s[q] == 'e' || s[q] == 'E'))
      ++q;
    if (q == p) throw std::runtime_error("json: bad token");
    v.type = Number;
    v.num = std::stod(s.substr(p, q - p));
    p = q;
    return v;
  }
};

inline std::string json_ints(const std::vector<int64_t> &v) {
  std::string s = "[";
  for (size_t i = 0; i < v.size(); ++i) {
    if (i) s += ",";
    s += std::to_string(v[i]);
  }
  return s + "]";
}

inline std::string json_str(const std::string &v) {
  std::string s = "\"";
  for (char c : v) {
    if (c == '"' || c == '\\') s += '\\';
    s += c;
  }
  return s + "\"";
}

}  // namespace ffb
