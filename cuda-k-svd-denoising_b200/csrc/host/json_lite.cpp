#include "json_lite.h"

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace ksvd_json {
namespace {

struct Parser {
  const std::string& s;
  size_t i = 0;
  std::string err;

  explicit Parser(const std::string& t) : s(t) {}

  void ws() {
    while (i < s.size()) {
      if (std::isspace(static_cast<unsigned char>(s[i]))) {
        ++i;
      } else if (s.compare(i, 2, "//") == 0) {  // tolerate line comments
        while (i < s.size() && s[i] != '\n') ++i;
      } else {
        break;
      }
    }
  }
  bool fail(const std::string& m) {
    if (err.empty()) err = m + " at offset " + std::to_string(i);
    return false;
  }
  bool lit(const char* w) {
    size_t n = std::char_traits<char>::length(w);
    if (s.compare(i, n, w) != 0) return false;
    i += n;
    return true;
  }
  bool str(std::string* out) {
    if (i >= s.size() || s[i] != '"') return fail("expected string");
    ++i;
    out->clear();
    while (i < s.size() && s[i] != '"') {
      char c = s[i++];
      if (c == '\\') {
        if (i >= s.size()) return fail("bad escape");
        char e = s[i++];
        switch (e) {
          case 'n': out->push_back('\n'); break;
          case 't': out->push_back('\t'); break;
          case 'r': out->push_back('\r'); break;
          case 'b': out->push_back('\b'); break;
          case 'f': out->push_back('\f'); break;
          case 'u': {
            if (i + 4 > s.size()) return fail("bad \\u escape");
            unsigned cp = unsigned(std::strtoul(s.substr(i, 4).c_str(), nullptr, 16));
            i += 4;
            if (cp < 0x80) {
              out->push_back(char(cp));
            } else if (cp < 0x800) {
              out->push_back(char(0xC0 | (cp >> 6)));
              out->push_back(char(0x80 | (cp & 0x3F)));
            } else {
              out->push_back(char(0xE0 | (cp >> 12)));
              out->push_back(char(0x80 | ((cp >> 6) & 0x3F)));
              out->push_back(char(0x80 | (cp & 0x3F)));
            }
            break;
          }
          default: out->push_back(e);
        }
      } else {
        out->push_back(c);
      }
    }
    if (i >= s.size()) return fail("unterminated string");
    ++i;
    return true;
  }
  bool value(Value* v) {
    ws();
    if (i >= s.size()) return fail("unexpected end");
    char c = s[i];
    if (c == '{') {
      ++i;
      v->kind = Value::Object;
      ws();
      if (i < s.size() && s[i] == '}') {
        ++i;
        return true;
      }
      for (;;) {
        ws();
        std::string k;
        if (!str(&k)) return false;
        ws();
        if (i >= s.size() || s[i] != ':') return fail("expected ':'");
        ++i;
        Value item;
        if (!value(&item)) return false;
        v->obj[k] = std::move(item);
        ws();
        if (i < s.size() && s[i] == ',') {
          ++i;
          continue;
        }
        if (i < s.size() && s[i] == '}') {
          ++i;
          return true;
        }
        return fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      ++i;
      v->kind = Value::Array;
      ws();
      if (i < s.size() && s[i] == ']') {
        ++i;
        return true;
      }
      for (;;) {
        Value item;
        if (!value(&item)) return false;
        v->arr.push_back(std::move(item));
        ws();
        if (i < s.size() && s[i] == ',') {
          ++i;
          continue;
        }
        if (i < s.size() && s[i] == ']') {
          ++i;
          return true;
        }
        return fail("expected ',' or ']'");
      }
    }
    if (c == '"') {
      v->kind = Value::String;
      return str(&v->str);
    }
    if (lit("true")) {
      v->kind = Value::Bool;
      v->b = true;
      return true;
    }
    if (lit("false")) {
      v->kind = Value::Bool;
      v->b = false;
      return true;
    }
    if (lit("null")) {
      v->kind = Value::Null;
      return true;
    }
    const char* b = s.c_str() + i;
    char* e = nullptr;
    double d = std::strtod(b, &e);
    if (e == b) return fail("unexpected character");
    i += size_t(e - b);
    v->kind = Value::Number;
    v->num = d;
    return true;
  }
};

}  // namespace

bool parse(const std::string& text, Value* out, std::string* err) {
  Parser p(text);
  *out = Value();
  if (!p.value(out)) {
    if (err) *err = p.err;
    return false;
  }
  p.ws();
  if (p.i != text.size()) {
    if (err) *err = "trailing characters at offset " + std::to_string(p.i);
    return false;
  }
  return true;
}

bool parse_file(const std::string& path, Value* out, std::string* err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    if (err) *err = "cannot open " + path;
    return false;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  return parse(ss.str(), out, err);
}

}  // namespace ksvd_json
