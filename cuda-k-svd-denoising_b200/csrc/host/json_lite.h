// Minimal JSON reader for the denoiser's config.json (objects, arrays,
// strings, numbers, booleans, null).  The reference uses the vendored jsonxx
// (src/lib/jsonLib/jsonxx.h); any parser that accepts the same keys will do.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace ksvd_json {

struct Value {
  enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<Value> arr;
  std::map<std::string, Value> obj;

  bool has(const std::string& k) const { return kind == Object && obj.count(k) != 0; }
  const Value* get(const std::string& k) const {
    if (kind != Object) return nullptr;
    auto it = obj.find(k);
    return it == obj.end() ? nullptr : &it->second;
  }
  // jsonxx-style typed getters with a default
  double number(const std::string& k, double dflt) const {
    const Value* v = get(k);
    return (v && v->kind == Number) ? v->num : dflt;
  }
  bool boolean(const std::string& k, bool dflt) const {
    const Value* v = get(k);
    return (v && v->kind == Bool) ? v->b : dflt;
  }
  std::string string(const std::string& k, const std::string& dflt) const {
    const Value* v = get(k);
    return (v && v->kind == String) ? v->str : dflt;
  }
};

// Parses text; on error returns false and sets *err.
bool parse(const std::string& text, Value* out, std::string* err);
bool parse_file(const std::string& path, Value* out, std::string* err);

}  // namespace ksvd_json
