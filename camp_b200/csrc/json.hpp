// Minimal JSON reader for CAMP input files (objects keep their key order,
// which decides reactant and product order in the packed reactions).
#pragma once

#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace campb {

struct Json {
  enum Kind { Null, Bool, Number, String, Array, Object };
  Kind kind = Null;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<Json> arr;
  std::vector<std::pair<std::string, Json>> obj;

  const Json* get(const std::string& key) const {
    for (const auto& kv : obj)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
  bool has(const std::string& key) const { return get(key) != nullptr; }
};

// Parses text; on error returns false with a message naming the offset.
bool parse_json(const std::string& text, Json* out, std::string* err);
bool read_json_file(const std::string& path, Json* out, std::string* err);

}  // namespace campb
