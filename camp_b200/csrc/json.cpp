// Minimal JSON reader (RFC 8259 values; \u escapes limited to the BMP).
#include "json.hpp"

#include <cstdlib>
#include <fstream>
#include <sstream>

namespace campb {

namespace {

struct Parser {
  const std::string& s;
  size_t i = 0;
  std::string err;

  explicit Parser(const std::string& text) : s(text) {}

  bool fail(const std::string& msg) {
    if (err.empty()) err = msg + " at offset " + std::to_string(i);
    return false;
  }
  void ws() {
    while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) ++i;
  }
  bool lit(const char* w) {
    size_t k = 0;
    while (w[k]) {
      if (i + k >= s.size() || s[i + k] != w[k]) return false;
      ++k;
    }
    i += k;
    return true;
  }
  static void utf8(unsigned cp, std::string* o) {
    if (cp < 0x80) {
      o->push_back((char)cp);
    } else if (cp < 0x800) {
      o->push_back((char)(0xC0 | (cp >> 6)));
      o->push_back((char)(0x80 | (cp & 0x3F)));
    } else {
      o->push_back((char)(0xE0 | (cp >> 12)));
      o->push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
      o->push_back((char)(0x80 | (cp & 0x3F)));
    }
  }
  bool string(std::string* o) {
    if (i >= s.size() || s[i] != '"') return fail("expected a string");
    ++i;
    while (i < s.size() && s[i] != '"') {
      char c = s[i++];
      if (c != '\\') {
        o->push_back(c);
        continue;
      }
      if (i >= s.size()) return fail("unterminated escape");
      char e = s[i++];
      switch (e) {
        case '"': o->push_back('"'); break;
        case '\\': o->push_back('\\'); break;
        case '/': o->push_back('/'); break;
        case 'b': o->push_back('\b'); break;
        case 'f': o->push_back('\f'); break;
        case 'n': o->push_back('\n'); break;
        case 'r': o->push_back('\r'); break;
        case 't': o->push_back('\t'); break;
        case 'u': {
          if (i + 4 > s.size()) return fail("short \\u escape");
          unsigned cp = (unsigned)std::strtoul(s.substr(i, 4).c_str(), nullptr, 16);
          i += 4;
          utf8(cp, o);
          break;
        }
        default: return fail("bad escape");
      }
    }
    if (i >= s.size()) return fail("unterminated string");
    ++i;
    return true;
  }
  bool value(Json* v) {
    ws();
    if (i >= s.size()) return fail("unexpected end");
    char c = s[i];
    if (c == '{') {
      v->kind = Json::Object;
      ++i;
      ws();
      if (i < s.size() && s[i] == '}') {
        ++i;
        return true;
      }
      for (;;) {
        ws();
        std::string key;
        if (!string(&key)) return false;
        ws();
        if (i >= s.size() || s[i] != ':') return fail("expected ':'");
        ++i;
        Json item;
        if (!value(&item)) return false;
        v->obj.emplace_back(std::move(key), std::move(item));
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
      v->kind = Json::Array;
      ++i;
      ws();
      if (i < s.size() && s[i] == ']') {
        ++i;
        return true;
      }
      for (;;) {
        Json item;
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
      v->kind = Json::String;
      return string(&v->str);
    }
    if (lit("true")) {
      v->kind = Json::Bool;
      v->b = true;
      return true;
    }
    if (lit("false")) {
      v->kind = Json::Bool;
      return true;
    }
    if (lit("null")) return true;
    // number
    const char* p = s.c_str() + i;
    char* end = nullptr;
    double d = std::strtod(p, &end);
    if (end == p) return fail("unexpected character");
    v->kind = Json::Number;
    v->num = d;
    i += (size_t)(end - p);
    return true;
  }
};

}  // namespace

bool parse_json(const std::string& text, Json* out, std::string* err) {
  Parser p(text);
  *out = Json();
  if (!p.value(out)) {
    *err = p.err;
    return false;
  }
  p.ws();
  if (p.i != text.size()) {
    *err = "trailing characters at offset " + std::to_string(p.i);
    return false;
  }
  return true;
}

bool read_json_file(const std::string& path, Json* out, std::string* err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    *err = "cannot open " + path;
    return false;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  if (!parse_json(ss.str(), out, err)) {
    *err = path + ": " + *err;
    return false;
  }
  return true;
}

}  // namespace campb
