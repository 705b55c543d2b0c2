#include "json.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <charconv>
#include <stdexcept>

namespace fdp {

bool Json::as_bool() const {
  if (t_ != Bool) throw std::runtime_error("JSON: expected a boolean");
  return b_;
}
int64_t Json::as_int() const {
  if (t_ != Int) throw std::runtime_error("JSON: expected an integer");
  return i_;
}
double Json::as_number() const {
  if (t_ == Int) return double(i_);
  if (t_ != Float) throw std::runtime_error("JSON: expected a number");
  return f_;
}
const std::string &Json::as_string() const {
  if (t_ != String) throw std::runtime_error("JSON: expected a string");
  return s_;
}
const std::vector<Json> &Json::items() const {
  if (t_ != Array) throw std::runtime_error("JSON: expected an array");
  return a_;
}
const std::map<std::string, Json> &Json::fields() const {
  if (t_ != Object) throw std::runtime_error("JSON: expected an object");
  return o_;
}
Json &Json::push(const Json &v) {
  if (t_ != Array) throw std::runtime_error("JSON: push on a non-array");
  a_.push_back(v);
  return *this;
}
Json &Json::set(const std::string &k, const Json &v) {
  if (t_ != Object) throw std::runtime_error("JSON: set on a non-object");
  o_[k] = v;
  return *this;
}
bool Json::has(const std::string &k) const { return t_ == Object && o_.count(k); }
const Json &Json::at(const std::string &k) const {
  auto it = fields().find(k);
  if (it == o_.end()) throw std::runtime_error("JSON: missing field " + k);
  return it->second;
}

std::string python_float_repr(double v) {
  if (!std::isfinite(v)) throw std::runtime_error("JSON: non-finite float");
  if (v == 0) return std::signbit(v) ? "-0.0" : "0.0";
  std::string sign;
  if (v < 0) {
    sign = "-";
    v = -v;
  }
  char buf[64];
  auto res = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::scientific);
  std::string sci(buf, res.ptr);
  const size_t e = sci.find('e');
  std::string mant = sci.substr(0, e);
  const int exp10 = atoi(sci.c_str() + e + 1);
  std::string digits;
  for (char c : mant)
    if (c != '.') digits += c;
  while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
  const int decpt = exp10 + 1;  // value = 0.DIGITS x 10^decpt
  std::string out;
  if (decpt > -4 && decpt <= 16) {
    const int nd = int(digits.size());
    if (decpt <= 0) out = "0." + std::string(size_t(-decpt), '0') + digits;
    else if (decpt >= nd) out = digits + std::string(size_t(decpt - nd), '0') + ".0";
    else out = digits.substr(0, size_t(decpt)) + "." + digits.substr(size_t(decpt));
  } else {
    out = digits.substr(0, 1);
    if (digits.size() > 1) out += "." + digits.substr(1);
    const int x = decpt - 1;
    char eb[16];
    snprintf(eb, sizeof(eb), "e%c%02d", x < 0 ? '-' : '+', x < 0 ? -x : x);
    out += eb;
  }
  return sign + out;
}

static void dump_string(std::string &out, const std::string &s) {
  out += '"';
  size_t i = 0;
  while (i < s.size()) {
    unsigned char c = (unsigned char)s[i];
    uint32_t cp;
    size_t len;
    if (c < 0x80) { cp = c; len = 1; }
    else if ((c >> 5) == 6 && i + 1 < s.size()) { cp = ((c & 0x1f) << 6) | (s[i + 1] & 0x3f); len = 2; }
    else if ((c >> 4) == 14 && i + 2 < s.size()) {
      cp = ((c & 0x0f) << 12) | ((s[i + 1] & 0x3f) << 6) | (s[i + 2] & 0x3f); len = 3;
    } else if ((c >> 3) == 30 && i + 3 < s.size()) {
      cp = ((c & 0x07) << 18) | ((s[i + 1] & 0x3f) << 12) | ((s[i + 2] & 0x3f) << 6) | (s[i + 3] & 0x3f); len = 4;
    } else throw std::runtime_error("JSON: invalid UTF-8 in string");
    i += len;
    char buf[16];
    switch (cp) {
      case '"': out += "\\\""; continue;
      case '\\': out += "\\\\"; continue;
      case '\n': out += "\\n"; continue;
      case '\r': out += "\\r"; continue;
      case '\t': out += "\\t"; continue;
      case '\b': out += "\\b"; continue;
      case '\f': out += "\\f"; continue;
      default: break;
    }
    if (cp < 0x20 || cp > 0x7e) {
      if (cp == 0x7f) { out += char(cp); continue; }
      if (cp >= 0x10000) {
        uint32_t v = cp - 0x10000;
        snprintf(buf, sizeof(buf), "\\u%04x\\u%04x", 0xd800 + (v >> 10), 0xdc00 + (v & 0x3ff));
      } else {
        snprintf(buf, sizeof(buf), "\\u%04x", cp);
      }
      out += buf;
    } else {
      out += char(cp);
    }
  }
  out += '"';
}

void Json::dump(std::string &out, int indent, int level) const {
  switch (t_) {
    case Null: out += "null"; return;
    case Bool: out += b_ ? "true" : "false"; return;
    case Int: out += std::to_string(i_); return;
    case Float: out += python_float_repr(f_); return;
    case String: dump_string(out, s_); return;
    case Array: {
      if (a_.empty()) { out += "[]"; return; }
      out += '[';
      for (size_t i = 0; i < a_.size(); ++i) {
        if (i) out += ',';
        if (indent) { out += '\n'; out += std::string(size_t(indent * (level + 1)), ' '); }
        a_[i].dump(out, indent, level + 1);
      }
      if (indent) { out += '\n'; out += std::string(size_t(indent * level), ' '); }
      out += ']';
      return;
    }
    case Object: {
      if (o_.empty()) { out += "{}"; return; }
      out += '{';
      bool first = true;
      for (auto &kv : o_) {
        if (!first) out += ',';
        first = false;
        if (indent) { out += '\n'; out += std::string(size_t(indent * (level + 1)), ' '); }
        dump_string(out, kv.first);
        out += indent ? ": " : ":";
        kv.second.dump(out, indent, level + 1);
      }
      if (indent) { out += '\n'; out += std::string(size_t(indent * level), ' '); }
      out += '}';
      return;
    }
  }
}

std::string Json::dump_compact() const {
  std::string s;
  dump(s, 0, 0);
  return s;
}
std::string Json::dump_indent2() const {
  std::string s;
  dump(s, 2, 0);
  return s;
}

namespace {
struct Parser {
  const std::string &t;
  size_t i = 0;
  explicit Parser(const std::string &text) : t(text) {}
  [[noreturn]] void fail(const char *m) {
    throw std::runtime_error(std::string("JSON parse error at byte ") + std::to_string(i) + ": " + m);
  }
  void ws() {
    while (i < t.size() && (t[i] == ' ' || t[i] == '\n' || t[i] == '\r' || t[i] == '\t')) ++i;
  }
  bool lit(const char *s) {
    size_t n = strlen(s);
    if (t.compare(i, n, s) == 0) { i += n; return true; }
    return false;
  }
  uint32_t hex4() {
    if (i + 4 > t.size()) fail("short \\u escape");
    uint32_t v = 0;
    for (int k = 0; k < 4; ++k) {
      char c = t[i++];
      v <<= 4;
      if (c >= '0' && c <= '9') v |= uint32_t(c - '0');
      else if (c >= 'a' && c <= 'f') v |= uint32_t(c - 'a' + 10);
      else if (c >= 'A' && c <= 'F') v |= uint32_t(c - 'A' + 10);
      else fail("bad \\u escape");
    }
    return v;
  }
  static void utf8(std::string &o, uint32_t cp) {
    if (cp < 0x80) o += char(cp);
    else if (cp < 0x800) { o += char(0xc0 | (cp >> 6)); o += char(0x80 | (cp & 0x3f)); }
    else if (cp < 0x10000) {
      o += char(0xe0 | (cp >> 12)); o += char(0x80 | ((cp >> 6) & 0x3f)); o += char(0x80 | (cp & 0x3f));
    } else {
      o += char(0xf0 | (cp >> 18)); o += char(0x80 | ((cp >> 12) & 0x3f));
      o += char(0x80 | ((cp >> 6) & 0x3f)); o += char(0x80 | (cp & 0x3f));
    }
  }
  std::string str() {
    if (t[i] != '"') fail("expected a string");
    ++i;
    std::string o;
    while (true) {
      if (i >= t.size()) fail("unterminated string");
      char c = t[i++];
      if (c == '"') break;
      if ((unsigned char)c < 0x20) fail("control character in string");
      if (c != '\\') { o += c; continue; }
      if (i >= t.size()) fail("bad escape");
      char e = t[i++];
      switch (e) {
        case '"': o += '"'; break;
        case '\\': o += '\\'; break;
        case '/': o += '/'; break;
        case 'b': o += '\b'; break;
        case 'f': o += '\f'; break;
        case 'n': o += '\n'; break;
        case 'r': o += '\r'; break;
        case 't': o += '\t'; break;
        case 'u': {
          uint32_t cp = hex4();
          if (cp >= 0xd800 && cp < 0xdc00 && i + 1 < t.size() && t[i] == '\\' && t[i + 1] == 'u') {
            i += 2;
            uint32_t lo = hex4();
            if (lo < 0xdc00 || lo > 0xdfff) fail("bad surrogate pair");
            cp = 0x10000 + ((cp - 0xd800) << 10) + (lo - 0xdc00);
          }
          utf8(o, cp);
          break;
        }
        default: fail("bad escape");
      }
    }
    return o;
  }
  Json num() {
    size_t s = i;
    if (t[i] == '-') ++i;
    if (i >= t.size() || !isdigit((unsigned char)t[i])) fail("bad number");
    if (t[i] == '0') ++i;
    else while (i < t.size() && isdigit((unsigned char)t[i])) ++i;
    bool is_float = false;
    if (i < t.size() && t[i] == '.') {
      is_float = true;
      ++i;
      if (i >= t.size() || !isdigit((unsigned char)t[i])) fail("bad fraction");
      while (i < t.size() && isdigit((unsigned char)t[i])) ++i;
    }
    if (i < t.size() && (t[i] == 'e' || t[i] == 'E')) {
      is_float = true;
      ++i;
      if (i < t.size() && (t[i] == '+' || t[i] == '-')) ++i;
      if (i >= t.size() || !isdigit((unsigned char)t[i])) fail("bad exponent");
      while (i < t.size() && isdigit((unsigned char)t[i])) ++i;
    }
    const std::string tok = t.substr(s, i - s);
    if (is_float) {
      double v = strtod(tok.c_str(), nullptr);
      if (!std::isfinite(v)) fail("float out of range");
      return Json::number(v);
    }
    int64_t v = 0;
    auto r = std::from_chars(tok.data(), tok.data() + tok.size(), v);
    if (r.ec != std::errc()) fail("integer out of range");
    return Json::integer(v);
  }
  Json value() {
    ws();
    if (i >= t.size()) fail("unexpected end");
    char c = t[i];
    if (c == '{') {
      ++i;
      Json o = Json::object();
      ws();
      if (i < t.size() && t[i] == '}') { ++i; return o; }
      while (true) {
        ws();
        if (i >= t.size() || t[i] != '"') fail("expected a key");
        std::string k = str();
        if (o.has(k)) fail(("duplicate JSON key: " + k).c_str());
        ws();
        if (i >= t.size() || t[i] != ':') fail("expected ':'");
        ++i;
        o.set(k, value());
        ws();
        if (i < t.size() && t[i] == ',') { ++i; continue; }
        if (i < t.size() && t[i] == '}') { ++i; return o; }
        fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      ++i;
      Json a = Json::array();
      ws();
      if (i < t.size() && t[i] == ']') { ++i; return a; }
      while (true) {
        a.push(value());
        ws();
        if (i < t.size() && t[i] == ',') { ++i; continue; }
        if (i < t.size() && t[i] == ']') { ++i; return a; }
        fail("expected ',' or ']'");
      }
    }
    if (c == '"') return Json::string(str());
    if (lit("null")) return Json::null();
    if (lit("true")) return Json::boolean(true);
    if (lit("false")) return Json::boolean(false);
    if (c == '-' || isdigit((unsigned char)c)) return num();
    fail("unexpected character (NaN and Infinity are rejected)");
  }
};
}  // namespace

Json Json::parse(const std::string &text) {
  Parser p(text);
  Json v = p.value();
  p.ws();
  if (p.i != text.size()) p.fail("trailing data");
  return v;
}

}  // namespace fdp
