// Minimal strict JSON for checkpoint V4 and the exact-result manifest.
//
// Serialisation reproduces Python's json.dumps(..., sort_keys=True,
// ensure_ascii=True) byte for byte, both the compact form
// (separators=(",", ":")) used for integrity digests and the indent=2 form used
// for files, so checkpoints written here verify under the reference runner
// (scripts/solve/exact_safety.py:146-165, 339-360) and vice versa.  Parsing is
// strict like exact_safety.py:167-186: duplicate keys, NaN/Infinity and
// trailing data are errors.
#pragma once
#include <stdint.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace fdp {

class Json {
 public:
  enum Type { Null, Bool, Int, Float, String, Array, Object };

  Json() : t_(Null) {}
  static Json null() { return Json(); }
  static Json boolean(bool b) { Json j; j.t_ = Bool; j.b_ = b; return j; }
  static Json integer(int64_t v) { Json j; j.t_ = Int; j.i_ = v; return j; }
  static Json number(double v) { Json j; j.t_ = Float; j.f_ = v; return j; }
  static Json string(const std::string &s) { Json j; j.t_ = String; j.s_ = s; return j; }
  static Json array() { Json j; j.t_ = Array; return j; }
  static Json object() { Json j; j.t_ = Object; return j; }

  Type type() const { return t_; }
  bool is(Type t) const { return t_ == t; }
  bool as_bool() const;
  int64_t as_int() const;
  double as_number() const;  // Int or Float
  const std::string &as_string() const;
  const std::vector<Json> &items() const;
  const std::map<std::string, Json> &fields() const;

  Json &push(const Json &v);                          // Array
  Json &set(const std::string &k, const Json &v);     // Object
  bool has(const std::string &k) const;
  const Json &at(const std::string &k) const;

  // Python-compatible text.
  std::string dump_compact() const;   // sort_keys, separators=(",", ":")
  std::string dump_indent2() const;   // sort_keys, indent=2

  static Json parse(const std::string &text);  // throws std::runtime_error

 private:
  void dump(std::string &out, int indent, int level) const;
  Type t_;
  bool b_ = false;
  int64_t i_ = 0;
  double f_ = 0;
  std::string s_;
  std::vector<Json> a_;
  std::map<std::string, Json> o_;
};

// Python repr() of a finite double.
std::string python_float_repr(double v);

}  // namespace fdp
