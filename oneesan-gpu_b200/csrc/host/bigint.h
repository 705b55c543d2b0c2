// Unsigned arbitrary-precision integers for the exact CRT driver: CRT
// reconstruction of a few hundred bits, the checkerboard-strip path bound and
// decimal text.  Little-endian base-2^32 limbs, no leading zero limbs.
#pragma once
#include <stdint.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

namespace fdp {

class BigUint {
 public:
  BigUint() = default;
  explicit BigUint(uint64_t v) {
    while (v) {
      d_.push_back(uint32_t(v));
      v >>= 32;
    }
  }

  bool is_zero() const { return d_.empty(); }

  size_t bit_length() const {
    if (d_.empty()) return 0;
    uint32_t top = d_.back();
    size_t b = 0;
    while (top) { ++b; top >>= 1; }
    return (d_.size() - 1) * 32 + b;
  }

  static int compare(const BigUint &a, const BigUint &b) {
    if (a.d_.size() != b.d_.size()) return a.d_.size() < b.d_.size() ? -1 : 1;
    for (size_t i = a.d_.size(); i-- > 0;)
      if (a.d_[i] != b.d_[i]) return a.d_[i] < b.d_[i] ? -1 : 1;
    return 0;
  }
  friend bool operator<(const BigUint &a, const BigUint &b) { return compare(a, b) < 0; }
  friend bool operator<=(const BigUint &a, const BigUint &b) { return compare(a, b) <= 0; }
  friend bool operator>(const BigUint &a, const BigUint &b) { return compare(a, b) > 0; }
  friend bool operator==(const BigUint &a, const BigUint &b) { return compare(a, b) == 0; }
  friend bool operator!=(const BigUint &a, const BigUint &b) { return compare(a, b) != 0; }

  friend BigUint operator+(const BigUint &a, const BigUint &b) {
    BigUint r;
    const size_t n = std::max(a.d_.size(), b.d_.size());
    r.d_.resize(n + 1, 0);
    uint64_t carry = 0;
    for (size_t i = 0; i < n; ++i) {
      uint64_t s = carry + (i < a.d_.size() ? a.d_[i] : 0) + (i < b.d_.size() ? b.d_[i] : 0);
      r.d_[i] = uint32_t(s);
      carry = s >> 32;
    }
    r.d_[n] = uint32_t(carry);
    r.trim();
    return r;
  }

  friend BigUint operator*(const BigUint &a, const BigUint &b) {
    if (a.is_zero() || b.is_zero()) return BigUint();
    BigUint r;
    r.d_.assign(a.d_.size() + b.d_.size(), 0);
    for (size_t i = 0; i < a.d_.size(); ++i) {
      uint64_t carry = 0;
      for (size_t j = 0; j < b.d_.size(); ++j) {
        uint64_t t = uint64_t(a.d_[i]) * b.d_[j] + r.d_[i + j] + carry;
        r.d_[i + j] = uint32_t(t);
        carry = t >> 32;
      }
      size_t k = i + b.d_.size();
      while (carry) {
        uint64_t t = uint64_t(r.d_[k]) + carry;
        r.d_[k] = uint32_t(t);
        carry = t >> 32;
        ++k;
      }
    }
    r.trim();
    return r;
  }

  // Remainder and in-place quotient by a nonzero 32-bit divisor.
  uint32_t mod_u32(uint32_t m) const {
    if (!m) throw std::invalid_argument("division by zero");
    uint64_t rem = 0;
    for (size_t i = d_.size(); i-- > 0;) rem = ((rem << 32) | d_[i]) % m;
    return uint32_t(rem);
  }
  uint32_t divmod_u32(uint32_t m) {
    if (!m) throw std::invalid_argument("division by zero");
    uint64_t rem = 0;
    for (size_t i = d_.size(); i-- > 0;) {
      uint64_t cur = (rem << 32) | d_[i];
      d_[i] = uint32_t(cur / m);
      rem = cur % m;
    }
    trim();
    return uint32_t(rem);
  }

  std::string to_decimal() const {
    if (is_zero()) return "0";
    BigUint t = *this;
    std::vector<uint32_t> chunks;  // base 1e9, least significant first
    while (!t.is_zero()) chunks.push_back(t.divmod_u32(1000000000u));
    std::string s = std::to_string(chunks.back());
    char buf[16];
    for (size_t i = chunks.size() - 1; i-- > 0;) {
      snprintf(buf, sizeof(buf), "%09u", chunks[i]);
      s += buf;
    }
    return s;
  }

  static BigUint from_decimal(const std::string &s) {
    if (s.empty()) throw std::invalid_argument("empty decimal");
    BigUint r;
    for (char c : s) {
      if (c < '0' || c > '9') throw std::invalid_argument("non-decimal digit");
      r = r * BigUint(10) + BigUint(uint64_t(c - '0'));
    }
    return r;
  }

 private:
  void trim() {
    while (!d_.empty() && d_.back() == 0) d_.pop_back();
  }
  std::vector<uint32_t> d_;
};

}  // namespace fdp
