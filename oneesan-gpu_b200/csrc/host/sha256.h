// SHA-256 (FIPS 180-4) for checkpoint and result-manifest integrity digests.
#pragma once
#include <stdint.h>

#include <string>

namespace fdp {

class Sha256 {
 public:
  Sha256();
  void update(const void *data, size_t len);
  std::string hex_digest();  // finalises; 64 lowercase hex characters

 private:
  void block(const uint8_t *p);
  uint32_t h_[8];
  uint8_t buf_[64];
  size_t buf_len_ = 0;
  uint64_t total_ = 0;
};

std::string sha256_hex(const std::string &data);
// Digest of a whole file; throws std::runtime_error if it cannot be read.
std::string sha256_file(const std::string &path);

}  // namespace fdp
