// Exact-count machinery of the CRT driver: the CRT prime table, the rigorous
// checkerboard-strip path bound, CRT reconstruction, checkpoint V4 and the
// ONEESAN_EXACT_RESULT_V4 manifest.  Restates scripts/solve/path_bound.py,
// scripts/solve/solve_b300_exact.py:30-32 and scripts/solve/exact_safety.py of
// the reference with the same file formats.
#pragma once
#include <stdint.h>

#include <map>
#include <optional>
#include <string>
#include <vector>

#include "bigint.h"

namespace fdp {

// The `count` largest primes below 2^32, descending (path_bound.py:5-18 lists
// the first 48 of this sequence).
std::vector<uint32_t> crt_primes(int count);
bool is_prime_u32(uint32_t x);

// Rigorous checkerboard-strip upper bound on corner-to-corner simple paths of
// the n x n grid and the strip partition that attains it (path_bound.py:53-117).
BigUint checkerboard_strip_count(int height, int width);
BigUint simple_path_upper_bound(int n, std::vector<int> *partition, int max_strip_height = 9);
// Shortest prefix of crt_primes(48) whose product exceeds `bound`; throws if
// the 48 primes are not enough (path_bound.py:110-121).
std::vector<uint32_t> primes_for_bound(const BigUint &bound);

// One CRT step: x mod m combined with r mod p (solve_b300_exact.py:30-32).
void crt_step(BigUint &x, BigUint &m, uint32_t r, uint32_t p);

struct ResidueRecord {
  uint32_t residue = 0;
  bool has_wall = false;
  double wall_s = 0;
  bool has_log = false;
  std::string log;
};

struct SolverIdentity {
  std::string binary_name, binary_sha256, git_commit;
};

constexpr int kCheckpointFormat = 4;

// Load a V4 checkpoint: strict fields, SHA-256 integrity, same n and same
// solver binary digest (exact_safety.py:227-311).  A missing file is empty.
std::map<uint32_t, ResidueRecord> load_checkpoint(const std::string &path, int n, const SolverIdentity &id);
// Write a V4 checkpoint durably: temp file, fsync, rename, fsync directory
// (exact_safety.py:313-360).
void save_checkpoint(const std::string &path, int n, const SolverIdentity &id,
                     const std::map<uint32_t, ResidueRecord> &residues);
std::string checkpoint_payload_digest(const std::string &file_text);

// Exclusive non-blocking lock on <work>/.solve.lock; returns the fd (kept open
// for the process lifetime) or throws if another driver holds it.
int acquire_workdir_lock(const std::string &work);

// Checks of exact_safety.py:362-383.
void validate_exact_reconstruction(const BigUint &x, const BigUint &product, const BigUint &bound,
                                   const std::vector<std::pair<uint32_t, uint32_t>> &used);

// exact_manifest.json (ONEESAN_EXACT_RESULT_V4) then exact.txt, both durable
// (exact_safety.py:395-530, without build-provenance or admission files).
void write_exact_result(const std::string &work, int n, const BigUint &exact, const BigUint &bound,
                        const BigUint &product, const std::vector<uint32_t> &used,
                        const std::map<uint32_t, ResidueRecord> &residues, const SolverIdentity &id,
                        const std::string &checkpoint_path, double total_wall_s,
                        const std::vector<int> &strip_partition, std::string *exact_path,
                        std::string *manifest_path);

void durable_atomic_write(const std::string &path, const std::string &text);

}  // namespace fdp
