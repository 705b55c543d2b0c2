#include "exact.h"

#include <errno.h>
#include <fcntl.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <sys/file.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <fstream>
#include <set>
#include <sstream>
#include <stdexcept>

#include "json.h"
#include "sha256.h"

namespace fdp {

// ---- primes -------------------------------------------------------------------
static uint64_t mulmod64(uint64_t a, uint64_t b, uint64_t m) { return (unsigned __int128)a * b % m; }
static uint64_t powmod64(uint64_t a, uint64_t e, uint64_t m) {
  uint64_t r = 1;
  a %= m;
  while (e) {
    if (e & 1) r = mulmod64(r, a, m);
    a = mulmod64(a, a, m);
    e >>= 1;
  }
  return r;
}

// Deterministic Miller-Rabin: bases 2, 7, 61 decide every n < 4,759,123,141.
bool is_prime_u32(uint32_t n) {
  if (n < 2) return false;
  for (uint32_t q : {2u, 3u, 5u, 7u, 11u, 13u, 61u})
    if (n % q == 0) return n == q;
  uint64_t d = n - 1;
  int s = 0;
  while (!(d & 1)) { d >>= 1; ++s; }
  for (uint64_t a : {2ull, 7ull, 61ull}) {
    uint64_t x = powmod64(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool comp = true;
    for (int i = 1; i < s; ++i) {
      x = mulmod64(x, x, n);
      if (x == n - 1) { comp = false; break; }
    }
    if (comp) return false;
  }
  return true;
}

std::vector<uint32_t> crt_primes(int count) {
  std::vector<uint32_t> out;
  for (uint64_t x = 0xffffffffull; out.size() < size_t(count) && x > 1; --x)
    if (is_prime_u32(uint32_t(x))) out.push_back(uint32_t(x));
  return out;
}

// ---- checkerboard-strip bound ---------------------------------------------------
// Two adjacent columns of `height` face bits are compatible unless some 2x2
// window is a checkerboard (path_bound.py:21-30).
static bool strip_compatible(uint32_t x, uint32_t y, int height) {
  for (int r = 0; r + 1 < height; ++r) {
    const uint32_t a = (x >> r) & 1, b = (x >> (r + 1)) & 1, c = (y >> r) & 1, d = (y >> (r + 1)) & 1;
    if (a != b && c != d && a != c) return false;
  }
  return true;
}

BigUint checkerboard_strip_count(int height, int width) {
  const uint32_t states = 1u << height, mask = states - 1;
  // Orbits under bit complement and vertical reflection (path_bound.py:33-50).
  std::vector<int> orbit_of(states, -1);
  std::vector<uint32_t> reps;
  std::vector<int> sizes;
  for (uint32_t x = 0; x < states; ++x) {
    if (orbit_of[x] >= 0) continue;
    uint32_t refl = 0;
    for (int b = 0; b < height; ++b)
      if ((x >> b) & 1) refl |= 1u << (height - 1 - b);
    std::set<uint32_t> orb = {x, x ^ mask, refl, refl ^ mask};
    const int idx = int(reps.size());
    reps.push_back(x);
    sizes.push_back(int(orb.size()));
    for (uint32_t y : orb) orbit_of[y] = idx;
  }
  // Edge weights: compatible members of each destination orbit.
  std::vector<std::vector<std::pair<int, uint64_t>>> nxt(reps.size());
  for (size_t i = 0; i < reps.size(); ++i) {
    std::map<int, uint64_t> w;
    for (uint32_t y = 0; y < states; ++y)
      if (strip_compatible(reps[i], y, height)) w[orbit_of[y]] += 1;
    for (auto &kv : w) nxt[i].push_back(kv);
  }
  std::vector<BigUint> dp(reps.size(), BigUint(1));
  for (int step = 1; step < width; ++step) {
    std::vector<BigUint> nd(reps.size());
    for (size_t i = 0; i < reps.size(); ++i) {
      BigUint s;
      for (auto &ow : nxt[i]) s = s + dp[size_t(ow.first)] * BigUint(ow.second);
      nd[i] = s;
    }
    dp.swap(nd);
  }
  BigUint total;
  for (size_t i = 0; i < reps.size(); ++i) total = total + dp[i] * BigUint(uint64_t(sizes[i]));
  return total;
}

BigUint simple_path_upper_bound(int n, std::vector<int> *partition, int max_strip_height) {
  if (partition) partition->clear();
  if (n < 1) return BigUint(1);
  const int hmax = std::min(max_strip_height, n);
  std::vector<BigUint> strip(size_t(hmax) + 1);
  for (int h = 1; h <= hmax; ++h) strip[size_t(h)] = checkerboard_strip_count(h, n);
  std::vector<bool> have(size_t(n) + 1, false);
  std::vector<BigUint> best(size_t(n) + 1);
  std::vector<std::vector<int>> parts(size_t(n) + 1);
  have[0] = true;
  best[0] = BigUint(1);
  for (int rows = 1; rows <= n; ++rows)
    for (int h = 1; h <= hmax; ++h) {
      if (h > rows || !have[size_t(rows - h)]) continue;
      BigUint cand = best[size_t(rows - h)] * strip[size_t(h)];
      if (!have[size_t(rows)] || cand < best[size_t(rows)]) {
        best[size_t(rows)] = cand;
        have[size_t(rows)] = true;
        parts[size_t(rows)] = parts[size_t(rows - h)];
        parts[size_t(rows)].push_back(h);
      }
    }
  if (partition) *partition = parts[size_t(n)];
  return best[size_t(n)];
}

std::vector<uint32_t> primes_for_bound(const BigUint &bound) {
  BigUint product(1);
  std::vector<uint32_t> out;
  for (uint32_t p : crt_primes(48)) {
    out.push_back(p);
    product = product * BigUint(p);
    if (product > bound) return out;
  }
  throw std::runtime_error("CRT prime capacity insufficient: product has " + std::to_string(product.bit_length()) +
                           " bits, bound has " + std::to_string(bound.bit_length()) + " bits");
}

// ---- CRT ------------------------------------------------------------------------
static uint32_t inv_mod(uint32_t a, uint32_t p) {
  int64_t t = 0, nt = 1, r = p, nr = a % p;
  while (nr) {
    int64_t q = r / nr;
    int64_t tmp = t - q * nt; t = nt; nt = tmp;
    tmp = r - q * nr; r = nr; nr = tmp;
  }
  if (r != 1) throw std::runtime_error("CRT moduli are not coprime");
  if (t < 0) t += p;
  return uint32_t(t);
}

void crt_step(BigUint &x, BigUint &m, uint32_t r, uint32_t p) {
  const uint32_t xr = x.mod_u32(p);
  const uint64_t diff = (uint64_t(r) + p - xr) % p;
  const uint64_t t = diff * inv_mod(m.mod_u32(p), p) % p;
  x = x + m * BigUint(t);
  m = m * BigUint(p);
}

// ---- durable files ------------------------------------------------------------------
static std::string dirname_of(const std::string &path) {
  const size_t s = path.rfind('/');
  return s == std::string::npos ? "." : (s == 0 ? "/" : path.substr(0, s));
}

void durable_atomic_write(const std::string &path, const std::string &text) {
  const std::string tmp = path + ".tmp";
  int fd = open(tmp.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
  if (fd < 0) throw std::runtime_error("cannot write " + tmp + ": " + strerror(errno));
  size_t off = 0;
  while (off < text.size()) {
    ssize_t w = write(fd, text.data() + off, text.size() - off);
    if (w < 0) {
      if (errno == EINTR) continue;
      close(fd);
      unlink(tmp.c_str());
      throw std::runtime_error("write failed on " + tmp);
    }
    off += size_t(w);
  }
  if (fsync(fd) != 0) {
    close(fd);
    unlink(tmp.c_str());
    throw std::runtime_error("fsync failed on " + tmp);
  }
  close(fd);
  if (rename(tmp.c_str(), path.c_str()) != 0) {
    unlink(tmp.c_str());
    throw std::runtime_error("rename failed for " + path);
  }
  int dfd = open(dirname_of(path).c_str(), O_RDONLY | O_DIRECTORY);
  if (dfd >= 0) {
    fsync(dfd);
    close(dfd);
  }
}

static std::string read_file(const std::string &path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot read exact checkpoint " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

static bool file_exists(const std::string &path) {
  struct stat st;
  return stat(path.c_str(), &st) == 0;
}

static bool is_hex64(const std::string &s) {
  if (s.size() != 64) return false;
  for (char c : s)
    if (!((c >= '0' && c <= '9') || (c >= 'a' && c <= 'f'))) return false;
  return true;
}

// ---- checkpoint V4 ---------------------------------------------------------------------
static Json identity_json(const SolverIdentity &id) {
  Json s = Json::object();
  s.set("binary_name", Json::string(id.binary_name));
  s.set("binary_sha256", Json::string(id.binary_sha256));
  s.set("git_commit", Json::string(id.git_commit));
  return s;
}

static std::string digest_without(const Json &data, const char *field) {
  Json payload = Json::object();
  for (auto &kv : data.fields())
    if (kv.first != field) payload.set(kv.first, kv.second);
  return sha256_hex(payload.dump_compact());
}

std::string checkpoint_payload_digest(const std::string &file_text) {
  return digest_without(Json::parse(file_text), "checkpoint_sha256");
}

static void validate_residue(uint64_t modulus, int64_t residue, const std::string &source) {
  if (modulus < 2) throw std::runtime_error(source + ": invalid modulus " + std::to_string(modulus));
  if (residue < 0 || uint64_t(residue) >= modulus)
    throw std::runtime_error(source + ": residue " + std::to_string(residue) + " is outside canonical range [0, " +
                             std::to_string(modulus) + ")");
}

std::map<uint32_t, ResidueRecord> load_checkpoint(const std::string &path, int n, const SolverIdentity &id) {
  std::map<uint32_t, ResidueRecord> out;
  if (!file_exists(path)) return out;
  Json data;
  try {
    data = Json::parse(read_file(path));
  } catch (const std::exception &e) {
    throw std::runtime_error("malformed exact checkpoint " + path + ": " + e.what());
  }
  if (!data.is(Json::Object)) throw std::runtime_error("checkpoint " + path + ": root must be a JSON object");
  if (!data.has("format_version"))
    throw std::runtime_error("checkpoint " + path +
                             " has no compatible solver fingerprint/integrity format; move/delete the legacy "
                             "checkpoint and recompute residues");
  if (!data.at("format_version").is(Json::Int) || !data.has("n") || !data.at("n").is(Json::Int))
    throw std::runtime_error("checkpoint " + path + ": format_version and n must be JSON integers");
  if (data.at("format_version").as_int() != kCheckpointFormat)
    throw std::runtime_error("checkpoint " + path +
                             " has no compatible solver fingerprint/integrity format; move/delete the legacy "
                             "checkpoint and recompute residues");
  if (!data.has("checkpoint_sha256") || !data.at("checkpoint_sha256").is(Json::String) ||
      data.at("checkpoint_sha256").as_string().size() != 64)
    throw std::runtime_error("checkpoint " + path + " has no compatible integrity checksum");
  if (digest_without(data, "checkpoint_sha256") != data.at("checkpoint_sha256").as_string())
    throw std::runtime_error("checkpoint " + path + ": SHA-256 integrity checksum mismatch");
  if (data.at("n").as_int() != n)
    throw std::runtime_error("checkpoint " + path + " belongs to n=" + std::to_string(data.at("n").as_int()) +
                             ", expected n=" + std::to_string(n));
  const std::set<std::string> expected = {"format_version", "n", "solver", "admission_certificate", "residues",
                                          "checkpoint_sha256"};
  for (auto &kv : data.fields())
    if (!expected.count(kv.first)) throw std::runtime_error("checkpoint " + path + ": unknown field " + kv.first);
  for (auto &k : expected)
    if (!data.has(k)) throw std::runtime_error("checkpoint " + path + ": missing field " + k);
  const Json &solver = data.at("solver");
  if (!solver.is(Json::Object) || solver.fields().size() != 3 || !solver.has("binary_name") ||
      !solver.has("binary_sha256") || !solver.has("git_commit"))
    throw std::runtime_error("checkpoint " + path + ": solver identity fields mismatch");
  for (auto &kv : solver.fields())
    if (!kv.second.is(Json::String))
      throw std::runtime_error("checkpoint " + path + ": solver identity values must be strings");
  const std::string &sha = solver.at("binary_sha256").as_string();
  if (!is_hex64(sha)) throw std::runtime_error("checkpoint " + path + ": invalid solver binary SHA-256");
  if (sha != id.binary_sha256)
    throw std::runtime_error("checkpoint " + path + ": solver binary changed ('" + sha + "' != '" +
                             id.binary_sha256 + "')");
  if (!data.at("admission_certificate").is(Json::Null))
    throw std::runtime_error("checkpoint " + path + ": admission certificate changed (this driver admits none)");
  const Json &raw = data.at("residues");
  if (!raw.is(Json::Object)) throw std::runtime_error("checkpoint " + path + ": residues must be an object");
  for (auto &kv : raw.fields()) {
    const std::string &key = kv.first;
    bool digits = !key.empty();
    for (char c : key) digits = digits && c >= '0' && c <= '9';
    if (!digits || (key.size() > 1 && key[0] == '0') || key.size() > 10)
      throw std::runtime_error("checkpoint " + path + ": non-canonical modulus key '" + key + "'");
    const uint64_t modulus = std::stoull(key);
    if (modulus > 0xffffffffull) throw std::runtime_error("checkpoint " + path + ": modulus key too large");
    const Json &rec = kv.second;
    const std::string src = "checkpoint modulus " + key;
    if (!rec.is(Json::Object)) throw std::runtime_error(src + ": record must be an object");
    for (auto &f : rec.fields())
      if (f.first != "residue" && f.first != "wall_s" && f.first != "log")
        throw std::runtime_error(src + ": unknown field " + f.first);
    if (!rec.has("residue")) throw std::runtime_error(src + ": missing residue");
    if (!rec.at("residue").is(Json::Int)) throw std::runtime_error(src + ": residue must be a JSON integer");
    validate_residue(modulus, rec.at("residue").as_int(), src);
    ResidueRecord r;
    r.residue = uint32_t(rec.at("residue").as_int());
    if (rec.has("wall_s")) {
      const Json &w = rec.at("wall_s");
      if (!(w.is(Json::Int) || w.is(Json::Float))) throw std::runtime_error(src + ": wall_s must be numeric");
      const double v = w.as_number();
      if (!std::isfinite(v) || v < 0) throw std::runtime_error(src + ": wall_s must be finite and nonnegative");
      r.has_wall = true;
      r.wall_s = v;
    }
    if (rec.has("log")) {
      if (!rec.at("log").is(Json::String)) throw std::runtime_error(src + ": log must be a string");
      r.has_log = true;
      r.log = rec.at("log").as_string();
    }
    out[uint32_t(modulus)] = r;
  }
  return out;
}

void save_checkpoint(const std::string &path, int n, const SolverIdentity &id,
                     const std::map<uint32_t, ResidueRecord> &residues) {
  Json res = Json::object();
  for (auto &kv : residues) {
    validate_residue(kv.first, kv.second.residue, "checkpoint modulus " + std::to_string(kv.first));
    Json rec = Json::object();
    rec.set("residue", Json::integer(kv.second.residue));
    if (kv.second.has_wall) rec.set("wall_s", Json::number(kv.second.wall_s));
    if (kv.second.has_log) rec.set("log", Json::string(kv.second.log));
    res.set(std::to_string(kv.first), rec);
  }
  Json payload = Json::object();
  payload.set("format_version", Json::integer(kCheckpointFormat));
  payload.set("n", Json::integer(n));
  payload.set("solver", identity_json(id));
  payload.set("admission_certificate", Json::null());
  payload.set("residues", res);
  payload.set("checkpoint_sha256", Json::string(sha256_hex(payload.dump_compact())));
  durable_atomic_write(path, payload.dump_indent2() + "\n");
}

int acquire_workdir_lock(const std::string &work) {
  const std::string p = work + "/.solve.lock";
  int fd = open(p.c_str(), O_RDWR | O_CREAT | O_APPEND, 0644);
  if (fd < 0) throw std::runtime_error("cannot open " + p);
  if (flock(fd, LOCK_EX | LOCK_NB) != 0) {
    close(fd);
    throw std::runtime_error("work directory is already in use: " + work);
  }
  return fd;
}

void validate_exact_reconstruction(const BigUint &x, const BigUint &product, const BigUint &bound,
                                   const std::vector<std::pair<uint32_t, uint32_t>> &used) {
  if (product <= bound)
    throw std::runtime_error("CRT capacity insufficient: M=" + product.to_decimal() +
                             " <= path_bound=" + bound.to_decimal());
  if (x > bound)
    throw std::runtime_error("CRT reconstruction violates rigorous path bound: exact=" + x.to_decimal() +
                             ", bound=" + bound.to_decimal());
  for (auto &pr : used) {
    validate_residue(pr.first, pr.second, "final modulus " + std::to_string(pr.first));
    if (x.mod_u32(pr.first) != pr.second)
      throw std::runtime_error("CRT reconstruction failed final congruence check for modulus " +
                               std::to_string(pr.first));
  }
}

void write_exact_result(const std::string &work, int n, const BigUint &exact, const BigUint &bound,
                        const BigUint &product, const std::vector<uint32_t> &used,
                        const std::map<uint32_t, ResidueRecord> &residues, const SolverIdentity &id,
                        const std::string &checkpoint_path, double total_wall_s,
                        const std::vector<int> &strip_partition, std::string *exact_path,
                        std::string *manifest_path) {
  std::set<uint32_t> uniq(used.begin(), used.end());
  if (uniq.size() != used.size()) throw std::runtime_error("exact result contains duplicate CRT moduli");
  BigUint prod(1);
  std::vector<std::pair<uint32_t, uint32_t>> used_res;
  for (uint32_t p : used) {
    auto it = residues.find(p);
    if (it == residues.end()) throw std::runtime_error("exact result is missing residue for modulus " + std::to_string(p));
    prod = prod * BigUint(p);
    used_res.push_back({p, it->second.residue});
  }
  if (prod != product) throw std::runtime_error("CRT modulus product mismatch before finalization");
  validate_exact_reconstruction(exact, product, bound, used_res);
  if (!file_exists(checkpoint_path))
    throw std::runtime_error("cannot finalize exact result without checkpoint: " + checkpoint_path);
  if (!std::isfinite(total_wall_s) || total_wall_s < 0)
    throw std::runtime_error("total solver wall time must be finite and nonnegative");
  Json congr = Json::array();
  double wall_sum = 0;
  for (uint32_t p : used) {
    const ResidueRecord &r = residues.at(p);
    Json item = Json::object();
    item.set("modulus", Json::integer(p));
    item.set("residue", Json::integer(r.residue));
    item.set("wall_s", Json::number(r.has_wall ? r.wall_s : 0.0));
    if (r.has_log) item.set("log", Json::string(r.log));
    wall_sum += r.has_wall ? r.wall_s : 0.0;
    congr.push(item);
  }
  if (fabs(total_wall_s - wall_sum) > 1e-9 + 1e-12 * fabs(wall_sum))
    throw std::runtime_error("solver wall-time sum mismatch before finalization");
  const std::string mpath = work + "/exact_manifest.json", epath = work + "/exact.txt";
  char wall_txt[64];
  snprintf(wall_txt, sizeof(wall_txt), "%.9f", total_wall_s);
  const std::string exact_text = "n=" + std::to_string(n) + "\nexact=" + exact.to_decimal() +
                                 "\nbound_bits=" + std::to_string(bound.bit_length()) +
                                 "\nmodulus_bits=" + std::to_string(product.bit_length()) +
                                 "\nprimes_used=" + std::to_string(used.size()) +
                                 "\nsolver_wall_s_sum=" + wall_txt + "\nmanifest_file=exact_manifest.json\n";
  Json parts = Json::array();
  for (int h : strip_partition) parts.push(Json::integer(h));
  Json m = Json::object();
  m.set("format", Json::string("ONEESAN_EXACT_RESULT_V4"));
  m.set("n", Json::integer(n));
  m.set("exact_decimal", Json::string(exact.to_decimal()));
  m.set("path_bound_decimal", Json::string(bound.to_decimal()));
  m.set("bound_bits", Json::integer(int64_t(bound.bit_length())));
  m.set("bound_method", Json::string("checkerboard_strip_v1"));
  m.set("strip_partition", parts);
  m.set("modulus_product_decimal", Json::string(product.to_decimal()));
  m.set("modulus_bits", Json::integer(int64_t(product.bit_length())));
  m.set("primes_used", Json::integer(int64_t(used.size())));
  m.set("congruences", congr);
  m.set("solver", identity_json(id));
  m.set("solver_wall_s_sum", Json::number(total_wall_s));
  m.set("checkpoint_file", Json::string(checkpoint_path.substr(checkpoint_path.rfind('/') + 1)));
  m.set("checkpoint_sha256", Json::string(sha256_file(checkpoint_path)));
  m.set("exact_file", Json::string("exact.txt"));
  m.set("exact_sha256", Json::string(sha256_hex(exact_text)));
  m.set("build_provenance_file", Json::null());
  m.set("build_provenance_sha256", Json::null());
  m.set("admission_certificate_file", Json::null());
  m.set("admission_certificate_sha256", Json::null());
  m.set("admission_certificate_schema", Json::null());
  m.set("manifest_sha256", Json::string(sha256_hex(m.dump_compact())));
  // The manifest goes first; exact.txt is the completion marker.
  durable_atomic_write(mpath, m.dump_indent2() + "\n");
  durable_atomic_write(epath, exact_text);
  if (exact_path) *exact_path = epath;
  if (manifest_path) *manifest_path = mpath;
}

}  // namespace fdp
