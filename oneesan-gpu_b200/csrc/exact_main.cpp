// oneesan_exact: checkpointed exact CRT driver (the reference's
// scripts/solve/solve_b300_exact_batch.py:70-268 behaviour, in C++).
//
//   oneesan_exact n [--work-dir DIR] [--max-runs K] [--lanes L]
//                   [--binary PATH --target-mib X --max-window Y --gpus G]
//
// 1. rigorous checkerboard-strip bound -> shortest CRT prime prefix;
// 2. lock the work directory, load checkpoint V4 (strict, binary-bound);
// 3. compute the missing residues -- in process through the C ABI
//    (fdp_run_sync, `lanes` residues per pass) or, with --binary, by running a
//    solver process with the reference argv and parsing its stdout lines as
//    strictly as scripts/solve/solver_output.py;
// 4. save the checkpoint after every residue;
// 5. once the contiguous prime prefix exceeds the bound: reconstruct, check
//    bound and congruences, cross-check every drop-one subset, write
//    exact_manifest.json (ONEESAN_EXACT_RESULT_V4) and exact.txt.
// Exit codes: 0 done (or --max-runs partial), 2 partial, 1 error.
#include <dlfcn.h>
#include <errno.h>
#include <math.h>
#include <regex.h>
#include <signal.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <sys/wait.h>
#include <unistd.h>

#include <chrono>
#include <map>
#include <regex>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/oneesan_fdp.h"
#include "host/exact.h"
#include "host/sha256.h"

using namespace fdp;

namespace {

struct Args {
  int n = 0;
  std::string work, binary;
  int max_runs = 0, lanes = 0, target_mib = 16384, max_window = 14, gpus = 1;
};

[[noreturn]] void die(const std::string &m) {
  fprintf(stderr, "%s\n", m.c_str());
  exit(1);
}

Args parse_args(int argc, char **argv) {
  Args a;
  std::vector<std::string> pos;
  for (int i = 1; i < argc; ++i) {
    std::string s = argv[i];
    auto val = [&](const char *name) -> std::string {
      if (i + 1 >= argc) die(std::string("missing value for ") + name);
      return argv[++i];
    };
    if (s == "--work-dir") a.work = val("--work-dir");
    else if (s == "--max-runs") a.max_runs = atoi(val("--max-runs").c_str());
    else if (s == "--lanes") a.lanes = atoi(val("--lanes").c_str());
    else if (s == "--binary") a.binary = val("--binary");
    else if (s == "--target-mib") a.target_mib = atoi(val("--target-mib").c_str());
    else if (s == "--max-window") a.max_window = atoi(val("--max-window").c_str());
    else if (s == "--gpus") a.gpus = atoi(val("--gpus").c_str());
    else if (!s.empty() && s[0] == '-') die("unknown option " + s);
    else pos.push_back(s);
  }
  if (pos.size() != 1) die("usage: oneesan_exact n [--work-dir DIR] [--max-runs K] [--lanes L] [--binary PATH]");
  a.n = atoi(pos[0].c_str());
  if (a.n < 2 || a.n > FDP_MAX_N) die("n must be in 2..27");
  if (a.max_runs < 0) die("--max-runs must be nonnegative");
  if (a.lanes < 0 || a.lanes > FDP_MAX_LANES) die("--lanes must be in 1..16");
  if (a.target_mib < 1) die("--target-mib must be at least 1");
  if (a.max_window < 1) die("--max-window must be at least 1");
  if (a.gpus < 0 || a.gpus > 8) die("--gpus must be in 0..8");
  if (a.work.empty()) a.work = "work/b200_exact_n" + std::to_string(a.n);
  return a;
}

void mkdirs(const std::string &path) {
  std::string cur;
  for (size_t i = 0; i <= path.size(); ++i) {
    if (i == path.size() || path[i] == '/') {
      if (!cur.empty()) mkdir(cur.c_str(), 0755);
    }
    if (i < path.size()) cur += path[i];
  }
}

std::string library_path() {
  Dl_info info{};
  if (dladdr(reinterpret_cast<void *>(&fdp_version), &info) && info.dli_fname) return info.dli_fname;
  return "";
}

std::string base_name(const std::string &p) {
  const size_t s = p.rfind('/');
  return s == std::string::npos ? p : p.substr(s + 1);
}

// Contiguous prefix reconstruction (solve_b300_exact_batch.py:30-40).
void reconstruct(const std::vector<uint32_t> &prefix, const std::map<uint32_t, ResidueRecord> &res, BigUint &x,
                 BigUint &m, double &wall, std::vector<uint32_t> *used) {
  x = BigUint();
  m = BigUint(1);
  wall = 0;
  if (used) used->clear();
  for (uint32_t p : prefix) {
    auto it = res.find(p);
    if (it == res.end()) break;
    crt_step(x, m, it->second.residue, p);
    wall += it->second.has_wall ? it->second.wall_s : 0.0;
    if (used) used->push_back(p);
  }
}

// Strict result-line parser (scripts/solve/solver_output.py:25-74).
struct Result {
  uint64_t n, residue, modulus;
  double wall;
};
bool parse_result_line(const std::string &line, Result *out) {
  static const std::regex uint_re("(?:0|[1-9][0-9]*)");
  static const std::regex float_re("(?:0|[1-9][0-9]*)(?:\\.[0-9]+)?(?:[eE][+-]?[0-9]+)?");
  const char *keys[4] = {"n", "residue", "modulus", "wall_s"};
  std::map<std::string, std::string> vals;
  size_t i = 0;
  while (i < line.size()) {
    while (i < line.size() && isspace((unsigned char)line[i])) ++i;
    size_t j = i;
    while (j < line.size() && !isspace((unsigned char)line[j])) ++j;
    const std::string tok = line.substr(i, j - i);
    i = j;
    for (const char *k : keys) {
      const std::string pre = std::string(k) + "=";
      if (tok.compare(0, pre.size(), pre) == 0) {
        if (vals.count(k)) throw std::runtime_error(std::string("duplicate solver result field: ") + k);
        vals[k] = tok.substr(pre.size());
        break;
      }
    }
  }
  if (!vals.count("residue") && !vals.count("modulus") && !vals.count("wall_s")) return false;
  for (const char *k : keys)
    if (!vals.count(k)) throw std::runtime_error(std::string("incomplete solver result fields: missing ") + k);
  for (const char *k : {"n", "residue", "modulus"})
    if (!std::regex_match(vals[k], uint_re)) throw std::runtime_error(std::string("non-canonical solver ") + k);
  if (!std::regex_match(vals["wall_s"], float_re)) throw std::runtime_error("invalid solver wall_s syntax");
  for (const char *k : {"n", "residue", "modulus"})
    if (vals[k].size() > 19) throw std::runtime_error(std::string("solver ") + k + " out of range");
  out->n = std::stoull(vals["n"]);
  out->residue = std::stoull(vals["residue"]);
  out->modulus = std::stoull(vals["modulus"]);
  out->wall = strtod(vals["wall_s"].c_str(), nullptr);
  if (out->n < 1) throw std::runtime_error("invalid solver n");
  if (out->modulus < 2) throw std::runtime_error("invalid solver modulus");
  if (!std::isfinite(out->wall) || out->wall < 0) throw std::runtime_error("solver wall_s must be finite and nonnegative");
  return true;
}

int finish(const Args &a, const BigUint &bound, const std::vector<uint32_t> &prefix,
           const std::map<uint32_t, ResidueRecord> &res, const std::vector<int> &strips, const SolverIdentity &id,
           const std::string &checkpoint) {
  BigUint x, m;
  double wall;
  std::vector<uint32_t> all;
  reconstruct(prefix, res, x, m, wall, &all);
  if (m <= bound) throw std::runtime_error("finish called before CRT capacity reached");
  std::vector<std::pair<uint32_t, uint32_t>> used_res;
  for (uint32_t p : all) used_res.push_back({p, res.at(p).residue});
  validate_exact_reconstruction(x, m, bound, used_res);
  // Moduli actually needed: the shortest prefix whose product exceeds the bound.
  std::vector<uint32_t> used;
  BigUint mm(1), xx;
  double wall_used = 0;
  for (uint32_t p : all) {
    used.push_back(p);
    crt_step(xx, mm, res.at(p).residue, p);
    wall_used += res.at(p).has_wall ? res.at(p).wall_s : 0.0;
    if (mm > bound) break;
  }
  // Cross-check: every subset that drops one modulus reconstructs the same
  // integer whenever its product still exceeds it.
  int checked = 0, agree = 0;
  for (size_t drop = 0; drop < used.size(); ++drop) {
    BigUint sx, sm(1);
    for (size_t k = 0; k < used.size(); ++k)
      if (k != drop) crt_step(sx, sm, res.at(used[k]).residue, used[k]);
    if (sm <= xx) continue;
    ++checked;
    if (sx == xx) ++agree;
    else throw std::runtime_error("CRT cross-check failed when dropping modulus " + std::to_string(used[drop]));
  }
  fprintf(stderr, "crt cross-check: %d of %d drop-one subsets reconstruct the same integer\n", agree, checked);
  std::string epath, mpath;
  write_exact_result(a.work, a.n, xx, bound, mm, used, res, id, checkpoint, wall_used, strips, &epath, &mpath);
  printf("n=%d\nexact=%s\nbound_bits=%zu\nmodulus_bits=%zu\nprimes_used=%zu\nsolver_wall_s_sum=%.9f\n", a.n,
         xx.to_decimal().c_str(), bound.bit_length(), mm.bit_length(), used.size(), wall_used);
  printf("result_file=%s\nmanifest_file=%s\n", epath.c_str(), mpath.c_str());
  fflush(stdout);
  return 0;
}

void run_in_process(const Args &a, const std::vector<uint32_t> &missing, std::map<uint32_t, ResidueRecord> &res,
                    const std::string &checkpoint, const SolverIdentity &id) {
  fdp_ctx *ctx = nullptr;
  fdp_status s = fdp_create(&ctx, 0);
  if (s != FDP_OK) throw std::runtime_error(std::string("fdp_create: ") + fdp_last_error());
  const int lanes = a.lanes ? a.lanes : (int(missing.size()) < FDP_MAX_LANES ? int(missing.size()) : FDP_MAX_LANES);
  for (size_t done = 0; done < missing.size(); done += size_t(lanes)) {
    const int L = int(missing.size() - done) < lanes ? int(missing.size() - done) : lanes;
    fdp_problem pr{a.n, L, missing.data() + done, L};
    std::vector<uint32_t> out(static_cast<size_t>(L), 0u);
    fdp_run_stats st{};
    auto t0 = std::chrono::steady_clock::now();
    s = fdp_run_sync(ctx, &pr, out.data(), &st);
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (s != FDP_OK) {
      std::string err = fdp_last_error();
      fdp_destroy(ctx);
      throw std::runtime_error("fdp_run_sync failed (status " + std::to_string(int(s)) + "): " + err);
    }
    for (int i = 0; i < L; ++i) {
      const uint32_t p = missing[done + size_t(i)];
      ResidueRecord r;
      r.residue = out[size_t(i)];
      r.has_wall = true;
      r.wall_s = wall / L;
      res[p] = r;
      save_checkpoint(checkpoint, a.n, id, res);
      printf("backend=b200-fdp-pull n=%d residue=%u modulus=%u lanes=%d batch_device_s=%.6f wall_s=%.6f\n", a.n,
             r.residue, p, L, st.device_s, r.wall_s);
      fflush(stdout);
    }
  }
  fdp_destroy(ctx);
}

void run_binary(const Args &a, const std::vector<uint32_t> &missing, std::map<uint32_t, ResidueRecord> &res,
                const std::string &checkpoint, const SolverIdentity &id) {
  std::vector<std::string> argv_s = {a.binary, std::to_string(a.n), std::to_string(a.target_mib),
                                     std::to_string(a.max_window), std::to_string(a.gpus)};
  for (uint32_t p : missing) argv_s.push_back(std::to_string(p));
  std::vector<char *> argv_c;
  for (auto &s : argv_s) argv_c.push_back(const_cast<char *>(s.c_str()));
  argv_c.push_back(nullptr);
  int fds[2];
  if (pipe(fds) != 0) throw std::runtime_error("pipe failed");
  fflush(stdout);
  pid_t pid = fork();
  if (pid < 0) throw std::runtime_error("fork failed");
  if (pid == 0) {
    dup2(fds[1], 1);
    close(fds[0]);
    close(fds[1]);
    execv(a.binary.c_str(), argv_c.data());
    _exit(127);
  }
  close(fds[1]);
  FILE *in = fdopen(fds[0], "r");
  std::set<uint32_t> want(missing.begin(), missing.end()), seen;
  auto fail = [&](const std::string &m) {
    kill(pid, SIGTERM);
    fclose(in);
    waitpid(pid, nullptr, 0);
    throw std::runtime_error(m);
  };
  char *buf = nullptr;
  size_t cap = 0;
  ssize_t len;
  while ((len = getline(&buf, &cap, in)) > 0) {
    std::string line(buf, size_t(len));
    fputs(line.c_str(), stdout);
    fflush(stdout);
    Result r;
    bool is_result = false;
    try {
      is_result = parse_result_line(line, &r);
    } catch (const std::exception &e) {
      free(buf);
      fail(std::string("invalid batch solver result line: ") + e.what());
    }
    if (!is_result) continue;
    if (r.n != uint64_t(a.n)) { free(buf); fail("batch binary returned n=" + std::to_string(r.n) + ", expected n=" + std::to_string(a.n)); }
    if (r.modulus > 0xffffffffull || !want.count(uint32_t(r.modulus))) { free(buf); fail("batch binary returned unexpected modulus " + std::to_string(r.modulus)); }
    if (seen.count(uint32_t(r.modulus))) { free(buf); fail("batch binary returned duplicate modulus " + std::to_string(r.modulus)); }
    if (r.residue >= r.modulus) { free(buf); fail("batch solver modulus " + std::to_string(r.modulus) + ": residue outside canonical range"); }
    ResidueRecord rec;
    rec.residue = uint32_t(r.residue);
    rec.has_wall = true;
    rec.wall_s = r.wall;
    res[uint32_t(r.modulus)] = rec;
    seen.insert(uint32_t(r.modulus));
    save_checkpoint(checkpoint, a.n, id, res);
  }
  free(buf);
  fclose(in);
  int status = 0;
  waitpid(pid, &status, 0);
  const int rc = WIFEXITED(status) ? WEXITSTATUS(status) : 128 + (WIFSIGNALED(status) ? WTERMSIG(status) : 0);
  if (rc != 0)
    throw std::runtime_error("batch solver failed, rc=" + std::to_string(rc) + "; completed this invocation=" +
                             std::to_string(seen.size()) + "/" + std::to_string(missing.size()));
  if (seen.size() != want.size()) throw std::runtime_error("batch solver exited without all residues");
}

}  // namespace

int main(int argc, char **argv) {
  Args a = parse_args(argc, argv);
  try {
    std::vector<int> strips;
    const BigUint bound = simple_path_upper_bound(a.n, &strips);
    const std::vector<uint32_t> prefix = primes_for_bound(bound);
    std::string sp;
    for (size_t i = 0; i < strips.size(); ++i) sp += (i ? ", " : "") + std::to_string(strips[i]);
    fprintf(stderr, "rigorous path bound: <=%s (%zu bits), strips=[%s], CRT primes=%zu\n", bound.to_decimal().c_str(),
            bound.bit_length(), sp.c_str(), prefix.size());
    SolverIdentity id;
    const std::string solver = a.binary.empty() ? library_path() : a.binary;
    if (solver.empty()) throw std::runtime_error("cannot locate the solver library");
    id.binary_name = base_name(solver);
    id.binary_sha256 = sha256_file(solver);
    id.git_commit = "unknown";
    fprintf(stderr, "solver fingerprint: sha256=%s\n", id.binary_sha256.c_str());
    mkdirs(a.work);
    acquire_workdir_lock(a.work);  // held until exit
    const std::string checkpoint = a.work + "/checkpoint.json";
    std::map<uint32_t, ResidueRecord> res = load_checkpoint(checkpoint, a.n, id);
    std::set<uint32_t> pref(prefix.begin(), prefix.end());
    for (auto &kv : res)
      if (!pref.count(kv.first)) throw std::runtime_error("checkpoint contains unexpected modulus " + std::to_string(kv.first));
    BigUint x, m;
    double wall;
    reconstruct(prefix, res, x, m, wall, nullptr);
    if (m > bound) return finish(a, bound, prefix, res, strips, id, checkpoint);
    std::vector<uint32_t> missing;
    for (uint32_t p : prefix)
      if (!res.count(p)) missing.push_back(p);
    if (a.max_runs && missing.size() > size_t(a.max_runs)) missing.resize(size_t(a.max_runs));
    if (missing.empty()) {
      fprintf(stderr, "partial: CRT bits=%zu bound_bits=%zu\n", m.bit_length(), bound.bit_length());
      return a.max_runs ? 0 : 2;
    }
    fprintf(stderr, "batch run: %zu residue(s), first=%u, last=%u\n", missing.size(), missing.front(), missing.back());
    if (a.binary.empty()) run_in_process(a, missing, res, checkpoint, id);
    else run_binary(a, missing, res, checkpoint, id);
    reconstruct(prefix, res, x, m, wall, nullptr);
    if (m > bound) return finish(a, bound, prefix, res, strips, id, checkpoint);
    fprintf(stderr, "partial: CRT bits=%zu bound_bits=%zu; cached=%zu\n", m.bit_length(), bound.bit_length(), res.size());
    return a.max_runs ? 0 : 2;
  } catch (const std::exception &e) {
    fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}
