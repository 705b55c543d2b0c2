// oneesan_solver: the reference solver's process contract on top of libfdp.
//
//   oneesan_solver n target_mib max_window gpus mod1 [mod2 ...]
//
// Argument positions follow GB.cu:2090-2101 (pinned by
// tests/test_solver_contract.py:21-33 of the reference); target_mib and
// max_window are accepted for compatibility (this engine needs no scratch
// arena and no window limit).  One stdout line per modulus, in argument order,
// with the tokens n= residue= modulus= ... wall_s= in that order (GB.cu:2257),
// parsable by scripts/solve/solver_output.py:25-74.  Exit codes: 1 bad
// arguments or CUDA error, 2 GPU count, 5 HBM (GB.cu:2098-2184).
//
// Environment:
//   FDP_LANES=k         residues per pass (1 = plain, default min(#moduli,16))
//   FDP_AUTOTUNE=1      pick residues per pass, panel strategy and CTA size with
//                       fdp_autotune before solving (FDP_LANES caps the lanes)
//   GRIDFP_PLAN_ONLY=1  print PLAN lines and exit 0 without touching a GPU
//                       (GB.cu:2117-2168)
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <string>
#include <vector>

#include "../../include/oneesan_fdp.h"

static int exit_code(fdp_status s) {
  switch (s) {
    case FDP_OK: return 0;
    case FDP_ERR_GPU_COUNT: return 2;
    case FDP_ERR_HBM: return 5;
    case FDP_ERR_WINDOW: return 4;
    default: return 1;
  }
}

int main(int argc, char **argv) {
  int n = argc > 1 ? atoi(argv[1]) : 16;
  int target_mib = argc > 2 ? atoi(argv[2]) : 16384;
  int max_window = argc > 3 ? atoi(argv[3]) : 14;
  int requested = argc > 4 ? atoi(argv[4]) : 0;
  std::vector<uint32_t> mods;
  for (int i = 5; i < argc; ++i) {
    char *end = nullptr;
    unsigned long long raw = strtoull(argv[i], &end, 10);
    if (!end || *end || raw < 2 || raw > 0xffffffffull) {
      fprintf(stderr, "modulus must be in [2, 4294967295], got %s\n", argv[i]);
      return 1;
    }
    mods.push_back(uint32_t(raw));
  }
  if (mods.empty()) mods.push_back(4294967291u);
  if (n < 1 || n > FDP_MAX_N) {
    fprintf(stderr, "n=1..%d\n", FDP_MAX_N);
    return 1;
  }
  int lanes = int(mods.size()) < FDP_MAX_LANES ? int(mods.size()) : FDP_MAX_LANES;
  if (const char *e = getenv("FDP_LANES")) {
    int v = atoi(e);
    if (v < 1 || v > FDP_MAX_LANES) {
      fprintf(stderr, "FDP_LANES must be 1..%d\n", FDP_MAX_LANES);
      return 1;
    }
    lanes = v;
  }
  fdp_problem pr{n, int(mods.size()), mods.data(), lanes};
  fdp_plan_out plan{};
  fdp_status s = fdp_plan(&pr, ~0ull, &plan);
  if (s != FDP_OK) {
    fprintf(stderr, "plan: %s\n", fdp_last_error());
    return exit_code(s);
  }
  if (const char *e = getenv("GRIDFP_PLAN_ONLY"); e && atoi(e) != 0) {
    // One `PLAN n=` line of key=value tokens, the memory plan the reference's
    // autotuner reads (scripts/run/autotune.py:189-200): it requires exactly
    // one such line with n= and gpus= equal to its request, and admits a
    // configuration when scratch_fits=1 and max(dp_peak_gib, row6_peak_gib)
    // plus its reserve fits every device's free memory.  This engine runs on
    // one GPU: a request for more is planned as not fitting.
    const int gpus = requested > 0 ? requested : 1;
    const double gib = double(1ull << 30);
    fprintf(stderr,
            "PLAN n=%d W=%d gpus=%d main=%llu blocked=%llu auth_gib=%.6f lanes=%d passes=%d index_bits=%d "
            "init_rows=%d state_gib=%.6f scratch_gib=0 table_mib=%.3f total_gib=%.6f dp_peak_gib=%.6f "
            "row6_peak_gib=%.6f rows=%d cells_per_row=%d alg_bytes_per_residue=%llu transitions_per_residue=%llu "
            "scratch_limit_mib=%d max_window=%d scratch_fits=%d\n",
            n, plan.width, gpus, (unsigned long long)plan.main_states, (unsigned long long)plan.blocked_states,
            double(plan.main_states + plan.blocked_states) * 4.0 / gib, plan.lanes, plan.passes, plan.index_bits,
            plan.init_rows, double(plan.state_bytes) / gib, double(plan.table_bytes) / (1 << 20),
            double(plan.total_bytes) / gib, double(plan.sweep_peak_bytes) / gib, double(plan.init_peak_bytes) / gib,
            plan.rows, plan.cells_per_row, (unsigned long long)plan.alg_bytes_per_residue,
            (unsigned long long)plan.transitions_per_residue, target_mib, max_window, gpus == 1 ? 1 : 0);
    fprintf(stderr, "PLAN crt_moduli=%zu", mods.size());
    for (uint32_t m : mods) fprintf(stderr, " %u:ok", m);
    fprintf(stderr, "\n");
    return 0;
  }
  if (requested > 1) {
    fprintf(stderr, "this engine runs on one GPU; gpus=%d requested\n", requested);
    return 2;
  }
  fdp_ctx *ctx = nullptr;
  if ((s = fdp_create(&ctx, 0)) != FDP_OK) {
    fprintf(stderr, "fdp_create: %s\n", fdp_last_error());
    return exit_code(s);
  }
  if (const char *e = getenv("FDP_AUTOTUNE"); e && atoi(e) != 0 && n >= 3) {
    fdp_problem tp{n, int(mods.size()), mods.data(), lanes};
    fdp_autotune_result ar{};
    static char js[1 << 16];
    s = fdp_autotune(ctx, &tp, ~0ull, 2, &ar, js, sizeof(js));
    if (s != FDP_OK) {
      fprintf(stderr, "fdp_autotune: %s\n", fdp_last_error());
      fdp_destroy(ctx);
      return exit_code(s);
    }
    fprintf(stderr, "autotune %s\n", js);
    lanes = ar.lanes;
  }
  int rc = 0;
  for (size_t done = 0; done < mods.size(); done += size_t(lanes)) {
    const int L = int(mods.size() - done) < lanes ? int(mods.size() - done) : lanes;
    fdp_problem chunk{n, L, mods.data() + done, L};
    std::vector<uint32_t> res(size_t(L), 0);
    fdp_run_stats st{};
    auto t0 = std::chrono::steady_clock::now();
    s = fdp_run_sync(ctx, &chunk, res.data(), &st);
    double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (s != FDP_OK) {
      fprintf(stderr, "fdp_run_sync: %s\n", fdp_last_error());
      rc = exit_code(s);
      break;
    }
    for (int i = 0; i < L; ++i) {
      printf("backend=b200-fdp-pull n=%d residue=%u modulus=%u residue_index=%zu residues_total=%zu gpus=1 "
             "main_states=%llu blocked_states=%llu lanes=%d batch_device_s=%.6f batch_wall_s=%.6f "
             "capture_s=%.6f wall_s=%.6f\n",
             n, res[size_t(i)], mods[done + size_t(i)], done + size_t(i), mods.size(),
             (unsigned long long)plan.main_states, (unsigned long long)plan.blocked_states, L, st.device_s, wall,
             st.capture_s, wall / L);
      fflush(stdout);
    }
  }
  fdp_destroy(ctx);
  return rc;
}
