// Autotuner: memory admission from the plan, timed row sweeps per candidate
// (1 warm-up + `repeats`, median), estimated device seconds per residue, and a
// known-residue check of the winner (n = 9 mod 4294967291 = 2674633373, the
// value published in scripts/test/groupbatch-runtime.py:17 of the reference).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/oneesan_fdp.h"
#include "fdp_api_internal.h"
#include "fdp_host.h"

namespace {

double median(std::vector<double> v) {
  std::sort(v.begin(), v.end());
  const size_t n = v.size();
  return n % 2 ? v[n / 2] : 0.5 * (v[n / 2 - 1] + v[n / 2]);
}

int panel_count(int lanes) {
  int n = 0;
  for (int l = 0; l < lanes; ++n) l += (lanes - l >= 8) ? 8 : (lanes - l >= 4) ? 4 : (lanes - l >= 2) ? 2 : 1;
  return n;
}

}  // namespace

extern "C" fdp_status fdp_autotune(fdp_ctx *c, const fdp_problem *pr, uint64_t budget, int repeats,
                                   fdp_autotune_result *out, char *json_out, size_t json_cap) {
  if (!c || !pr || !out || pr->n < 3 || pr->n > FDP_MAX_N || pr->k < 1 || !pr->moduli) return FDP_ERR_ARGS;
  if (repeats < 1) repeats = 1;
  const int max_lanes = std::max(1, std::min({pr->lanes > 0 ? pr->lanes : FDP_MAX_LANES, pr->k, FDP_MAX_LANES}));
  // Candidate residues-per-pass values.
  std::vector<int> lane_opts;
  for (int L : {1, 2, 4, 7, 8, 12, 14, 16})
    if (L <= max_lanes) lane_opts.push_back(L);
  if (std::find(lane_opts.begin(), lane_opts.end(), max_lanes) == lane_opts.end()) lane_opts.push_back(max_lanes);
  const int k = pr->k;
  for (int L = 1; L <= max_lanes; ++L)  // an even split of k into passes
    if ((k + L - 1) / L * L == k && std::find(lane_opts.begin(), lane_opts.end(), L) == lane_opts.end() && L >= 4)
      lane_opts.push_back(L);
  std::sort(lane_opts.begin(), lane_opts.end());
  fdp_tuning saved{};
  fdp_get_tuning(c, &saved);
  const int W = pr->n + 1, rows = fdp::sweep_rows(W);
  std::string js = "{\"n\":" + std::to_string(pr->n) + ",\"k\":" + std::to_string(k) + ",\"candidates\":[";
  bool first = true;
  fdp_autotune_result best{};
  best.s_per_residue = INFINITY;
  int tried = 0, rejected = 0;
  std::vector<double> cell_ms(size_t(W) + 1);
  for (int L : lane_opts) {
    fdp_problem cand{pr->n, L, pr->moduli, L};
    fdp_plan_out plan{};
    if (fdp_plan(&cand, budget, &plan) != FDP_OK || !plan.fits) {
      ++rejected;
      char buf[160];
      snprintf(buf, sizeof(buf), "%s{\"lanes\":%d,\"status\":\"memory-rejected\",\"state_bytes\":%llu}",
               first ? "" : ",", L, (unsigned long long)plan.state_bytes);
      js += buf;
      first = false;
      continue;
    }
    const int npanels = panel_count(L);
    for (int split = 0; split <= (npanels > 1 ? 1 : 0); ++split)
      for (int block : {128, 256}) {
        fdp_tuning t = saved;
        t.block = block;
        t.grid = 0;
        t.split_panels = split;
        fdp_status s = fdp_set_tuning(c, &t);
        std::vector<double> samples;
        for (int r = 0; r <= repeats && s == FDP_OK; ++r) {
          s = fdp_time_cells(c, &cand, 1, cell_ms.data());
          double row = 0;
          for (int p = 1; p < W; ++p) row += cell_ms[size_t(p)];
          if (r > 0) samples.push_back(row);
        }
        ++tried;
        char buf[320];
        if (s != FDP_OK) {
          snprintf(buf, sizeof(buf), "%s{\"lanes\":%d,\"split_panels\":%d,\"block\":%d,\"status\":\"failed\"}",
                   first ? "" : ",", L, split, block);
          js += buf;
          first = false;
          if (s == FDP_ERR_HBM) continue;
          fdp_set_tuning(c, &saved);
          return s;
        }
        const double row = median(samples);
        const int passes = (k + L - 1) / L;
        // Each pass sweeps the rows the row-k initialiser does not fill
        // (its own fill is left out of the estimate); spread over k residues.
        const int swept = rows - (plan.init_rows >= 2 ? plan.init_rows - 1 : 0);
        const double spr = row * 1e-3 * swept * passes / k;
        snprintf(buf, sizeof(buf),
                 "%s{\"lanes\":%d,\"split_panels\":%d,\"block\":%d,\"status\":\"ok\",\"row_ms\":%.4f,"
                 "\"s_per_residue\":%.6f,\"passes\":%d}",
                 first ? "" : ",", L, split, block, row, spr, passes);
        js += buf;
        first = false;
        if (spr < best.s_per_residue) {
          best.lanes = L;
          best.passes = passes;
          best.tuning = t;
          best.row_ms = row;
          best.s_per_residue = spr;
        }
      }
  }
  if (!std::isfinite(best.s_per_residue)) {
    fdp_set_tuning(c, &saved);
    fdp_set_last_error("autotune: no candidate fits the HBM budget");
    return FDP_ERR_HBM;
  }
  fdp_status s = fdp_set_tuning(c, &best.tuning);
  // Known-residue check of the chosen launch configuration.
  if (s == FDP_OK) {
    const uint32_t m = 4294967291u;
    std::vector<uint32_t> mods(size_t(best.lanes), m), res(size_t(best.lanes));
    fdp_problem chk{9, best.lanes, mods.data(), best.lanes};
    fdp_run_stats st{};
    s = fdp_run_sync(c, &chk, res.data(), &st);
    if (s == FDP_OK)
      for (uint32_t r : res)
        if (r != 2674633373u) {
          fdp_set_tuning(c, &saved);
          fdp_set_last_error("autotune: WRONG RESIDUE in the known-answer check");
          return FDP_ERR_CUDA;
        }
  }
  if (s != FDP_OK) return s;
  best.residues_per_hour = 3600.0 / best.s_per_residue;
  best.candidates = tried;
  best.rejected_memory = rejected;
  char tail[320];
  snprintf(tail, sizeof(tail),
           "],\"best\":{\"lanes\":%d,\"passes\":%d,\"split_panels\":%d,\"block\":%d,\"row_ms\":%.4f,"
           "\"s_per_residue\":%.6f,\"residues_per_hour\":%.3f},\"known_residue_check\":\"ok\"}",
           best.lanes, best.passes, best.tuning.split_panels, best.tuning.block, best.row_ms, best.s_per_residue,
           best.residues_per_hour);
  js += tail;
  if (json_out && json_cap) {
    const size_t n = std::min(json_cap - 1, js.size());
    memcpy(json_out, js.data(), n);
    json_out[n] = 0;
  }
  *out = best;
  return FDP_OK;
}
