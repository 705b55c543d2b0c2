// Request loop with continuous batching (fdp_server_* / fdp_submit / fdp_poll).
//
// One device pool of the configured budget is reserved at start and carved by
// a first-fit allocator, so admission never calls cudaMalloc.  A scheduler
// thread: (1) retires requests whose completion event has fired, freeing
// their pool range and slot; (2) admits queued requests in arrival order while
// a slot and pool memory are free, letting smaller requests pass a blocked head
// until the head has waited max_bypass_s; (3) captures each admitted request's
// whole computation (every pass of `lanes` residues: zero, row-0 init, row
// sweeps, first-row dot, residue copy) as one CUDA graph and launches it on the
// slot's own stream.  Requests on different slots therefore overlap on the
// GPU.  An admitted request whose moduli fill less than one pass takes along
// later queued requests of the same n while their moduli fit its lanes, so
// one pass serves them all (a residue does not depend on the other lanes).
// Every wait is bounded: the scheduler sleeps at most 200 us between
// event polls, and fdp_wait returns FDP_TIMEOUT after its limit.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/oneesan_fdp.h"
#include "fdp_api_internal.h"
#include "fdp_host.h"
#include "fdp_launch.h"

namespace {

using Clock = std::chrono::steady_clock;
double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

constexpr uint64_t kAlign = 256;
constexpr int kMaxModuliPerRequest = 64;

// First-fit allocator over [0, size) with coalescing frees.
struct PoolAlloc {
  uint64_t size = 0, used = 0, peak = 0;
  std::map<uint64_t, uint64_t> free_;  // offset -> length
  void reset(uint64_t s) {
    size = s;
    used = peak = 0;
    free_.clear();
    if (s) free_[0] = s;
  }
  bool alloc(uint64_t len, uint64_t *off) {
    len = (len + kAlign - 1) / kAlign * kAlign;
    for (auto it = free_.begin(); it != free_.end(); ++it)
      if (it->second >= len) {
        *off = it->first;
        const uint64_t rest = it->second - len, roff = it->first + len;
        free_.erase(it);
        if (rest) free_[roff] = rest;
        used += len;
        peak = std::max(peak, used);
        return true;
      }
    return false;
  }
  void release(uint64_t off, uint64_t len) {
    len = (len + kAlign - 1) / kAlign * kAlign;
    used -= len;
    auto it = free_.emplace(off, len).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

struct Job {
  uint64_t id = 0;
  int n = 0, lanes = 1, passes = 1, slot = -1;
  std::vector<uint32_t> mods, residues;
  uint64_t bytes = 0, off = 0;
  // LAUNCHING: admitted (slot and pool range reserved), being captured and
  // launched by the scheduler with the lock released.
  enum State { QUEUED, LAUNCHING, RUNNING, DONE, FAILED } state = QUEUED;
  fdp_status status = FDP_OK;
  std::string error;
  Clock::time_point t_submit, t_admit, t_done;
  cudaGraphExec_t exec = nullptr;
  double device_s = 0;
  // Queued requests of the same n whose moduli fit this request's one pass:
  // they ride in its lanes (batch = its moduli, then each rider's).
  std::vector<Job *> riders;
  std::vector<uint32_t> batch;
};

// Bytes of one request in the pool: the state for `lanes` residues, then the
// dot-product accumulators (256 bytes), and the device residues with the
// request's error word 128 bytes after them (256 bytes).
uint64_t request_bytes(int n, int lanes) {
  const int W = n + 1;
  const uint64_t M = fdp::main_states(W), D = fdp::blocked_states(W);
  const uint64_t a = (4ull * M * lanes + kAlign - 1) / kAlign * kAlign;
  const uint64_t b = (4ull * D * lanes + kAlign - 1) / kAlign * kAlign;
  return a + b + 2 * kAlign;
}

}  // namespace

struct fdp_server {
  fdp_ctx *ctx = nullptr;
  fdp_server_config cfg{};
  char *pool = nullptr;
  PoolAlloc alloc;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> ev_start, ev_done;
  std::vector<uint32_t *> pinned;  // per slot, kMaxModuliPerRequest residues, then the error word
  std::vector<Job *> slot_job;
  std::deque<uint64_t> queue;
  std::map<uint64_t, std::unique_ptr<Job>> jobs;
  std::mutex mu;
  std::condition_variable cv;
  std::thread th;
  bool stopping = false;
  uint64_t next_id = 1, submitted = 0, completed = 0, failed = 0;
  int running = 0, peak_running = 0;

  void fail(Job *j, fdp_status s, const std::string &msg) {
    j->state = Job::FAILED;
    j->status = s;
    j->error = msg;
    j->t_done = Clock::now();
    ++failed;
  }

  // Capture and launch every pass of job j on its slot's stream.
  fdp_status launch(Job *j) {
    const int slot = j->slot;
    cudaStream_t s = streams[size_t(slot)];
    const fdp::DevTables *t = nullptr;
    fdp_status st = fdp_prepare_pass(ctx, j->n + 1, &t);
    if (st != FDP_OK) return st;
    const int W = j->n + 1;
    const uint64_t M = fdp::main_states(W);
    char *base = pool + j->off;
    uint32_t *main = reinterpret_cast<uint32_t *>(base);
    uint32_t *blk = reinterpret_cast<uint32_t *>(base + (4ull * M * j->lanes + kAlign - 1) / kAlign * kAlign);
    char *small = base + j->bytes - 2 * kAlign;
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(small);
    uint32_t *dres = reinterpret_cast<uint32_t *>(small + kAlign);
    unsigned int *derr = reinterpret_cast<unsigned int *>(small + kAlign + 128);
    unsigned int *herr = reinterpret_cast<unsigned int *>(pinned[size_t(slot)] + kMaxModuliPerRequest);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fdp_cuda_status(e, "serve: begin capture");
    fdp_status es = fdp_cuda_status(fdp_enqueue_err_reset(derr, s), "serve: error word");
    uint64_t launches = 0;
    const std::vector<uint32_t> &mods = j->batch.empty() ? j->mods : j->batch;
    for (int done = 0; done < int(mods.size()) && es == FDP_OK; done += j->lanes) {
      const int L = std::min(j->lanes, int(mods.size()) - done);
      es = fdp_enqueue_pass(ctx, *t, L, mods.data() + done, main, blk, acc, dres, pinned[size_t(slot)] + done,
                            derr, s, &launches);
    }
    if (es == FDP_OK) es = fdp_cuda_status(fdp_enqueue_err_read(herr, derr, s), "serve: error word");
    e = cudaStreamEndCapture(s, &g);
    if (es != FDP_OK) {
      if (g) cudaGraphDestroy(g);
      return es;
    }
    if (e != cudaSuccess) return fdp_cuda_status(e, "serve: end capture");
    e = cudaGraphInstantiate(&j->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fdp_cuda_status(e, "serve: instantiate");
    cudaEventRecord(ev_start[size_t(slot)], s);
    e = cudaGraphLaunch(j->exec, s);
    if (e != cudaSuccess) return fdp_cuda_status(e, "serve: graph launch");
    e = cudaEventRecord(ev_done[size_t(slot)], s);
    if (e != cudaSuccess) return fdp_cuda_status(e, "serve: event");
    return FDP_OK;
  }

  void retire(int slot, bool ok, cudaError_t err) {
    Job *j = slot_job[size_t(slot)];
    slot_job[size_t(slot)] = nullptr;
    --running;
    alloc.release(j->off, j->bytes);
    if (j->exec) cudaGraphExecDestroy(j->exec);
    j->exec = nullptr;
    const unsigned int herr = pinned[size_t(slot)][kMaxModuliPerRequest];
    float ms = 0;
    if (ok && !herr) cudaEventElapsedTime(&ms, ev_start[size_t(slot)], ev_done[size_t(slot)]);
    const Clock::time_point now = Clock::now();
    size_t at = 0;  // the leader's residues, then each rider's, in batch order
    std::vector<Job *> all{j};
    all.insert(all.end(), j->riders.begin(), j->riders.end());
    for (Job *r : all) {
      r->t_done = now;
      if (ok && herr) {
        fail(r, FDP_ERR_CUDA, "serve: a bounded wait on the device gave up; the residues are invalid");
      } else if (ok) {
        r->device_s = ms * 1e-3;
        r->residues.assign(pinned[size_t(slot)] + at, pinned[size_t(slot)] + at + r->mods.size());
        r->state = Job::DONE;
        ++completed;
      } else {
        fail(r, FDP_ERR_CUDA, std::string("serve: request failed: ") + cudaGetErrorString(err));
      }
      at += r->mods.size();
    }
  }

  void loop() {
    cudaSetDevice(ctx->device);
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
      // (1) completions
      for (int s = 0; s < int(slot_job.size()); ++s) {
        if (!slot_job[size_t(s)]) continue;
        cudaError_t q = cudaEventQuery(ev_done[size_t(s)]);
        if (q == cudaErrorNotReady) continue;
        retire(s, q == cudaSuccess, q);
      }
      if (stopping) {
        for (uint64_t id : queue) fail(jobs[id].get(), FDP_ERR_ARGS, "server stopped before admission");
        queue.clear();
        if (!running) break;
      }
      // (2) admission, arrival order with bounded backfill.  A request is
      // taken off the queue with its slot and pool range reserved under the
      // lock; its tables, capture, instantiation and launch then run with the
      // lock released, so fdp_submit / fdp_poll / fdp_wait never wait for
      // them.  Only this thread changes slots and the pool.
      while (running < cfg.max_active) {
        const Clock::time_point now = Clock::now();
        Job *j = nullptr;
        int slot = -1;
        for (int s = 0; s < int(slot_job.size()); ++s)
          if (!slot_job[size_t(s)]) { slot = s; break; }
        if (slot < 0) break;
        std::vector<Job *> riders;
        for (auto it = queue.begin(); it != queue.end(); ++it) {
          Job *q = jobs[*it].get();
          // Later queued requests of the same n ride in q's one pass while
          // their moduli fit its lanes.
          int total = int(q->mods.size());
          if (total < cfg.max_lanes)
            for (auto jt = std::next(it); jt != queue.end() && total < cfg.max_lanes; ++jt) {
              Job *r = jobs[*jt].get();
              if (r->n == q->n && total + int(r->mods.size()) <= cfg.max_lanes) {
                riders.push_back(r);
                total += int(r->mods.size());
              }
            }
          uint64_t off = 0;
          uint64_t bytes = riders.empty() ? q->bytes : request_bytes(q->n, total);
          bool got = alloc.alloc(bytes, &off);
          if (!got && !riders.empty()) {  // the batch does not fit: the request alone
            riders.clear();
            total = int(q->mods.size());
            bytes = q->bytes;
            got = alloc.alloc(bytes, &off);
          }
          if (got) {
            q->off = off;
            q->bytes = bytes;
            if (!riders.empty()) {
              q->lanes = total;
              q->passes = 1;
              q->batch = q->mods;
              for (Job *r : riders) q->batch.insert(q->batch.end(), r->mods.begin(), r->mods.end());
            }
            j = q;
            queue.erase(it);
            break;
          }
          riders.clear();
          if (it == queue.begin() && secs(q->t_submit, now) > cfg.max_bypass_s) break;  // reserve for the head
        }
        if (!j) break;
        if (!riders.empty()) {
          std::deque<uint64_t> rest;
          for (uint64_t id : queue) {
            bool rides = false;
            for (Job *r : riders) rides = rides || r->id == id;
            if (!rides) rest.push_back(id);
          }
          queue.swap(rest);
          for (Job *r : riders) {
            r->slot = slot;
            r->t_admit = now;
            r->lanes = j->lanes;
            r->passes = 1;
            r->state = Job::LAUNCHING;
          }
          j->riders = riders;
        }
        j->slot = slot;
        j->t_admit = now;
        j->state = Job::LAUNCHING;
        slot_job[size_t(slot)] = j;
        ++running;
        peak_running = std::max(peak_running, running);
        lk.unlock();
        const fdp_status st = launch(j);
        const std::string why = st != FDP_OK ? std::string(fdp_last_error()) : std::string();
        lk.lock();
        if (st != FDP_OK) {
          slot_job[size_t(slot)] = nullptr;
          --running;
          alloc.release(j->off, j->bytes);
          if (j->exec) cudaGraphExecDestroy(j->exec);
          j->exec = nullptr;
          fail(j, st, "serve: launch failed: " + why);
          for (Job *r : j->riders) fail(r, st, "serve: launch failed: " + why);
        } else {
          j->state = Job::RUNNING;
          for (Job *r : j->riders) r->state = Job::RUNNING;
        }
      }
      cv.notify_all();  // wake fdp_wait callers
      if (!running && queue.empty() && !stopping) cv.wait(lk);
      else cv.wait_for(lk, std::chrono::microseconds(200));
    }
    cv.notify_all();
  }
};

extern "C" fdp_status fdp_server_start(fdp_ctx *c, const fdp_server_config *cfg) {
  if (!c || !cfg) return FDP_ERR_ARGS;
  if (c->server) {
    fdp_set_last_error("server already running on this context");
    return FDP_ERR_ARGS;
  }
  if (cfg->max_active < 1 || cfg->max_active > 64 || cfg->max_lanes < 1 || cfg->max_lanes > FDP_MAX_LANES ||
      cfg->hbm_budget_bytes < (1u << 20)) {
    fdp_set_last_error("server: need 1 <= max_active <= 64, 1 <= max_lanes <= 16, budget >= 1 MiB");
    return FDP_ERR_ARGS;
  }
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fdp_cuda_status(e, "cudaSetDevice");
  auto sv = std::make_unique<fdp_server>();
  sv->ctx = c;
  sv->cfg = *cfg;
  if (sv->cfg.max_bypass_s <= 0) sv->cfg.max_bypass_s = 30.0;
  e = cudaMalloc(&sv->pool, cfg->hbm_budget_bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    fdp_set_last_error("server: cannot reserve the HBM budget");
    return FDP_ERR_HBM;
  }
  sv->alloc.reset(cfg->hbm_budget_bytes);
  const size_t S = size_t(cfg->max_active);
  sv->streams.resize(S);
  sv->ev_start.resize(S);
  sv->ev_done.resize(S);
  sv->pinned.resize(S);
  sv->slot_job.assign(S, nullptr);
  fdp_status st = FDP_OK;
  for (size_t i = 0; i < S && st == FDP_OK; ++i) {
    st = fdp_cuda_status(cudaStreamCreateWithFlags(&sv->streams[i], cudaStreamNonBlocking), "server stream");
    if (st == FDP_OK) st = fdp_cuda_status(cudaEventCreate(&sv->ev_start[i]), "server event");
    if (st == FDP_OK) st = fdp_cuda_status(cudaEventCreate(&sv->ev_done[i]), "server event");
    if (st == FDP_OK)
      st = fdp_cuda_status(cudaMallocHost(&sv->pinned[i], sizeof(uint32_t) * (kMaxModuliPerRequest + 1)),
                           "server pinned");
  }
  if (st != FDP_OK) {
    for (size_t i = 0; i < S; ++i) {
      if (sv->streams[i]) cudaStreamDestroy(sv->streams[i]);
      if (sv->ev_start[i]) cudaEventDestroy(sv->ev_start[i]);
      if (sv->ev_done[i]) cudaEventDestroy(sv->ev_done[i]);
      if (sv->pinned[i]) cudaFreeHost(sv->pinned[i]);
    }
    cudaFree(sv->pool);
    return st;
  }
  fdp_server *raw = sv.release();
  c->server = raw;
  raw->th = std::thread([raw] { raw->loop(); });
  return FDP_OK;
}

void fdp_server_shutdown(fdp_ctx *c) {
  fdp_server *sv = c ? c->server : nullptr;
  if (!sv) return;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stopping = true;
  }
  sv->cv.notify_all();
  if (sv->th.joinable()) sv->th.join();
  cudaSetDevice(c->device);
  for (size_t i = 0; i < sv->streams.size(); ++i) {
    cudaStreamSynchronize(sv->streams[i]);
    cudaStreamDestroy(sv->streams[i]);
    cudaEventDestroy(sv->ev_start[i]);
    cudaEventDestroy(sv->ev_done[i]);
    cudaFreeHost(sv->pinned[i]);
  }
  cudaFree(sv->pool);
  c->server = nullptr;
  delete sv;
}

extern "C" fdp_status fdp_server_stop(fdp_ctx *c) {
  if (!c) return FDP_ERR_ARGS;
  if (!c->server) return FDP_ERR_NOT_FOUND;
  fdp_server_shutdown(c);
  return FDP_OK;
}

extern "C" fdp_status fdp_submit(fdp_ctx *c, const fdp_problem *pr, uint64_t *id) {
  if (!c || !pr || !id) return FDP_ERR_ARGS;
  fdp_server *sv = c->server;
  if (!sv) {
    fdp_set_last_error("submit: no server running (fdp_server_start)");
    return FDP_ERR_NOT_FOUND;
  }
  if (pr->n < 1 || pr->n > FDP_MAX_N || pr->k < 1 || pr->k > kMaxModuliPerRequest || !pr->moduli) {
    fdp_set_last_error("submit: need 1 <= n <= 27 and 1 <= k <= 64 moduli");
    return FDP_ERR_ARGS;
  }
  for (int i = 0; i < pr->k; ++i)
    if (pr->moduli[i] < 2) {
      fdp_set_last_error("submit: modulus must be in [2, 2^32-1]");
      return FDP_ERR_MODULUS;
    }
  auto j = std::make_unique<Job>();
  j->n = pr->n;
  j->mods.assign(pr->moduli, pr->moduli + pr->k);
  j->lanes = std::min(sv->cfg.max_lanes, pr->k);
  j->passes = (pr->k + j->lanes - 1) / j->lanes;
  j->bytes = request_bytes(pr->n, j->lanes);
  if (j->bytes > sv->alloc.size) {
    fdp_set_last_error("submit: request needs more device memory than the whole HBM budget");
    return FDP_ERR_HBM;
  }
  j->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stopping) return FDP_ERR_NOT_FOUND;
    j->id = sv->next_id++;
    *id = j->id;
    sv->queue.push_back(j->id);
    sv->jobs[j->id] = std::move(j);
    ++sv->submitted;
  }
  sv->cv.notify_all();
  return FDP_OK;
}

static fdp_status take_result(fdp_server *sv, uint64_t id, uint32_t *out, fdp_request_info *info) {
  auto it = sv->jobs.find(id);
  if (it == sv->jobs.end()) return FDP_ERR_NOT_FOUND;
  Job *j = it->second.get();
  if (j->state == Job::QUEUED || j->state == Job::LAUNCHING || j->state == Job::RUNNING) return FDP_PENDING;
  if (info) {
    info->queue_s = j->slot >= 0 || j->state == Job::DONE ? secs(j->t_submit, j->t_admit) : secs(j->t_submit, j->t_done);
    info->run_s = j->state == Job::DONE ? secs(j->t_admit, j->t_done) : 0.0;
    info->latency_s = secs(j->t_submit, j->t_done);
    info->device_s = j->device_s;
    info->lanes = j->lanes;
    info->passes = j->passes;
    info->state_bytes = j->bytes;
  }
  fdp_status st = j->state == Job::DONE ? FDP_OK : j->status;
  if (st == FDP_OK && out) std::copy(j->residues.begin(), j->residues.end(), out);
  if (st != FDP_OK) fdp_set_last_error(j->error.c_str());
  sv->jobs.erase(it);
  return st;
}

extern "C" fdp_status fdp_poll(fdp_ctx *c, uint64_t id, uint32_t *out, fdp_request_info *info) {
  if (!c || !c->server) return FDP_ERR_NOT_FOUND;
  std::lock_guard<std::mutex> lk(c->server->mu);
  return take_result(c->server, id, out, info);
}

extern "C" fdp_status fdp_wait(fdp_ctx *c, uint64_t id, int timeout_ms, uint32_t *out, fdp_request_info *info) {
  if (!c || !c->server) return FDP_ERR_NOT_FOUND;
  fdp_server *sv = c->server;
  const Clock::time_point limit = Clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
  std::unique_lock<std::mutex> lk(sv->mu);
  while (true) {
    fdp_status st = take_result(sv, id, out, info);
    if (st != FDP_PENDING) return st;
    if (Clock::now() >= limit) return FDP_TIMEOUT;
    sv->cv.wait_until(lk, std::min(limit, Clock::now() + std::chrono::milliseconds(5)));
  }
}

extern "C" fdp_status fdp_server_get_stats(fdp_ctx *c, fdp_server_stats *st) {
  if (!c || !st) return FDP_ERR_ARGS;
  if (!c->server) return FDP_ERR_NOT_FOUND;
  fdp_server *sv = c->server;
  std::lock_guard<std::mutex> lk(sv->mu);
  st->submitted = sv->submitted;
  st->completed = sv->completed;
  st->failed = sv->failed;
  st->queued = sv->queue.size();
  st->running = uint64_t(sv->running);
  st->pool_bytes = sv->alloc.size;
  st->bytes_in_use = sv->alloc.used;
  st->peak_bytes_in_use = sv->alloc.peak;
  st->peak_running = sv->peak_running;
  return FDP_OK;
}
