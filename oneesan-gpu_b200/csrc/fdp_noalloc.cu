// First-row dot product that allocates no device memory.
//
// Who needs it: callers that hand all device memory to their own allocator up
// front -- a serving process that reserves its HBM budget in one pool, or a
// framework with a caching allocator that owns the GPU -- cannot let a library
// call cudaMalloc: the call would fail once the pool has taken the memory, or
// steal from the budget the pool enforces, and cudaMalloc / cudaFree may
// synchronise the device in the middle of the caller's stream work.  Those
// callers own the state vectors and the output and need the residue read-out
// to touch nothing else.
//
// This is a variant of the first-row dot product (the only kernel of the
// library that needs scratch: 64-bit accumulators, one per lane).  Here the
// accumulators live in a file-scope device array of fixed size instead of a
// buffer the library allocates.  Limits: width <= 28 and lanes <= 16.
//
// Set-up: the first call on a device (with that device current) looks up the
// device address of the array with cudaGetSymbolAddress and keeps it for the
// life of the process; do that first call before any stream capture.  The
// address belongs to the device's primary context: a caller that destroys it
// (cudaDeviceReset) must not call this entry point again in the same process.
// Host code must never pass the array's name itself to a kernel: in host code
// it is a host-side stand-in, not a device address.  The kernel builds the
// canonical-rank count table in its own shared memory, so nothing else is
// uploaded.
//
// Every call on a device shares the same accumulators and they keep the last
// call's contents; each call clears them on its stream before use.  Calls
// whose work overlaps on the GPU (different streams, or different host
// threads) race on the accumulators and give wrong residues: serialise them.
#include <mutex>
#include <string>

#include "../../include/oneesan_fdp.h"
#include "fdp_api_internal.h"
#include "fdp_host.h"
#include "fdp_item.cuh"

#define FDP_NOALLOC_MAX_LANES 16
#define FDP_NOALLOC_MAX_DEVICES 64

namespace {

using ull = unsigned long long;

// Scratch: the dot product's per-lane 64-bit accumulators (128 bytes).
static __device__ __align__(256) ull g_noalloc_acc[FDP_NOALLOC_MAX_LANES];

struct DeviceSetup {
  bool ready = false;
  ull *acc = nullptr;  // device address of g_noalloc_acc
};
std::mutex g_setup_mu;
DeviceSetup g_setup[FDP_NOALLOC_MAX_DEVICES];

struct Mods {
  uint32_t m[FDP_NOALLOC_MAX_LANES];
};

template <int K>
__global__ void __launch_bounds__(256) noalloc_dot_kernel(const uint32_t *main, uint64_t mstates, ull *acc_out,
                                                          int W) {
  __shared__ ull sH[FDP_MAXW + 1][FDP_HT];
  __shared__ ull red[8][K];
  // H[w][h]: words of w symbols from height h down to 0 (N keeps the height,
  // R lowers it, L raises it), built row by row: the canonical-rank counts.
  if (threadIdx.x < FDP_HT) sH[0][threadIdx.x] = threadIdx.x == 0 ? 1ull : 0ull;
  __syncthreads();
  for (int w = 1; w <= FDP_MAXW; ++w) {
    const int h = int(threadIdx.x);
    if (h < FDP_HT)
      sH[w][h] = sH[w - 1][h] + (h > 0 ? sH[w - 1][h - 1] : 0ull) + (h + 1 < FDP_HT ? sH[w - 1][h + 1] : 0ull);
    __syncthreads();
  }
  const uint64_t total = 1ull << (W - 1);
  ull acc[K];
#pragma unroll
  for (int i = 0; i < K; ++i) acc[i] = 0;
  for (uint64_t mask = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; mask < total;
       mask += uint64_t(gridDim.x) * blockDim.x) {
    const ull rk = fdp::rank_dev<ull>(fdp::first_row_state_dev(mask, W), W, sH);
    uint32_t v[K];
    fdp::ld_lanes<K>(main, mstates, size_t(rk), v);
#pragma unroll
    for (int i = 0; i < K; ++i) acc[i] += v[i];
  }
#pragma unroll
  for (int i = 0; i < K; ++i) {
    ull v = acc[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][i] = v;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    ull v = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) v += red[w][threadIdx.x];
    atomicAdd(acc_out + threadIdx.x, v);
  }
}

__global__ void noalloc_finalize_kernel(const ull *acc, uint32_t *out, Mods mods, int k) {
  const int i = threadIdx.x;
  if (i < k) out[i] = uint32_t(acc[i] % mods.m[i]);
}

template <int K>
cudaError_t launch_dot(const DeviceSetup &s, const uint32_t *main, int W, cudaStream_t st) {
  const uint64_t total = 1ull << (W - 1);
  uint64_t blocks = (total + 255) / 256;
  if (blocks > 1184) blocks = 1184;
  noalloc_dot_kernel<K><<<unsigned(blocks), 256, 0, st>>>(main, fdp::main_states(W), s.acc, W);
  return cudaGetLastError();
}

cudaError_t dispatch_dot(int K, const DeviceSetup &s, const uint32_t *main, int W, cudaStream_t st) {
  switch (K) {
    case 1: return launch_dot<1>(s, main, W, st);
    case 2: return launch_dot<2>(s, main, W, st);
    case 3: return launch_dot<3>(s, main, W, st);
    case 4: return launch_dot<4>(s, main, W, st);
    case 5: return launch_dot<5>(s, main, W, st);
    case 6: return launch_dot<6>(s, main, W, st);
    case 7: return launch_dot<7>(s, main, W, st);
    case 8: return launch_dot<8>(s, main, W, st);
    case 9: return launch_dot<9>(s, main, W, st);
    case 10: return launch_dot<10>(s, main, W, st);
    case 11: return launch_dot<11>(s, main, W, st);
    case 12: return launch_dot<12>(s, main, W, st);
    case 13: return launch_dot<13>(s, main, W, st);
    case 14: return launch_dot<14>(s, main, W, st);
    case 15: return launch_dot<15>(s, main, W, st);
    case 16: return launch_dot<16>(s, main, W, st);
    default: return cudaErrorInvalidValue;
  }
}

fdp_status fail(cudaError_t e, const char *what) {
  std::string m = std::string("fdp_first_row_dot_noalloc: ") + what + ": " + cudaGetErrorString(e);
  fdp_set_last_error(m.c_str());
  return FDP_ERR_CUDA;
}

// Once per device, with that device current: resolve the array's device
// address.
fdp_status setup_device(int dev, DeviceSetup **out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  DeviceSetup &s = g_setup[dev];
  if (!s.ready) {
    cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&s.acc), g_noalloc_acc);
    if (e != cudaSuccess) return fail(e, "cudaGetSymbolAddress(accumulators)");
    s.ready = true;
  }
  *out = &s;
  return FDP_OK;
}

}  // namespace

extern "C" fdp_status fdp_first_row_dot_noalloc(int width, int lanes, const uint32_t *moduli, const uint32_t *d_main,
                                                uint32_t *d_residues, void *stream) {
  if (width < 2 || width > FDP_MAXW) {
    fdp_set_last_error("fdp_first_row_dot_noalloc: width must be in 2..28");
    return FDP_ERR_ARGS;
  }
  if (lanes < 1 || lanes > FDP_NOALLOC_MAX_LANES) {
    fdp_set_last_error("fdp_first_row_dot_noalloc: lanes must be in 1..16 (the fixed scratch holds 16 accumulators)");
    return FDP_ERR_ARGS;
  }
  if (!moduli || !d_main || !d_residues) {
    fdp_set_last_error("fdp_first_row_dot_noalloc: null pointer");
    return FDP_ERR_ARGS;
  }
  if (!fdp::panel_aligned(lanes, d_main)) {
    fdp_set_last_error("fdp_first_row_dot_noalloc: d_main must be aligned to one word of the widest lane panel "
                       "(32 bytes for 8 or more lanes, 16 for 4-7, 8 for 2-3)");
    return FDP_ERR_ARGS;
  }
  Mods mods{};
  for (int i = 0; i < lanes; ++i) {
    if (moduli[i] < 2) {
      fdp_set_last_error("fdp_first_row_dot_noalloc: modulus must be in [2, 2^32-1]");
      return FDP_ERR_MODULUS;
    }
    mods.m[i] = moduli[i];
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= FDP_NOALLOC_MAX_DEVICES) {
    fdp_set_last_error("fdp_first_row_dot_noalloc: device index above 63");
    return FDP_ERR_GPU_COUNT;
  }
  DeviceSetup *s = nullptr;
  fdp_status st = setup_device(dev, &s);
  if (st != FDP_OK) return st;
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  if ((e = cudaMemsetAsync(s->acc, 0, sizeof(ull) * lanes, cs)) != cudaSuccess) return fail(e, "clear accumulators");
  if ((e = dispatch_dot(lanes, *s, d_main, width, cs)) != cudaSuccess) return fail(e, "dot kernel");
  noalloc_finalize_kernel<<<1, 32, 0, cs>>>(s->acc, d_residues, mods, lanes);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "finalize kernel");
  return FDP_OK;
}
