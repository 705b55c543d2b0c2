// Explicit instantiations of the cell / first-row kernels for K in
// [FDP_K_LO, FDP_K_HI]; the build compiles this file once per K range so the
// 2 x 16 kernel variants build in parallel.
#include <map>
#include <mutex>

#include "fdp_kernels.cuh"
#include "fdp_launch.h"

#ifndef FDP_K_LO
#define FDP_K_LO 1
#endif
#ifndef FDP_K_HI
#define FDP_K_HI 16
#endif

namespace fdp {

// Per-device launch state of one kernel variant: the dynamic shared-memory
// limit is raised once per device to the largest layout of the largest CTA,
// and the occupancy of every (CTA size, shared-memory size) is resolved on
// first use on that device.
constexpr int kInstMaxDevices = 64;

struct VariantState {
  bool limit_set = false;
  std::map<uint64_t, int> per_sm;  // (block, dynamic shared bytes) -> resident CTAs per SM
};

template <typename Idx, int K>
cudaError_t launch_cell_t(const CellArgs &a, const LaunchCfg &cfg, cudaStream_t s) {
  static std::mutex mu;
  static VariantState state[kInstMaxDevices];
  if (cfg.block < 32 || cfg.block > 256 || cfg.block % 32) return cudaErrorInvalidValue;
  if (a.W < 2 || a.W > FDP_MAXW) return cudaErrorInvalidValue;
  const int compact = a.compact == 2 ? 2 : (a.compact && a.lane_items <= FDP_REC_MAX_ITEMS ? 1 : 0);
  const size_t smem = cell_smem_bytes<Idx, K>(cfg.block, a.W, compact, a.lane_items);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kInstMaxDevices) return cudaErrorInvalidDevice;
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    VariantState &v = state[dev];
    if (!v.limit_set) {
      size_t most = cell_smem_bytes<Idx, K>(256, FDP_MAXW, 1, FDP_REC_MAX_ITEMS);
      const size_t carry = cell_smem_bytes<Idx, K>(256, FDP_MAXW, 2, 0);
      if (carry > most) most = carry;
      e = cudaFuncSetAttribute(cell_kernel<Idx, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(most));
      if (e != cudaSuccess) return e;
      e = cudaFuncSetAttribute(cell_stream_kernel<Idx, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(most));
      if (e != cudaSuccess) return e;
      v.limit_set = true;
    }
    int &slot = v.per_sm[(uint64_t(a.compact ? 1 : 0) << 62) | (uint64_t(cfg.block) << 32) | uint64_t(smem)];
    if (slot == 0) {
      e = a.compact ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&slot, cell_kernel<Idx, K>, cfg.block, smem)
                    : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&slot, cell_stream_kernel<Idx, K>, cfg.block, smem);
      if (e != cudaSuccess) {
        slot = 0;
        return e;
      }
      if (slot < 1) slot = 1;
    }
    per_sm = slot;
  }
  int grid = cfg.grid > 0 ? cfg.grid : device_sm_count() * per_sm;
  const uint64_t per_block = uint64_t(cfg.block) * uint64_t(a.lane_items < 1 ? 1 : a.lane_items);
  const uint64_t need = (a.items + per_block - 1) / per_block;
  if (uint64_t(grid) > need) grid = int(need ? need : 1);
  if (a.compact) cell_kernel<Idx, K><<<grid, cfg.block, smem, s>>>(a);
  else cell_stream_kernel<Idx, K><<<grid, cfg.block, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename Idx, int K>
cudaError_t launch_first_row_t(const FirstRowArgs &a, bool dot, cudaStream_t s) {
  const uint64_t total = 1ull << (a.W - 1);
  uint64_t blocks = (total + 255) / 256;
  const uint64_t cap = uint64_t(device_sm_count()) * 8;
  if (blocks > cap) blocks = cap;
  if (dot) first_row_dot_kernel<Idx, K><<<unsigned(blocks), 256, 0, s>>>(a);
  else first_row_init_kernel<Idx, K><<<unsigned(blocks), 256, 0, s>>>(a);
  return cudaGetLastError();
}

#define FDP_INST(K)                                                                              \
  template cudaError_t launch_cell_t<uint32_t, K>(const CellArgs &, const LaunchCfg &, cudaStream_t); \
  template cudaError_t launch_cell_t<uint64_t, K>(const CellArgs &, const LaunchCfg &, cudaStream_t); \
  template cudaError_t launch_first_row_t<uint32_t, K>(const FirstRowArgs &, bool, cudaStream_t);    \
  template cudaError_t launch_first_row_t<uint64_t, K>(const FirstRowArgs &, bool, cudaStream_t);

#if FDP_K_LO <= 1 && 1 <= FDP_K_HI
FDP_INST(1)
#endif
#if FDP_K_LO <= 2 && 2 <= FDP_K_HI
FDP_INST(2)
#endif
#if FDP_K_LO <= 3 && 3 <= FDP_K_HI
FDP_INST(3)
#endif
#if FDP_K_LO <= 4 && 4 <= FDP_K_HI
FDP_INST(4)
#endif
#if FDP_K_LO <= 5 && 5 <= FDP_K_HI
FDP_INST(5)
#endif
#if FDP_K_LO <= 6 && 6 <= FDP_K_HI
FDP_INST(6)
#endif
#if FDP_K_LO <= 7 && 7 <= FDP_K_HI
FDP_INST(7)
#endif
#if FDP_K_LO <= 8 && 8 <= FDP_K_HI
FDP_INST(8)
#endif
#if FDP_K_LO <= 9 && 9 <= FDP_K_HI
FDP_INST(9)
#endif
#if FDP_K_LO <= 10 && 10 <= FDP_K_HI
FDP_INST(10)
#endif
#if FDP_K_LO <= 11 && 11 <= FDP_K_HI
FDP_INST(11)
#endif
#if FDP_K_LO <= 12 && 12 <= FDP_K_HI
FDP_INST(12)
#endif
#if FDP_K_LO <= 13 && 13 <= FDP_K_HI
FDP_INST(13)
#endif
#if FDP_K_LO <= 14 && 14 <= FDP_K_HI
FDP_INST(14)
#endif
#if FDP_K_LO <= 15 && 15 <= FDP_K_HI
FDP_INST(15)
#endif
#if FDP_K_LO <= 16 && 16 <= FDP_K_HI
FDP_INST(16)
#endif

}  // namespace fdp
