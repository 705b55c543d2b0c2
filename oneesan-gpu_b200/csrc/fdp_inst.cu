// Explicit instantiations of the cell / first-row kernels for K in
// [FDP_K_LO, FDP_K_HI]; the build compiles this file once per K range so the
// 2 x 16 kernel variants build in parallel.
#include "fdp_kernels.cuh"
#include "fdp_launch.h"

#ifndef FDP_K_LO
#define FDP_K_LO 1
#endif
#ifndef FDP_K_HI
#define FDP_K_HI 16
#endif

namespace fdp {

template <typename Idx, int K>
cudaError_t launch_cell_t(const CellArgs &a, const LaunchCfg &cfg, cudaStream_t s) {
  const int rec_items = a.compact ? a.lane_items : 0;  // <= FDP_REC_MAX_ITEMS (launch_cell)
  const size_t smem = cell_smem_bytes<Idx, K>(cfg.block, rec_items);
  // Per-variant state, resolved on first use (the device is the same for the
  // life of the process in this library's contexts): the shared-memory limit
  // is raised to the largest record store once, and occupancy is known for
  // every record size.
  static int configured_block = 0, per_sm[FDP_REC_MAX_ITEMS + 1] = {};
  if (configured_block != cfg.block) {
    const size_t most = cell_smem_bytes<Idx, K>(cfg.block, FDP_REC_MAX_ITEMS);
    cudaError_t e = cudaFuncSetAttribute(cell_kernel<Idx, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(most));
    if (e != cudaSuccess) return e;
    for (int c = 0; c <= FDP_REC_MAX_ITEMS; ++c) {
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[c], cell_kernel<Idx, K>, cfg.block,
                                                        cell_smem_bytes<Idx, K>(cfg.block, c));
      if (e != cudaSuccess) return e;
      if (per_sm[c] < 1) per_sm[c] = 1;
    }
    configured_block = cfg.block;
  }
  int grid = cfg.grid > 0 ? cfg.grid : device_sm_count() * per_sm[rec_items];
  const uint64_t per_block = uint64_t(cfg.block) * uint64_t(a.lane_items < 1 ? 1 : a.lane_items);
  const uint64_t need = (a.items + per_block - 1) / per_block;
  if (uint64_t(grid) > need) grid = int(need ? need : 1);
  cell_kernel<Idx, K><<<grid, cfg.block, smem, s>>>(a);
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
