// Row-k initialiser on the device (fdp_rowinit_dev.cu): fills the state after
// row rows-1 of width W into the target space of height cap `cap`.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fdp {

// Upload the automaton and the fill plan for (W, rows, cap) on the current
// device, once; must run outside stream capture.
cudaError_t prepare_row_init(int W, int rows, int cap);

// Scratch words per lane the fill needs (two prefix and two suffix levels).
uint64_t row_init_scratch(int W, int rows, int cap);

// Enqueue the fill of `main` (L lanes, panel layout, the target space's
// states) on `s`, using `scratch` (scratch_words words, not overlapping main).
cudaError_t enqueue_row_init(int W, int rows, int cap, int L, const uint32_t *mods, uint32_t *main,
                             uint32_t *scratch, uint64_t scratch_words, cudaStream_t s, uint64_t *launches);

}  // namespace fdp
