// Row-k initialiser on the device (fdp_rowinit_dev.cu): fills the state after
// row rows-1 of width W into the target space of height cap `cap`.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fdp {

// Upload the automaton and the fill plan for (W, rows, cap) on the current
// device, once; must run outside stream capture.
cudaError_t prepare_row_init(int W, int rows, int cap);

// Rows of vertices the initialiser fills by default for width W (0: none):
// seven from width 18 up, six from width 14 (measured at n = 22: 7 rows
// 18.40 s, 6 rows 18.84 s, 5 rows 19.78 s per pass of 14 residues, none 22.23 s).
int auto_row_init_rows(int W);

// Scratch words per lane the fill needs (two prefix and two suffix levels).
uint64_t row_init_scratch(int W, int rows, int cap);

// Device bytes of the fill's resident tables (automaton, prefix trie).
uint64_t row_init_tables(int W, int rows, int cap);

// Enqueue the fill of `main` (L lanes, panel layout, the target space's
// states) on `s`, using `scratch` (scratch_words words, not overlapping main).
// tensor: the products on the tensor cores (tcgen05, 8-bit limbs) instead of
// the CUDA cores; a tensor-core product whose bounded wait gives up writes a
// nonzero value to the caller's device word `err` (required when tensor), and
// its residues are then invalid.
cudaError_t enqueue_row_init(int W, int rows, int cap, int L, const uint32_t *mods, uint32_t *main,
                             uint32_t *scratch, uint64_t scratch_words, bool tensor, unsigned int *err,
                             cudaStream_t s, uint64_t *launches);

}  // namespace fdp
