// Transition-matrix and invariant-measure launches (csr.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace b12g {

// CSR of P -> CSR of P^T (columns >= n_cols are dropped); rows of P^T list sources in
// ascending order.  work: n_cols + 1 u32; tile_sums: compact_tiles(n_cols + 1) u32.
cudaError_t transpose_csr(const uint32_t* rowptr, const uint32_t* cols, const double* vals, const uint32_t* n_rows,
                          const uint32_t* nnz, uint32_t max_rows, uint64_t max_nnz, uint32_t n_cols,
                          uint32_t* tptr, uint32_t* trows, double* tvals, uint32_t* work, uint32_t* tile_sums,
                          const uint32_t* n_cols_dev, cudaStream_t s);

// the rows of P^T of one length class (1: 9..64 entries, 2: more), ascending; the count
// ends up in pos[n] (flag, pos: n + 1 u32; list: n u32; n_dev: device copy of n)
cudaError_t class_rows(const uint32_t* tptr, uint32_t n, uint32_t cls, uint32_t* flag, uint32_t* pos,
                       uint32_t* list, const uint32_t* n_dev, uint32_t* tile_sums, cudaStream_t s);

// power iteration on the CSR of P^T with the medium and long rows listed by class_rows
// (both lists nullptr: every row gets one thread); sync_words: 65 u32 (barrier count at
// 0, generation at 32, error at 64: bit 1 = barrier timeout); partial: partial_cap doubles.
// start: the first iterate (nullptr: uniform); change: nullptr, or measure_partial_slots()
// / 2 doubles, zeroed by the caller, that receive per launch block the L1 change made by
// the last iteration (their sum is |v_iters - v_(iters-1)|_1)
cudaError_t invariant_measure(const uint32_t* tptr, const uint32_t* trows, const double* tvals,
                              const uint32_t* mid_list, uint32_t n_mid, const uint32_t* long_list, uint32_t n_long,
                              uint32_t n, uint32_t iters, double* w0, double* w1, double* partial,
                              uint32_t partial_cap, double* out, unsigned* sync_words, cudaStream_t s,
                              uint64_t nnz = 0, const double* start = nullptr, double* change = nullptr);
int measure_partial_slots();
// true when invariant_measure keeps a matrix of nnz entries whose longest row of P^T has
// max_row entries on chip (one block per SM; it then reads no row-class lists)
bool measure_on_chip(uint64_t nnz, uint32_t max_row, uint32_t partial_cap);
// *out = the longest row of the n rows of tptr (asynchronous)
cudaError_t max_row_length(const uint32_t* tptr, uint32_t n, uint32_t* out, cudaStream_t s);

}  // namespace b12g
