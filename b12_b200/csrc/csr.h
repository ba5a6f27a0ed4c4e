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

// power iteration on the CSR of P^T; sync_words: 3 u32 (barrier count, generation,
// error: bit 1 = barrier timeout); partial: partial_cap doubles
cudaError_t invariant_measure(const uint32_t* tptr, const uint32_t* trows, const double* tvals, uint32_t n,
                              uint32_t iters, double* w0, double* w1, double* partial, uint32_t partial_cap,
                              double* out, unsigned* sync_words, cudaStream_t s);
int measure_partial_slots();

}  // namespace b12g
