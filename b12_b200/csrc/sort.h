// Radix sort and sorted-set operations on 64-bit box codes (sort.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace b12g {

// u32 cells of the sort's scratch (look-back status words, digit histograms, tile
// counters) for up to max_n keys; the scratch must be 8-byte aligned
uint64_t sort_scratch_u32(uint64_t max_n);

// kernel launches of one sort of `bits` bits (the histogram pass + one pass a digit)
int sort_launches(int bits);

// onesweep sort of the low `bits` bits of *n <= max_n keys; the result is in keys or alt
// (*sorted tells which).  scratch: sort_scratch_u32(max_n) u32.  A look-back that gives
// up sets bit 2 of *error (the result is then not sorted).
cudaError_t radix_sort_u64(uint64_t* keys, uint64_t* alt, const uint32_t* n, uint32_t max_n, int bits,
                           uint32_t* scratch, uint32_t* error, uint64_t** sorted, cudaStream_t s);

// the same with a u32 value per key moved along (stable); *sorted_vals tells where the
// values ended up (vals or valt)
cudaError_t radix_sort_u64_values(uint64_t* keys, uint64_t* alt, uint32_t* vals, uint32_t* valt, const uint32_t* n,
                                  uint32_t max_n, int bits, uint32_t* scratch, uint32_t* error, uint64_t** sorted,
                                  uint32_t** sorted_vals, cudaStream_t s);

// distinct values of a sorted array, in order; flag and pos: max_n + 1 u32
cudaError_t unique_sorted_u64(const uint64_t* keys, const uint32_t* n, uint32_t max_n, uint64_t* out, uint32_t* n_out,
                              uint32_t* flag, uint32_t* pos, uint32_t* scan_tiles, cudaStream_t s);

// merge two sorted arrays (equal values: a first); a's flags are ANDed with a_keep,
// entries of b get flags fb
cudaError_t merge_sorted(const uint64_t* a, const uint8_t* fa, const uint32_t* na, uint8_t a_keep, const uint64_t* b,
                         uint8_t fb, const uint32_t* nb, uint32_t max_total, uint64_t* out, uint8_t* fout,
                         uint32_t* n_out, cudaStream_t s);

}  // namespace b12g
