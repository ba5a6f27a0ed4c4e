// LSD radix sort of 64-bit keys (box codes), 8-bit digits, and the set operations the
// continuation needs on sorted code arrays: unique and merge.
//
// One pass over a digit = three steps: every 4096-key tile counts its digits
// (histogram kernel), the digit-major table of tile counts is scanned, and every tile
// scatters its keys, stably ranked within the tile (warp ballots on equal digits in
// key order, then a prefix over the tile's warps).  This replaces the reference's
// thrust::sort / sort_by_key on codes (helpFunctions.hpp:40-98 via sortBoxes, used by
// insertByIterators at ImplicitBoxTree.hpp:1832-1875).
#include <utility>

#include "kernels.h"
#include "sort.h"

namespace b12g {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kRounds = 16;                       // keys per thread per tile
constexpr uint32_t kTile = kThreads * kRounds;    // 4096
constexpr int kBins = 256;

int grid_for(uint64_t work, int per_block, int blocks_per_sm)
{
  const uint64_t want = (work + per_block - 1) / per_block;
  const uint64_t cap = uint64_t(device_sm_count()) * blocks_per_sm;
  return int(want < 1 ? 1 : (want < cap ? want : cap));
}

// key index of (warp w, round r, lane) within a tile: each warp owns 512 consecutive keys
__device__ __forceinline__ uint32_t tile_index(int w, int r, int lane) { return uint32_t(w * 512 + r * 32 + lane); }

__global__ void __launch_bounds__(kThreads) digit_hist_kernel(const uint64_t* keys, const uint32_t* n_ptr, int shift,
                                                              uint32_t* tile_hist)
{
  __shared__ uint32_t h[kBins];
  const uint32_t n = *n_ptr;
  const uint32_t tiles = (n + kTile - 1) / kTile;
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    for (int i = threadIdx.x; i < kBins; i += kThreads) h[i] = 0;
    __syncthreads();
    for (int r = 0; r < kRounds; ++r) {
      const uint32_t i = t * kTile + r * kThreads + threadIdx.x;
      if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xFFu], 1u);
    }
    __syncthreads();
    // digit-major: all tiles of digit 0, then digit 1, ...
    for (int d = threadIdx.x; d < kBins; d += kThreads) tile_hist[size_t(d) * tiles + t] = h[d];
    __syncthreads();
  }
}

template<bool kValues>
__global__ void __launch_bounds__(kThreads) digit_scatter_kernel(const uint64_t* keys, const uint32_t* vals,
                                                                 const uint32_t* n_ptr, int shift,
                                                                 const uint32_t* offsets, uint64_t* out,
                                                                 uint32_t* vout)
{
  __shared__ uint32_t wcount[kWarps][kBins];     // per-warp running digit counts
  __shared__ uint32_t wbase[kWarps][kBins];      // exclusive prefix over warps, + tile offset
  const uint32_t n = *n_ptr;
  const uint32_t tiles = (n + kTile - 1) / kTile;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    for (int i = threadIdx.x; i < kWarps * kBins; i += kThreads) (&wcount[0][0])[i] = 0;
    __syncthreads();
    uint64_t key[kRounds];
    uint32_t val[kValues ? kRounds : 1];
    uint32_t rank[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
      const uint32_t i = t * kTile + tile_index(w, r, lane);
      const bool valid = i < n;
      key[r] = valid ? keys[i] : 0ull;
      if constexpr (kValues) val[r] = valid ? vals[i] : 0u;
      const uint32_t d = valid ? uint32_t((key[r] >> shift) & 0xFFu) : 0xFFFFFFFFu;
      const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
      const uint32_t before = valid ? wcount[w][d] : 0u;
      rank[r] = before + __popc(peers & ((1u << lane) - 1u));
      __syncwarp();
      if (valid && lane == 31 - __clz(peers)) wcount[w][d] = before + __popc(peers);
      __syncwarp();
    }
    __syncthreads();
    // prefix over the tile's warps per digit, plus the global offset of this tile's digit
    for (int d = threadIdx.x; d < kBins; d += kThreads) {
      uint32_t run = offsets[size_t(d) * tiles + t];
      for (int q = 0; q < kWarps; ++q) {
        wbase[q][d] = run;
        run += wcount[q][d];
      }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
      const uint32_t i = t * kTile + tile_index(w, r, lane);
      if (i < n) {
        const uint32_t p = wbase[w][(key[r] >> shift) & 0xFFu] + rank[r];
        out[p] = key[r];
        if constexpr (kValues) vout[p] = val[r];
      }
    }
    __syncthreads();
  }
}

// unique of a sorted array: flag heads, scan, scatter
__global__ void head_flag_kernel(const uint64_t* keys, const uint32_t* n_ptr, uint32_t* flag)
{
  const uint32_t n = *n_ptr;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void head_scatter_kernel(const uint64_t* keys, const uint32_t* n_ptr, const uint32_t* pos, uint64_t* out,
                                    uint32_t* n_out)
{
  const uint32_t n = *n_ptr;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (i == 0 || keys[i] != keys[i - 1]) out[pos[i]] = keys[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = pos[n];
}

// merge of two sorted, disjoint code arrays by rank: a[i] goes to i + |{b < a[i]}|,
// b[j] to j + |{a < b[j]}|; the new entries (b) get flags `fb`
__device__ __forceinline__ uint32_t lower_bound_u64(const uint64_t* v, uint32_t n, uint64_t x)
{
  uint32_t lo = 0, len = n;
  while (len > 0) {
    const uint32_t half = len >> 1;
    if (v[lo + half] < x) { lo += half + 1; len -= half + 1; }
    else len = half;
  }
  return lo;
}

__global__ void merge_kernel(const uint64_t* a, const uint8_t* fa, const uint32_t* na_ptr, const uint64_t* b,
                             uint8_t fb, const uint32_t* nb_ptr, uint64_t* out, uint8_t* fout, uint32_t* n_out)
{
  const uint32_t na = *na_ptr, nb = *nb_ptr;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < na + nb; i += stride) {
    if (i < na) {
      const uint32_t p = i + lower_bound_u64(b, nb, a[i]);
      out[p] = a[i];
      fout[p] = fa[i];
    } else {
      const uint32_t j = i - na;
      const uint32_t p = j + lower_bound_u64(a, na, b[j]);
      out[p] = b[j];
      fout[p] = fb;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = na + nb;
}

__global__ void set_u32_kernel(uint32_t* p, uint32_t v) { *p = v; }

}  // namespace

uint64_t sort_scratch_u32(uint64_t max_n)
{
  const uint64_t tiles = (max_n + kTile - 1) / kTile;
  return tiles * kBins + 1;
}

cudaError_t radix_sort_u64(uint64_t* keys, uint64_t* alt, const uint32_t* n, uint32_t max_n, int bits,
                           uint32_t* hist, uint32_t* offsets, uint32_t* scan_tiles, uint32_t* count_tmp,
                           uint64_t** sorted, cudaStream_t s)
{
  // *n must equal max_n: the digit-major table has 256 x tiles(max_n) cells, and
  // count_tmp[0] tells the scan how many
  const uint32_t tiles = (max_n + kTile - 1) / kTile;
  set_u32_kernel<<<1, 1, 0, s>>>(count_tmp, tiles * kBins);
  const int g = grid_for(uint64_t(tiles) * kTile, kTile, 4);
  uint64_t* src = keys;
  uint64_t* dst = alt;
  for (int shift = 0; shift < bits; shift += 8) {
    digit_hist_kernel<<<g, kThreads, 0, s>>>(src, n, shift, hist);
    cudaError_t e = exclusive_scan_u32(hist, offsets, count_tmp, scan_tiles, uint32_t(tiles) * kBins, s);
    if (e != cudaSuccess) return e;
    digit_scatter_kernel<false><<<g, kThreads, 0, s>>>(src, nullptr, n, shift, offsets, dst, nullptr);
    uint64_t* t = src;
    src = dst;
    dst = t;
  }
  *sorted = src;
  return cudaGetLastError();
}

cudaError_t radix_sort_u64_values(uint64_t* keys, uint64_t* alt, uint32_t* vals, uint32_t* valt, const uint32_t* n,
                                  uint32_t max_n, int bits, uint32_t* hist, uint32_t* offsets, uint32_t* scan_tiles,
                                  uint32_t* count_tmp, uint64_t** sorted, uint32_t** sorted_vals, cudaStream_t s)
{
  const uint32_t tiles = (max_n + kTile - 1) / kTile;
  set_u32_kernel<<<1, 1, 0, s>>>(count_tmp, tiles * kBins);
  const int g = grid_for(uint64_t(tiles) * kTile, kTile, 4);
  uint64_t* src = keys;
  uint64_t* dst = alt;
  uint32_t* vsrc = vals;
  uint32_t* vdst = valt;
  for (int shift = 0; shift < bits; shift += 8) {
    digit_hist_kernel<<<g, kThreads, 0, s>>>(src, n, shift, hist);
    cudaError_t e = exclusive_scan_u32(hist, offsets, count_tmp, scan_tiles, uint32_t(tiles) * kBins, s);
    if (e != cudaSuccess) return e;
    digit_scatter_kernel<true><<<g, kThreads, 0, s>>>(src, vsrc, n, shift, offsets, dst, vdst);
    std::swap(src, dst);
    std::swap(vsrc, vdst);
  }
  *sorted = src;
  *sorted_vals = vsrc;
  return cudaGetLastError();
}

cudaError_t unique_sorted_u64(const uint64_t* keys, const uint32_t* n, uint32_t max_n, uint64_t* out, uint32_t* n_out,
                              uint32_t* flag, uint32_t* pos, uint32_t* scan_tiles, cudaStream_t s)
{
  const int g = grid_for(max_n, kThreads, 8);
  head_flag_kernel<<<g, kThreads, 0, s>>>(keys, n, flag);
  cudaError_t e = exclusive_scan_u32(flag, pos, n, scan_tiles, max_n, s);
  if (e != cudaSuccess) return e;
  head_scatter_kernel<<<g, kThreads, 0, s>>>(keys, n, pos, out, n_out);
  return cudaGetLastError();
}

cudaError_t merge_sorted(const uint64_t* a, const uint8_t* fa, const uint32_t* na, const uint64_t* b, uint8_t fb,
                         const uint32_t* nb, uint32_t max_total, uint64_t* out, uint8_t* fout, uint32_t* n_out,
                         cudaStream_t s)
{
  merge_kernel<<<grid_for(max_total, kThreads, 8), kThreads, 0, s>>>(a, fa, na, b, fb, nb, out, fout, n_out);
  return cudaGetLastError();
}

}  // namespace b12g
