// Onesweep LSD radix sort of 64-bit keys (box codes), 8-bit digits, and the set
// operations the continuation needs on sorted code arrays: unique and merge.
//
// The sort follows the onesweep scheme of Adinets and Merrill ("Onesweep: A Faster
// Least Significant Digit Radix Sort for GPUs", 2022): one histogram pass counts every
// digit position of every key at once; then each digit takes ONE pass in which a tile
// of 4096 keys (tile number drawn from an atomic counter, so that lower tiles are always
// already running) ranks its keys stably in shared memory, publishes its per-digit
// count, stages its keys in digit order in shared memory, adds its predecessors' counts
// by decoupled look-back (a predecessor that has already published its inclusive prefix
// ends the walk), and writes its keys out from shared memory, so a warp's stores are
// runs of consecutive addresses.  Every look-back wait is bounded: a tile that gives up sets bit 2 of the
// caller's error word (the caller reports a timeout) and the result is not used.
// This replaces the reference's thrust::sort / sort_by_key on codes
// (helpFunctions.hpp:40-98 via sortBoxes, used by insertByIterators at
// ImplicitBoxTree.hpp:1832-1875).
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
constexpr int kMaxPasses = 8;
constexpr uint64_t kAggregate = 1ull << 62;       // status word: tile count published
constexpr uint64_t kInclusive = 2ull << 62;       // status word: inclusive prefix published
constexpr uint64_t kFlagMask = 3ull << 62;
constexpr uint32_t kLookbackPolls = 1u << 20;     // polls of one predecessor before giving up
// predecessor status words loaded together in the look-back: every tile of a wave
// publishes its counts at about the same time, so a tile walks back over the wave's
// earlier tiles until one has its inclusive prefix; 32 a round take the last tile of a
// wave of 296 (two blocks a SM) there in 4 rounds, 8 a round in 9
constexpr int kLookbackBatch = 32;

int grid_for(uint64_t work, int per_block, int blocks_per_sm)
{
  const uint64_t want = (work + per_block - 1) / per_block;
  const uint64_t cap = uint64_t(device_sm_count()) * blocks_per_sm;
  return int(want < 1 ? 1 : (want < cap ? want : cap));
}

// Scratch layout (u64 words): [status region 0: tiles x 256][status region 1: tiles x 256]
// [histograms: kMaxPasses x 256 (u32 pairs)][tile counters: kMaxPasses (u32)]
struct SortScratch
{
  uint64_t* status[2];
  uint32_t* hist;       // kMaxPasses x kBins
  uint32_t* counter;    // kMaxPasses
};

SortScratch carve(uint32_t* base, uint32_t tiles)
{
  SortScratch sc;
  uint64_t* w = reinterpret_cast<uint64_t*>(base);
  sc.status[0] = w;
  sc.status[1] = w + size_t(tiles) * kBins;
  sc.hist = reinterpret_cast<uint32_t*>(w + 2 * size_t(tiles) * kBins);
  sc.counter = sc.hist + kMaxPasses * kBins;
  return sc;
}

// every digit of every key, all passes at once (one read of the keys)
__global__ void __launch_bounds__(kThreads) onesweep_hist_kernel(const uint64_t* __restrict__ keys,
                                                                 const uint32_t* n_ptr, int passes, uint32_t* hist)
{
  __shared__ uint32_t h[kMaxPasses * kBins];
  for (int i = threadIdx.x; i < passes * kBins; i += kThreads) h[i] = 0;
  __syncthreads();
  const uint32_t n = *n_ptr;
  for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
    const uint64_t k = __ldg(keys + i);
    for (int p = 0; p < passes; ++p) atomicAdd(&h[p * kBins + int((k >> (8 * p)) & 0xFFu)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kBins; i += kThreads)
    if (h[i]) atomicAdd(hist + i, h[i]);
}

// exclusive scan of one value per thread over the block (256 threads)
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_sums)
{
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) warp_sums[w] = x;
  __syncthreads();
  uint32_t before = 0;
  for (int q = 0; q < w; ++q) before += warp_sums[q];
  __syncthreads();
  return before + x - v;
}

// key index of (warp w, round r, lane) within a tile: each warp owns 512 consecutive keys
__device__ __forceinline__ uint32_t tile_index(int w, int r, int lane) { return uint32_t(w * 512 + r * 32 + lane); }

template<bool kValues>
__global__ void __launch_bounds__(kThreads, 2) onesweep_pass_kernel(const uint64_t* __restrict__ keys,
                                                                 const uint32_t* __restrict__ vals,
                                                                 const uint32_t* n_ptr, int pass, SortScratch sc,
                                                                 uint64_t* out, uint32_t* vout, uint32_t* error)
{
  static_assert(kBins == kThreads, "one thread per digit");
  __shared__ uint32_t wcount[kWarps][kBins];   // per-warp digit counts, then per-warp digit bases in the tile
  __shared__ uint32_t s_gofs[kBins];           // global position of the tile's first key of digit d, minus
                                               // that key's staging index
  __shared__ uint32_t warp_sums[kWarps];
  __shared__ uint32_t s_tile;
  __shared__ __align__(16) uint64_t s_key[kTile];   // the tile in digit order (then its values, as u32)
  __shared__ uint8_t s_dig[kTile];                  // digit of each staged key

  const uint32_t n = *n_ptr;
  const uint32_t tiles = (n + kTile - 1) / kTile;
  if (threadIdx.x == 0) s_tile = atomicAdd(sc.counter + pass, 1u);
  for (int i = threadIdx.x; i < kWarps * kBins; i += kThreads) (&wcount[0][0])[i] = 0;
  __syncthreads();
  const uint32_t t = s_tile;
  if (t >= tiles) return;
  const int shift = 8 * pass;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t first = t * kTile;
  const uint32_t tile_n = min(kTile, n - first);

  // 1. stable ranks within each warp's 512 keys
  uint64_t key[kRounds];
  uint32_t val[kValues ? kRounds : 1];
  uint32_t rank[kRounds];
#pragma unroll
  for (int r = 0; r < kRounds; ++r) {             // all loads first: 16 in flight per thread
    const uint32_t li = tile_index(w, r, lane);
    key[r] = li < tile_n ? __ldcs(keys + first + li) : 0ull;
    if constexpr (kValues) val[r] = li < tile_n ? __ldcs(vals + first + li) : 0u;
  }
#pragma unroll
  for (int r = 0; r < kRounds; ++r) {
    const bool valid = tile_index(w, r, lane) < tile_n;
    const uint32_t d = valid ? uint32_t((key[r] >> shift) & 0xFFu) : 0xFFFFFFFFu;
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
    const uint32_t before = valid ? wcount[w][d] : 0u;
    rank[r] = before + __popc(peers & ((1u << lane) - 1u));
    __syncwarp();
    if (valid && lane == 31 - __clz(peers)) wcount[w][d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();

  // 2. thread d owns digit d: the tile's count, published at once for the successors
  const int d = threadIdx.x;
  uint32_t cnt = 0;
  for (int q = 0; q < kWarps; ++q) {
    const uint32_t c = wcount[q][d];
    wcount[q][d] = cnt;                  // the warp's first rank among the tile's keys of digit d
    cnt += c;
  }
  uint64_t* status = sc.status[pass & 1] + size_t(t) * kBins;
  {
    const uint64_t word = (t == 0 ? kInclusive : kAggregate) | cnt;
    __stcg(reinterpret_cast<unsigned long long*>(status + d), (unsigned long long)word);
  }
  // the other region is the next pass's: clear this tile's slots (the pass before, which
  // used it, has finished)
  __stcg(reinterpret_cast<unsigned long long*>(sc.status[(pass + 1) & 1] + size_t(t) * kBins + d), 0ull);
  const uint32_t digit_base = block_exclusive_scan(sc.hist[pass * kBins + d], warp_sums);
  const uint32_t tile_start = block_exclusive_scan(cnt, warp_sums);   // digit d's first staging index
  for (int q = 0; q < kWarps; ++q) wcount[q][d] += tile_start;
  __syncthreads();

  // 3. stage the tile in digit order (the positions are the tile's own), before the
  // look-back, so that the keys' registers are free while it runs
  uint32_t pos[kValues ? kRounds : 1];
#pragma unroll
  for (int r = 0; r < kRounds; ++r) {
    const uint32_t li = tile_index(w, r, lane);
    uint32_t p = kTile;
    if (li < tile_n) {
      const uint32_t dg = uint32_t((key[r] >> shift) & 0xFFu);
      p = wcount[w][dg] + rank[r];
      if (p < kTile) {
        s_key[p] = key[r];
        s_dig[p] = uint8_t(dg);
      }
    }
    if constexpr (kValues) pos[r] = p;
  }

  // 4. decoupled look-back over the preceding tiles for digit d, kLookbackBatch tiles at
  // a time: their status words are loaded together (one memory latency per batch, not
  // one per tile), then taken nearest first; a tile that has not published yet is polled
  // (bounded) before the walk goes past it
  uint32_t excl = 0;
  if (t > 0) {
    const uint64_t* region = sc.status[pass & 1] + d;
    int64_t j = int64_t(t) - 1;
    bool done = false;
    while (!done && j >= 0) {
      uint64_t v[kLookbackBatch];
#pragma unroll
      for (int q = 0; q < kLookbackBatch; ++q)
        v[q] = j - q >= 0 ? *reinterpret_cast<const volatile unsigned long long*>(region + size_t(j - q) * kBins)
                          : kInclusive;
#pragma unroll
      for (int q = 0; q < kLookbackBatch; ++q) {
        if (done) break;
        if (j - q < 0) { done = true; break; }
        const volatile unsigned long long* src =
            reinterpret_cast<const volatile unsigned long long*>(region + size_t(j - q) * kBins);
        uint32_t polls = 0;
        while ((v[q] & kFlagMask) == 0) {
          if (++polls > kLookbackPolls) break;
          v[q] = *src;
        }
        if ((v[q] & kFlagMask) == 0) { atomicOr(error, 2u); done = true; break; }
        excl += uint32_t(v[q]);
        if ((v[q] & kFlagMask) == kInclusive) done = true;
      }
      j -= kLookbackBatch;
    }
    __threadfence();
    __stcg(reinterpret_cast<unsigned long long*>(status + d), (unsigned long long)(kInclusive | (excl + cnt)));
  }
  s_gofs[d] = digit_base + excl - tile_start;
  __syncthreads();

  // 5. write runs of consecutive addresses
  // (a position past n would mean inconsistent counts: recorded as a capacity error, not written)
  for (uint32_t i = threadIdx.x; i < tile_n; i += kThreads) {
    const uint32_t g = s_gofs[s_dig[i]] + i;
    if (g < n) out[g] = s_key[i];
    else atomicOr(error, 1u);
  }
  if constexpr (kValues) {
    // the values take the same positions, staged in the keys' place
    uint32_t* s_val = reinterpret_cast<uint32_t*>(s_key);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRounds; ++r)
      if (pos[r] < kTile) s_val[pos[r]] = val[r];
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < tile_n; i += kThreads) {
      const uint32_t g = s_gofs[s_dig[i]] + i;
      if (g < n) vout[g] = s_val[i];
    }
  }
}

template<bool kValues>
cudaError_t onesweep(uint64_t* keys, uint64_t* alt, uint32_t* vals, uint32_t* valt, const uint32_t* n,
                     uint32_t max_n, int bits, uint32_t* scratch, uint32_t* error, uint64_t** sorted,
                     uint32_t** sorted_vals, cudaStream_t s)
{
  const uint32_t tiles = (max_n + kTile - 1) / kTile;
  const int passes = (bits + 7) / 8 < 1 ? 1 : ((bits + 7) / 8 > kMaxPasses ? kMaxPasses : (bits + 7) / 8);
  const SortScratch sc = carve(scratch, tiles);
  // status region 0 (the first pass's), histograms and tile counters start at zero
  cudaError_t e = cudaMemsetAsync(sc.status[0], 0, size_t(tiles) * kBins * sizeof(uint64_t), s);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(sc.hist, 0, (kMaxPasses * kBins + kMaxPasses) * sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  onesweep_hist_kernel<<<grid_for(max_n, kThreads * 16, 4), kThreads, 0, s>>>(keys, n, passes, sc.hist);
  uint64_t* src = keys;
  uint64_t* dst = alt;
  uint32_t* vsrc = vals;
  uint32_t* vdst = valt;
  const unsigned grid = tiles < 1 ? 1u : tiles;
  for (int p = 0; p < passes; ++p) {
    onesweep_pass_kernel<kValues><<<grid, kThreads, 0, s>>>(src, vsrc, n, p, sc, dst, vdst, error);
    std::swap(src, dst);
    if constexpr (kValues) std::swap(vsrc, vdst);
  }
  *sorted = src;
  if (sorted_vals) *sorted_vals = vsrc;
  return cudaGetLastError();
}

}  // namespace

uint64_t sort_scratch_u32(uint64_t max_n)
{
  const uint64_t tiles = (max_n + kTile - 1) / kTile;
  return 2 * (2 * tiles * kBins) + kMaxPasses * kBins + kMaxPasses + 4;
}

int sort_launches(int bits)
{
  const int passes = (bits + 7) / 8 < 1 ? 1 : ((bits + 7) / 8 > kMaxPasses ? kMaxPasses : (bits + 7) / 8);
  return 1 + passes;
}

cudaError_t radix_sort_u64(uint64_t* keys, uint64_t* alt, const uint32_t* n, uint32_t max_n, int bits,
                           uint32_t* scratch, uint32_t* error, uint64_t** sorted, cudaStream_t s)
{
  return onesweep<false>(keys, alt, nullptr, nullptr, n, max_n, bits, scratch, error, sorted, nullptr, s);
}

cudaError_t radix_sort_u64_values(uint64_t* keys, uint64_t* alt, uint32_t* vals, uint32_t* valt, const uint32_t* n,
                                  uint32_t max_n, int bits, uint32_t* scratch, uint32_t* error, uint64_t** sorted,
                                  uint32_t** sorted_vals, cudaStream_t s)
{
  return onesweep<true>(keys, alt, vals, valt, n, max_n, bits, scratch, error, sorted, sorted_vals, s);
}

namespace {

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

// Merge of two sorted code arrays (merge path: Odeh, Green, Mwassi, Shmueli, Birk,
// "Merge Path - Parallel Merging Made Simple", 2012).  The output is cut into tiles of
// kMergeTile positions; two warps of the tile's block find its first and last a-element
// by a 33-way co-rank search on the global arrays (a few rounds of loads, the range being
// at most the shorter array), the tile's a- and b-runs are staged in shared memory, every
// thread merges kMergeItems consecutive outputs after a co-rank search in shared memory
// and stores them with vector stores.  Equal keys take a first.  a's flags
// are ANDed with `a_keep`; b's entries get flags `fb`.
constexpr int kMergeThreads = 256;
constexpr int kMergeItems = 8;
constexpr uint32_t kMergeTile = kMergeThreads * kMergeItems;

// the number of a-elements among the first d outputs (one thread)
__device__ __forceinline__ uint32_t co_rank(const uint64_t* a, uint32_t na, const uint64_t* b, uint32_t nb, uint32_t d)
{
  uint32_t lo = d > nb ? d - nb : 0, hi = d < na ? d : na;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] <= b[d - 1 - mid]) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// the same by a whole warp: each round tests 32 evenly spaced candidates of the range
// (the predicate a[i] <= b[d-1-i] holds for a prefix of it) and keeps the gap where it
// turns false
__device__ __forceinline__ uint32_t co_rank_warp(const uint64_t* a, uint32_t na, const uint64_t* b, uint32_t nb,
                                                 uint32_t d, int lane)
{
  uint32_t lo = d > nb ? d - nb : 0, hi = d < na ? d : na;
  while (hi - lo > 32) {
    const uint64_t span = hi - lo;
    const uint32_t m = lo + uint32_t(span * uint64_t(lane + 1) / 33ull);     // lo <= m < hi, increasing
    const bool p = __ldg(a + m) <= __ldg(b + (d - 1 - m));
    const int c = __popc(__ballot_sync(0xFFFFFFFFu, p));
    const uint32_t m_lo = __shfl_sync(0xFFFFFFFFu, m, c > 0 ? c - 1 : 0);
    const uint32_t m_hi = __shfl_sync(0xFFFFFFFFu, m, c < 32 ? c : 31);
    if (c > 0) lo = m_lo + 1;
    if (c < 32) hi = m_hi;
  }
  const uint32_t m = lo + uint32_t(lane);
  const bool p = m < hi && __ldg(a + m) <= __ldg(b + (d - 1 - m));
  return lo + uint32_t(__popc(__ballot_sync(0xFFFFFFFFu, p)));
}

__global__ void __launch_bounds__(kMergeThreads) merge_path_kernel(const uint64_t* __restrict__ a,
                                                                   const uint8_t* __restrict__ fa,
                                                                   const uint32_t* na_ptr, uint8_t a_keep,
                                                                   const uint64_t* __restrict__ b, uint8_t fb,
                                                                   const uint32_t* nb_ptr,
                                                                   uint64_t* __restrict__ out,
                                                                   uint8_t* __restrict__ fout, uint32_t* n_out)
{
  __shared__ uint64_t s_in[kMergeTile];     // the tile's a-run, then its b-run
  __shared__ uint8_t s_fa[kMergeTile];
  __shared__ uint32_t s_split[2];
  const uint32_t na = *na_ptr, nb = *nb_ptr, total = na + nb;
  const uint32_t tiles = (total + kMergeTile - 1) / kMergeTile;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const uint32_t d0 = t * kMergeTile, d1 = min(d0 + kMergeTile, total);
    if (w < 2) {
      const uint32_t r = co_rank_warp(a, na, b, nb, w == 0 ? d0 : d1, lane);
      if (lane == 0) s_split[w] = r;
    }
    __syncthreads();
    const uint32_t i0 = s_split[0], i1 = s_split[1];
    const uint32_t j0 = d0 - i0, j1 = d1 - i1;
    const uint32_t la = i1 - i0, lb = j1 - j0;
    const uint32_t len = la + lb;
    // all loads of the tile first (kMergeItems per thread), then the shared-memory stores
    uint64_t v[kMergeItems];
    uint8_t f[kMergeItems];
#pragma unroll
    for (int q = 0; q < kMergeItems; ++q) {
      const uint32_t k = threadIdx.x + uint32_t(q) * kMergeThreads;
      v[q] = 0;
      f[q] = 0;
      if (k < la) {
        v[q] = __ldg(a + i0 + k);
        f[q] = __ldg(fa + i0 + k);
      } else if (k < len) {
        v[q] = __ldg(b + j0 + (k - la));
      }
    }
#pragma unroll
    for (int q = 0; q < kMergeItems; ++q) {
      const uint32_t k = threadIdx.x + uint32_t(q) * kMergeThreads;
      if (k < len) s_in[k] = v[q];
      if (k < la) s_fa[k] = f[q] & a_keep;
    }
    __syncthreads();
    const uint32_t dl = min(threadIdx.x * uint32_t(kMergeItems), len);
    uint32_t ia = co_rank(s_in, la, s_in + la, lb, dl);
    uint32_t ib = dl - ia;
    uint64_t o[kMergeItems];
    uint8_t of[kMergeItems];
#pragma unroll
    for (int q = 0; q < kMergeItems; ++q) {
      const bool take_a = ib >= lb || (ia < la && s_in[ia] <= s_in[la + ib]);
      o[q] = take_a ? s_in[ia < la ? ia : 0] : s_in[la + ib];
      of[q] = take_a ? s_fa[ia < la ? ia : 0] : fb;
      if (take_a) ++ia;
      else ++ib;
    }
    // a thread's outputs are consecutive: 16-byte stores of its codes, one 8-byte store of
    // its flags (tile starts are multiples of kMergeTile, so both are aligned)
    if (dl + kMergeItems <= len) {
      uint4* op = reinterpret_cast<uint4*>(out + d0 + dl);
#pragma unroll
      for (int q = 0; q < kMergeItems; q += 2)
        op[q / 2] = make_uint4(uint32_t(o[q]), uint32_t(o[q] >> 32), uint32_t(o[q + 1]), uint32_t(o[q + 1] >> 32));
      uint64_t fw = 0;
#pragma unroll
      for (int q = 0; q < kMergeItems; ++q) fw |= uint64_t(of[q]) << (8 * q);
      *reinterpret_cast<uint64_t*>(fout + d0 + dl) = fw;
    } else {
#pragma unroll
      for (int q = 0; q < kMergeItems; ++q)
        if (dl + q < len) {
          out[d0 + dl + q] = o[q];
          fout[d0 + dl + q] = of[q];
        }
    }
    __syncthreads();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = total;
}

}  // namespace

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

cudaError_t merge_sorted(const uint64_t* a, const uint8_t* fa, const uint32_t* na, uint8_t a_keep, const uint64_t* b,
                         uint8_t fb, const uint32_t* nb, uint32_t max_total, uint64_t* out, uint8_t* fout,
                         uint32_t* n_out, cudaStream_t s)
{
  const uint64_t tiles = (uint64_t(max_total) + kMergeTile - 1) / kMergeTile;
  const uint64_t cap = uint64_t(device_sm_count()) * 5;   // resident blocks a SM (48 registers)
  const unsigned grid = unsigned(tiles < 1 ? 1 : (tiles < cap ? tiles : cap));
  merge_path_kernel<<<grid, kMergeThreads, 0, s>>>(a, fa, na, a_keep, b, fb, nb, out, fout, n_out);
  return cudaGetLastError();
}

}  // namespace b12g
