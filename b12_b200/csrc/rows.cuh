// Transition-row helpers shared by the single-tree and batched row kernels: a warp
// sorts the <= 128 target indices of one source box in shared memory and emits the
// row's (column, count) runs in column order.
#pragma once

#include "kernels.h"

namespace b12g {

__device__ __forceinline__ void warp_bitonic_128(uint32_t* s, int lane)
{
#pragma unroll 1
  for (int k = 2; k <= 128; k <<= 1) {
#pragma unroll 1
    for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int c = lane + 32 * q;                           // comparator 0..63
        const int i = ((c & ~(j - 1)) << 1) | (c & (j - 1));    // insert a zero bit at log2(j)
        const int l = i | j;
        const bool up = (i & k) == 0;
        const uint32_t x = s[i], y = s[l];
        if ((x > y) == up) { s[i] = y; s[l] = x; }
      }
      __syncwarp();
    }
  }
}

// The warp's 128 keys are in s (targets, kLostKey for points that left the domain,
// kPadKey beyond P).  Sorts them, writes the runs to col/cnt (at most P entries) and
// returns their number.  bounds: 4 words of the warp's shared memory.
__device__ __forceinline__ uint32_t row_emit_sorted(uint32_t* s, uint32_t* bounds, int lane, uint32_t P,
                                                    int keep_lost, uint32_t lost_col, uint32_t* col, uint32_t* cnt)
{
    if (lane < 4) bounds[lane] = 0;
    __syncwarp();
    warp_bitonic_128(s, lane);

    // run boundaries: position p starts a run if p == 0 or s[p] != s[p-1]
    uint32_t nib = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int p = lane * 4 + r;
      if (p == 0 || s[p] != s[p - 1]) nib |= 1u << r;
    }
    atomicOr(&bounds[lane >> 3], nib << ((lane & 7) * 4));
    __syncwarp();

    const uint32_t ws[4] = {bounds[0], bounds[1], bounds[2], bounds[3]};
    uint32_t cols[4], cnts[4], emit = 0;
    bool take[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int p = lane * 4 + r;
      const uint32_t key = s[p];
      take[r] = ((nib >> r) & 1u) && key != kPadKey && (key != kLostKey || keep_lost);
      // the run ends at the next boundary after p (or at P, where the padding starts)
      int end = int(P);
      bool found = false;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int first = q * 32, from = p + 1;
        if (found || from >= first + 32) continue;
        const uint32_t m = from > first ? ws[q] & (0xFFFFFFFFu << (from - first)) : ws[q];
        if (m) { end = min(int(P), first + __ffs(m) - 1); found = true; }
      }
      cols[r] = key == kLostKey ? lost_col : key;
      cnts[r] = uint32_t(end - p);
      emit += take[r] ? 1u : 0u;
    }
    // warp exclusive scan of emit counts
    uint32_t off = emit;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, off, d);
      if (lane >= d) off += v;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, off, 31);
    off -= emit;
#pragma unroll
    for (int r = 0; r < 4; ++r)
      if (take[r]) { col[off] = cols[r]; cnt[off] = cnts[r]; ++off; }
    __syncwarp();
    return total;
}

// The same runs, found by taking the warp's smallest remaining key and its count until
// none is left: a box's points fall into a few boxes (about 6.5 on average for Lorenz at
// depth 27), so this usually ends after a few rounds.  A row with more than kMinRounds
// distinct keys sorts the rest with row_emit_sorted.  Same arguments and results.
constexpr int kMinRounds = 16;

__device__ __forceinline__ uint32_t row_emit(uint32_t* s, uint32_t* bounds, int lane, uint32_t P, int keep_lost,
                                             uint32_t lost_col, uint32_t* col, uint32_t* cnt)
{
  __syncwarp();
  uint32_t k0 = s[lane], k1 = s[lane + 32], k2 = s[lane + 64], k3 = s[lane + 96];
  const uint32_t stop = keep_lost ? kPadKey : kLostKey;
  uint32_t total = 0;
#pragma unroll 1
  for (int round = 0; round < kMinRounds; ++round) {
    const uint32_t m = __reduce_min_sync(0xFFFFFFFFu, min(min(k0, k1), min(k2, k3)));
    if (m >= stop) return total;
    const uint32_t c = uint32_t(k0 == m) + uint32_t(k1 == m) + uint32_t(k2 == m) + uint32_t(k3 == m);
    const uint32_t count = __reduce_add_sync(0xFFFFFFFFu, c);
    if (lane == 0) {
      col[total] = m == kLostKey ? lost_col : m;
      cnt[total] = count;
    }
    ++total;
    k0 = k0 == m ? kPadKey : k0;
    k1 = k1 == m ? kPadKey : k1;
    k2 = k2 == m ? kPadKey : k2;
    k3 = k3 == m ? kPadKey : k3;
  }
  // many distinct keys: sort what is left (the keys taken are padding now)
  s[lane] = k0;
  s[lane + 32] = k1;
  s[lane + 64] = k2;
  s[lane + 96] = k3;
  __syncwarp();
  return total + row_emit_sorted(s, bounds, lane, P, keep_lost, lost_col, col + total, cnt + total);
}

}  // namespace b12g
