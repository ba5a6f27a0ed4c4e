// Leaf-array kernels: flag updates, subdivision split, stream compaction, scans.
// All kernels read element counts from device memory and run grid-stride loops over a
// persistent-sized grid, so a sequence of them needs no host round trip and can be
// captured in a CUDA graph.
#include <algorithm>

#include "kernels.h"

namespace b12g {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = kCompactTile / kThreads;  // 16 elements per thread per tile

__device__ __forceinline__ bool has_all(uint8_t f, uint8_t check) { return uint8_t(f & check) == check; }

// block-wide sum of one value per thread (all threads must call)
__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* red)
{
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, d);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  uint32_t t = 0;
  for (int i = 0; i < int(blockDim.x >> 5); ++i) t += red[i];
  return t;
}

// block-wide exclusive scan of one value per thread; returns the prefix, *total the sum
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t* red, uint32_t* total)
{
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
    if (lane >= d) x += y;
  }
  __syncthreads();
  if (lane == 31) red[w] = x;
  __syncthreads();
  uint32_t before = 0, all = 0;
  for (int i = 0; i < int(blockDim.x >> 5); ++i) {
    const uint32_t r = red[i];
    before += i < w ? r : 0u;
    all += r;
  }
  *total = all;
  return before + x - v;
}

int grid_for(uint64_t work, int per_block, int blocks_per_sm)
{
  const uint64_t want = (work + per_block - 1) / per_block;
  const uint64_t cap = uint64_t(device_sm_count()) * blocks_per_sm;
  return int(std::max<uint64_t>(1, std::min(want, cap)));
}

// ---------------------------------------------------------------------------------
__global__ void apply_hits_kernel(uint8_t* flags, uint8_t* hit, const uint32_t* n_ptr, uint8_t f, uint32_t* changed)
{
  __shared__ uint32_t red[32];
  const uint32_t n = *n_ptr;
  const uint32_t stride = gridDim.x * blockDim.x;
  uint32_t c = 0;
  const uint32_t iters = (n + stride - 1) / stride;
  for (uint32_t it = 0, i = blockIdx.x * blockDim.x + threadIdx.x; it < iters; ++it, i += stride) {
    if (i < n && hit[i]) {
      const uint8_t old = flags[i];
      c += has_all(old, f) ? 0u : 1u;
      flags[i] = old | f;
      hit[i] = 0;
    }
  }
  c = block_sum(c, red);
  if (threadIdx.x == 0 && c) atomicAdd(changed, c);
}

// op 0: set f (count boxes lacking f); 1: unset f (count boxes having any of f);
// 2: change u -> f (count boxes having all of u)
__global__ void flag_op_kernel(uint8_t* flags, const uint32_t* n_ptr, int op, uint8_t u, uint8_t f, uint32_t* changed)
{
  __shared__ uint32_t red[32];
  const uint32_t n = *n_ptr;
  const uint32_t stride = gridDim.x * blockDim.x;
  uint32_t c = 0;
  const uint32_t iters = (n + stride - 1) / stride;
  for (uint32_t it = 0, i = blockIdx.x * blockDim.x + threadIdx.x; it < iters; ++it, i += stride) {
    if (i >= n) continue;
    const uint8_t old = flags[i];
    if (op == 0) { c += has_all(old, f) ? 0u : 1u; flags[i] = old | f; }
    else if (op == 1) { c += (old & f) ? 1u : 0u; flags[i] = old & uint8_t(~f); }
    else if (has_all(old, u)) { ++c; flags[i] = uint8_t((old & ~u) | f); }
  }
  c = block_sum(c, red);
  if (threadIdx.x == 0 && c && changed) atomicAdd(changed, c);
}

__global__ void count_flags_kernel(const uint8_t* flags, const uint32_t* n_ptr, uint8_t f, uint32_t* count)
{
  __shared__ uint32_t red[32];
  const uint32_t n = *n_ptr;
  const uint32_t stride = gridDim.x * blockDim.x;
  uint32_t c = 0;
  const uint32_t iters = (n + stride - 1) / stride;
  for (uint32_t it = 0, i = blockIdx.x * blockDim.x + threadIdx.x; it < iters; ++it, i += stride)
    if (i < n && has_all(flags[i], f)) ++c;
  c = block_sum(c, red);
  if (threadIdx.x == 0 && c) atomicAdd(count, c);
}

// subdivide: incrementDepthBy(1) + computeOtherHalf (Box.hpp:140-147, 234-239); the
// children of a sorted parent array, written adjacently, are sorted
__global__ void split_kernel(const uint64_t* code, const uint8_t* flags, const uint32_t* n_ptr, uint64_t* out_code,
                             uint8_t* out_flags, uint32_t* n_out)
{
  const uint32_t n = *n_ptr;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t c = code[i] << 1;
    const uint8_t f = flags[i];
    reinterpret_cast<ulonglong2*>(out_code)[i] = make_ulonglong2(c, c | 1u);
    out_flags[2 * i] = f;
    out_flags[2 * i + 1] = f;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = 2 * n;
}

// ---------------------------------------------------------------------------------
// leaf lookup table: linear-probing inserts with a 64-bit CAS on the key word (guessing
// an empty slot is zero, else retrying with the old-tag value the CAS returned); a CAS
// that loses to another insert sees the current tag and moves on, so every insert ends
// within the table size
// ---------------------------------------------------------------------------------
// The keys are the leaves' packed per-dimension indices (pack_bits at `depth`), also
// written to h.pk for the image kernels.
template<int D>
__global__ void hash_build_kernel(const uint64_t* codes, const uint32_t* n_ptr, int depth, LeafHash h,
                                  uint32_t* error)
{
  const uint32_t n = *n_ptr;
  const int l = table_log2(h, n);
  if (l > int(h.log2_cap)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(error, 1u);
    return;
  }
  const uint64_t mask = (1ull << l) - 1ull;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint64_t code = codes[i];
    uint32_t bits[D];
#pragma unroll
    for (int j = 0; j < D; ++j) bits[j] = deinterleave<D>(code, depth, j);
    const uint64_t pk = pack_bits<D>(bits, depth);
    h.pk[i] = pk;
    const unsigned long long key = (uint64_t(h.tag) << 56) | pk;
    uint64_t s = hash_slot(pk, l);
    bool done = false;
    unsigned long long expect = 0;   // first guess for a slot: never used
    for (uint64_t step = 0; step <= 2 * mask + 64 && !done; ++step) {
      unsigned long long* kw = reinterpret_cast<unsigned long long*>(&h.slots[s].x);
      const unsigned long long cur = atomicCAS(kw, expect, key);
      if (cur == expect) {           // an empty slot (tag 0 or an old tag) now holds the key
        h.slots[s].y = i;
        done = true;
      } else if ((cur >> 56) != h.tag) {
        expect = cur;                // empty under an old tag: try it again with its value
      } else {
        s = (s + 1) & mask;
        expect = 0;
      }
    }
    if (!done) atomicOr(error, 1u);
  }
}

// ---------------------------------------------------------------------------------
// compaction: tile counts -> single-block tile scan -> ordered scatter
// ---------------------------------------------------------------------------------
// element count; 0 (with error bit 0) if the children do not fit the hit mask
__device__ __forceinline__ uint32_t compact_n(const CompactArgs& a)
{
  if (!a.children) return *a.n;
  const uint64_t c = 2ull * *a.n;
  return c <= a.hit_cap ? uint32_t(c) : 0u;
}

// Each thread owns a run of 16 consecutive elements (kItems), so a tile of kCompactTile
// elements is one pass of the block: the keep bits of a run come from one 16-byte load
// of the hit mask (children) or of the flags, and the block needs one scan per tile.
static_assert(kItems == 16, "a thread's run is one 16-byte vector of mask bytes");

// keep bits of the run starting at `base` (bit j: element base + j)
__device__ __forceinline__ uint32_t run_mask(const CompactArgs& a, uint32_t base, uint32_t n, bool vec)
{
  const uint8_t* src = a.children ? a.hit : a.flags;
  uint32_t m = 0;
  if (vec && base + 16 <= n) {
    const uint4 v = *reinterpret_cast<const uint4*>(src + base);
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const uint8_t byte = uint8_t(w[j >> 2] >> (8 * (j & 3)));
      const bool keep = a.children ? byte != 0 : has_all(byte, a.keep_flags);
      m |= uint32_t(keep) << j;
    }
  } else {
    for (int j = 0; j < 16; ++j) {
      const uint32_t i = base + j;
      if (i >= n) break;
      const bool keep = a.children ? src[i] != 0 : has_all(src[i], a.keep_flags);
      m |= uint32_t(keep) << j;
    }
  }
  return m;
}

__global__ void __launch_bounds__(kThreads) compact_count_kernel(const CompactArgs a, uint32_t* tile_counts)
{
  __shared__ uint32_t red[32];
  const uint32_t n = compact_n(a);
  const uint32_t tiles = (n + kCompactTile - 1) / kCompactTile;
  const bool vec = a.vec != 0;
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const uint32_t base = t * kCompactTile + threadIdx.x * kItems;
    const uint32_t c = __popc(run_mask(a, base, n, vec));
    const uint32_t total = block_sum(c, red);
    if (threadIdx.x == 0) tile_counts[t] = total;
  }
}

// one block: exclusive scan of the tile counts; total -> *n_out.  Each thread sums a
// contiguous group of tiles first, so the block scans once.
// the compaction's totals once the survivors' count (carry) is known: the counts, the
// last rank and the capacity check (one thread)
__device__ __forceinline__ void compact_finish(const CompactArgs& a, uint32_t n, uint32_t carry)
{
  if (carry > a.out_cap || (a.children && 2ull * *a.n > a.hit_cap)) atomicOr(a.error, 1u);
  if (a.out_rank) a.out_rank[n] = carry;
  if (carry > a.out_cap) carry = a.out_cap;
  *a.n_out = carry;
  if (a.n_out2) *a.n_out2 = carry;
}

__global__ void compact_scan_kernel(const CompactArgs a, const uint32_t* tile_counts, uint32_t* tile_offsets)
{
  __shared__ uint32_t red[32];
  const uint32_t n = compact_n(a);
  const uint32_t tiles = (n + kCompactTile - 1) / kCompactTile;
  const uint32_t per = (tiles + blockDim.x - 1) / blockDim.x;
  const uint32_t first = threadIdx.x * per, last = min(tiles, first + per);
  uint32_t mine = 0;
  for (uint32_t t = first; t < last; ++t) mine += tile_counts[t];
  uint32_t carry;
  uint32_t off = block_exclusive(mine, red, &carry);
  for (uint32_t t = first; t < last; ++t) {
    const uint32_t v = tile_counts[t];
    tile_offsets[t] = off;
    off += v;
  }
  if (threadIdx.x == 0) compact_finish(a, n, carry);
}

// survivors of a tile staged in shared memory in order, then written out coalesced.
// tile_offsets null: each block sums the counts of the tiles before its own (few tiles),
// and the block of the last tile writes the totals the scan kernel would have
__global__ void __launch_bounds__(kThreads) compact_scatter_kernel(const CompactArgs a, const uint32_t* tile_offsets,
                                                                   const uint32_t* tile_counts)
{
  __shared__ uint32_t red[32];
  __shared__ uint64_t s_code[kCompactTile];     // codes, or kept indices in out_index mode
  __shared__ uint8_t s_flags[kCompactTile];
  const uint32_t n = compact_n(a);
  const uint32_t tiles = (n + kCompactTile - 1) / kCompactTile;
  const bool vec = a.vec != 0;
  if (!tile_offsets && tiles == 0 && blockIdx.x == 0 && threadIdx.x == 0) compact_finish(a, n, 0);
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    uint32_t off;
    if (tile_offsets) {
      off = tile_offsets[t];
    } else {
      uint32_t b = 0;
      for (uint32_t q = threadIdx.x; q < t; q += kThreads) b += tile_counts[q];
      off = block_sum(b, red);
    }
    const uint32_t base = t * kCompactTile + threadIdx.x * kItems;
    const uint32_t m = run_mask(a, base, n, vec);
    uint32_t total;
    uint32_t at = block_exclusive(__popc(m), red, &total);
    if (!tile_offsets && t + 1 == tiles && threadIdx.x == 0) compact_finish(a, n, off + total);
    if (a.out_rank) {
      // rank of element base + j: survivors before it
      uint32_t r[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) r[j] = off + at + __popc(m & ((1u << j) - 1u));
      if (base + 16 <= n && vec) {
        uint4* dst = reinterpret_cast<uint4*>(a.out_rank + base);
#pragma unroll
        for (int q = 0; q < 4; ++q) dst[q] = make_uint4(r[4 * q], r[4 * q + 1], r[4 * q + 2], r[4 * q + 3]);
      } else {
        for (int j = 0; j < 16 && base + j < n; ++j) a.out_rank[base + j] = r[j];
      }
    }
    if (a.children) {
      // the mask is consumed: clear it for the next step
      if (base + 16 <= n && vec) *reinterpret_cast<uint4*>(a.hit + base) = make_uint4(0, 0, 0, 0);
      else
        for (int j = 0; j < 16 && base + j < n; ++j) a.hit[base + j] = 0;
    }
    // stage this run's survivors at their tile positions
    uint32_t mm = m;
    if (a.children && !a.out_index && vec && m && base + 16 <= n) {
      // the run's 8 parents: 64 bytes of codes and 8 of flags in four + one vector loads
      const uint4* pc = reinterpret_cast<const uint4*>(a.code + (base >> 1));
      uint64_t pcode[8];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint4 v = pc[q];
        pcode[2 * q] = (uint64_t(v.y) << 32) | v.x;
        pcode[2 * q + 1] = (uint64_t(v.w) << 32) | v.z;
      }
      const uint2 fv = *reinterpret_cast<const uint2*>(a.flags + (base >> 1));
      const uint8_t keep_mask = uint8_t(~a.clear_flags);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        if (!((m >> j) & 1u)) continue;
        const uint32_t fw = (j >> 1) < 4 ? fv.x : fv.y;
        s_code[at] = (pcode[j >> 1] << 1) | uint64_t(j & 1);
        s_flags[at] = uint8_t(fw >> (8 * ((j >> 1) & 3))) & keep_mask;
        ++at;
      }
      mm = 0;
    }
    while (mm) {
      const int j = __ffs(mm) - 1;
      const uint32_t i = base + j;
      if (a.out_index) {
        s_code[at] = i;
      } else if (a.children) {
        s_code[at] = (a.code[i >> 1] << 1) | uint64_t(i & 1u);
        s_flags[at] = a.flags[i >> 1] & uint8_t(~a.clear_flags);
      } else {
        s_code[at] = a.code[i];
        s_flags[at] = a.flags[i] & uint8_t(~a.clear_flags);
      }
      ++at;
      mm &= mm - 1;
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < total; x += kThreads) {
      const uint32_t pos = off + x;
      if (pos >= a.out_cap) break;
      if (a.out_index) {
        a.out_index[pos] = uint32_t(s_code[x]);
      } else {
        a.out_code[pos] = s_code[x];
        a.out_flags[pos] = s_flags[x];
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------
// exclusive scan u32 -> u32 with out[n] = total
// ---------------------------------------------------------------------------------
__global__ void scan_tiles_kernel(const uint32_t* in, const uint32_t* n_ptr, uint32_t* tile_sums)
{
  __shared__ uint32_t red[32];
  const uint32_t n = *n_ptr;
  const uint32_t tiles = (n + kCompactTile - 1) / kCompactTile;
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    uint32_t c = 0;
    for (int k = 0; k < kItems; ++k) {
      const uint32_t i = t * kCompactTile + k * kThreads + threadIdx.x;
      if (i < n) c += in[i];
    }
    c = block_sum(c, red);
    if (threadIdx.x == 0) tile_sums[t] = c;
  }
}

__global__ void scan_tile_offsets_kernel(const uint32_t* n_ptr, uint32_t* tile_sums, uint32_t* out)
{
  __shared__ uint32_t red[32];
  const uint32_t n = *n_ptr;
  const uint32_t tiles = (n + kCompactTile - 1) / kCompactTile;
  uint32_t carry = 0;
  for (uint32_t base = 0; base < tiles; base += blockDim.x) {
    const uint32_t t = base + threadIdx.x;
    const uint32_t v = t < tiles ? tile_sums[t] : 0u;
    uint32_t total;
    const uint32_t ex = block_exclusive(v, red, &total);
    __syncthreads();
    if (t < tiles) tile_sums[t] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) out[n] = carry;
}

// each thread takes 16 consecutive elements of the tile (four 16-byte loads when `vec`:
// both arrays 16-byte aligned), so a tile costs one block scan of the threads' sums
__global__ void scan_down_kernel(const uint32_t* in, const uint32_t* n_ptr, const uint32_t* tile_offsets, uint32_t* out,
                                 int vec)
{
  __shared__ uint32_t red[32];
  const uint32_t n = *n_ptr;
  const uint32_t tiles = (n + kCompactTile - 1) / kCompactTile;
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const uint32_t i0 = t * kCompactTile + threadIdx.x * kItems;
    const bool whole = vec && i0 + kItems <= n;
    uint32_t v[kItems];
    if (whole) {
#pragma unroll
      for (int q = 0; q < kItems / 4; ++q) {
        const uint4 x = reinterpret_cast<const uint4*>(in + i0)[q];
        v[4 * q] = x.x;
        v[4 * q + 1] = x.y;
        v[4 * q + 2] = x.z;
        v[4 * q + 3] = x.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < kItems; ++k) v[k] = i0 + k < n ? in[i0 + k] : 0u;
    }
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k) sum += v[k];
    uint32_t total;
    uint32_t run = tile_offsets[t] + block_exclusive(sum, red, &total);
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
      const uint32_t x = v[k];
      v[k] = run;
      run += x;
    }
    if (whole) {
#pragma unroll
      for (int q = 0; q < kItems / 4; ++q)
        reinterpret_cast<uint4*>(out + i0)[q] = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    } else {
#pragma unroll
      for (int k = 0; k < kItems; ++k)
        if (i0 + k < n) out[i0 + k] = v[k];
    }
  }
}

}  // namespace

int device_sm_count()
{
  static int sms[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (!sms[dev]) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    sms[dev] = v > 0 ? v : 1;
  }
  return sms[dev];
}

cudaError_t apply_hits(uint8_t* flags, uint8_t* hit, const uint32_t* n, uint8_t f, uint32_t* changed, uint32_t max_n,
                       cudaStream_t s)
{
  apply_hits_kernel<<<grid_for(max_n, kThreads, 8), kThreads, 0, s>>>(flags, hit, n, f, changed);
  return cudaGetLastError();
}

cudaError_t flag_op(uint8_t* flags, const uint32_t* n, int op, uint8_t u, uint8_t f, uint32_t* changed,
                    uint32_t max_n, cudaStream_t s)
{
  flag_op_kernel<<<grid_for(max_n, kThreads, 8), kThreads, 0, s>>>(flags, n, op, u, f, changed);
  return cudaGetLastError();
}

cudaError_t count_flags(const uint8_t* flags, const uint32_t* n, uint8_t f, uint32_t* count, uint32_t max_n,
                        cudaStream_t s)
{
  count_flags_kernel<<<grid_for(max_n, kThreads, 8), kThreads, 0, s>>>(flags, n, f, count);
  return cudaGetLastError();
}

cudaError_t split_codes(const uint64_t* code, const uint8_t* flags, const uint32_t* n, uint64_t* out_code,
                        uint8_t* out_flags, uint32_t* n_out, uint32_t max_n, cudaStream_t s)
{
  split_kernel<<<grid_for(max_n, kThreads, 8), kThreads, 0, s>>>(code, flags, n, out_code, out_flags, n_out);
  return cudaGetLastError();
}

cudaError_t build_leaf_hash(const uint64_t* codes, const uint32_t* n, int depth, int dim, LeafHash h, uint32_t* error,
                            uint32_t max_n, cudaStream_t s)
{
  const int g = grid_for(max_n, kThreads, 8);
  switch (dim) {
    case 2: hash_build_kernel<2><<<g, kThreads, 0, s>>>(codes, n, depth, h, error); break;
    case 3: hash_build_kernel<3><<<g, kThreads, 0, s>>>(codes, n, depth, h, error); break;
    case 4: hash_build_kernel<4><<<g, kThreads, 0, s>>>(codes, n, depth, h, error); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}


constexpr uint64_t kLocalScanTiles = 4096;

int compact_launches(bool children, uint32_t max_in)
{
  const uint64_t elems = children ? 2ull * max_in : uint64_t(max_in);
  return (elems + kCompactTile - 1) / kCompactTile <= kLocalScanTiles ? 2 : 3;
}

cudaError_t compact(const CompactArgs& args, const CompactScratch& sc, uint32_t max_in, cudaStream_t s)
{
  CompactArgs a = args;
  // 16-byte runs of the mask and of the ranks need 16-byte aligned arrays
  const uintptr_t mask = uintptr_t(a.children ? static_cast<const void*>(a.hit) : a.flags);
  a.vec = (mask % 16 == 0 && uintptr_t(a.out_rank) % 16 == 0 && uintptr_t(a.code) % 16 == 0 &&
           uintptr_t(a.flags) % 8 == 0) ? 1 : 0;
  const uint64_t elems = a.children ? 2ull * max_in : uint64_t(max_in);
  const int g = grid_for(elems, kCompactTile, 4);
  compact_count_kernel<<<g, kThreads, 0, s>>>(a, sc.tile_counts);
  // up to kLocalScanTiles tiles every scatter block sums the counts before its tile
  // itself (at most 16 loads a thread): no scan launch between the two
  const bool local = (elems + kCompactTile - 1) / kCompactTile <= kLocalScanTiles;
  if (!local) compact_scan_kernel<<<1, 1024, 0, s>>>(a, sc.tile_counts, sc.tile_offsets);
  compact_scatter_kernel<<<g, kThreads, 0, s>>>(a, local ? nullptr : sc.tile_offsets, sc.tile_counts);
  return cudaGetLastError();
}

cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, const uint32_t* n, uint32_t* tile_sums,
                               uint32_t max_n, cudaStream_t s)
{
  const int g = grid_for(max_n, kCompactTile, 4);
  scan_tiles_kernel<<<g, kThreads, 0, s>>>(in, n, tile_sums);
  scan_tile_offsets_kernel<<<1, 1024, 0, s>>>(n, tile_sums, out);
  const int vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15u) == 0;
  scan_down_kernel<<<g, kThreads, 0, s>>>(in, n, tile_sums, out, vec);
  return cudaGetLastError();
}

}  // namespace b12g
