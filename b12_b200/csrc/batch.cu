// Batched subdivision: many independent instances of the subdivision loop
// (subdivision.m:18-45) - one map kind and grid, per-instance map parameters and
// depths - advanced in lockstep, one persistent launch per subdivision step for all of
// them.
//
// Layout: instances are ordered by depth, deepest first, so the instances still
// subdividing at step k are a prefix of the order.  Their leaves are concatenated in
// one code array with per-instance offsets.  A step runs:
//   1. a lookup table over (instance, parent code);
//   2. the box-image kernel: a device work queue of fixed-size point chunks over all
//      instances' (implicit) children, claimed by the persistent blocks with one atomic
//      per chunk; a chunk's points find their instance by binary search in shared memory;
//   3. per-instance survivor counts, then one ordered compaction of all children;
//   4. new offsets; instances whose depth is reached move to the final arena.
// All launches read their sizes from device memory: the whole run is one CUDA graph.
// The image kernel's block size, points per thread and chunk size are chosen by timing
// the candidates on the first run (autotuner).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "batch.h"
#include "rows.cuh"
#include "tree.h"

using namespace b12g;
using namespace b12g::host;

namespace {


__device__ __forceinline__ uint32_t find_instance(const uint32_t* off_s, uint32_t n_inst, uint64_t x)
{
  // largest i with off_s[i] <= x
  uint32_t lo = 0, len = n_inst;
  while (len > 1) {
    const uint32_t half = len >> 1;
    lo = (off_s[lo + half] <= x) ? lo + half : lo;
    len -= half;
  }
  return lo;
}

__device__ __forceinline__ uint64_t inst_key(uint32_t inst, uint64_t code) { return (uint64_t(inst) << 32) | code; }

__global__ void batch_hash_build_kernel(const uint64_t* codes, const uint32_t* off, uint32_t n_inst, LeafHash h,
                                        uint32_t code_cap, uint32_t* error)
{
  __shared__ uint32_t off_s[kMaxInstances + 1];
  for (uint32_t i = threadIdx.x; i <= n_inst; i += blockDim.x) off_s[i] = off[i];
  __syncthreads();
  const uint32_t n = off_s[n_inst];
  const int l = hash_log2(n);
  if (n > code_cap || l > int(h.log2_cap)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(error, 1u);
    return;
  }
  const uint64_t mask = (1ull << l) - 1ull;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const uint64_t code = inst_key(find_instance(off_s, n_inst, p), codes[p]);
    const unsigned long long key = (uint64_t(h.tag) << 56) | code;
    uint64_t s = hash_slot(code, l);
    bool done = false;
    for (uint64_t step = 0; step <= 2 * mask + 64 && !done; ++step) {
      unsigned long long* kw = reinterpret_cast<unsigned long long*>(&h.slots[s].x);
      const unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(kw);
      if ((cur >> 56) != h.tag) {
        if (atomicCAS(kw, cur, key) == cur) { h.slots[s].y = p; done = true; }
        continue;
      }
      s = (s + 1) & mask;
    }
    if (!done) atomicOr(error, 1u);
  }
}

template<class Map, class Grid>
__device__ __forceinline__ void load_batch_points(const GridParams& g, uint64_t P, double* pts)
{
  for (uint32_t idx = threadIdx.x; idx < uint32_t(P) * Map::D; idx += blockDim.x) {
    const int j = int(idx / uint32_t(P));
    pts[idx] = Grid::table_value(g, g.coord, idx - uint32_t(j) * uint32_t(P), j);
  }
}

// maps that can integrate W states interleaved in one thread
template<class Map> struct Multi {
  static constexpr bool kOk = false;
  template<int W, int D>
  static __device__ __forceinline__ void apply(const MapParams&, const double (&)[W][D], double (&)[W][D]) {}
};
template<class A> struct Multi<LorenzMap<A>> {
  static constexpr bool kOk = true;
  template<int W, int D>
  static __device__ __forceinline__ void apply(const MapParams& m, const double (&x)[W][D], double (&y)[W][D])
  {
    lorenz_apply_multi<A, W>(m, x, y);
  }
};

template<> struct Multi<ForcedDuffingMap> {
  static constexpr bool kOk = true;
  template<int W, int D>
  static __device__ __forceinline__ void apply(const MapParams& m, const double (&x)[W][D], double (&y)[W][D])
  {
    duffing_apply_multi<W>(m, x, y);
  }
};

// the image of child point (child c of the concatenated children, grid index k)
template<class Map, class Grid, int W>
struct BatchPoint {
  static constexpr int D = Map::D;
  // W points: child[w], k[w]; returns their children-level targets (global child index,
  // kInvalidIndex when the image box is no child of a leaf, kOutsideIndex when the image
  // left the domain) and their instances
  // inst[w]: the instance of child[w] (the caller tracks it along its points)
  static __device__ __forceinline__ void run(const BatchArgs& a, const uint32_t* off_s, const double* pts,
                                             const uint64_t (&child)[W], const uint32_t (&k)[W],
                                             const bool (&act)[W], uint32_t (&target)[W],
                                             const uint32_t (&inst)[W])
  {
    double x[W][D], y[W][D];
    int dep[W];
    MapParams mp[W];
    const bool uni = a.inst_depth == nullptr;   // one depth: the launch's constants
#pragma unroll
    for (int w = 0; w < W; ++w) {
      dep[w] = uni ? a.depth : int(a.inst_depth[inst[w]]);
      const uint64_t c = child[w];
      const uint64_t code = act[w] ? ((a.codes[c >> 1] << 1) | (c & 1u)) : 0ull;
      double cc[D], r[D];
      if (uni) {
#pragma unroll
        for (int j = 0; j < D; ++j) box_axis(a.dom, a.dc.ax[j], j, deinterleave<D>(code, a.depth, j), cc[j], r[j]);
      } else {
        box_coordinates<D>(a.dom, code, dep[w], cc, r);
      }
#pragma unroll
      for (int j = 0; j < D; ++j) x[w][j] = __dadd_rn(cc[j], __dmul_rn(pts[j * uint32_t(a.points) + k[w]], r[j]));
      mp[w] = a.map;
#pragma unroll
      for (int q = 0; q < 6; ++q) mp[w].p[q] = a.params[size_t(inst[w]) * 6 + q];
    }
    if constexpr (W > 1 && Multi<Map>::kOk) {
      // the interleaved integrator needs one parameter set: the W points share it
      // when they share an instance, else fall back to one at a time
      bool same = true;
#pragma unroll
      for (int w = 1; w < W; ++w) same = same && inst[w] == inst[0];
      if (same) {
        Multi<Map>::template apply<W, D>(mp[0], x, y);
      } else {
#pragma unroll
        for (int w = 0; w < W; ++w) Map::apply(mp[w], x[w], y[w]);
      }
    } else {
#pragma unroll
      for (int w = 0; w < W; ++w) Map::apply(mp[w], x[w], y[w]);
    }
#pragma unroll
    for (int w = 0; w < W; ++w) {
      uint64_t tcode = 0;
      bool inside = false;
      if (uni) {
        uint32_t tb[D];
        inside = act[w] && point_bits<D>(a.dom, a.dc, y[w], tb);
        if (inside) tcode = code_of_bits<D>(a.dc, tb, a.depth);
      } else {
        inside = act[w] && point_code<D>(a.dom, y[w], dep[w], tcode);
      }
      uint32_t t = act[w] ? kOutsideIndex : kInvalidIndex;
      if (inside) {
        const uint32_t p = hash_locate(a.hash, off_s[a.n_inst], inst_key(inst[w], tcode >> 1));
        t = p != kInvalidIndex ? 2u * p + uint32_t(tcode & 1u) : kInvalidIndex;
      }
      target[w] = t;
    }
  }
};

constexpr uint32_t kBatchTable = 2048;

template<class Map, class Grid, int W>
__global__ void __launch_bounds__(512) batch_image_kernel(const BatchArgs a)
{
  __shared__ uint32_t off_s[kMaxInstances + 1];
  __shared__ double pts[kBatchTable];
  __shared__ uint32_t item_s;
  for (uint32_t i = threadIdx.x; i <= a.n_inst; i += blockDim.x) off_s[i] = a.off[i];
  load_batch_points<Map, Grid>(a.grid, a.points, pts);
  __syncthreads();
  const uint64_t children = 2ull * off_s[a.n_inst];
  if (children > a.hit_cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(a.error, 1u);
    return;
  }
  const uint64_t P = a.points;
  const uint64_t total = children * P;
  const int lane = threadIdx.x & 31;
  const uint64_t span = uint64_t(blockDim.x) * W;
  for (;;) {
    if (threadIdx.x == 0) item_s = atomicAdd(a.queue, 1u);
    __syncthreads();
    const uint64_t start = uint64_t(item_s) * a.chunk;
    __syncthreads();
    if (start >= total) break;
    const uint64_t end = min(total, start + a.chunk);
    // this thread's points g_w = start + threadIdx.x + w * blockDim.x + trip * span as
    // (child, k) = (g / P, g % P), divided once per chunk and then advanced by span, with
    // their instance found once and then followed along the (increasing) children
    uint64_t child[W];
    uint32_t k[W], inst[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
      const uint64_t g = start + threadIdx.x + uint64_t(w) * blockDim.x;
      if (total <= 0xFFFFFFFFull - span) {
        child[w] = uint32_t(g) / uint32_t(P);
        k[w] = uint32_t(g) - uint32_t(child[w]) * uint32_t(P);
      } else {
        child[w] = g / P;
        k[w] = uint32_t(g - child[w] * P);
      }
      inst[w] = find_instance(off_s, a.n_inst, child[w] >> 1);
    }
    const uint64_t dchild = span / P;
    const uint32_t dk = uint32_t(span - dchild * P);
    for (uint64_t base = start + threadIdx.x - lane; base < end; base += span) {
      uint32_t target[W];
      bool act[W];
#pragma unroll
      for (int w = 0; w < W; ++w) act[w] = base + lane + uint64_t(w) * blockDim.x < end;
      BatchPoint<Map, Grid, W>::run(a, off_s, pts, child, k, act, target, inst);
#pragma unroll
      for (int w = 0; w < W; ++w) {
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, target[w]);
        if (act[w] && target[w] < kOutsideIndex && lane == __ffs(peers) - 1) a.hit[target[w]] = 1;
      }
      if (a.targets) {
        // the instances finishing in this step keep every point's target for their
        // transition matrix
#pragma unroll
        for (int w = 0; w < W; ++w) {
          if (!act[w]) continue;
          const uint64_t tb = a.tgt_base[inst[w]];
          if (tb != ~0ull) a.targets[tb + (child[w] - 2ull * off_s[inst[w]]) * P + k[w]] = target[w];
        }
      }
#pragma unroll
      for (int w = 0; w < W; ++w) {
        child[w] += dchild;
        k[w] += dk;
        if (k[w] >= P) { k[w] -= uint32_t(P); ++child[w]; }
        while (inst[w] + 1 < a.n_inst && (child[w] >> 1) >= off_s[inst[w] + 1]) ++inst[w];
      }
    }
  }
}


// survivors per instance (children with a hit), one block per instance
__global__ void inst_count_kernel(const uint8_t* hit, const uint32_t* off, uint32_t* cnt, uint64_t hit_cap,
                                  uint32_t* error)
{
  __shared__ uint32_t red[32];
  const uint32_t i = blockIdx.x;
  const uint64_t b = 2ull * off[i], e = 2ull * off[i + 1];
  if (e > hit_cap || b > e) {
    // capacity exceeded upstream: report it and leave this instance's count at zero
    if (threadIdx.x == 0) { cnt[i] = 0; atomicOr(error, 1u); }
    return;
  }
  uint32_t c = 0;
  for (uint64_t x = b + threadIdx.x; x < e; x += blockDim.x) c += hit[x] ? 1u : 0u;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, d);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (uint32_t w = 0; w < blockDim.x / 32; ++w) t += red[w];
    cnt[i] = t;
  }
}

// one block: new offsets = exclusive scan of the counts; the step's counts recorded;
// the instances [a_next, n_inst) are finished: they get consecutive regions of the
// final arena starting at *fin_base (fin_lo, fin_len per sorted position)
__global__ void inst_offsets_kernel(const uint32_t* cnt, uint32_t n_inst, uint32_t a_next, uint32_t* new_off,
                                    uint32_t* step_counts, uint32_t* fin_lo, uint32_t* fin_len, uint32_t* fin_base,
                                    uint32_t code_cap, uint32_t* error)
{
  __shared__ uint32_t part[1024];
  const uint32_t per = (n_inst + blockDim.x - 1) / blockDim.x;
  const uint32_t b = min(n_inst, threadIdx.x * per), e = min(n_inst, b + per);
  uint32_t s = 0;
  for (uint32_t i = b; i < e; ++i) s += cnt[i];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (uint32_t t = 0; t < blockDim.x; ++t) { const uint32_t v = part[t]; part[t] = run; run += v; }
    new_off[n_inst] = run;
    if (run > code_cap) atomicOr(error, 1u);
  }
  __syncthreads();
  uint32_t run = part[threadIdx.x];
  for (uint32_t i = b; i < e; ++i) {
    new_off[i] = run;
    step_counts[i] = cnt[i];
    run += cnt[i];
  }
  __syncthreads();
  const uint32_t base = *fin_base;
  for (uint32_t i = a_next + threadIdx.x; i < n_inst; i += blockDim.x) {
    fin_lo[i] = base + (new_off[i] - new_off[a_next]);
    fin_len[i] = cnt[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) *fin_base = base + (new_off[n_inst] - new_off[a_next]);
}

__global__ void copy_finished_kernel(const uint64_t* code, const uint8_t* flags, const uint32_t* new_off,
                                     uint32_t a_next, uint32_t n_inst, const uint32_t* fin_lo, uint64_t* fin_code,
                                     uint8_t* fin_flags, uint32_t fin_cap, uint32_t code_cap, uint32_t* error)
{
  const uint32_t b = new_off[a_next], e = min(new_off[n_inst], code_cap);
  const uint32_t dst = fin_lo[a_next];
  for (uint32_t i = b + blockIdx.x * blockDim.x + threadIdx.x; i < e; i += gridDim.x * blockDim.x) {
    const uint32_t d = dst + (i - b);
    if (d < fin_cap) { fin_code[d] = code[i]; fin_flags[d] = flags[i]; }
    else atomicOr(error, 1u);
  }
}

template<class Map, class Grid>
__global__ void __launch_bounds__(256) batch_rows_kernel(const BatchRowArgs a)
{
  constexpr int D = Map::D;
  __shared__ uint32_t off_s[kMaxInstances + 1];
  __shared__ double pts[kBatchTable];
  __shared__ uint32_t keys[8][128];
  __shared__ uint32_t bounds[8][4];
  for (uint32_t i = threadIdx.x; i <= a.n_inst; i += blockDim.x) off_s[i] = a.off[i];
  load_batch_points<Map, Grid>(a.grid, a.points, pts);
  __syncthreads();
  const uint32_t nrows = off_s[a.n_inst];
  const uint32_t P = uint32_t(a.points);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t* s = keys[w];
  for (uint32_t row = blockIdx.x * 8 + w; row < nrows; row += gridDim.x * 8) {
    const uint32_t inst = find_instance(off_s, a.n_inst, row);   // arena index
    const uint32_t sp = a.inst_of[inst];                          // sorted position
    const int depth = a.depths[sp];
    const uint64_t code = a.codes[row];
    const uint32_t n_i = off_s[inst + 1] - off_s[inst];
    MapParams mp = a.map;
#pragma unroll
    for (int q = 0; q < 6; ++q) mp.p[q] = a.params[size_t(sp) * 6 + q];
    double cc[D], r[D];
    box_coordinates<D>(a.dom, code, depth, cc, r);
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
      const uint32_t k = uint32_t(lane) + 32u * q;
      uint32_t key = kPadKey;
      if (k < P) {
        double x[D], y[D];
#pragma unroll
        for (int j = 0; j < D; ++j) x[j] = __dadd_rn(cc[j], __dmul_rn(pts[j * P + k], r[j]));
        Map::apply(mp, x, y);
        uint64_t tcode = 0;
        uint32_t t = kInvalidIndex;
        if (point_code<D>(a.dom, y, depth, tcode)) {
          const uint32_t g = hash_locate(a.hash, nrows, inst_key(inst, tcode));
          if (g != kInvalidIndex) t = g - off_s[inst];
        } else if (a.codes[off_s[inst] + n_i - 1] == 0) {
          t = n_i - 1;   // a point outside the domain is found in a last leaf of code 0
        }
        key = t == kInvalidIndex ? kLostKey : t;
      }
      s[lane + 32 * q] = key;
    }
    const uint32_t total = row_emit(s, bounds[w], lane, P, a.keep_lost, n_i + 1, a.stage_col + size_t(row) * P,
                                    a.stage_cnt + size_t(row) * P);
    if (lane == 0) a.row_count[row] = total;
    __syncwarp();
  }
}

// transition rows from stored targets: a warp per child of a finishing instance; the
// child is a row when it survived (its rank advances), a target is a column when its
// child survived, and its column is its rank within the instance
__global__ void __launch_bounds__(256) target_rows_kernel(const TargetRowArgs a)
{
  __shared__ uint32_t off_s[kMaxInstances + 1];
  __shared__ uint32_t keys[8][128];
  __shared__ uint32_t bounds[8][4];
  for (uint32_t i = threadIdx.x; i <= a.n_inst; i += blockDim.x) off_s[i] = a.child_off[i];
  __syncthreads();
  const uint32_t total = off_s[a.n_inst];
  const uint32_t P = a.points;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t* s = keys[w];
  for (uint32_t j = blockIdx.x * 8 + w; j < total; j += gridDim.x * 8) {
    const uint32_t q = find_instance(off_s, a.n_inst, j);
    const uint32_t cb = a.child_base[q];
    const uint32_t c = cb + (j - off_s[q]);
    const uint32_t r0 = a.rank[cb];
    const uint32_t rc = a.rank[c];
    if (a.rank[c + 1] == rc) continue;            // not a survivor: no row (warp-uniform)
    const uint32_t n_i = a.rank[cb + (off_s[q + 1] - off_s[q])] - r0;
    const uint32_t row = a.row_off[q] + (rc - r0);
    // a point outside the domain is found in a last leaf of code 0
    const bool zero_leaf = a.arena[a.row_off[q] + n_i - 1] == 0;
    // every load of the row goes out before any is used: the targets, then their ranks
    uint32_t tg[4], lo[4], hi[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t k = uint32_t(lane) + 32u * u;
      tg[u] = k < P ? a.targets[size_t(j) * P + k] : kInvalidIndex;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const bool in = tg[u] < kOutsideIndex;
      lo[u] = in ? a.rank[tg[u]] : 0u;
      hi[u] = in ? a.rank[tg[u] + 1] : 0u;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t k = uint32_t(lane) + 32u * u, t = tg[u];
      uint32_t key = kPadKey;
      if (k < P) {
        if (t < kOutsideIndex) key = hi[u] != lo[u] ? lo[u] - r0 : kLostKey;
        else key = (t == kOutsideIndex && zero_leaf) ? n_i - 1 : kLostKey;
      }
      s[lane + 32 * u] = key;
    }
    const uint32_t cnt = row_emit(s, bounds[w], lane, P, a.keep_lost, n_i + 1, a.stage_col + size_t(row) * P,
                                  a.stage_cnt + size_t(row) * P);
    if (lane == 0) a.row_count[row] = cnt;
    __syncwarp();
  }
}

// dispatch over (map, arith, grid); the batched kernels take table grids only
template<class F>
cudaError_t batch_dispatch(uint32_t map_kind, uint32_t arith, uint32_t grid_kind, F&& f)
{
  auto with_grid = [&](auto map_tag) -> cudaError_t {
    switch (grid_kind) {
      case B12G_GRID_INNER: return f(decltype(map_tag){}, InnerGrid{});
      case B12G_GRID_FULL: return f(decltype(map_tag){}, FullGrid{});
      default: return cudaErrorInvalidValue;
    }
  };
  switch (map_kind) {
    case B12G_MAP_HENON: return arith == B12G_ARITH_STRICT ? with_grid(HenonMap{}) : cudaErrorInvalidValue;
    case B12G_MAP_LORENZ:
      return arith == B12G_ARITH_FMA ? with_grid(LorenzMap<Fused>{}) : with_grid(LorenzMap<Strict>{});
    case B12G_MAP_FORCED_DUFFING:
      return arith == B12G_ARITH_STRICT ? with_grid(ForcedDuffingMap{}) : cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
  }
}

int batch_grid(const void* kernel, int threads)
{
  int b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, 0);
  return device_sm_count() * (b > 0 ? b : 1);
}

}  // namespace

namespace b12g {

cudaError_t launch_batch_image(uint32_t map_kind, uint32_t arith, uint32_t grid_kind, const Tuning& tu,
                               const BatchArgs& args, cudaStream_t s)
{
  BatchArgs a = args;
  if (!a.inst_depth) {
    int dim = 0;
    batch_dispatch(map_kind, arith, grid_kind, [&](auto map, auto) -> cudaError_t {
      dim = decltype(map)::D;
      return cudaSuccess;
    });
    if (dim > 0) fill_depth_const(a.dom, dim, a.depth, a.dc);
  }
  return batch_dispatch(map_kind, arith, grid_kind, [&](auto map, auto grid) -> cudaError_t {
    using Map = decltype(map);
    using Grid = decltype(grid);
    if constexpr (Map::D <= 2) {
      // four points per thread only for the two-dimensional maps (register budget)
      if (tu.ppt == 4) {
        const void* k = (const void*)batch_image_kernel<Map, Grid, 4>;
        batch_image_kernel<Map, Grid, 4><<<batch_grid(k, int(tu.threads)), tu.threads, 0, s>>>(a);
        return cudaGetLastError();
      }
    }
    if (tu.ppt >= 2) {
      const void* k = (const void*)batch_image_kernel<Map, Grid, 2>;
      batch_image_kernel<Map, Grid, 2><<<batch_grid(k, int(tu.threads)), tu.threads, 0, s>>>(a);
    } else {
      const void* k = (const void*)batch_image_kernel<Map, Grid, 1>;
      batch_image_kernel<Map, Grid, 1><<<batch_grid(k, int(tu.threads)), tu.threads, 0, s>>>(a);
    }
    return cudaGetLastError();
  });
}

cudaError_t launch_batch_rows(uint32_t map_kind, uint32_t arith, uint32_t grid_kind, const BatchRowArgs& a,
                              uint32_t max_rows, cudaStream_t s)
{
  return batch_dispatch(map_kind, arith, grid_kind, [&](auto map, auto grid) -> cudaError_t {
    using Map = decltype(map);
    using Grid = decltype(grid);
    const void* k = (const void*)batch_rows_kernel<Map, Grid>;
    const int g = std::max(1, std::min<int>(batch_grid(k, 256), int((uint64_t(max_rows) + 7) / 8)));
    batch_rows_kernel<Map, Grid><<<g, 256, 0, s>>>(a);
    return cudaGetLastError();
  });
}

cudaError_t launch_target_rows(const TargetRowArgs& a, uint32_t max_children, cudaStream_t s)
{
  if (max_children == 0) return cudaSuccess;
  const int g = std::max(1, std::min<int>(batch_grid((const void*)target_rows_kernel, 256),
                                          int((uint64_t(max_children) + 7) / 8)));
  target_rows_kernel<<<g, 256, 0, s>>>(a);
  return cudaGetLastError();
}

bool batch_supported(uint32_t map_kind, uint32_t arith, uint32_t grid_kind)
{
  return batch_dispatch(map_kind, arith, grid_kind, [](auto, auto) { return cudaSuccess; }) == cudaSuccess;
}

cudaError_t launch_batch_hash(const uint64_t* codes, const uint32_t* off, uint32_t n_inst, LeafHash h,
                              uint32_t code_cap, uint32_t* error, cudaStream_t s)
{
  batch_hash_build_kernel<<<device_sm_count() * 4, 256, 0, s>>>(codes, off, n_inst, h, code_cap, error);
  return cudaGetLastError();
}

cudaError_t launch_inst_count(const uint8_t* hit, const uint32_t* off, uint32_t n_inst, uint32_t* cnt,
                              uint64_t hit_cap, uint32_t* error, cudaStream_t s)
{
  if (n_inst > 0) inst_count_kernel<<<n_inst, 256, 0, s>>>(hit, off, cnt, hit_cap, error);
  return cudaGetLastError();
}

}  // namespace b12g

namespace {

// autotuning results, per (device, map, arith, grid)
std::mutex g_tune_mu;
std::map<uint64_t, Tuning> g_tuned;

uint64_t tune_key(int dev, uint32_t map, uint32_t arith, uint32_t grid)
{
  return (uint64_t(dev) << 48) | (uint64_t(map) << 32) | (uint64_t(arith) << 16) | grid;
}

}  // namespace

namespace b12g {

Tuning batch_tuning(int device, uint32_t map_kind, uint32_t arith, uint32_t grid_kind, uint32_t dim)
{
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tuned.find(tune_key(device, map_kind, arith, grid_kind));
    if (it != g_tuned.end()) return it->second;
  }
  // the shapes the tuner picks on B200 for these maps: the two-dimensional maps keep four
  // points per thread in flight, Lorenz one
  Tuning t{};
  if (dim <= 2 && map_kind == B12G_MAP_FORCED_DUFFING) t.ppt = 4;
  return t;
}

}  // namespace b12g

namespace {

}  // namespace

// ------------------------------------------------------------------------ host side
struct b12g_batch {
  template<class T> using Buf = b12g::host::Buf<T>;
  int device = 0;
  cudaStream_t stream = nullptr;
  b12g_domain domain{};
  Domain dom{};
  b12g_scheme scheme{};
  MapParams mp{};
  GridParams gp{};
  uint64_t P = 0;
  uint32_t N = 0;
  uint8_t max_depth = 0;
  std::vector<uint32_t> order;         // sorted position -> instance
  std::vector<uint32_t> pos;           // instance -> sorted position
  std::vector<uint8_t> depth_sorted;
  std::vector<uint32_t> active;        // active[k] = instances with depth >= k (k = 0..max_depth+1)
  Buf<double> params;                  // sorted order
  Buf<uint8_t> depths;                 // sorted order
  Buf<uint64_t> code[2];
  Buf<uint8_t> flags[2];
  Buf<uint8_t> hit;
  Buf<uint32_t> off[2];
  Buf<uint32_t> cnt, step_counts, ctr, tiles_a, tiles_b, fin_lo, fin_len, arena_off, arena_inst;
  Buf<ulonglong2> hash;
  uint32_t hash_log2 = 0;
  Buf<uint64_t> fin_code;
  Buf<uint8_t> fin_flags;
  uint64_t cap = 0, fin_cap = 0;
  Tuning tuning{};
  bool tuned = false;
  cudaGraphExec_t graph = nullptr;
  uint64_t graph_kernels = 0;
  bool ran = false;
  std::vector<uint32_t> h_step_counts;  // max_depth x N (sorted order)
  std::vector<uint32_t> h_fin_lo, h_fin_len;   // per sorted position
  std::vector<uint32_t> h_arena_off, h_arena_inst, h_arena_of;  // arena order
  // transition matrices
  Buf<uint32_t> stage_col, stage_cnt, row_count, rowptr, cols;
  Buf<double> vals;
  uint64_t nnz = 0;
  bool has_tm = false;
  int tm_invalid = 0;
  std::vector<uint32_t> h_rowptr_arena; // rowptr at arena_off[a]
  uint32_t* h_ctr = nullptr;
};

namespace {

enum : int { B_ERROR = 0, B_QUEUE = 1, B_FINBASE = 2, B_TOTAL = 3, B_TMP = 4, B_COUNT = 64 };

b12g_status batch_reserve(b12g_batch* b, uint64_t cap)
{
  if (cap > 0x7FFFFFF0ull) return fail(B12G_ERR_CAPACITY, "batch capacity above 2^31 boxes");
  for (int q = 0; q < 2; ++q) {
    ST(b->code[q].ensure(cap, "batch codes"));
    ST(b->flags[q].ensure(cap, "batch flags"));
  }
  if (b->hit.n < 2 * cap) {
    ST(b->hit.ensure(2 * cap, "batch hit mask"));
    CK(cudaMemsetAsync(b->hit.p, 0, b->hit.n, b->stream));
  }
  const size_t most = std::max<size_t>(b->hit.n, 2 * cap) + 1;
  ST(b->tiles_a.ensure(compact_tiles(most) + 2, "batch tiles"));
  ST(b->tiles_b.ensure(compact_tiles(most) + 2, "batch tiles"));
  uint32_t l = 6;
  while ((1ull << l) < 2ull * cap) ++l;
  if (!b->hash.p || l > b->hash_log2) {
    b->hash.release();
    ST(b->hash.ensure(size_t(1) << l, "batch lookup table"));
    b->hash_log2 = l;
  }
  ST(b->fin_code.ensure(cap, "batch final leaves"));
  ST(b->fin_flags.ensure(cap, "batch final leaves"));
  b->cap = cap;
  b->fin_cap = std::min(b->fin_code.n, b->fin_flags.n);
  return B12G_OK;
}

b12g_status batch_read(b12g_batch* b, int first, int count)
{
  CK(cudaMemcpyAsync(b->h_ctr + first, b->ctr.p + first, count * 4, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return B12G_OK;
}

// initial state: every instance is the surrounding box with SD set (setFlags(SD))
b12g_status batch_reset(b12g_batch* b)
{
  std::vector<uint32_t> off(b->N + 1);
  for (uint32_t i = 0; i <= b->N; ++i) off[i] = i;
  CK(cudaMemcpyAsync(b->off[0].p, off.data(), (b->N + 1) * 4, cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemsetAsync(b->code[0].p, 0, size_t(b->N) * 8, b->stream));
  CK(cudaMemsetAsync(b->flags[0].p, B12G_SD, b->N, b->stream));
  CK(cudaMemsetAsync(b->ctr.p, 0, B_COUNT * 4, b->stream));
  CK(cudaMemsetAsync(b->fin_len.p, 0, b->N * 4, b->stream));
  CK(cudaMemsetAsync(b->hit.p, 0, b->hit.n, b->stream));
  CK(cudaMemsetAsync(b->fin_lo.p, 0, b->N * 4, b->stream));
  CK(cudaMemsetAsync(b->hash.p, 0, b->hash.n * sizeof(ulonglong2), b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return B12G_OK;
}

// the launches of subdivision step k (1-based) reading offsets from off[k & 1 ^ 1]
cudaError_t build_step_hash(b12g_batch* b, uint32_t k)
{
  const uint32_t A = b->active[k];
  const int in = (k - 1) & 1;
  const LeafHash h{b->hash.p, k, b->hash_log2};
  batch_hash_build_kernel<<<device_sm_count() * 4, 256, 0, b->stream>>>(
      b->code[in].p, b->off[in].p, A, h, uint32_t(std::min<uint64_t>(b->cap, 0xFFFFFFFFu)), b->ctr.p + B_ERROR);
  return cudaGetLastError();
}

cudaError_t enqueue_step(b12g_batch* b, uint32_t k, const Tuning& tu, bool with_hash = true)
{
  const uint32_t A = b->active[k], a_next = b->active[k + 1];
  const int in = (k - 1) & 1, out = k & 1;
  const LeafHash h{b->hash.p, k, b->hash_log2};
  const uint32_t capu = uint32_t(std::min<uint64_t>(b->cap, 0xFFFFFFFFu));
  if (with_hash) {
    cudaError_t e0 = build_step_hash(b, k);
    if (e0 != cudaSuccess) return e0;
  }
  cudaMemsetAsync(b->ctr.p + B_QUEUE, 0, 4, b->stream);
  BatchArgs a{};
  a.dom = b->dom;
  a.map = b->mp;
  a.grid = b->gp;
  a.points = b->P;
  a.params = b->params.p;
  a.depths = b->depths.p;
  a.n_inst = A;
  a.off = b->off[in].p;
  a.codes = b->code[in].p;
  a.depth = int(k);
  a.hash = h;
  a.hit = b->hit.p;
  a.hit_cap = uint32_t(std::min<size_t>(b->hit.n, 0xFFFFFFFFu));
  a.queue = b->ctr.p + B_QUEUE;
  a.chunk = tu.chunk;
  a.error = b->ctr.p + B_ERROR;
  cudaError_t e = launch_batch_image(b->scheme.map.kind, b->scheme.map.arith, b->scheme.grid.kind, tu, a, b->stream);
  if (e != cudaSuccess) return e;
  if (A > 0) inst_count_kernel<<<A, 256, 0, b->stream>>>(b->hit.p, b->off[in].p, b->cnt.p, b->hit.n,
                                                         b->ctr.p + B_ERROR);
  // all active instances' children, in instance order, compacted by the hit mask
  CompactArgs ca{};
  ca.code = b->code[in].p;
  ca.flags = b->flags[in].p;
  ca.n = b->off[in].p + A;
  ca.hit = b->hit.p;
  ca.children = 1;
  ca.hit_cap = a.hit_cap;
  ca.out_code = b->code[out].p;
  ca.out_flags = b->flags[out].p;
  ca.n_out = b->ctr.p + B_TOTAL;
  ca.out_cap = capu;
  ca.error = b->ctr.p + B_ERROR;
  e = compact(ca, {b->tiles_a.p, b->tiles_b.p}, capu, b->stream);
  if (e != cudaSuccess) return e;
  inst_offsets_kernel<<<1, 1024, 0, b->stream>>>(b->cnt.p, A, a_next, b->off[out].p,
                                                 b->step_counts.p + size_t(k - 1) * b->N, b->fin_lo.p,
                                                 b->fin_len.p, b->ctr.p + B_FINBASE, capu, b->ctr.p + B_ERROR);
  if (a_next < A) {
    copy_finished_kernel<<<device_sm_count() * 2, 256, 0, b->stream>>>(
        b->code[out].p, b->flags[out].p, b->off[out].p, a_next, A, b->fin_lo.p, b->fin_code.p, b->fin_flags.p,
        uint32_t(std::min<uint64_t>(b->fin_cap, 0xFFFFFFFFu)), capu, b->ctr.p + B_ERROR);
  }
  return cudaGetLastError();
}

// kernels per step in the graph: hash, image, count, the compaction's, offsets, (copy)
uint64_t step_kernels(const b12g_batch* b, uint32_t k)
{
  const uint32_t capu = uint32_t(std::min<uint64_t>(b->cap, 0xFFFFFFFFu));
  return 4 + compact_launches(true, capu) + (b->active[k + 1] < b->active[k] ? 1 : 0);
}

// time every candidate shape on the batch's own steps (first run) and keep the fastest
b12g_status autotune(b12g_batch* b)
{
  const Tuning all[] = {{256, 1, 8192}, {256, 2, 8192}, {128, 1, 8192}, {512, 1, 16384}, {256, 1, 32768},
                        {256, 2, 32768}, {256, 4, 8192}, {128, 4, 8192}};
  std::vector<Tuning> cands;
  for (const Tuning& t : all)
    if (t.ppt < 4 || b->domain.dim <= 2) cands.push_back(t);   // 4 points per thread: 2-D maps only
  std::vector<double> total(cands.size(), 0.0);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  ST(batch_reset(b));
  for (uint32_t k = 1; k <= b->max_depth; ++k) {
    const uint32_t A = b->active[k];
    const int in = (k - 1) & 1;
    // the step's point count decides whether it is worth timing
    uint32_t parents = 0;
    CK(cudaMemcpyAsync(&parents, b->off[in].p + A, 4, cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    if (2ull * parents * b->P >= (1ull << 22)) {
      for (size_t c = 0; c < total.size(); ++c) {
        BatchArgs a{};
        a.dom = b->dom; a.map = b->mp; a.grid = b->gp; a.points = b->P; a.params = b->params.p;
        a.depths = b->depths.p; a.n_inst = A; a.off = b->off[in].p; a.codes = b->code[in].p; a.depth = int(k);
        a.hash = LeafHash{b->hash.p, k, b->hash_log2}; a.hit = b->hit.p;
        a.hit_cap = uint32_t(std::min<size_t>(b->hit.n, 0xFFFFFFFFu)); a.queue = b->ctr.p + B_QUEUE;
        a.chunk = cands[c].chunk; a.error = b->ctr.p + B_ERROR;
        // the lookup table of step k is built once, before the first trial
        if (c == 0) CK(build_step_hash(b, k));
        CK(cudaMemsetAsync(b->ctr.p + B_QUEUE, 0, 4, b->stream));
        cudaEventRecord(e0, b->stream);
        CK(launch_batch_image(b->scheme.map.kind, b->scheme.map.arith, b->scheme.grid.kind, cands[c], a, b->stream));
        cudaEventRecord(e1, b->stream);
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        total[c] += ms;
      }
    }
    // the real step (with the default shape; the hit marks of the trials are the same)
    CK(enqueue_step(b, k, b->tuning, /*with_hash=*/!(2ull * parents * b->P >= (1ull << 22))));
    CK(cudaStreamSynchronize(b->stream));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  size_t best = 0;
  for (size_t c = 1; c < total.size(); ++c)
    if (total[c] > 0.0 && total[c] < total[best]) best = c;
  if (total[best] > 0.0) b->tuning = cands[best];
  b->tuned = true;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tuned[tune_key(b->device, b->scheme.map.kind, b->scheme.map.arith, b->scheme.grid.kind)] = b->tuning;
  return B12G_OK;
}

b12g_status batch_collect(b12g_batch* b)
{
  const uint32_t N = b->N;
  b->h_step_counts.assign(size_t(b->max_depth) * N, 0);
  b->h_fin_lo.assign(N, 0);
  b->h_fin_len.assign(N, 0);
  CK(cudaMemcpyAsync(b->h_step_counts.data(), b->step_counts.p, b->h_step_counts.size() * 4, cudaMemcpyDeviceToHost,
                     b->stream));
  CK(cudaMemcpyAsync(b->h_fin_lo.data(), b->fin_lo.p, N * 4, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaMemcpyAsync(b->h_fin_len.data(), b->fin_len.p, N * 4, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  // arena order: instances in the order their regions were appended (by start offset;
  // an empty region is placed where it was written, which keeps the offsets prefix-summed)
  b->h_arena_inst.resize(N);
  for (uint32_t q = 0; q < N; ++q) b->h_arena_inst[q] = q;
  std::stable_sort(b->h_arena_inst.begin(), b->h_arena_inst.end(), [&](uint32_t x, uint32_t y) {
    return b->h_fin_lo[x] < b->h_fin_lo[y] || (b->h_fin_lo[x] == b->h_fin_lo[y] && b->h_fin_len[x] < b->h_fin_len[y]);
  });
  b->h_arena_off.assign(N + 1, 0);
  b->h_arena_of.assign(N, 0);
  for (uint32_t a = 0; a < N; ++a) {
    const uint32_t q = b->h_arena_inst[a];
    b->h_arena_of[q] = a;
    b->h_arena_off[a] = b->h_fin_lo[q];
    b->h_arena_off[a + 1] = b->h_fin_lo[q] + b->h_fin_len[q];
  }
  for (uint32_t a = 0; a < N; ++a)
    if (b->h_arena_off[a + 1] != b->h_arena_off[a] + b->h_fin_len[b->h_arena_inst[a]] ||
        (a + 1 < N && b->h_arena_off[a + 1] != b->h_fin_lo[b->h_arena_inst[a + 1]]))
      return fail(B12G_ERR_CUDA, "batch: final regions are not contiguous");
  ST(b->arena_off.ensure(N + 1, "arena offsets"));
  ST(b->arena_inst.ensure(N, "arena instances"));
  CK(cudaMemcpyAsync(b->arena_off.p, b->h_arena_off.data(), (N + 1) * 4, cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->arena_inst.p, b->h_arena_inst.data(), N * 4, cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return B12G_OK;
}

}  // namespace

extern "C" {

b12g_status b12g_batch_create(const b12g_domain* domain, const b12g_scheme* scheme, uint32_t n, const double* params,
                              const uint8_t* depths, b12g_batch** out)
{
  if (!domain || !scheme || !params || !depths || !out) return fail(B12G_ERR_INVALID, "NULL argument");
  if (n == 0 || n > kMaxInstances) return fail(B12G_ERR_INVALID, "1..%u instances", kMaxInstances);
  if (domain->dim < 1 || domain->dim > B12G_MAX_DIM) return fail(B12G_ERR_INVALID, "dim must be 1..4");
  if (scheme->flags_to_check != 0 || scheme->depth != B12G_LEAF_DEPTH)
    return fail(B12G_ERR_INVALID, "the batched subdivision maps every leaf");
  if (scheme->grid.kind != B12G_GRID_INNER && scheme->grid.kind != B12G_GRID_FULL)
    return fail(B12G_ERR_INVALID, "the batched path takes inner or full grids");
  const bool ok = batch_dispatch(scheme->map.kind, scheme->map.arith, scheme->grid.kind,
                                 [](auto, auto) { return cudaSuccess; }) == cudaSuccess;
  if (!ok || !image_supported(scheme->map.kind, scheme->map.arith, scheme->grid.kind, domain->dim))
    return fail(B12G_ERR_INVALID, "unsupported map/arith/grid/dimension for the batch");
  for (uint32_t i = 0; i < n; ++i)
    if (depths[i] < 1 || depths[i] > 32) return fail(B12G_ERR_INVALID, "instance depths must be 1..32");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(B12G_ERR_NO_DEVICE, "no CUDA device");
  }
  // the tree helpers validate the scheme and build map/grid parameters
  b12g_tree* probe = nullptr;
  ST(b12g_tree_create(domain, &probe));
  Prepared pr;
  b12g_status st = prepare(probe, scheme, pr);
  if (st != B12G_OK) { b12g_tree_destroy(probe); return st; }
  if (pr.P * domain->dim > kBatchTable || pr.P > kMaxRowPoints) {
    b12g_tree_destroy(probe);
    return fail(B12G_ERR_CAPACITY, "the batched path takes up to %u grid points per box", kMaxRowPoints);
  }
  b12g_batch* b = new b12g_batch();
  cudaGetDevice(&b->device);
  b->domain = *domain;
  b->dom = probe->dom;
  b->scheme = *scheme;
  b->mp = pr.a.map;
  b->gp = pr.a.grid;
  b->P = pr.P;
  b->N = n;
  std::vector<double> table;
  if (scheme->map.kind == B12G_MAP_FORCED_DUFFING) {
    table.resize(2 * size_t(scheme->map.steps) + 1);
    cudaMemcpy(table.data(), probe->table.p, table.size() * 8, cudaMemcpyDeviceToHost);
  }
  b12g_tree_destroy(probe);
  st = B12G_OK;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    st = cuda_fail(cudaGetLastError(), "stream");
  // deepest first, stable by instance index
  b->order.resize(n);
  for (uint32_t i = 0; i < n; ++i) b->order[i] = i;
  std::stable_sort(b->order.begin(), b->order.end(), [&](uint32_t x, uint32_t y) { return depths[x] > depths[y]; });
  b->pos.resize(n);
  b->depth_sorted.resize(n);
  std::vector<double> ps(size_t(n) * 6);
  for (uint32_t q = 0; q < n; ++q) {
    b->pos[b->order[q]] = q;
    b->depth_sorted[q] = depths[b->order[q]];
    for (int j = 0; j < 6; ++j) ps[size_t(q) * 6 + j] = params[size_t(b->order[q]) * 6 + j];
  }
  b->max_depth = b->depth_sorted[0];
  b->active.assign(b->max_depth + 2, 0);
  for (uint32_t k = 0; k <= uint32_t(b->max_depth) + 1; ++k)
    for (uint32_t q = 0; q < n; ++q) b->active[k] += b->depth_sorted[q] >= k ? 1u : 0u;
  if (st == B12G_OK && cudaMallocHost(&b->h_ctr, B_COUNT * 4) != cudaSuccess) st = cuda_fail(cudaGetLastError(), "pinned");
  if (st == B12G_OK) st = b->params.ensure(ps.size(), "batch params");
  if (st == B12G_OK) st = b->depths.ensure(n, "batch depths");
  if (st == B12G_OK) st = b->off[0].ensure(n + 1, "batch offsets");
  if (st == B12G_OK) st = b->off[1].ensure(n + 1, "batch offsets");
  if (st == B12G_OK) st = b->cnt.ensure(n, "batch counts");
  if (st == B12G_OK) st = b->step_counts.ensure(size_t(b->max_depth) * n, "batch step counts");
  if (st == B12G_OK) st = b->fin_lo.ensure(n, "batch final offsets");
  if (st == B12G_OK) st = b->fin_len.ensure(n, "batch final offsets");
  if (st == B12G_OK) st = b->ctr.ensure(B_COUNT, "batch counters");
  if (st == B12G_OK) {
    cudaMemcpy(b->params.p, ps.data(), ps.size() * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(b->depths.p, b->depth_sorted.data(), n, cudaMemcpyHostToDevice);
    cudaMemset(b->step_counts.p, 0, size_t(b->max_depth) * n * 4);
  }
  if (st == B12G_OK && !table.empty()) {
    double* tp = nullptr;
    if (cudaMalloc(&tp, table.size() * 8) != cudaSuccess) st = cuda_fail(cudaGetLastError(), "table");
    else {
      cudaMemcpy(tp, table.data(), table.size() * 8, cudaMemcpyHostToDevice);
      b->mp.table = tp;
    }
  }
  if (st == B12G_OK) st = batch_reserve(b, std::max<uint64_t>(1ull << 22, 4ull * n));
  // start from the family's usual shape; the first run tunes it unless this process has
  b->tuning = batch_tuning(b->device, scheme->map.kind, scheme->map.arith, scheme->grid.kind, domain->dim);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tuned.find(tune_key(b->device, scheme->map.kind, scheme->map.arith, scheme->grid.kind));
    if (it != g_tuned.end()) { b->tuning = it->second; b->tuned = true; }
  }
  if (st != B12G_OK) {
    b12g_batch_destroy(b);
    return st;
  }
  *out = b;
  return B12G_OK;
}

b12g_status b12g_batch_destroy(b12g_batch* b)
{
  if (!b) return B12G_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->mp.table) cudaFree(const_cast<double*>(b->mp.table));
  b->params.release(); b->depths.release(); b->hit.release(); b->cnt.release(); b->step_counts.release();
  b->ctr.release(); b->tiles_a.release(); b->tiles_b.release(); b->fin_lo.release(); b->fin_len.release();
  b->arena_off.release(); b->arena_inst.release(); b->hash.release();
  b->fin_code.release(); b->fin_flags.release(); b->stage_col.release(); b->stage_cnt.release();
  b->row_count.release(); b->rowptr.release(); b->cols.release(); b->vals.release();
  for (int q = 0; q < 2; ++q) { b->code[q].release(); b->flags[q].release(); b->off[q].release(); }
  if (b->h_ctr) cudaFreeHost(b->h_ctr);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return B12G_OK;
}

b12g_status b12g_batch_run(b12g_batch* b)
{
  if (!b) return fail(B12G_ERR_INVALID, "NULL batch");
  for (int attempt = 0; attempt < 10; ++attempt) {
    if (!b->tuned) {
      ST(autotune(b));
    } else {
      if (!b->graph) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t err = cudaSuccess;
        b->graph_kernels = 0;
        for (uint32_t k = 1; k <= b->max_depth && err == cudaSuccess; ++k) {
          err = enqueue_step(b, k, b->tuning);
          b->graph_kernels += step_kernels(b, k);
        }
        cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
        if (err != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(err, "batch capture"); }
        if (e2 != cudaSuccess) return cuda_fail(e2, "batch end capture");
        cudaError_t e3 = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) { b->graph = nullptr; return cuda_fail(e3, "batch instantiate"); }
      }
      ST(batch_reset(b));
      CK(cudaGraphLaunch(b->graph, b->stream));
      count_launches(b->graph_kernels);
    }
    ST(batch_read(b, 0, B_COUNT));
    if (b->h_ctr[B_ERROR] & 1u) {
      // capacity: grow 4x and run again (graph re-captured with the new buffers)
      if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
      ST(batch_reserve(b, b->cap * 4));
      continue;
    }
    ST(batch_collect(b));
    b->ran = true;
    b->has_tm = false;
    return B12G_OK;
  }
  return fail(B12G_ERR_CAPACITY, "batch run: capacity retries exhausted");
}

b12g_status b12g_batch_counts(b12g_batch* b, uint32_t i, uint32_t* counts)
{
  if (!b || !counts || i >= b->N) return fail(B12G_ERR_INVALID, "bad argument");
  if (!b->ran) return fail(B12G_ERR_INVALID, "batch has not run");
  const uint32_t q = b->pos[i];
  for (uint32_t k = 0; k < b->depth_sorted[q]; ++k) counts[k] = b->h_step_counts[size_t(k) * b->N + q];
  // a step that removed every box leaves the surrounding box (insertSurroundingBoxIfEmpty)
  bool empty = false;
  for (uint32_t k = 0; k < b->depth_sorted[q]; ++k) {
    if (counts[k] == 0) empty = true;
    if (empty) counts[k] = 1;
  }
  return B12G_OK;
}

b12g_status b12g_batch_leaves(b12g_batch* b, uint32_t i, uint64_t* codes, uint8_t* flags, uint32_t* n, uint8_t* depth)
{
  if (!b || i >= b->N) return fail(B12G_ERR_INVALID, "bad argument");
  if (!b->ran) return fail(B12G_ERR_INVALID, "batch has not run");
  const uint32_t q = b->pos[i];
  const uint32_t lo = b->h_fin_lo[q], hi = lo + b->h_fin_len[q];
  if (hi == lo) {
    if (n) *n = 1;
    if (depth) *depth = 0;
    if (codes) codes[0] = 0;
    if (flags) flags[0] = B12G_NONE;
    return B12G_OK;
  }
  if (n) *n = hi - lo;
  if (depth) *depth = b->depth_sorted[q];
  if (codes) CK(cudaMemcpyAsync(codes, b->fin_code.p + lo, size_t(hi - lo) * 8, cudaMemcpyDeviceToHost, b->stream));
  if (flags) CK(cudaMemcpyAsync(flags, b->fin_flags.p + lo, hi - lo, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return B12G_OK;
}

b12g_status b12g_batch_transition_matrices(b12g_batch* b, int absolute, int invalid_column)
{
  if (!b) return fail(B12G_ERR_INVALID, "NULL batch");
  if (!b->ran) return fail(B12G_ERR_INVALID, "batch has not run");
  const uint32_t rows = b->h_arena_off[b->N];
  const uint64_t stage = uint64_t(rows) * b->P;
  ST(b->stage_col.ensure(std::max<uint64_t>(stage, 1), "batch staging"));
  ST(b->stage_cnt.ensure(std::max<uint64_t>(stage, 1), "batch staging"));
  ST(b->row_count.ensure(rows + 1, "batch row counts"));
  ST(b->rowptr.ensure(rows + 1, "batch rowptr"));
  ST(b->tiles_a.ensure(compact_tiles(rows + 1) + 2, "batch tiles"));
  // lookup table over the final leaves, keyed by (instance, code)
  uint32_t l = 6;
  while ((1ull << l) < 2ull * std::max<uint32_t>(rows, 1)) ++l;
  if (l > b->hash_log2) {
    b->hash.release();
    ST(b->hash.ensure(size_t(1) << l, "batch lookup table"));
    b->hash_log2 = l;
  }
  CK(cudaMemsetAsync(b->hash.p, 0, b->hash.n * sizeof(ulonglong2), b->stream));
  const LeafHash h{b->hash.p, 1, b->hash_log2};
  batch_hash_build_kernel<<<device_sm_count() * 4, 256, 0, b->stream>>>(
      b->fin_code.p, b->arena_off.p, b->N, h, uint32_t(std::min<uint64_t>(b->fin_cap, 0xFFFFFFFFu)),
      b->ctr.p + B_ERROR);
  BatchRowArgs ra{};
  ra.dom = b->dom;
  ra.map = b->mp;
  ra.grid = b->gp;
  ra.points = b->P;
  ra.params = b->params.p;
  ra.depths = b->depths.p;
  ra.n_inst = b->N;
  ra.off = b->arena_off.p;
  ra.inst_of = b->arena_inst.p;
  ra.codes = b->fin_code.p;
  ra.hash = h;
  ra.keep_lost = invalid_column ? 1 : 0;
  ra.stage_col = b->stage_col.p;
  ra.stage_cnt = b->stage_cnt.p;
  ra.row_count = b->row_count.p;
  CK(launch_batch_rows(b->scheme.map.kind, b->scheme.map.arith, b->scheme.grid.kind, ra, rows, b->stream));
  CK(exclusive_scan_u32(b->row_count.p, b->rowptr.p, b->arena_off.p + b->N, b->tiles_a.p, rows, b->stream));
  uint32_t nnz = 0;
  CK(cudaMemcpyAsync(&nnz, b->rowptr.p + rows, 4, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  ST(b->cols.ensure(std::max<uint32_t>(nnz, 1), "batch cols"));
  ST(b->vals.ensure(std::max<uint32_t>(nnz, 1), "batch vals"));
  CK(gather_rows(b->stage_col.p, b->stage_cnt.p, uint32_t(b->P), b->row_count.p, b->rowptr.p, b->arena_off.p + b->N,
                 b->cols.p, b->vals.p, absolute, double(b->P), rows, b->stream));
  count_launches(7);
  b->h_rowptr_arena.assign(b->N + 1, 0);
  for (uint32_t a = 0; a <= b->N; ++a)
    CK(cudaMemcpyAsync(&b->h_rowptr_arena[a], b->rowptr.p + b->h_arena_off[a], 4, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  ST(batch_read(b, 0, 1));
  if (b->h_ctr[B_ERROR] & 1u) return fail(B12G_ERR_CAPACITY, "batch transition matrices: lookup table overflow");
  b->nnz = nnz;
  b->has_tm = true;
  b->tm_invalid = invalid_column;
  return B12G_OK;
}

b12g_status b12g_batch_csr(b12g_batch* b, uint32_t i, uint32_t* rowptr, uint32_t* cols, double* vals, uint32_t* n_rows,
                           uint64_t* nnz)
{
  if (!b || i >= b->N) return fail(B12G_ERR_INVALID, "bad argument");
  if (!b->has_tm) return fail(B12G_ERR_INVALID, "no transition matrices computed");
  const uint32_t a = b->h_arena_of[b->pos[i]];
  const uint32_t lo = b->h_arena_off[a], hi = b->h_arena_off[a + 1];
  const uint32_t e0 = b->h_rowptr_arena[a], e1 = b->h_rowptr_arena[a + 1];
  if (n_rows) *n_rows = hi - lo;
  if (nnz) *nnz = e1 - e0;
  if (rowptr) {
    std::vector<uint32_t> r(hi - lo + 1);
    CK(cudaMemcpyAsync(r.data(), b->rowptr.p + lo, r.size() * 4, cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    for (size_t x = 0; x < r.size(); ++x) rowptr[x] = r[x] - e0;
  }
  if (cols && e1 > e0) CK(cudaMemcpyAsync(cols, b->cols.p + e0, size_t(e1 - e0) * 4, cudaMemcpyDeviceToHost, b->stream));
  if (vals && e1 > e0) CK(cudaMemcpyAsync(vals, b->vals.p + e0, size_t(e1 - e0) * 8, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return B12G_OK;
}

b12g_status b12g_batch_info(b12g_batch* b, uint64_t* box_images, uint64_t* final_boxes, uint64_t* nnz,
                            uint32_t* threads, uint32_t* points_per_thread, uint32_t* chunk)
{
  if (!b) return fail(B12G_ERR_INVALID, "NULL batch");
  if (box_images) {
    // every subdivision step images the children of the instance's boxes: 2 x previous count
    uint64_t s = 0;
    if (b->ran)
      for (uint32_t q = 0; q < b->N; ++q) {
        uint64_t prev = 1;
        for (uint32_t k = 0; k < b->depth_sorted[q]; ++k) {
          s += 2 * prev;
          prev = b->h_step_counts[size_t(k) * b->N + q];
        }
      }
    *box_images = s;
  }
  if (final_boxes) *final_boxes = b->ran ? b->h_arena_off[b->N] : 0;
  if (nnz) *nnz = b->has_tm ? b->nnz : 0;
  if (threads) *threads = b->tuning.threads;
  if (points_per_thread) *points_per_thread = b->tuning.ppt;
  if (chunk) *chunk = b->tuning.chunk;
  return B12G_OK;
}

b12g_status b12g_batch_stream(b12g_batch* b, void** stream)
{
  if (!b || !stream) return fail(B12G_ERR_INVALID, "NULL argument");
  *stream = (void*)b->stream;
  return B12G_OK;
}

}  // extern "C"
