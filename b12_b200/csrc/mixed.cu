// Trees whose leaves have different depths.
//
// The reference stores every leaf with its own depth and keeps the leaves in the order
// of isStrictlyPreceding (Box.hpp:124-135): by the comparable bit pattern
// getComparableBitPattern (Box.hpp:67-73) - the code moved to the top of 64 bits with
// 0111...1 below it - and, for equal patterns, deeper first.  A point is located by
// thrust::lower_bound over the leaves followed by ComputeSearchIndexFunctor
// (Functors.hpp:289-315): the leaf before the lower bound, or the one at it, that lies
// on the point's path (hasSamePath, Box.hpp:75-83).
//
// A tree enters this mode when an operation would give its leaves different depths (a
// subdivision of some of the leaves, a load of such leaves) and leaves it again when an
// operation leaves one depth behind.  The operations of the box-image path keep their
// reference semantics here: flags on the leaves, count, depth, subdivide, remove,
// setFlagsByIterators, searchByIterators, transitionMatrixForLeaves.  Leaf lookups are
// binary searches over the comparable patterns (a mixed tree has no single-depth table).
#include <algorithm>
#include <cstring>
#include <vector>

#include "rows.cuh"
#include "tree.h"

using namespace b12g;
using namespace b12g::host;

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kTable = 2048;   // doubles of the per-block grid-point table

int grid_for_n(uint64_t n, int per_thread = 1)
{
  const uint64_t want = (n + uint64_t(kThreads) * per_thread - 1) / (uint64_t(kThreads) * per_thread);
  const uint64_t cap = uint64_t(device_sm_count()) * 8;
  return int(std::max<uint64_t>(1, std::min(want, cap)));
}

__host__ __device__ __forceinline__ uint64_t comparable(uint64_t code, uint32_t depth)
{
  const uint32_t shift = 64u - depth;           // getComparableBitPattern with safe shifts
  const uint64_t high = shift >= 64 ? 0ull : (code << shift);
  const uint64_t fill = shift >= 2 ? ((1ull << (shift - 1)) - 1ull) : 0ull;
  return high | fill;
}

// hasSamePath of a depth-64 point and a leaf: the leaf's code is the point's prefix
__device__ __forceinline__ bool on_path(uint64_t p64, uint64_t code, uint32_t depth)
{
  const uint32_t shift = 64u - depth;
  return (shift >= 64 ? 0ull : (p64 >> shift)) == code;
}

// search of one point among the leaves (ImplicitBoxTree.hpp:2394-2432, leaf branch)
__device__ __forceinline__ uint32_t locate_mixed(const uint64_t* __restrict__ cmp, const uint64_t* __restrict__ code,
                                                 const uint8_t* __restrict__ dep, uint32_t n, bool valid,
                                                 uint64_t p64)
{
  if (n == 0) return kInvalidIndex;
  if (!valid) {
    // the invalid box shares its path with a last leaf of code 0
    return __ldg(code + n - 1) == 0 ? n - 1 : kInvalidIndex;
  }
  // lower bound: first leaf that does not strictly precede the depth-64 point box
  uint32_t lo = 0, len = n;
  while (len > 0) {
    const uint32_t half = len >> 1;
    if (__ldg(cmp + lo + half) < p64) {
      lo += half + 1;
      len -= half + 1;
    } else {
      len = half;
    }
  }
  const uint32_t a = lo > 0 ? lo - 1 : 0;
  const uint32_t b = lo < n - 1 ? lo : n - 1;
  if (on_path(p64, __ldg(code + a), __ldg(dep + a))) return lo > 0 ? lo - 1 : 0;
  if (on_path(p64, __ldg(code + b), __ldg(dep + b))) return lo;
  return kInvalidIndex;
}

__global__ void comparable_kernel(const uint64_t* code, const uint8_t* dep, uint32_t n, uint64_t* cmp)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    cmp[i] = comparable(code[i], dep[i]);
}

__global__ void depth_range_kernel(const uint8_t* dep, uint32_t n, uint32_t* range)
{
  uint32_t lo = 255, hi = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    lo = min(lo, uint32_t(dep[i]));
    hi = max(hi, uint32_t(dep[i]));
  }
  atomicMin(range, lo);
  atomicMax(range + 1, hi);
}

// 1 where the leaf starts a new box at `d` (count(depth), ImplicitBoxTree.hpp:1061-1095)
__global__ void new_box_kernel(const uint64_t* code, const uint8_t* dep, uint32_t n, uint32_t d, uint32_t* count)
{
  uint32_t c = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (dep[i] < d) continue;
    const uint64_t pre = code[i] >> (dep[i] - d);
    bool fresh = i == 0 || dep[i - 1] < d;
    if (!fresh) fresh = (code[i - 1] >> (dep[i - 1] - d)) != pre;
    c += fresh;
  }
  if (c) atomicAdd(count, c);
}

// subdivide: a flagged leaf below depth 64 becomes its two halves in place (order kept)
__global__ void split_count_kernel(const uint8_t* flags, const uint8_t* dep, uint32_t n, uint8_t f, uint32_t* cnt)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    cnt[i] = (uint8_t(flags[i] & f) == f && dep[i] < 64) ? 2u : 1u;
}

__global__ void split_scatter_kernel(const uint64_t* code, const uint8_t* flags, const uint8_t* dep, uint32_t n,
                                     const uint32_t* pos, uint64_t* out_code, uint8_t* out_flags, uint8_t* out_dep)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t p = pos[i];
    if (pos[i + 1] - p == 2) {
      out_code[p] = code[i] << 1;
      out_code[p + 1] = (code[i] << 1) | 1ull;
      out_flags[p] = out_flags[p + 1] = flags[i];
      out_dep[p] = out_dep[p + 1] = uint8_t(dep[i] + 1);
    } else {
      out_code[p] = code[i];
      out_flags[p] = flags[i];
      out_dep[p] = dep[i];
    }
  }
}

// keep marks of remove(flags) and of a scheme's source filter: all of f set
__global__ void keep_kernel(const uint8_t* flags, uint32_t n, uint8_t f, uint32_t* keep)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    keep[i] = uint8_t(flags[i] & f) == f ? 1u : 0u;
}

__global__ void keep_scatter_kernel(const uint64_t* code, const uint8_t* flags, const uint8_t* dep, uint32_t n,
                                    const uint32_t* pos, uint64_t* out_code, uint8_t* out_flags, uint8_t* out_dep,
                                    uint32_t* out_index)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t p = pos[i];
    if (pos[i + 1] == p) continue;
    if (out_index) {
      out_index[p] = i;
    } else {
      out_code[p] = code[i];
      out_flags[p] = flags[i];
      out_dep[p] = dep[i];
    }
  }
}

__global__ void apply_hits_kernel(uint8_t* flags, uint8_t* hit, uint32_t n, uint8_t f, uint32_t* changed)
{
  uint32_t c = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!hit[i]) continue;
    hit[i] = 0;
    c += uint8_t(flags[i] & f) != f;
    flags[i] |= f;
  }
  if (c) atomicAdd(changed, c);
}

// ---------------------------------------------------------------------------- images
struct MixedArgs {
  Domain dom;
  MapParams map;
  GridParams grid;
  uint64_t points;
  const uint64_t* code;
  const uint8_t* dep;
  const uint64_t* cmp;
  uint32_t n;                  // leaves
  const uint32_t* src;         // source leaves (nullptr: every leaf)
  uint32_t n_src;
  uint8_t* hit;                // Hit: marks of the leaves hit
  uint32_t* out;               // Search: leaf index of every point
  // transition rows
  uint32_t* stage_col;
  uint32_t* stage_cnt;
  uint32_t* row_count;
  int keep_lost;
  uint32_t lost_col;
};

template<class Grid, int D>
__device__ __forceinline__ bool load_table(const GridParams& g, uint64_t P, double* pts)
{
  const bool table = Grid::kTable && P * D <= kTable;
  if (table) {
    for (uint32_t idx = threadIdx.x; idx < uint32_t(P) * D; idx += blockDim.x) {
      const int j = int(idx / uint32_t(P));
      pts[idx] = Grid::table_value(g, g.coord, idx - uint32_t(j) * uint32_t(P), j);
    }
  } else {
    for (uint32_t i = threadIdx.x; i < 64; i += blockDim.x) pts[i] = g.coord[i];
  }
  __syncthreads();
  return table;
}

// the leaf the image of point k of source leaf `leaf` lands in (point index g)
template<class Map, class Grid>
__device__ __forceinline__ uint32_t image_of(const MixedArgs& a, const double* pts, bool table, uint32_t leaf,
                                             uint32_t k, uint64_t g)
{
  constexpr int D = Map::D;
  double c[D], r[D], gp[D], x[D], y[D];
  box_coordinates<D>(a.dom, __ldg(a.code + leaf), int(__ldg(a.dep + leaf)), c, r);
  if (Grid::kTable && table) {
#pragma unroll
    for (int j = 0; j < D; ++j) gp[j] = pts[j * uint32_t(a.points) + k];
  } else {
    Grid::template point<D>(a.grid, pts, g, k, gp);
  }
#pragma unroll
  for (int j = 0; j < D; ++j) x[j] = __dadd_rn(c[j], __dmul_rn(gp[j], r[j]));
  Map::apply(a.map, x, y);
  uint64_t p64 = 0;
  const bool valid = point_code<D>(a.dom, y, 64, p64);
  return locate_mixed(a.cmp, a.code, a.dep, a.n, valid, p64);
}

template<class Map, class Grid, bool kSearch>
__global__ void __launch_bounds__(kThreads) mixed_image_kernel(const MixedArgs a)
{
  __shared__ double pts[kTable];
  const bool table = load_table<Grid, Map::D>(a.grid, a.points, pts);
  const uint64_t P = a.points;
  const uint64_t total = uint64_t(a.n_src) * P;
  for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < total; g += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t rank = g / P;
    const uint32_t k = uint32_t(g - rank * P);
    const uint32_t leaf = a.src ? __ldg(a.src + rank) : uint32_t(rank);
    const uint32_t t = image_of<Map, Grid>(a, pts, table, leaf, k, g);
    if constexpr (kSearch) a.out[g] = t;
    else if (t != kInvalidIndex) a.hit[t] = 1;
  }
}

// a warp per leaf: its P <= 128 targets sorted and run-length counted (as for uniform trees)
template<class Map, class Grid>
__global__ void __launch_bounds__(kThreads) mixed_rows_kernel(const MixedArgs a)
{
  constexpr int kWarps = kThreads / 32;
  __shared__ double pts[kTable];
  __shared__ uint32_t keys[kWarps][128];
  __shared__ uint32_t bounds[kWarps][4];
  const bool table = load_table<Grid, Map::D>(a.grid, a.points, pts);
  const uint32_t P = uint32_t(a.points);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t* s = keys[w];
  for (uint32_t row = blockIdx.x * kWarps + w; row < a.n; row += gridDim.x * kWarps) {
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
      const uint32_t k = uint32_t(lane) + 32u * q;
      uint32_t key = kPadKey;
      if (k < P) {
        const uint32_t t = image_of<Map, Grid>(a, pts, table, row, k, uint64_t(row) * P + k);
        key = t == kInvalidIndex ? kLostKey : t;
      }
      s[lane + 32 * q] = key;
    }
    const uint32_t total = row_emit(s, bounds[w], lane, P, a.keep_lost, a.lost_col, a.stage_col + size_t(row) * P,
                                    a.stage_cnt + size_t(row) * P);
    if (lane == 0) a.row_count[row] = total;
    __syncwarp();
  }
}

template<class F>
cudaError_t dispatch(uint32_t map_kind, uint32_t arith, uint32_t grid_kind, uint32_t dim, F&& f)
{
  auto with_grid = [&](auto map_tag) -> cudaError_t {
    using Map = decltype(map_tag);
    if (dim != uint32_t(Map::D)) return cudaErrorInvalidValue;
    switch (grid_kind) {
      case B12G_GRID_INNER: return f(Map{}, InnerGrid{});
      case B12G_GRID_FULL: return f(Map{}, FullGrid{});
      case B12G_GRID_PHILOX: return f(Map{}, PhiloxGrid{});
      default: return cudaErrorInvalidValue;
    }
  };
  switch (map_kind) {
    case B12G_MAP_HENON: return arith == B12G_ARITH_STRICT ? with_grid(HenonMap{}) : cudaErrorInvalidValue;
    case B12G_MAP_LORENZ:
      return arith == B12G_ARITH_FMA ? with_grid(LorenzMap<Fused>{}) : with_grid(LorenzMap<Strict>{});
    case B12G_MAP_COUPLED_DUFFING:
      return arith == B12G_ARITH_STRICT ? with_grid(CoupledDuffingMap{}) : cudaErrorInvalidValue;
    case B12G_MAP_FORCED_DUFFING:
      return arith == B12G_ARITH_STRICT ? with_grid(ForcedDuffingMap{}) : cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
  }
}

// ---------------------------------------------------------------------------- host helpers
uint8_t* dep_cur(b12g_tree* t) { return t->dep[t->cur].p; }

b12g_status ensure_dep(b12g_tree* t, uint64_t n)
{
  for (int q = 0; q < 2; ++q) ST(t->dep[q].grow_keep(std::max<uint64_t>(n, 1), q == t->cur ? t->n : 0, t->stream,
                                                     "leaf depths"));
  return B12G_OK;
}

// exclusive scan of n u32 marks into pos (n + 1 entries, pos[n] = total)
b12g_status scan_marks(b12g_tree* t, const uint32_t* marks, uint32_t* pos, uint32_t n, uint32_t* total)
{
  ST(t->tiles_a.ensure(compact_tiles(uint64_t(n) + 1) + 2, "tiles"));
  ST(set_ctr(t, C_TMP, n));
  CK(exclusive_scan_u32(marks, pos, t->ctr.p + C_TMP, t->tiles_a.p, n, t->stream));
  CK(cudaMemcpyAsync(t->h_ctr + C_TMP, pos + n, 4, cudaMemcpyDeviceToHost, t->stream));
  ST(sync(t, "scan"));
  count_launches(3);
  *total = t->h_ctr[C_TMP];
  return B12G_OK;
}

b12g_status refresh_comparable(b12g_tree* t)
{
  ST(t->cmp.ensure(std::max<uint32_t>(t->n, 1), "comparable patterns"));
  comparable_kernel<<<grid_for_n(t->n), kThreads, 0, t->stream>>>(t->codes(), dep_cur(t), t->n, t->cmp.p);
  count_launches(1);
  return B12G_OK;
}

// the scheme's source leaves: every leaf with all the scheme's flags
b12g_status mixed_sources(b12g_tree* t, const b12g_scheme* sc, const uint32_t** src, uint32_t* n_src)
{
  if (sc->flags_to_check == 0) {
    *src = nullptr;
    *n_src = t->n;
    return B12G_OK;
  }
  ST(t->row_count.ensure(uint64_t(t->n) + 1, "source marks"));
  ST(t->rowptr.ensure(uint64_t(t->n) + 1, "source positions"));
  ST(t->src.ensure(std::max<uint32_t>(t->n, 1), "source list"));
  keep_kernel<<<grid_for_n(t->n), kThreads, 0, t->stream>>>(t->flg(), t->n, sc->flags_to_check, t->row_count.p);
  uint32_t total = 0;
  ST(scan_marks(t, t->row_count.p, t->rowptr.p, t->n, &total));
  keep_scatter_kernel<<<grid_for_n(t->n), kThreads, 0, t->stream>>>(nullptr, nullptr, nullptr, t->n, t->rowptr.p,
                                                                     nullptr, nullptr, nullptr, t->src.p);
  count_launches(2);
  *src = t->src.p;
  *n_src = total;
  return B12G_OK;
}

b12g_status mixed_args(b12g_tree* t, const b12g_scheme* sc, MixedArgs& a)
{
  if (sc && sc->depth != B12G_LEAF_DEPTH)
    return fail(B12G_ERR_UNSUPPORTED_MIXED_DEPTH, "the scheme of a tree of mixed depths maps its leaves (depth 255)");
  Prepared pr;
  ST(prepare(t, sc, pr));
  a = MixedArgs{};
  a.dom = pr.a.dom;
  a.map = pr.a.map;
  a.grid = pr.a.grid;
  a.points = pr.P;
  a.code = t->codes();
  a.dep = dep_cur(t);
  a.n = t->n;
  ST(refresh_comparable(t));
  a.cmp = t->cmp.p;
  return B12G_OK;
}

}  // namespace

namespace b12g {
namespace host {

b12g_status mixed_enter(b12g_tree* t)
{
  if (t->mixed) return B12G_OK;
  ST(ensure_dep(t, std::max<uint64_t>(t->code[0].n, t->n)));
  CK(cudaMemsetAsync(dep_cur(t), t->depth, t->n, t->stream));
  t->mixed = true;
  return sync(t, "mixed depths");
}

// back to one depth when every leaf has the same one
b12g_status mixed_settle(b12g_tree* t)
{
  if (!t->mixed) return B12G_OK;
  ST(set_ctr(t, C_TMP, 255));
  ST(set_ctr(t, C_TMP + 1, 0));
  depth_range_kernel<<<grid_for_n(t->n), kThreads, 0, t->stream>>>(dep_cur(t), t->n, t->ctr.p + C_TMP);
  count_launches(1);
  ST(read_ctr(t, C_TMP, 2));
  if (t->h_ctr[C_TMP] == t->h_ctr[C_TMP + 1]) {
    t->depth = uint8_t(t->h_ctr[C_TMP]);
    t->mixed = false;
  } else {
    t->depth = uint8_t(t->h_ctr[C_TMP + 1]);
  }
  return B12G_OK;
}

b12g_status mixed_load(b12g_tree* t, const uint64_t* codes, const uint8_t* depths, const uint8_t* flags, uint32_t n)
{
  // the leaves must be in the reference's order and no leaf may contain another
  for (uint32_t i = 0; i < n; ++i) {
    if (depths[i] > 64) return fail(B12G_ERR_INVALID, "depth %u above the maximal depth 64", depths[i]);
    if (depths[i] < 64 && (codes[i] >> depths[i]) != 0) return fail(B12G_ERR_INVALID, "code %u has bits above its depth", i);
    if (i) {
      const uint64_t a = comparable(codes[i - 1], depths[i - 1]), b = comparable(codes[i], depths[i]);
      const uint32_t d = std::min(depths[i - 1], depths[i]);
      const bool nested = (d == 0) || ((codes[i - 1] >> (depths[i - 1] - d)) == (codes[i] >> (depths[i] - d)));
      if (!(a < b) || nested) return fail(B12G_ERR_INVALID, "leaves %u and %u are out of order or nested", i - 1, i);
    }
  }
  ST(reserve(t, n));
  ST(ensure_dep(t, std::max<uint64_t>(t->code[0].n, n)));
  CK(cudaMemcpyAsync(t->codes(), codes, size_t(n) * 8, cudaMemcpyHostToDevice, t->stream));
  CK(cudaMemcpyAsync(t->flg(), flags, n, cudaMemcpyHostToDevice, t->stream));
  CK(cudaMemcpyAsync(dep_cur(t), depths, n, cudaMemcpyHostToDevice, t->stream));
  t->n = n;
  t->mixed = true;
  ST(set_ctr(t, t->ncur, n));
  ST(sync(t, "load leaves"));
  return mixed_settle(t);
}

b12g_status mixed_count(b12g_tree* t, uint8_t depth, uint32_t* count)
{
  if (depth == 0) {
    *count = 1;
    return B12G_OK;
  }
  if (depth == B12G_LEAF_DEPTH) {
    *count = t->n;
    return B12G_OK;
  }
  ST(set_ctr(t, C_TMP, 0));
  new_box_kernel<<<grid_for_n(t->n), kThreads, 0, t->stream>>>(t->codes(), dep_cur(t), t->n, depth, t->ctr.p + C_TMP);
  count_launches(1);
  ST(read_ctr(t, C_TMP, 1));
  *count = t->h_ctr[C_TMP];
  return B12G_OK;
}

b12g_status mixed_leaves(b12g_tree* t, uint64_t* codes, uint8_t* depths, uint8_t* flags)
{
  if (codes) CK(cudaMemcpyAsync(codes, t->codes(), size_t(t->n) * 8, cudaMemcpyDeviceToHost, t->stream));
  if (flags) CK(cudaMemcpyAsync(flags, t->flg(), t->n, cudaMemcpyDeviceToHost, t->stream));
  if (depths) CK(cudaMemcpyAsync(depths, dep_cur(t), t->n, cudaMemcpyDeviceToHost, t->stream));
  return sync(t, "leaves");
}

// subdivide (ImplicitBoxTree.hpp:2884-2929): every leaf below depth 64 with all flags
// set becomes its two halves, which take its place in the order (the halves of a leaf
// sort between its neighbours); returns the leaves with all flags set
b12g_status mixed_subdivide(b12g_tree* t, uint8_t flags, uint32_t* n_subdivided)
{
  const uint32_t n = t->n;
  ST(set_ctr(t, C_CAND, 0));
  CK(count_flags(t->flg(), t->dn(), flags, t->ctr.p + C_CAND, n, t->stream));
  ST(t->row_count.ensure(uint64_t(n) + 1, "split counts"));
  ST(t->rowptr.ensure(uint64_t(n) + 1, "split positions"));
  split_count_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(t->flg(), dep_cur(t), n, flags, t->row_count.p);
  count_launches(2);
  uint32_t total = 0;
  ST(scan_marks(t, t->row_count.p, t->rowptr.p, n, &total));
  ST(read_ctr(t, C_CAND, 1));
  if (n_subdivided) *n_subdivided = t->h_ctr[C_CAND];
  if (total == n) return B12G_OK;
  ST(reserve(t, total));
  const int o = 1 - t->cur, no = 1 - t->ncur;
  split_scatter_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(t->codes(), t->flg(), dep_cur(t), n, t->rowptr.p,
                                                                    t->code[o].p, t->flags[o].p, t->dep[o].p);
  count_launches(1);
  t->cur = o;
  t->ncur = no;
  t->n = total;
  ST(set_ctr(t, t->ncur, total));
  ST(sync(t, "subdivide"));
  return mixed_settle(t);
}

b12g_status mixed_remove(b12g_tree* t, uint8_t flags, uint32_t* n_removed)
{
  const uint32_t n = t->n;
  ST(t->row_count.ensure(uint64_t(n) + 1, "keep marks"));
  ST(t->rowptr.ensure(uint64_t(n) + 1, "keep positions"));
  keep_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(t->flg(), n, flags, t->row_count.p);
  count_launches(1);
  uint32_t kept = 0;
  ST(scan_marks(t, t->row_count.p, t->rowptr.p, n, &kept));
  const int o = 1 - t->cur, no = 1 - t->ncur;
  keep_scatter_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(t->codes(), t->flg(), dep_cur(t), n, t->rowptr.p,
                                                                   t->code[o].p, t->flags[o].p, t->dep[o].p, nullptr);
  count_launches(1);
  t->cur = o;
  t->ncur = no;
  t->n = kept;
  ST(set_ctr(t, t->ncur, kept));
  ST(sync(t, "remove"));
  if (n_removed) *n_removed = n - kept;
  if (kept == 0) return set_root(t, B12G_NONE);  // insertSurroundingBoxIfEmpty; one depth again
  return mixed_settle(t);
}

b12g_status mixed_set_flags_by_image(b12g_tree* t, const b12g_scheme* sc, uint8_t flags, uint8_t depth,
                                     uint32_t* n_changed)
{
  if (depth != B12G_LEAF_DEPTH)
    return fail(B12G_ERR_UNSUPPORTED_MIXED_DEPTH, "images flag the leaves (depth 255) of a tree of mixed depths");
  MixedArgs a;
  ST(mixed_args(t, sc, a));
  ST(mixed_sources(t, sc, &a.src, &a.n_src));
  if (t->hit.n < t->n) {
    // the hit marks are all clear between calls (apply_hits clears what it reads)
    ST(t->hit.ensure(t->n, "hit marks"));
    CK(cudaMemsetAsync(t->hit.p, 0, t->hit.n, t->stream));
  }
  a.hit = t->hit.p;
  CK(dispatch(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, [&](auto map, auto grid) -> cudaError_t {
    mixed_image_kernel<decltype(map), decltype(grid), false>
        <<<grid_for_n(uint64_t(a.n_src) * a.points), kThreads, 0, t->stream>>>(a);
    return cudaGetLastError();
  }));
  ST(set_ctr(t, C_CHANGED, 0));
  apply_hits_kernel<<<grid_for_n(t->n), kThreads, 0, t->stream>>>(t->flg(), t->hit.p, t->n, flags,
                                                                   t->ctr.p + C_CHANGED);
  count_launches(2);
  ST(read_ctr(t, C_CHANGED, 1));
  if (n_changed) *n_changed = t->h_ctr[C_CHANGED];
  return B12G_OK;
}

// leaf index of every point of every source leaf into t->out (device); *n_points
b12g_status mixed_search(b12g_tree* t, const b12g_scheme* sc, uint64_t* n_points)
{
  MixedArgs a;
  ST(mixed_args(t, sc, a));
  ST(mixed_sources(t, sc, &a.src, &a.n_src));
  const uint64_t np = uint64_t(a.n_src) * a.points;
  ST(t->out.ensure(std::max<uint64_t>(np, 1), "search output"));
  a.out = t->out.p;
  CK(dispatch(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, [&](auto map, auto grid) -> cudaError_t {
    mixed_image_kernel<decltype(map), decltype(grid), true><<<grid_for_n(np), kThreads, 0, t->stream>>>(a);
    return cudaGetLastError();
  }));
  count_launches(1);
  *n_points = np;
  return B12G_OK;
}

// the transition rows of every leaf into the tree's staging arrays (rows = leaves)
b12g_status mixed_rows(b12g_tree* t, const b12g_scheme* sc, int invalid_column)
{
  MixedArgs a;
  ST(mixed_args(t, sc, a));
  const uint64_t stage = uint64_t(t->n) * a.points;
  ST(t->stage_col.ensure(stage, "row staging"));
  ST(t->stage_cnt.ensure(stage, "row staging"));
  ST(t->row_count.ensure(uint64_t(t->n) + 1, "row counts"));
  a.stage_col = t->stage_col.p;
  a.stage_cnt = t->stage_cnt.p;
  a.row_count = t->row_count.p;
  a.keep_lost = invalid_column ? 1 : 0;
  a.lost_col = t->n + 1;
  a.n_src = t->n;
  CK(dispatch(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, [&](auto map, auto grid) -> cudaError_t {
    mixed_rows_kernel<decltype(map), decltype(grid)>
        <<<std::max(1, std::min<int>(int((t->n + 7) / 8), device_sm_count() * 8)), kThreads, 0, t->stream>>>(a);
    return cudaGetLastError();
  }));
  count_launches(1);
  return B12G_OK;
}

}  // namespace host
}  // namespace b12g
