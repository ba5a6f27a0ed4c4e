// Fused box-image kernels: per test point, box centre -> grid point -> map -> depth-d
// code -> leaf index, all in FP64 registers.  This is the reference's
// GridPointsFunctor (Functors.hpp:476-511) consumed by thrust::lower_bound and
// ComputeSearchIndexFunctor (ImplicitBoxTree.hpp:2394-2432), evaluated once per point
// instead of twice and without the point stream ever being stored.
#include "kernels.h"
#include "rows.cuh"

namespace b12g {

namespace {

constexpr int kThreads = 256;

// the source box of point (rank, k) and the leaf index its image lands in
template<class Map, class Grid>
struct PointImage {
  static constexpr int D = Map::D;

  // per-dimension indices of source box `leaf` at a.depth (in children mode: child
  // leaf & 1 of leaf leaf >> 1): from the packed keys the lookup table was built from,
  // else from the code
  static __device__ __forceinline__ void source_bits(const ImageArgs& a, uint32_t leaf, uint32_t (&bits)[D])
  {
    if (a.hash.pk) {
      if (a.children) {
        unpack_bits_k<D>(__ldg(a.hash.pk + (leaf >> 1)), a.dc.kp, bits);
        const int jd = a.dc.jd;                    // the last bisection splits dimension jd
#pragma unroll
        for (int j = 0; j < D; ++j)                // (no dynamic index: the array stays in registers)
          if (j == jd) bits[j] = (bits[j] << 1) | (leaf & 1u);
      } else {
        unpack_bits_k<D>(__ldg(a.hash.pk + leaf), a.dc.k, bits);
      }
      return;
    }
    const uint64_t code =
        a.children ? ((__ldg(a.codes + (leaf >> 1)) << 1) | uint64_t(leaf & 1u)) : __ldg(a.codes + leaf);
#pragma unroll
    for (int j = 0; j < D; ++j) bits[j] = deinterleave<D>(code, a.depth, j);
  }

  // returns whether the image point lies in the domain; `tbits` its box's per-dimension
  // indices at a.depth.  `pts` is the block's grid-point table (dimension-major, P
  // entries per dimension) when the grid has one, else the 1-D coordinate table.
  // the same from the source box's centre (its radius is the launch's)
  static __device__ __forceinline__ bool image_at(const ImageArgs& a, const double* pts, bool use_table,
                                                  const double (&c)[D], uint64_t i, uint32_t k, uint32_t (&tbits)[D])
  {
    double g[D], x[D], y[D];
    if (Grid::kTable && use_table) {
#pragma unroll
      for (int j = 0; j < D; ++j) g[j] = pts[j * uint32_t(a.points) + k];
    } else {
      Grid::template point<D>(a.grid, pts, i, k, g);
    }
#pragma unroll
    for (int j = 0; j < D; ++j) x[j] = __dadd_rn(c[j], __dmul_rn(g[j], a.dc.ax[j].rk));
    Map::apply(a.map, x, y);
    return point_bits<D>(a.dom, a.dc, y, tbits);
  }

  static __device__ __forceinline__ bool image(const ImageArgs& a, const double* pts, bool use_table,
                                               const uint32_t (&sbits)[D], uint64_t i, uint32_t k,
                                               uint32_t (&tbits)[D])
  {
    double c[D], r;
#pragma unroll
    for (int j = 0; j < D; ++j) box_axis(a.dom, a.dc.ax[j], j, sbits[j], c[j], r);
    return image_at(a, pts, use_table, c, i, k, tbits);
  }

  // centre of source `rank` from the launch's table
  static __device__ __forceinline__ void source_centre(const ImageArgs& a, uint64_t rank, double (&c)[D])
  {
    const double2* p = reinterpret_cast<const double2*>(a.src_c + kSrcStride * rank);
    const double2 c01 = __ldg(p);
    c[0] = c01.x;
    if (D > 1) c[D > 1 ? 1 : 0] = c01.y;
    if (D > 2) {
      const double2 c23 = __ldg(p + 1);
      c[D > 2 ? 2 : 0] = c23.x;
      if (D > 3) c[D > 3 ? 3 : 0] = c23.y;
    }
  }

  static __device__ __forceinline__ uint32_t target(const ImageArgs& a, uint32_t n, bool valid,
                                                    const uint32_t (&tbits)[D])
  {
    if (!a.children) return find_leaf_bits<D>(a.hash, a.codes, n, valid, tbits, a.depth, a.dc.k);
    if (!valid) return kInvalidIndex;
    const int jd = a.dc.jd;
    uint32_t pbits[D], child = 0;
#pragma unroll
    for (int j = 0; j < D; ++j) {
      pbits[j] = j == jd ? tbits[j] >> 1 : tbits[j];
      if (j == jd) child = tbits[j] & 1u;
    }
    const uint32_t p = find_leaf_bits<D>(a.hash, a.codes, n, true, pbits, a.depth - 1, a.dc.kp);
    return p == kInvalidIndex ? kInvalidIndex : 2u * p + child;
  }
};

constexpr uint32_t kPointTable = 2048;  // doubles of grid-point table per block (16 KB)
constexpr int kChunkTrips = 4;          // points per lane in a chunk of the image kernel's work queue

// fills `pts` with the P x D grid points when they fit (returns true), else with the
// 1-D coordinates for the per-point path
template<class Grid, int D>
__device__ __forceinline__ bool load_points(const GridParams& g, uint64_t P, double* pts)
{
  const bool table = Grid::kTable && P * D <= kPointTable;
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

template<class Map, class Grid, ImageMode M>
__global__ void __launch_bounds__(kThreads, 6) image_points_kernel(const ImageArgs a)
{
  using PI = PointImage<Map, Grid>;
  __shared__ double pts[kPointTable];
  const bool table = load_points<Grid, Map::D>(a.grid, a.points, pts);

  const uint32_t n = *a.n_leaves;
  const uint32_t nboxes = M == ImageMode::Mark ? a.n_src_value : a.n_src ? *a.n_src : (a.children ? 2u * n : n);
  const uint64_t P = a.points;
  const uint32_t P32 = uint32_t(P);
  const uint64_t total = uint64_t(nboxes) * P;
  const int lane = threadIdx.x & 31;
  if (M == ImageMode::Hit && a.children && 2ull * n > a.hit_cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(a.error, 1u);
    return;
  }
  // One point of the launch: g = rank * P + k (the source's rank among the sources, the
  // point's index in its box).  Every lane of the warp calls it the same number of times
  // (inactive lanes with active = false), so that the warp collectives stay converged.
  auto point = [&](uint64_t g, uint32_t rank, uint32_t k, bool active) {
    uint32_t t = kInvalidIndex;
    uint32_t tbits[Map::D];
    bool valid = false;
    if (active) {
      if constexpr (M == ImageMode::Insert || M == ImageMode::Mark) {   // these carry their source centres
        double c[Map::D];
        PI::source_centre(a, rank, c);
        valid = PI::image_at(a, pts, table, c, g, uint32_t(k), tbits);
      } else {
        const uint32_t leaf = a.src ? __ldg(a.src + rank) : uint32_t(rank);
        uint32_t sbits[Map::D];
        PI::source_bits(a, leaf, sbits);
        valid = PI::image(a, pts, table, sbits, g, uint32_t(k), tbits);
      }
      if constexpr (M != ImageMode::Mark) t = PI::target(a, n, valid, tbits);
    }
    if constexpr (M == ImageMode::Hit) {
      // one store per distinct target in the warp
      const unsigned peers = __match_any_sync(0xFFFFFFFFu, t);
      if (active && t != kInvalidIndex && lane == __ffs(peers) - 1) a.hit[t] = 1;
      if (a.targets && active) {
        if (g < a.targets_cap) a.targets[g] = valid ? t : kOutsideIndex;
        else *a.targets_over = 1;
      }
    } else if constexpr (M == ImageMode::Search) {
      if (active) a.out[g] = t;
    } else if constexpr (M == ImageMode::Mark) {
      // the image's box, unless its bit is set already (a stale read only sends the point
      // on to the atomic), deduplicated within the warp; the lane whose atomic sets the bit
      // marks the box in `fresh`, and the warp counts its new boxes with one atomic
      uint64_t code = kInvalidCode;
      bool fresh = false;
      if (active && valid) {
        code = code_of_bits<Map::D>(a.dc, tbits, a.depth);
        fresh = !((a.bits[code >> 5] >> uint32_t(code & 31u)) & 1u);
      }
      const unsigned peers = __match_any_sync(0xFFFFFFFFu, fresh ? code : kInvalidCode) & __ballot_sync(0xFFFFFFFFu, fresh);
      bool leader = fresh && lane == __ffs(peers) - 1;
      if (leader) {
        const uint32_t m = 1u << uint32_t(code & 31u);
        leader = !(atomicOr(a.bits + (code >> 5), m) & m);
        if (leader) atomicOr(a.fresh + (code >> 5), m);
      }
      const unsigned lead_mask = __ballot_sync(0xFFFFFFFFu, leader);
      if (lane == 0 && lead_mask) atomicAdd(a.cand_count, uint32_t(__popc(lead_mask)));
    } else {
      // candidates: valid images that are not leaves, as packed keys (the caller turns them
      // into codes); deduplicated within the warp and appended with one atomic per warp
      if (a.hit) {
        const unsigned hp = __match_any_sync(0xFFFFFFFFu, t);
        if (active && t != kInvalidIndex && lane == __ffs(hp) - 1) a.hit[t] = 1;
      }
      const bool is_cand = active && valid && t == kInvalidIndex;
      const uint64_t tcode = is_cand ? pack_bits_k<Map::D>(tbits, a.dc.k) : 0ull;
      const uint64_t key = is_cand ? tcode : kInvalidCode;
      // (the lowest candidate lane of each key leads: a non-candidate lane may share the
      // all-ones key)
      const unsigned peers = __match_any_sync(0xFFFFFFFFu, key) & __ballot_sync(0xFFFFFFFFu, is_cand);
      bool leader = is_cand && lane == __ffs(peers) - 1;
      if (a.claim && leader) leader = hash_claim(a.hash, tcode, a.error);
      const unsigned lead_mask = __ballot_sync(0xFFFFFFFFu, leader);
      uint32_t slot = 0;
      if (lane == 0 && lead_mask) slot = atomicAdd(a.cand_count, uint32_t(__popc(lead_mask)));
      slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
      if (leader) {
        const uint32_t pos = slot + __popc(lead_mask & ((1u << lane) - 1u));
        if (pos < a.cand_cap) a.cand[pos] = tcode;
        else atomicOr(a.error, 1u);
      }
    }
  };

  // A device work queue (a.work, zeroed by launch_image): every warp takes chunks of 32 x
  // kChunkTrips consecutive points until none is left, so that warps that run ahead take
  // more work and the SM stays full to the end (a static split leaves the slower warps
  // alone at the end: 47 % of the warp slots were active on average, of 75 % possible).
  constexpr uint64_t kChunk = 32ull * kChunkTrips;
  const uint64_t chunks = (total + kChunk - 1) / kChunk;
  for (;;) {
    unsigned long long c = 0;
    if (lane == 0) c = atomicAdd(a.work, 1ull);
    c = __shfl_sync(0xFFFFFFFFu, c, 0);
    if (c >= chunks) break;
    // (sources and points per box both fit 32 bits: the rank and the point index do)
    const uint64_t g = c * kChunk + uint64_t(lane);
    uint32_t rank, k;
    if (total <= 0xFFFFFFFFull - kChunk) {
      rank = uint32_t(g) / P32;
      k = uint32_t(g) - rank * P32;
    } else {
      rank = uint32_t(g / P);
      k = uint32_t(g - uint64_t(rank) * P);
    }
#pragma unroll 1
    for (int j = 0; j < kChunkTrips; ++j) {
      const uint64_t gj = g + 32ull * uint64_t(j);
      point(gj, rank, k, gj < total);
      k += 32;
      while (k >= P32) { k -= P32; ++rank; }
    }
  }
}

// ---------------------------------------------------------------------------------
// transition rows: warp per source box; the box's P <= 128 targets are sorted in
// shared memory and run-length counted, giving the row's (column, count) pairs in
// column order - the reference's packed (row, col) radix sort plus reverse
// inclusive_scan_by_key and unique_by_key (ImplicitBoxTree.hpp:3007-3038) done per row
// ---------------------------------------------------------------------------------
constexpr int kRowWarps = kThreads / 32;

template<class Map, class Grid>
__global__ void __launch_bounds__(kThreads) transition_rows_kernel(const RowArgs ra)
{
  using PI = PointImage<Map, Grid>;
  const ImageArgs& a = ra.img;
  __shared__ double pts[kPointTable];
  __shared__ uint32_t keys[kRowWarps][128];
  __shared__ uint32_t bounds[kRowWarps][4];
  const bool table = load_points<Grid, Map::D>(a.grid, a.points, pts);

  const uint32_t n = *a.n_leaves;
  const uint32_t nrows = a.n_src ? *a.n_src : n;
  const uint32_t P = uint32_t(a.points);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t* s = keys[w];
  const uint32_t warps = gridDim.x * kRowWarps;

  for (uint32_t row = blockIdx.x * kRowWarps + w; row < nrows; row += warps) {
    const uint32_t leaf = a.src ? __ldg(a.src + row) : row;
    uint32_t sbits[Map::D];
    PI::source_bits(a, leaf, sbits);
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
      const uint32_t k = uint32_t(lane) + 32u * q;
      uint32_t key = kPadKey;
      if (k < P) {
        uint32_t tbits[Map::D];
        const bool valid = PI::image(a, pts, table, sbits, uint64_t(row) * P + k, k, tbits);
        const uint32_t t = PI::target(a, n, valid, tbits);
        key = t == kInvalidIndex ? kLostKey : t;
      }
      s[lane + 32 * q] = key;
    }
    const uint32_t total = row_emit(s, bounds[w], lane, P, ra.keep_lost, ra.lost_col,
                                    ra.stage_col + size_t(row) * P, ra.stage_cnt + size_t(row) * P);
    if (lane == 0) ra.row_count[row] = total;
    __syncwarp();
  }
}

template<class Map, class Grid>
cudaError_t launch_image_t(ImageMode mode, const ImageArgs& a, uint64_t max_points, cudaStream_t s)
{
  static int blocks_per_sm[4] = {0, 0, 0, 0};
  const int m = int(mode);
  if (!blocks_per_sm[m]) {
    int b = 0;
    if (mode == ImageMode::Hit)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, image_points_kernel<Map, Grid, ImageMode::Hit>, kThreads, 0);
    else if (mode == ImageMode::Search)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, image_points_kernel<Map, Grid, ImageMode::Search>, kThreads, 0);
    else if (mode == ImageMode::Insert)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, image_points_kernel<Map, Grid, ImageMode::Insert>, kThreads, 0);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, image_points_kernel<Map, Grid, ImageMode::Mark>, kThreads, 0);
    blocks_per_sm[m] = b > 0 ? b : 1;
  }
  const uint64_t want = (max_points + kThreads - 1) / kThreads;
  const uint64_t cap = uint64_t(device_sm_count()) * blocks_per_sm[m];
  const unsigned grid = unsigned(want < 1 ? 1 : (want < cap ? want : cap));
  if (mode == ImageMode::Hit) image_points_kernel<Map, Grid, ImageMode::Hit><<<grid, kThreads, 0, s>>>(a);
  else if (mode == ImageMode::Search) image_points_kernel<Map, Grid, ImageMode::Search><<<grid, kThreads, 0, s>>>(a);
  else if (mode == ImageMode::Insert) image_points_kernel<Map, Grid, ImageMode::Insert><<<grid, kThreads, 0, s>>>(a);
  else image_points_kernel<Map, Grid, ImageMode::Mark><<<grid, kThreads, 0, s>>>(a);
  return cudaGetLastError();
}

template<class Map, class Grid>
cudaError_t launch_rows_t(const RowArgs& a, uint32_t max_rows, cudaStream_t s)
{
  static int blocks_per_sm = 0;
  if (!blocks_per_sm) {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, transition_rows_kernel<Map, Grid>, kThreads, 0);
    blocks_per_sm = b > 0 ? b : 1;
  }
  const uint64_t want = (uint64_t(max_rows) + kRowWarps - 1) / kRowWarps;
  const uint64_t cap = uint64_t(device_sm_count()) * blocks_per_sm;
  const unsigned grid = unsigned(want < 1 ? 1 : (want < cap ? want : cap));
  transition_rows_kernel<Map, Grid><<<grid, kThreads, 0, s>>>(a);
  return cudaGetLastError();
}

// (map, arith, grid) dispatch; each map has a fixed dimension
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

// a warp per child of the step that stored the targets: the child is a row when it
// survived (its rank advances); a target is a column when its child survived, at the
// child's rank; a point that left the domain is found in a last leaf of code 0
__global__ void __launch_bounds__(kThreads) stored_rows_kernel(const StoredRowArgs a)
{
  __shared__ uint32_t keys[kRowWarps][128];
  __shared__ uint32_t bounds[kRowWarps][4];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t* s = keys[w];
  const uint32_t P = a.points, n = a.n_leaves;
  const bool zero_leaf = n > 0 && __ldg(a.codes + n - 1) == 0;
  for (uint32_t c = blockIdx.x * kRowWarps + w; c < a.n_children; c += gridDim.x * kRowWarps) {
    const uint32_t row = __ldg(a.rank + c);
    if (__ldg(a.rank + c + 1) == row) continue;        // removed: no row (warp-uniform)
    // every load of the row goes out before any is used: the targets, then their ranks
    uint32_t tg[4], lo[4], hi[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t k = uint32_t(lane) + 32u * q;
      tg[q] = k < P ? __ldg(a.targets + size_t(c) * P + k) : kInvalidIndex;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const bool in = tg[q] < kOutsideIndex;
      lo[q] = in ? __ldg(a.rank + tg[q]) : 0u;
      hi[q] = in ? __ldg(a.rank + tg[q] + 1) : 0u;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t k = uint32_t(lane) + 32u * q, t = tg[q];
      uint32_t key = kPadKey;
      if (k < P) {
        if (t < kOutsideIndex) key = hi[q] != lo[q] ? lo[q] : kLostKey;
        else key = (t == kOutsideIndex && zero_leaf) ? n - 1 : kLostKey;
      }
      s[lane + 32 * q] = key;
    }
    const uint32_t total = row_emit(s, bounds[w], lane, P, a.keep_lost, n + 1, a.stage_col + size_t(row) * P,
                                    a.stage_cnt + size_t(row) * P);
    if (lane == 0) a.row_count[row] = total;
    __syncwarp();
  }
}

}  // namespace

cudaError_t launch_stored_rows(const StoredRowArgs& a, cudaStream_t s)
{
  if (a.n_children == 0) return cudaSuccess;
  const uint64_t want = (uint64_t(a.n_children) + kRowWarps - 1) / kRowWarps;
  const uint64_t cap = uint64_t(device_sm_count()) * 8;
  stored_rows_kernel<<<unsigned(want < cap ? want : cap), kThreads, 0, s>>>(a);
  return cudaGetLastError();
}

bool image_supported(uint32_t map_kind, uint32_t arith, uint32_t grid_kind, uint32_t dim)
{
  return dispatch(map_kind, arith, grid_kind, dim, [](auto, auto) { return cudaSuccess; }) == cudaSuccess;
}

cudaError_t launch_image(uint32_t map_kind, uint32_t arith, uint32_t grid_kind, uint32_t dim, ImageMode mode,
                         const ImageArgs& a, uint64_t max_points, cudaStream_t s)
{
  if (!a.work) return cudaErrorInvalidValue;     // the image kernel takes its points from a work queue
  const cudaError_t e = cudaMemsetAsync(a.work, 0, sizeof(unsigned long long), s);   // the queue starts empty
  if (e != cudaSuccess) return e;
  ImageArgs b = a;
  fill_depth_const(b.dom, int(dim), b.depth, b.dc);
  return dispatch(map_kind, arith, grid_kind, dim, [&](auto map, auto grid) {
    return launch_image_t<decltype(map), decltype(grid)>(mode, b, max_points, s);
  });
}

cudaError_t launch_rows(uint32_t map_kind, uint32_t arith, uint32_t grid_kind, uint32_t dim, const RowArgs& a,
                        uint32_t max_rows, cudaStream_t s)
{
  RowArgs b = a;
  fill_depth_const(b.img.dom, int(dim), b.img.depth, b.img.dc);
  return dispatch(map_kind, arith, grid_kind, dim, [&](auto map, auto grid) {
    return launch_rows_t<decltype(map), decltype(grid)>(b, max_rows, s);
  });
}

}  // namespace b12g
