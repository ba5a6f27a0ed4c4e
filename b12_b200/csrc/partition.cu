// Entry points for a tree whose leaves are range-partitioned over several ranks.
//
// Every rank holds a contiguous run of the leaves in the reference's order.  One
// subdivision step images the local leaves (b12g_image_point_boxes), sends each point box
// to the rank whose code range holds it, and that rank flags the leaves hit
// (b12g_set_flags_by_point_boxes, the setFlagsByIterators of ImplicitBoxTree.hpp:2167-2196
// over point boxes) or reports their indices for the transition matrix
// (b12g_search_point_boxes, searchByIterators of ImplicitBoxTree.hpp:2394-2432).  The
// rows of a rank's leaves are assembled from global target indices by
// b12g_transition_rows, the run-length step of transitionMatrixForLeaves
// (ImplicitBoxTree.hpp:2934-3159).  All buffers here are device memory: they are what
// the collectives between the ranks move.
#include <algorithm>
#include <vector>

#include "rows.cuh"
#include "sort.h"
#include "tree.h"

using namespace b12g;
using namespace b12g::host;

namespace {

constexpr int kThreads = 256;

int grid_for(uint64_t n, int per_block)
{
  const uint64_t want = (n + per_block - 1) / per_block;
  return int(std::max<uint64_t>(1, std::min<uint64_t>(want, uint64_t(device_sm_count()) * 8)));
}

__global__ void value_present_kernel(const uint32_t* __restrict__ v, uint64_t n, uint32_t x, uint32_t* found)
{
  bool f = false;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    f |= __ldg(v + i) == x;
  if (__syncthreads_or(f) && threadIdx.x == 0) *found = 1;
}

// a warp per row: the row's P <= 128 targets (column indices, or B12G_INVALID_INDEX for
// points that left the domain) sorted and run-length counted, as for a whole tree
__global__ void __launch_bounds__(kThreads) partition_rows_kernel(const uint32_t* __restrict__ targets, uint32_t n,
                                                               uint32_t P, int keep_lost, uint32_t lost_col,
                                                               uint32_t* stage_col, uint32_t* stage_cnt,
                                                               uint32_t* row_count)
{
  constexpr int kWarps = kThreads / 32;
  __shared__ uint32_t keys[kWarps][128];
  __shared__ uint32_t bounds[kWarps][4];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t* s = keys[w];
  for (uint32_t row = blockIdx.x * kWarps + w; row < n; row += gridDim.x * kWarps) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t k = uint32_t(lane) + 32u * q;
      uint32_t key = kPadKey;
      if (k < P) {
        const uint32_t t = __ldg(targets + size_t(row) * P + k);
        key = t == kInvalidIndex ? kLostKey : t;
      }
      s[lane + 32 * q] = key;
    }
    const uint32_t total = row_emit(s, bounds[w], lane, P, keep_lost, lost_col, stage_col + size_t(row) * P,
                                    stage_cnt + size_t(row) * P);
    if (lane == 0) row_count[row] = total;
    __syncwarp();
  }
}

// The rank that owns each point box: a valid box goes to the last run whose first
// depth-64 code is at or below its code (unsigned order), a box that left the domain to
// the last run.  keys[i] = owner, vals[i] = i (for the stable partition), cnt[owner]++.
constexpr int kMaxRuns = 1024;

__global__ void __launch_bounds__(kThreads) route_owner_kernel(const uint64_t* __restrict__ codes,
                                                               const uint8_t* __restrict__ valid, uint32_t n,
                                                               const uint64_t* __restrict__ starts,
                                                               const uint32_t* __restrict__ ranks, uint32_t n_runs,
                                                               uint32_t world, uint64_t* keys, uint32_t* vals,
                                                               uint32_t* cnt)
{
  __shared__ uint64_t s_start[kMaxRuns];
  __shared__ uint32_t s_rank[kMaxRuns];
  __shared__ uint32_t s_cnt[kMaxRuns];
  for (uint32_t r = threadIdx.x; r < n_runs; r += blockDim.x) {
    s_start[r] = starts[r];
    s_rank[r] = ranks[r];
  }
  for (uint32_t r = threadIdx.x; r < world; r += blockDim.x) s_cnt[r] = 0;
  __syncthreads();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t run = n_runs - 1;
    if (valid[i]) {
      // first run whose start is above the code, minus one (run 0 starts at or below every code)
      const uint64_t c = codes[i];
      uint32_t lo = 0, len = n_runs;
      while (len > 0) {
        const uint32_t half = len >> 1;
        if (s_start[lo + half] <= c) { lo += half + 1; len -= half + 1; }
        else len = half;
      }
      run = lo > 0 ? lo - 1 : 0;
    }
    const uint32_t owner = s_rank[run];
    keys[i] = owner;
    vals[i] = i;
    atomicAdd(&s_cnt[owner], 1u);
  }
  __syncthreads();
  for (uint32_t r = threadIdx.x; r < world; r += blockDim.x)
    if (s_cnt[r]) atomicAdd(cnt + r, s_cnt[r]);
}

// the point boxes in owner order (stable): perm[p] is the point box at position p
__global__ void route_gather_kernel(const uint32_t* __restrict__ perm, uint32_t n, const uint64_t* __restrict__ codes,
                                    const uint8_t* __restrict__ valid, uint64_t* out_codes, uint8_t* out_valid,
                                    uint32_t* slot)
{
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const uint32_t i = __ldg(perm + p);
    out_codes[p] = __ldg(codes + i);
    out_valid[p] = __ldg(valid + i);
    if (slot) slot[i] = p;
  }
}

}  // namespace

namespace b12g {

cudaError_t value_present(const uint32_t* v, uint64_t n, uint32_t x, uint32_t* found, cudaStream_t s)
{
  if (n == 0) return cudaSuccess;
  value_present_kernel<<<grid_for(n, kThreads * 4), kThreads, 0, s>>>(v, n, x, found);
  return cudaGetLastError();
}

}  // namespace b12g

extern "C" {

b12g_status b12g_image_point_boxes(b12g_tree* t, const b12g_scheme* sc, uint64_t* codes, uint8_t* valid,
                                   uint64_t capacity, uint64_t* n_points)
{
  if (!t || !sc || !n_points) return fail(B12G_ERR_INVALID, "NULL argument");
  return mixed_image_point_boxes(t, sc, codes, valid, capacity, n_points);
}

b12g_status b12g_image_distinct_point_boxes(b12g_tree* t, const b12g_scheme* sc, uint8_t depth, uint64_t* codes,
                                            uint8_t* valid, uint64_t capacity, uint64_t* n_boxes)
{
  if (!t || !sc || !n_boxes) return fail(B12G_ERR_INVALID, "NULL argument");
  if (depth > 64) return fail(B12G_ERR_INVALID, "depth %u above 64", depth);
  return mixed_image_point_boxes(t, sc, codes, valid, capacity, n_boxes, true, depth);
}

b12g_status b12g_search_point_boxes(b12g_tree* t, const uint64_t* codes, const uint8_t* valid, uint64_t n,
                                    uint32_t* index)
{
  if (!t || (n && !index)) return fail(B12G_ERR_INVALID, "NULL argument");
  return mixed_point_box_search(t, codes, valid, n, index, 0, nullptr);
}

b12g_status b12g_set_flags_by_point_boxes(b12g_tree* t, const uint64_t* codes, const uint8_t* valid, uint64_t n,
                                          uint8_t flags, uint32_t* n_changed)
{
  if (!t) return fail(B12G_ERR_INVALID, "NULL tree");
  return mixed_point_box_search(t, codes, valid, n, nullptr, flags, n_changed);
}

b12g_status b12g_transition_rows(b12g_tree* t, const uint32_t* targets, uint32_t points_per_row, uint32_t n_columns,
                                 int absolute, int invalid_column, b12g_csr** out)
{
  if (!t || !out || !targets) return fail(B12G_ERR_INVALID, "NULL argument");
  const uint32_t P = points_per_row;
  if (P == 0 || P > kMaxRowPoints)
    return fail(B12G_ERR_CAPACITY, "transition rows support 1 to %u points per box", kMaxRowPoints);
  if (n_columns == 0 || n_columns >= kLostKey - 1) return fail(B12G_ERR_INVALID, "%u columns", n_columns);
  const uint32_t n = t->n;
  const uint64_t stage = uint64_t(n) * P;
  ST(t->stage_col.ensure_room(stage, "row staging"));
  ST(t->stage_cnt.ensure_room(stage, "row staging"));
  ST(t->row_count.ensure_room(uint64_t(n) + 1, "row counts"));
  ST(t->rowptr.ensure_room(uint64_t(n) + 1, "row pointers"));
  partition_rows_kernel<<<grid_for(n, kThreads / 32), kThreads, 0, t->stream>>>(
      targets, n, P, invalid_column ? 1 : 0, n_columns + 1, t->stage_col.p, t->stage_cnt.p, t->row_count.p);
  CK(cudaGetLastError());
  count_launches(1);
  return finish_rows(t, P, n_columns, absolute, invalid_column, out);
}

b12g_status b12g_route_point_boxes(b12g_tree* t, const uint64_t* codes, const uint8_t* valid, uint64_t n,
                                   const uint64_t* run_starts, const uint32_t* run_ranks, uint32_t n_runs,
                                   uint32_t world, uint64_t* out_codes, uint8_t* out_valid, uint32_t* slot,
                                   uint64_t* counts)
{
  if (!t || !run_starts || !run_ranks || !counts || (n && (!codes || !valid || !out_codes || !out_valid)))
    return fail(B12G_ERR_INVALID, "NULL argument");
  if (world == 0 || world > uint32_t(kMaxRuns) || n_runs == 0 || n_runs > world)
    return fail(B12G_ERR_INVALID, "%u runs over %u ranks (1 <= runs <= ranks <= %d)", n_runs, world, kMaxRuns);
  for (uint32_t r = 0; r < n_runs; ++r) {
    if (run_ranks[r] >= world || (r > 0 && (run_ranks[r] <= run_ranks[r - 1] || run_starts[r] <= run_starts[r - 1])))
      return fail(B12G_ERR_INVALID, "runs must have ascending ranks below %u and ascending starts", world);
  }
  if (n > 0xFFFFFFF0ull) return fail(B12G_ERR_CAPACITY, "at most 2^32-16 point boxes per exchange");
  const uint32_t m = uint32_t(n);
  cudaStream_t s = t->stream;
  ST(t->route_runs.ensure(size_t(n_runs) * 3, "route runs"));
  ST(t->route_cnt.ensure(world + 1, "route counts"));
  std::vector<uint32_t> host_runs(size_t(n_runs) * 3);
  for (uint32_t r = 0; r < n_runs; ++r) {
    host_runs[2 * r] = uint32_t(run_starts[r]);
    host_runs[2 * r + 1] = uint32_t(run_starts[r] >> 32);
    host_runs[2 * size_t(n_runs) + r] = run_ranks[r];
  }
  CK(cudaMemcpyAsync(t->route_runs.p, host_runs.data(), host_runs.size() * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(t->route_cnt.p, 0, (world + 1) * 4, s));
  std::vector<uint32_t> cnt(world, 0);
  if (m > 0) {
    // the exchanges of a subdivision grow by about 1.6x a step: room for 3x, so that the
    // buffers are reallocated every third step at most
    for (int q = 0; q < 2; ++q) {
      ST(t->ins_key[q].ensure_room(m, "route keys", 3));
      ST(t->ins_idx[q].ensure_room(m, "route order", 3));
    }
    const uint64_t cells = sort_scratch_u32(m);
    ST(t->sort_idx.ensure_room(cells + 8, "route sort", 3));
    const uint64_t* starts = reinterpret_cast<const uint64_t*>(t->route_runs.p);
    const uint32_t* ranks = t->route_runs.p + 2 * size_t(n_runs);
    route_owner_kernel<<<grid_for(m, kThreads * 4), kThreads, 0, s>>>(codes, valid, m, starts, ranks, n_runs, world,
                                                                      t->ins_key[0].p, t->ins_idx[0].p,
                                                                      t->route_cnt.p);
    CK(cudaGetLastError());
    // a stable partition by owner: one onesweep pass per 8 bits of the rank
    const int bits = world <= 256 ? 8 : 16;
    uint32_t* n_dev = t->route_cnt.p + world;
    CK(cudaMemcpyAsync(n_dev, &m, 4, cudaMemcpyHostToDevice, s));
    uint64_t* skeys = nullptr;
    uint32_t* perm = nullptr;
    CK(radix_sort_u64_values(t->ins_key[0].p, t->ins_key[1].p, t->ins_idx[0].p, t->ins_idx[1].p, n_dev, m, bits,
                             t->sort_idx.p, t->ctr.p + C_ERROR, &skeys, &perm, s));
    route_gather_kernel<<<grid_for(m, kThreads * 4), kThreads, 0, s>>>(perm, m, codes, valid, out_codes, out_valid,
                                                                       slot);
    CK(cudaGetLastError());
    count_launches(2 + uint64_t(sort_launches(bits)));
    CK(cudaMemcpyAsync(cnt.data(), t->route_cnt.p, world * 4, cudaMemcpyDeviceToHost, s));
  }
  ST(sync(t, "route point boxes"));
  ST(check_error(t, "route point boxes"));
  for (uint32_t r = 0; r < world; ++r) counts[r] = cnt[r];
  return B12G_OK;
}

b12g_status b12g_leaf_at(b12g_tree* t, uint32_t index, uint64_t* code, uint8_t* depth, uint8_t* flags)
{
  if (!t) return fail(B12G_ERR_INVALID, "NULL tree");
  if (index >= t->n) return fail(B12G_ERR_INVALID, "leaf %u of %u", index, t->n);
  uint64_t c = 0;
  uint8_t d = t->depth, f = 0;
  CK(cudaMemcpyAsync(&c, t->codes() + index, 8, cudaMemcpyDeviceToHost, t->stream));
  CK(cudaMemcpyAsync(&f, t->flg() + index, 1, cudaMemcpyDeviceToHost, t->stream));
  if (t->mixed) CK(cudaMemcpyAsync(&d, t->dep[t->cur].p + index, 1, cudaMemcpyDeviceToHost, t->stream));
  ST(sync(t, "leaf"));
  if (code) *code = c;
  if (depth) *depth = d;
  if (flags) *flags = f;
  return B12G_OK;
}

b12g_status b12g_load_leaves_device(b12g_tree* t, const uint64_t* codes, const uint8_t* depths, const uint8_t* flags,
                                    uint32_t n)
{
  if (!t || (n && (!codes || !depths || !flags))) return fail(B12G_ERR_INVALID, "NULL argument");
  return mixed_load_device(t, codes, depths, flags, n);
}

}  // extern "C"
