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

#include "rows.cuh"
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
  ST(t->stage_col.ensure(stage, "row staging"));
  ST(t->stage_cnt.ensure(stage, "row staging"));
  ST(t->row_count.ensure(uint64_t(n) + 1, "row counts"));
  ST(t->rowptr.ensure(uint64_t(n) + 1, "row pointers"));
  partition_rows_kernel<<<grid_for(n, kThreads / 32), kThreads, 0, t->stream>>>(
      targets, n, P, invalid_column ? 1 : 0, n_columns + 1, t->stage_col.p, t->stage_cnt.p, t->row_count.p);
  CK(cudaGetLastError());
  count_launches(1);
  return finish_rows(t, P, n_columns, absolute, invalid_column, out);
}

b12g_status b12g_load_leaves_device(b12g_tree* t, const uint64_t* codes, const uint8_t* depths, const uint8_t* flags,
                                    uint32_t n)
{
  if (!t || (n && (!codes || !depths || !flags))) return fail(B12G_ERR_INVALID, "NULL argument");
  return mixed_load_device(t, codes, depths, flags, n);
}

}  // extern "C"
