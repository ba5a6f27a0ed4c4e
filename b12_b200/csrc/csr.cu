// Transition-matrix assembly and the invariant measure.
//
//   gather_rows        - packs the per-row (column, count) runs of the transition-row
//                        kernel into CSR (compressIndexVector, CooMatrix.hpp:14-56, and
//                        the count -> probability division of ImplicitBoxTree.hpp:3147-3158)
//   transpose          - CSR of P -> CSR of P^T with sources ascending in every row
//   invariant_measure  - FP64 power iteration v <- P^T v / |P^T v|_1 in one persistent
//                        cooperative launch with a bounded grid barrier
#include <cooperative_groups.h>

#include "kernels.h"
#include "csr.h"

namespace b12g {

namespace {

constexpr int kThreads = 256;

int grid_for(uint64_t work, int per_block, int blocks_per_sm)
{
  const uint64_t want = (work + per_block - 1) / per_block;
  const uint64_t cap = uint64_t(device_sm_count()) * blocks_per_sm;
  return int(want < 1 ? 1 : (want < cap ? want : cap));
}

__global__ void gather_rows_kernel(const uint32_t* stage_col, const uint32_t* stage_cnt, uint32_t stride,
                                   const uint32_t* row_count, const uint32_t* rowptr, const uint32_t* n_rows,
                                   uint32_t* cols, double* vals, int absolute, double points)
{
  const uint32_t n = *n_rows;
  const uint32_t lanes = gridDim.x * blockDim.x / 8;
  // 8 threads per row: rows hold a handful of entries
  for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) / 8; r < n; r += lanes) {
    const uint32_t c = row_count[r], base = rowptr[r];
    for (uint32_t e = threadIdx.x & 7; e < c; e += 8) {
      const size_t src = size_t(r) * stride + e;
      const uint32_t cnt = stage_cnt[src];
      cols[base + e] = stage_col[src];
      vals[base + e] = absolute ? double(cnt) : __ddiv_rn(double(cnt), points);
    }
  }
}

// ---- transpose -------------------------------------------------------------------
__global__ void col_hist_kernel(const uint32_t* cols, const uint32_t* nnz_ptr, uint32_t n_cols, uint32_t* hist)
{
  const uint32_t nnz = *nnz_ptr;
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x) {
    const uint32_t c = cols[e];
    if (c < n_cols) atomicAdd(hist + c, 1u);
  }
}

__global__ void transpose_fill_kernel(const uint32_t* rowptr, const uint32_t* cols, const double* vals,
                                      const uint32_t* n_rows, uint32_t n_cols, const uint32_t* tptr,
                                      uint32_t* cursor, uint32_t* trows, double* tvals)
{
  const uint32_t n = *n_rows;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    for (uint32_t e = rowptr[r]; e < rowptr[r + 1]; ++e) {
      const uint32_t c = cols[e];
      if (c >= n_cols) continue;
      const uint32_t pos = tptr[c] + atomicAdd(cursor + c, 1u);
      trows[pos] = r;
      tvals[pos] = vals[e];
    }
  }
}

// the atomic fill leaves each transposed row in arrival order: sort it by source
__global__ void transpose_sort_kernel(const uint32_t* tptr, uint32_t n_cols, uint32_t* trows, double* tvals)
{
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n_cols; c += gridDim.x * blockDim.x) {
    const uint32_t b = tptr[c], e = tptr[c + 1];
    for (uint32_t i = b + 1; i < e; ++i) {
      const uint32_t r = trows[i];
      const double v = tvals[i];
      uint32_t j = i;
      while (j > b && trows[j - 1] > r) { trows[j] = trows[j - 1]; tvals[j] = tvals[j - 1]; --j; }
      trows[j] = r;
      tvals[j] = v;
    }
  }
}

// ---- power iteration ----------------------------------------------------------------
// A sense-reversal grid barrier whose waits give up after a bounded number of polls;
// co-residency of all blocks is guaranteed by the cooperative launch.
constexpr unsigned long long kBarrierPolls = 1ull << 24;  // far beyond any real wait (~1 s)
constexpr int kMeasureThreads = 512;
constexpr int kRowLanes = 8;                                // lanes per row of P^T

__device__ bool grid_barrier(unsigned* count, unsigned* gen, unsigned* error)
{
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned* vgen = gen;
    const unsigned g = *vgen;
    __threadfence();
    if (atomicAdd(count, 1u) == gridDim.x - 1) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      unsigned long long polls = 0;
      while (*vgen == g) {
        if (++polls > kBarrierPolls) { atomicOr(error, 2u); ok = 0; break; }
        if ((polls & 1023u) == 0) __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok && !(*(volatile unsigned*)error & 2u);
}

struct MeasureArgs {
  const uint32_t* tptr;      // CSR of P^T
  const uint32_t* trows;
  const double* tvals;
  uint32_t n;
  uint32_t iters;
  double* w0;
  double* w1;
  double* partial;           // 2 x gridDim.x
  double* out;
  unsigned* bar_count;
  unsigned* bar_gen;
  unsigned* error;
};

// sum of the per-block partials in one fixed order, identical in every block
__device__ double sum_partials(const double* part, uint32_t nb, double* bcast)
{
  if (threadIdx.x < 32) {
    double x = 0.0;
    for (uint32_t i = threadIdx.x; i < nb; i += 32) x = __dadd_rn(x, __ldcg(part + i));
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) x = __dadd_rn(x, __shfl_xor_sync(0xFFFFFFFFu, x, d));
    if (threadIdx.x == 0) *bcast = x;
  }
  __syncthreads();
  return *bcast;
}

// v <- P^T v / |P^T v|_1; rows of P^T are handled by groups of 8 lanes; the previous
// iterate is scaled by 1/s on the fly, so one grid barrier per iteration suffices
__global__ void __launch_bounds__(kMeasureThreads) invariant_measure_kernel(const MeasureArgs a)
{
  __shared__ double red[kMeasureThreads / 32];
  __shared__ double bcast;
  const uint32_t n = a.n;
  const uint32_t lane8 = threadIdx.x & (kRowLanes - 1);
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) / kRowLanes;
  const uint32_t groups = gridDim.x * blockDim.x / kRowLanes;
  const double v0 = __ddiv_rn(1.0, double(n));
  double inv = 1.0;
  for (uint32_t it = 0; it < a.iters; ++it) {
    const double* wp = (it & 1u) ? a.w0 : a.w1;
    double* wc = (it & 1u) ? a.w1 : a.w0;
    double local = 0.0;
    // the loop runs over the warp's first group so that every lane of a warp takes the
    // same number of trips (the shuffles below need the whole warp)
    for (uint32_t jb = group & ~3u; jb < n; jb += groups) {
      const uint32_t j = jb + (group & 3u);
      const bool row = j < n;
      double acc = 0.0;
      const uint32_t b = row ? __ldg(a.tptr + j) : 0u, e = row ? __ldg(a.tptr + j + 1) : 0u;
      for (uint32_t k = b + lane8; k < e; k += kRowLanes) {
        const double v = it == 0 ? v0 : __dmul_rn(__ldcg(wp + __ldg(a.trows + k)), inv);
        acc = __fma_rn(__ldg(a.tvals + k), v, acc);
      }
#pragma unroll
      for (int d = kRowLanes / 2; d > 0; d >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xFFFFFFFFu, acc, d));
      if (lane8 == 0 && row) {
        __stcg(wc + j, acc);
        local = __dadd_rn(local, fabs(acc));
      }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) local = __dadd_rn(local, __shfl_xor_sync(0xFFFFFFFFu, local, d));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int i = 0; i < kMeasureThreads / 32; ++i) t = __dadd_rn(t, red[i]);
      __stcg(a.partial + (it & 1u) * gridDim.x + blockIdx.x, t);
    }
    if (!grid_barrier(a.bar_count, a.bar_gen, a.error)) return;
    inv = __ddiv_rn(1.0, sum_partials(a.partial + (it & 1u) * gridDim.x, gridDim.x, &bcast));
  }
  const double* wl = (a.iters & 1u) ? a.w0 : a.w1;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    a.out[j] = a.iters ? __dmul_rn(__ldcg(wl + j), inv) : v0;
}

}  // namespace

cudaError_t gather_rows(const uint32_t* stage_col, const uint32_t* stage_cnt, uint32_t stride,
                        const uint32_t* row_count, const uint32_t* rowptr, const uint32_t* n_rows, uint32_t* cols,
                        double* vals, int absolute, double points, uint32_t max_rows, cudaStream_t s)
{
  gather_rows_kernel<<<grid_for(uint64_t(max_rows) * 8, kThreads, 8), kThreads, 0, s>>>(
      stage_col, stage_cnt, stride, row_count, rowptr, n_rows, cols, vals, absolute, points);
  return cudaGetLastError();
}

cudaError_t transpose_csr(const uint32_t* rowptr, const uint32_t* cols, const double* vals, const uint32_t* n_rows,
                          const uint32_t* nnz, uint32_t max_rows, uint64_t max_nnz, uint32_t n_cols,
                          uint32_t* tptr, uint32_t* trows, double* tvals, uint32_t* work, uint32_t* tile_sums,
                          const uint32_t* n_cols_dev, cudaStream_t s)
{
  // work: n_cols + 1 counters
  cudaMemsetAsync(work, 0, (size_t(n_cols) + 1) * sizeof(uint32_t), s);
  col_hist_kernel<<<grid_for(max_nnz, kThreads, 8), kThreads, 0, s>>>(cols, nnz, n_cols, work);
  cudaError_t e = exclusive_scan_u32(work, tptr, n_cols_dev, tile_sums, n_cols, s);
  if (e != cudaSuccess) return e;
  cudaMemsetAsync(work, 0, (size_t(n_cols) + 1) * sizeof(uint32_t), s);
  transpose_fill_kernel<<<grid_for(max_rows, kThreads, 8), kThreads, 0, s>>>(rowptr, cols, vals, n_rows, n_cols,
                                                                             tptr, work, trows, tvals);
  transpose_sort_kernel<<<grid_for(n_cols, kThreads, 8), kThreads, 0, s>>>(tptr, n_cols, trows, tvals);
  return cudaGetLastError();
}

cudaError_t invariant_measure(const uint32_t* tptr, const uint32_t* trows, const double* tvals, uint32_t n,
                              uint32_t iters, double* w0, double* w1, double* partial, uint32_t partial_cap,
                              double* out, unsigned* sync_words, cudaStream_t s)
{
  static int blocks_per_sm = 0;
  if (!blocks_per_sm) {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, invariant_measure_kernel, kMeasureThreads, 0);
    blocks_per_sm = b > 0 ? (b < 2 ? b : 2) : 1;
  }
  int grid = grid_for(uint64_t(n) * kRowLanes, kMeasureThreads, blocks_per_sm);
  if (grid > int(partial_cap / 2)) grid = int(partial_cap / 2);
  if (grid < 1) grid = 1;
  cudaMemsetAsync(sync_words, 0, 3 * sizeof(unsigned), s);
  MeasureArgs a{tptr, trows, tvals, n, iters, w0, w1, partial, out, sync_words, sync_words + 1, sync_words + 2};
  void* params[] = {&a};
  return cudaLaunchCooperativeKernel((const void*)invariant_measure_kernel, dim3(grid), dim3(kMeasureThreads), params,
                                     0, s);
}

int measure_partial_slots()
{
  return 2 * device_sm_count() * 8;
}

}  // namespace b12g
