// Transition-matrix assembly and the invariant measure.
//
//   gather_rows        - packs the per-row (column, count) runs of the transition-row
//                        kernel into CSR (compressIndexVector, CooMatrix.hpp:14-56, and
//                        the count -> probability division of ImplicitBoxTree.hpp:3147-3158)
//   transpose          - CSR of P -> CSR of P^T with sources ascending in every row
//   invariant_measure  - FP64 power iteration v <- P^T v / |P^T v|_1 in one persistent
//                        cooperative launch with bounded grid barriers (and, with the
//                        matrix on chip, bounded waits between dependent blocks)
#include <cooperative_groups.h>

#include <mutex>

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

// the atomic fill leaves each transposed row in arrival order: sort it by source.  A warp
// per row: a row of up to 32 entries is held one entry a lane, and every entry goes to its
// rank (the entries before it in source order, ties by lane: the sources of a row are
// distinct); a longer row is sorted by insertion by one lane.
__global__ void transpose_sort_kernel(const uint32_t* tptr, uint32_t n_cols, uint32_t* trows, double* tvals)
{
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < n_cols; c += nwarps) {
    const uint32_t b = tptr[c], e = tptr[c + 1], len = e - b;
    if (len <= 1) continue;
    if (len <= 32) {
      const bool have = lane < len;
      const uint32_t r = have ? trows[b + lane] : 0u;
      const double v = have ? tvals[b + lane] : 0.0;
      uint32_t rank = 0;
      for (uint32_t j = 0; j < len; ++j) {
        const uint32_t rj = __shfl_sync(0xFFFFFFFFu, r, int(j));
        rank += rj < r || (rj == r && j < lane);
      }
      if (have) {
        trows[b + rank] = r;
        tvals[b + rank] = v;
      }
    } else if (lane == 0) {
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
}

// the longest row of P^T (*out must be 0 before)
__global__ void max_row_kernel(const uint32_t* tptr, uint32_t n, uint32_t* out)
{
  uint32_t m = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    m = max(m, tptr[i + 1] - tptr[i]);
  m = __reduce_max_sync(0xFFFFFFFFu, m);
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// ---- power iteration ----------------------------------------------------------------
// A sense-reversal grid barrier whose waits give up after a bounded number of polls;
// co-residency of all blocks is guaranteed by the cooperative launch.
constexpr unsigned long long kBarrierPolls = 1ull << 24;  // far beyond any real wait (~1 s)
constexpr int kMeasureThreads = 1024;
constexpr uint32_t kShortRow = 8;                           // rows of P^T with more entries get 8 lanes
constexpr uint32_t kMidRow = 64;                            // ... and with more than this a warp

struct MeasureArgs {
  const uint32_t* tptr;      // CSR of P^T
  const uint32_t* trows;
  const double* tvals;
  const uint32_t* mid_rows;  // rows longer than short_limit, up to kMidRow entries: 8 lanes each
  uint32_t n_mid;
  const uint32_t* long_rows; // longer rows: a warp each
  uint32_t n_long;
  uint32_t short_limit;      // kShortRow with row lists, else no limit
  uint32_t n;
  uint32_t iters;
  double* w0;
  double* w1;
  double* partial;           // 2 x gridDim.x
  double* out;
  unsigned* bar_count;
  unsigned* bar_gen;
  unsigned* error;
  double* totals;            // 2 slots: the L1 norm of the last two iterates
  unsigned gen_seen;         // completed barriers before the current one
  const double* start;       // first iterate (L1 norm 1), or nullptr: the uniform vector
  double* change;            // nullptr, or per block: sum of |v_k - v_(k-1)| of the last iteration
  unsigned* epoch;           // shared-memory kernel: per block, the iterations it has completed
  unsigned* dep_mask;        // shared-memory kernel: per block, kDepWords words: the blocks
                             // owning the sources its rows gather
};

// Grid barrier that also reduces: every block has written its partial sum; the last
// block to arrive adds all partials in one fixed order (lane-strided, then a fixed
// shuffle tree), publishes the total and releases the others, who poll a generation
// word with a bounded number of polls.  Returns false when a wait gave up.
__device__ bool barrier_sum(const MeasureArgs& a, const double* part, double* total_slot, double* total)
{
  __shared__ int last;
  __shared__ int ok;
  __shared__ double bcast;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    __threadfence();
    last = atomicAdd(a.bar_count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last) {
    if (threadIdx.x < 32) {
      double x = 0.0;
#pragma unroll 4
      for (uint32_t i = threadIdx.x; i < gridDim.x; i += 32) x = __dadd_rn(x, __ldcg(part + i));
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) x = __dadd_rn(x, __shfl_xor_sync(0xFFFFFFFFu, x, d));
      if (threadIdx.x == 0) {
        __stcg(total_slot, x);
        bcast = x;
        atomicExch(a.bar_count, 0u);
        __threadfence();
        atomicAdd(a.bar_gen, 1u);
      }
    }
  } else if (threadIdx.x == 0) {
    volatile unsigned* vgen = a.bar_gen;
    const unsigned g = a.gen_seen;
    unsigned long long polls = 0;
    while (*vgen == g) {
      if (++polls > kBarrierPolls) { atomicOr(a.error, 2u); ok = 0; break; }
    }
    __threadfence();
    bcast = __ldcg(total_slot);
  }
  __syncthreads();
  *total = bcast;
  return ok && !(*(volatile unsigned*)a.error & 2u);
}

__device__ __forceinline__ double iterate_value(const double* wp, const double* start, uint32_t src, uint32_t it,
                                                double v0, double inv)
{
  return it == 0 ? (start ? __ldg(start + src) : v0) : __dmul_rn(__ldcg(wp + src), inv);
}

// The result v = the last iterate scaled by 1/|.|_1 (the first iterate when iters == 0)
// and, when asked for, each block's part of |v - previous normalised iterate|_1 (the
// change made by the last iteration: the stopping test of a tolerance-driven run).
__device__ void write_result(const MeasureArgs& a, double inv, double inv_prev)
{
  __shared__ double red_c[32];
  const uint32_t n = a.n;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  const double v0 = __ddiv_rn(1.0, double(n));
  const double* wl = (a.iters & 1u) ? a.w0 : a.w1;     // iteration iters - 1
  const double* wq = (a.iters & 1u) ? a.w1 : a.w0;     // iteration iters - 2
  double c = 0.0;
  for (uint32_t j = tid; j < n; j += nthreads) {
    const double first = a.start ? __ldg(a.start + j) : v0;
    const double x = a.iters ? __dmul_rn(__ldcg(wl + j), inv) : first;
    a.out[j] = x;
    if (a.change && a.iters) {
      const double prev = a.iters >= 2 ? __dmul_rn(__ldcg(wq + j), inv_prev) : first;
      c = __dadd_rn(c, fabs(__dsub_rn(x, prev)));
    }
  }
  if (!a.change) return;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) c = __dadd_rn(c, __shfl_xor_sync(0xFFFFFFFFu, c, d));
  if ((threadIdx.x & 31) == 0) red_c[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (uint32_t i = 0; i < (blockDim.x >> 5); ++i) t = __dadd_rn(t, red_c[i]);
    a.change[blockIdx.x] = t;
  }
}

// sum of tvals[k] * v(trows[k]) over k = b + off, b + off + step, ... < e, with all
// index loads issued before the gathers (8 entries per round) so that a round costs two
// dependent memory latencies whatever its length
__device__ __forceinline__ double dot_strided(const MeasureArgs& a, const double* wp, uint32_t b, uint32_t e,
                                              uint32_t off, uint32_t step, uint32_t it, double v0, double inv)
{
  double acc = 0.0;
  for (uint32_t k0 = b + off; k0 < e; k0 += 8 * step) {
    uint32_t src[8];
    double val[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const uint32_t k = k0 + q * step;
      src[q] = k < e ? __ldg(a.trows + k) : 0u;
      val[q] = k < e ? __ldg(a.tvals + k) : 0.0;
    }
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = k0 + q * step < e ? iterate_value(wp, a.start, src[q], it, v0, inv) : 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) acc = __fma_rn(val[q], v[q], acc);
  }
  return acc;
}

// v <- P^T v / |P^T v|_1.  Rows of P^T are short (a target box has a handful of source
// boxes): rows of up to 8 entries get one thread, rows of up to 64 a group of 8 lanes,
// longer ones a warp, so that every row of an iteration is in flight at once and no
// thread walks a long dependent chain.  The previous iterate is scaled by 1/s on the
// fly, so one grid barrier per iteration suffices.
__global__ void __launch_bounds__(kMeasureThreads) invariant_measure_kernel(MeasureArgs a)
{
  __shared__ double red[kMeasureThreads / 32];
  const uint32_t n = a.n;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = tid >> 5, nwarps = nthreads >> 5;
  const uint32_t group = tid >> 3, ngroups = nthreads >> 3, lane8 = threadIdx.x & 7;
  const double v0 = __ddiv_rn(1.0, double(n));
  double inv = 1.0, inv_prev = 1.0;
  for (uint32_t it = 0; it < a.iters; ++it) {
    const double* wp = (it & 1u) ? a.w0 : a.w1;
    double* wc = (it & 1u) ? a.w1 : a.w0;
    double local = 0.0;
    // short rows: a thread each
    for (uint32_t j = tid; j < n; j += nthreads) {
      const uint32_t b = __ldg(a.tptr + j), e = __ldg(a.tptr + j + 1);
      if (e - b > a.short_limit) continue;
      const double acc = dot_strided(a, wp, b, e, 0u, 1u, it, v0, inv);
      __stcg(wc + j, acc);
      local = __dadd_rn(local, fabs(acc));
    }
    // medium rows: 8 lanes each (trip counts uniform per warp for the shuffles)
    for (uint32_t qb = group & ~3u; qb < a.n_mid; qb += ngroups) {
      const uint32_t q = qb + (group & 3u);
      const bool row = q < a.n_mid;
      const uint32_t j = row ? __ldg(a.mid_rows + q) : 0u;
      const uint32_t b = row ? __ldg(a.tptr + j) : 0u, e = row ? __ldg(a.tptr + j + 1) : 0u;
      double acc = dot_strided(a, wp, b, e, lane8, 8u, it, v0, inv);
#pragma unroll
      for (int d = 4; d > 0; d >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xFFFFFFFFu, acc, d));
      if (row && lane8 == 0) {
        __stcg(wc + j, acc);
        local = __dadd_rn(local, fabs(acc));
      }
    }
    // long rows: a warp each
    for (uint32_t q = warp; q < a.n_long; q += nwarps) {
      const uint32_t j = __ldg(a.long_rows + q);
      const uint32_t b = __ldg(a.tptr + j), e = __ldg(a.tptr + j + 1);
      double acc = dot_strided(a, wp, b, e, lane, 32u, it, v0, inv);
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xFFFFFFFFu, acc, d));
      if (lane == 0) {
        __stcg(wc + j, acc);
        local = __dadd_rn(local, fabs(acc));
      }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) local = __dadd_rn(local, __shfl_xor_sync(0xFFFFFFFFu, local, d));
    if (lane == 0) red[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int i = 0; i < kMeasureThreads / 32; ++i) t = __dadd_rn(t, red[i]);
      __stcg(a.partial + (it & 1u) * gridDim.x + blockIdx.x, t);
    }
    a.gen_seen = it;  // the generation counts completed barriers
    double s_it;
    if (!barrier_sum(a, a.partial + (it & 1u) * gridDim.x, a.totals + (it & 1u), &s_it)) return;
    inv_prev = inv;
    inv = __ddiv_rn(1.0, s_it);
  }
  write_result(a, inv, inv_prev);
}

// Grid barrier on a counter that only grows, in two halves for a caller that has work to
// start in between: the wait (every block publishes its partial sum and arrives with
// release semantics, then polls with acquire loads, bounded) and the total (every block
// adds all partials itself in one fixed order - lane-strided, then a fixed shuffle tree -
// so no block waits for a last arriver to publish it).  A block whose wait gives up sets
// error bit 1 and returns; the others then give up at their next wait, bounded as well.
__device__ bool barrier_wait(const MeasureArgs& a, uint32_t round)
{
  __syncthreads();
  bool ok = true;
  if (threadIdx.x == 0) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(a.bar_count) : "memory");
    const unsigned target = (round + 1u) * gridDim.x;
    unsigned long long polls = 0;
    unsigned seen;
    for (;;) {
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(seen) : "l"(a.bar_count) : "memory");
      if (seen >= target) break;
      if (++polls > kBarrierPolls) { atomicOr(a.error, 2u); ok = false; break; }
    }
  }
  return __syncthreads_and(ok);
}

// Point-to-point waits between barriers.  A block that has written its rows of an iterate
// publishes the count of iterations it has completed (release); before its next
// iteration a block waits (acquire, bounded) only for the blocks whose rows it gathers -
// their rows of the previous iterate must be written - and for the blocks that gather its
// rows - they must have read the previous iterate before it is overwritten (two buffers).
constexpr int kDepWords = 8;   // blocks the dependency masks can name: 256
constexpr uint32_t kEpochStride = 32;  // u32 words between two blocks' epochs: a 128-byte line each

__device__ __forceinline__ void epoch_publish(const MeasureArgs& a, unsigned done)
{
  __syncthreads();
  if (threadIdx.x == 0)
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(a.epoch + blockIdx.x * kEpochStride), "r"(done)
                 : "memory");
}

// thread j waits for block j when `waits` (j < gridDim.x, j named by this block's masks)
__device__ __forceinline__ bool epoch_wait(const MeasureArgs& a, bool waits, unsigned done)
{
  bool ok = true;
  if (waits) {
    unsigned long long polls = 0;
    unsigned seen;
    for (;;) {
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];"
                   : "=r"(seen)
                   : "l"(a.epoch + threadIdx.x * kEpochStride)
                   : "memory");
      if (seen >= done) break;
      if (++polls > kBarrierPolls) { atomicOr(a.error, 2u); ok = false; break; }
    }
  }
  return __syncthreads_and(ok);
}

// the block owning row s: the last j < nb with bnd[j] <= s (bnd ascending, bnd[0] = 0;
// block j owns the rows [bnd[j], bnd[j + 1]))
__device__ __forceinline__ uint32_t owner_block(const uint32_t* bnd, uint32_t nb, uint32_t s)
{
  uint32_t lo = 0, len = nb;
  while (len > 0) {
    const uint32_t half = len >> 1;
    if (bnd[lo + half] <= s) { lo += half + 1; len -= half + 1; }
    else len = half;
  }
  return lo - 1;
}

__device__ double barrier_total(const double* part)
{
  __shared__ double bcast;
  if (threadIdx.x < 32) {
    double x = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += 32) x = __dadd_rn(x, __ldcg(part + i));
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) x = __dadd_rn(x, __shfl_xor_sync(0xFFFFFFFFu, x, d));
    if (threadIdx.x == 0) bcast = x;
  }
  __syncthreads();
  const double total = bcast;
  __syncthreads();           // bcast is read by every thread before it can be written again
  return total;
}

// The shared-memory iteration sums an iterate's L1 norm (and the next iteration scales by
// its inverse) every kNormalisePeriod iterations and at the last two
constexpr uint32_t kNormalisePeriod = 8;

__device__ __forceinline__ bool measure_normalises(uint32_t it, uint32_t iters)
{
  return it % kNormalisePeriod == kNormalisePeriod - 1 || it + 2 >= iters;
}

// The same iteration with the matrix held on chip.  Block b owns the rows of P^T whose
// first entry lies in [b * per, (b + 1) * per) (per = nnz / blocks, rounded up), keeps
// their entries (source, value, row) in shared memory for all iterations, and gives each
// thread a run of at most kSmemChunk consecutive entries: one round of gathers of the
// previous iterate per iteration, whatever the row lengths.  A row split over several
// threads is summed by the thread holding its first entry, adding the other threads'
// parts in thread order, so the result does not depend on scheduling.  A grid barrier
// ends only the normalising iterations (every block needs every partial sum); the others
// end with the block's epoch, and the next iteration waits for the blocks it depends on.
constexpr int kSmemChunk = 13;
constexpr uint32_t kSmemEntries = uint32_t(kSmemChunk) * kMeasureThreads;
constexpr size_t kSmemMeasureBytes = size_t(kSmemEntries) * (8 + 4 + 4) + size_t(kMeasureThreads) * (8 + 4);

__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* a, uint32_t n, uint32_t x)
{
  uint32_t lo = 0, len = n;
  while (len > 0) {
    const uint32_t half = len >> 1;
    if (__ldg(a + lo + half) < x) { lo += half + 1; len -= half + 1; }
    else len = half;
  }
  return lo;
}

__global__ void __launch_bounds__(kMeasureThreads, 1) invariant_measure_smem_kernel(MeasureArgs a, uint32_t nnz)
{
  extern __shared__ __align__(16) unsigned char smem[];
  double* s_val = reinterpret_cast<double*>(smem);
  uint32_t* s_src = reinterpret_cast<uint32_t*>(s_val + kSmemEntries);
  uint32_t* s_row = s_src + kSmemEntries;
  double* s_head = reinterpret_cast<double*>(s_row + kSmemEntries);
  uint32_t* s_head_end = reinterpret_cast<uint32_t*>(s_head + kMeasureThreads);
  __shared__ double red[kMeasureThreads / 32];
  __shared__ uint32_t s_bnd[32 * kDepWords + 1];
  __shared__ uint32_t s_dep[kDepWords];
  const uint32_t n = a.n;
  const uint32_t t = threadIdx.x, lane = t & 31;
  const uint32_t per = (nnz + gridDim.x - 1) / gridDim.x;
  // every block's first row: lower bounds over the n + 1 row starts, at most n (a block
  // past the last entry gets no rows)
  if (t <= gridDim.x) s_bnd[t] = t == gridDim.x ? n : min(lower_bound_u32(a.tptr, n + 1, t * per), n);
  if (t < kDepWords) s_dep[t] = 0u;
  __syncthreads();
  const uint32_t r0 = s_bnd[blockIdx.x], r1 = max(r0, s_bnd[blockIdx.x + 1]);
  const uint32_t e0 = __ldg(a.tptr + r0), e1 = __ldg(a.tptr + r1);
  uint32_t nloc = e1 - e0;
  if (nloc > kSmemEntries) {
    // more entries than the host planned for: flag it and take part in the barriers only
    if (t == 0) atomicOr(a.error, 4u);
    nloc = 0;
  }
  for (uint32_t k = t; k < nloc; k += blockDim.x) {
    s_src[k] = __ldg(a.trows + e0 + k);
    s_val[k] = __ldg(a.tvals + e0 + k);
  }
  for (uint32_t r = r0 + t; r < r1; r += blockDim.x) {
    const uint32_t b = __ldg(a.tptr + r), e = __ldg(a.tptr + r + 1);
    if (b == e) { a.w0[r] = 0.0; a.w1[r] = 0.0; }   // no entries: 0 in every iterate
    if (nloc) for (uint32_t k = b; k < e; ++k) s_row[k - e0] = r;
  }
  __syncthreads();
  // this thread's run of entries and whether its first row began in an earlier run
  const uint32_t chunk = (nloc + blockDim.x - 1) / blockDim.x;
  const uint32_t k0 = min(t * chunk, nloc), k1 = min(k0 + chunk, nloc);
  const bool head_open = k0 < k1 && k0 > 0 && s_row[k0 - 1] == s_row[k0];
  const bool tail_open = k0 < k1 && k1 < nloc && s_row[k1] == s_row[k1 - 1];
  // the blocks owning this block's sources, published for the blocks whose rows they are
  {
    uint32_t m[kDepWords] = {};
    for (uint32_t k = k0; k < k1; ++k) {
      const uint32_t o = owner_block(s_bnd, gridDim.x, s_src[k]);
#pragma unroll
      for (int w = 0; w < kDepWords; ++w) m[w] |= (o >> 5) == uint32_t(w) ? 1u << (o & 31u) : 0u;
    }
#pragma unroll
    for (int w = 0; w < kDepWords; ++w) {
      m[w] = __reduce_or_sync(0xFFFFFFFFu, m[w]);
      if (lane == 0 && m[w]) atomicOr(s_dep + w, m[w]);
    }
  }
  __syncthreads();
  if (t < kDepWords) a.dep_mask[blockIdx.x * kDepWords + t] = s_dep[t];
  if (t == 0) a.epoch[blockIdx.x * kEpochStride] = 0u;
  uint32_t bars = 0;         // full barriers passed
  if (!barrier_wait(a, bars++)) return;
  const uint32_t me = blockIdx.x;
  const bool waits = t < gridDim.x && t != me &&
                     (((s_dep[t >> 5] >> (t & 31u)) & 1u) ||
                      ((__ldcg(a.dep_mask + t * kDepWords + (me >> 5)) >> (me & 31u)) & 1u));
  const double v0 = __ddiv_rn(1.0, double(n));
  double inv = 1.0, inv_prev = 1.0;
  uint32_t norms = 0;        // normalising iterations done: their partial sums alternate slots
  bool after_barrier = true;
  for (uint32_t it = 0; it < a.iters; ++it) {
    const double* wp = (it & 1u) ? a.w0 : a.w1;
    double* wc = (it & 1u) ? a.w1 : a.w0;
    double local = 0.0;
    double v[kSmemChunk];
    if (!after_barrier && !epoch_wait(a, waits, it)) return;
    // the gathers of the previous iterate go out first; when that iterate's L1 norm was
    // summed (the partial sums of the barrier before), it is read while they are in
    // flight and every value is scaled by its inverse exactly as iterate_value scales it;
    // the iterates between two normalisations are left unscaled (the same direction: the
    // scaling is linear; the last two iterates are always normalised, for the result and
    // its change)
#pragma unroll
    for (int q = 0; q < kSmemChunk; ++q) {
      const uint32_t k = k0 + q;
      v[q] = k < k1 ? (it == 0 ? (a.start ? __ldg(a.start + s_src[k]) : v0) : __ldcg(wp + s_src[k])) : 0.0;
    }
    if (it > 0 && measure_normalises(it - 1, a.iters)) {
      const double s_prev = barrier_total(a.partial + ((norms - 1u) & 1u) * gridDim.x);
      inv_prev = inv;
      inv = __ddiv_rn(1.0, s_prev);
#pragma unroll
      for (int q = 0; q < kSmemChunk; ++q) v[q] = __dmul_rn(v[q], inv);
    }
    // walk the run: a row that ends inside it is written here unless it began earlier
    uint32_t row = k0 < k1 ? s_row[k0] : 0u;
    double acc = 0.0, tail = 0.0;
    bool first = true;
#pragma unroll
    for (int q = 0; q < kSmemChunk; ++q) {
      const uint32_t k = k0 + q;
      if (k < k1) {
        const uint32_t r = s_row[k];
        if (r != row) {
          if (first && head_open) { s_head[t] = acc; s_head_end[t] = 1u; }
          else { __stcg(wc + row, acc); local = __dadd_rn(local, fabs(acc)); }
          first = false;
          row = r;
          acc = 0.0;
        }
        acc = __fma_rn(s_val[k], v[q], acc);
      }
    }
    if (k0 < k1) {
      if (first && head_open) { s_head[t] = acc; s_head_end[t] = tail_open ? 0u : 1u; }
      else if (tail_open) tail = acc;
      else { __stcg(wc + row, acc); local = __dadd_rn(local, fabs(acc)); }
    }
    __syncthreads();
    if (k0 < k1 && tail_open && !(first && head_open)) {
      // this run holds the row's first entry: add the later runs' parts in order
      double sum = tail;
      for (uint32_t j = t + 1; j < blockDim.x; ++j) {
        sum = __dadd_rn(sum, s_head[j]);
        if (s_head_end[j]) break;
      }
      __stcg(wc + row, sum);
      local = __dadd_rn(local, fabs(sum));
    }
    if (measure_normalises(it, a.iters)) {
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) local = __dadd_rn(local, __shfl_xor_sync(0xFFFFFFFFu, local, d));
      if (lane == 0) red[t >> 5] = local;
      __syncthreads();
      if (t == 0) {
        double sum = 0.0;
        for (int i = 0; i < kMeasureThreads / 32; ++i) sum = __dadd_rn(sum, red[i]);
        __stcg(a.partial + (norms & 1u) * gridDim.x + blockIdx.x, sum);
      }
      // every block reads the partial sums at the start of the next iteration; a slot is
      // written again only after the next barrier, which every reader passes afterwards
      if (!barrier_wait(a, bars++)) return;
      ++norms;
      after_barrier = true;
    } else {
      epoch_publish(a, it + 1u);
      after_barrier = false;
    }
  }
  if (a.iters) {
    // the last iteration normalises: a barrier ended it
    const double s_last = barrier_total(a.partial + ((norms - 1u) & 1u) * gridDim.x);
    inv_prev = inv;
    inv = __ddiv_rn(1.0, s_last);
  }
  write_result(a, inv, inv_prev);
}

// the rows of P^T of one length class (1: medium, 2: long), ascending (flag, scan, scatter)
__device__ __forceinline__ uint32_t row_class(const uint32_t* tptr, uint32_t j)
{
  const uint32_t len = tptr[j + 1] - tptr[j];
  return len <= kShortRow ? 0u : (len <= kMidRow ? 1u : 2u);
}

__global__ void class_flag_kernel(const uint32_t* tptr, uint32_t n, uint32_t cls, uint32_t* flag)
{
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    flag[j] = row_class(tptr, j) == cls ? 1u : 0u;
}

__global__ void class_scatter_kernel(const uint32_t* tptr, uint32_t n, uint32_t cls, const uint32_t* pos,
                                     uint32_t* list)
{
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    if (row_class(tptr, j) == cls) list[pos[j]] = j;
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
  transpose_sort_kernel<<<grid_for(uint64_t(n_cols) * 32, kThreads, 8), kThreads, 0, s>>>(tptr, n_cols, trows,
                                                                                           tvals);
  return cudaGetLastError();
}

cudaError_t class_rows(const uint32_t* tptr, uint32_t n, uint32_t cls, uint32_t* flag, uint32_t* pos,
                       uint32_t* list, const uint32_t* n_dev, uint32_t* tile_sums, cudaStream_t s)
{
  class_flag_kernel<<<grid_for(n, kThreads, 8), kThreads, 0, s>>>(tptr, n, cls, flag);
  cudaError_t e = exclusive_scan_u32(flag, pos, n_dev, tile_sums, n, s);
  if (e != cudaSuccess) return e;
  class_scatter_kernel<<<grid_for(n, kThreads, 8), kThreads, 0, s>>>(tptr, n, cls, pos, list);
  return cudaGetLastError();
}

namespace {

struct MeasureLaunch
{
  bool smem_ok;        // the shared-memory kernel may take kSmemMeasureBytes and fits one block per SM
  int blocks_per_sm;   // resident blocks per SM of the L2 kernel
};

std::mutex g_measure_mu;
int g_measure_ready[64] = {};
MeasureLaunch g_measure_cfg[64];

// Per device: cudaFuncSetAttribute applies to the device current when it runs, so the
// opt-in to the large shared memory is made once on every device that launches the
// kernel, with that device current, under a lock (server engines run on their own
// host threads).
MeasureLaunch measure_launch()
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { cudaGetLastError(); return {false, 1}; }
  std::lock_guard<std::mutex> lock(g_measure_mu);
  if (!g_measure_ready[dev]) {
    int b = 0;
    MeasureLaunch c;
    c.smem_ok = cudaFuncSetAttribute(invariant_measure_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(kSmemMeasureBytes)) == cudaSuccess &&
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, invariant_measure_smem_kernel, kMeasureThreads,
                                                              kSmemMeasureBytes) == cudaSuccess && b >= 1;
    cudaGetLastError();
    b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, invariant_measure_kernel, kMeasureThreads, 0);
    cudaGetLastError();
    c.blocks_per_sm = b > 0 ? b : 1;
    g_measure_cfg[dev] = c;
    g_measure_ready[dev] = 1;
  }
  return g_measure_cfg[dev];
}

}  // namespace

bool measure_on_chip(uint64_t nnz, uint32_t max_row, uint32_t partial_cap)
{
  const MeasureLaunch cfg = measure_launch();
  const uint32_t blocks = uint32_t(device_sm_count());
  // partial: 2 x blocks partial sums, 2 totals, then (as u32) the blocks' epochs, a
  // 128-byte line each, and their dependency masks
  const uint64_t slots = 2ull * blocks + 2 + (uint64_t(blocks) * kEpochStride + uint64_t(kDepWords) * blocks + 1) / 2;
  // a block's rows begin in its share of the entries and have at most kMidRow entries
  return cfg.smem_ok && max_row <= kMidRow && nnz > 0 && (nnz + blocks - 1) / blocks + kMidRow <= kSmemEntries &&
         blocks <= 32u * kDepWords && slots <= partial_cap;
}

cudaError_t max_row_length(const uint32_t* tptr, uint32_t n, uint32_t* out, cudaStream_t s)
{
  cudaMemsetAsync(out, 0, sizeof(uint32_t), s);
  max_row_kernel<<<grid_for(n, kThreads, 8), kThreads, 0, s>>>(tptr, n, out);
  return cudaGetLastError();
}

cudaError_t invariant_measure(const uint32_t* tptr, const uint32_t* trows, const double* tvals,
                              const uint32_t* mid_list, uint32_t n_mid, const uint32_t* long_list, uint32_t n_long,
                              uint32_t n, uint32_t iters, double* w0, double* w1, double* partial,
                              uint32_t partial_cap, double* out, unsigned* sync_words, cudaStream_t s, uint64_t nnz,
                              const double* start, double* change)
{
  // the matrix on chip: one block per SM, every block's rows within its shared memory
  // (a row of P^T has at most kMidRow entries when there are no long rows)
  const MeasureLaunch cfg = measure_launch();
  const uint32_t blocks = uint32_t(device_sm_count());
  const uint32_t epoch_words = blocks * kEpochStride;
  if (mid_list && long_list && n_long == 0 && measure_on_chip(nnz, 0u, partial_cap)) {
    cudaMemsetAsync(sync_words, 0, 65 * sizeof(unsigned), s);
    unsigned* words = reinterpret_cast<unsigned*>(partial + 2 * size_t(blocks) + 2);
    MeasureArgs a{tptr, trows, tvals, mid_list, n_mid, long_list, 0u, kShortRow, n, iters, w0, w1, partial, out,
                  sync_words, sync_words + 32, sync_words + 64, partial + 2 * size_t(blocks), 0u, start, change,
                  words, words + epoch_words};
    uint32_t nnz32 = uint32_t(nnz);
    void* params[] = {&a, &nnz32};
    return cudaLaunchCooperativeKernel((const void*)invariant_measure_smem_kernel, dim3(blocks),
                                       dim3(kMeasureThreads), params, kSmemMeasureBytes, s);
  }
  int grid = grid_for(n, kMeasureThreads, cfg.blocks_per_sm);
  if (grid > int(partial_cap / 2)) grid = int(partial_cap / 2);
  if (grid < 1) grid = 1;
  if (grid > int(partial_cap / 2) - 1) grid = int(partial_cap / 2) - 1;
  cudaMemsetAsync(sync_words, 0, 65 * sizeof(unsigned), s);
  // partial: 2 x grid per-block sums, then 2 totals
  // barrier words on separate 128-byte lines: arrival count, generation, error
  const bool lists = mid_list && long_list;
  MeasureArgs a{tptr, trows, tvals, mid_list, lists ? n_mid : 0u, long_list, lists ? n_long : 0u,
                lists ? kShortRow : 0xFFFFFFFFu, n, iters, w0, w1, partial, out, sync_words, sync_words + 32,
                sync_words + 64, partial + 2 * size_t(grid), 0u, start, change};
  void* params[] = {&a};
  return cudaLaunchCooperativeKernel((const void*)invariant_measure_kernel, dim3(grid), dim3(kMeasureThreads), params,
                                     0, s);
}

int measure_partial_slots()
{
  return 2 * device_sm_count() * 12;
}

}  // namespace b12g
