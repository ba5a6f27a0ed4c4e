// Job server: continuous batching of subdivision jobs (subdivision loop of
// subdivision.m:18-45 followed by transitionMatrixForLeaves) on one GPU.
//
// Jobs of one family (map kind, arithmetic, grid, domain, integrator step) share an
// engine: a host thread with its own CUDA stream that repeatedly runs a *tick* - one
// subdivision step of every job it holds, as one batched launch sequence (lookup table
// over (slot, code), persistent work-queue image kernel, per-job survivor counts, one
// ordered compaction).  A job admitted while others are running joins at the next tick
// as the surrounding box; a job whose depth is reached leaves at the end of the tick,
// gets its transition matrix from a batched row kernel, and its leaves and CSR stay
// resident on the device until the client releases them.  Engines of different
// families run concurrently on their own streams.
//
// Admission is by projected HBM footprint: a job is admitted when the projected bytes
// of every admitted and resident job plus its own stay under the server's cap;
// otherwise it waits (first come, first served within its family).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "batch.h"
#include "tree.h"

using namespace b12g;
using namespace b12g::host;

namespace {

constexpr uint32_t kMaxSlots = 2048;            // jobs per engine at once
constexpr uint64_t kInitialLeaves = 1u << 19;

double now_s()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// projected peak leaves of a job: growth per depth of the attractors of the three
// families with a margin, and never more than 2^depth
uint64_t projected_boxes(const b12g_job& j)
{
  double c = 4.0;
  if (j.map.kind == B12G_MAP_HENON) c = 2.5;
  else if (j.map.kind == B12G_MAP_LORENZ) c = 1.6;
  else if (j.map.kind == B12G_MAP_FORCED_DUFFING) c = 2.0;
  const double est = c * std::pow(1.6, double(j.depth));
  const double cap = std::ldexp(1.0, std::min<int>(int(j.depth), 62));
  return uint64_t(std::max(1.0, std::min(est, cap)));
}

uint64_t points_per_box(const b12g_job& j)
{
  if (j.grid.kind == B12G_GRID_PHILOX) return j.grid.points;
  uint64_t p = 1;
  for (uint32_t d = 0; d < j.domain.dim; ++d) p *= j.grid.n;
  return p;
}

// engine working set + resident result + transient row staging, per box
uint64_t projected_bytes(const b12g_job& j)
{
  return projected_boxes(j) * (160 + 8 * points_per_box(j));
}

struct Job {
  uint64_t id = 0;
  b12g_job spec{};
  double t_submit = 0.0, t_start = 0.0, t_done = 0.0;
  int state = B12G_JOB_WAITING;
  uint64_t reserved = 0;          // admitted bytes
  uint32_t depth_done = 0;        // subdivision steps done
  std::vector<uint32_t> counts;   // leaves after each step
  // resident result: one block from the server's pool holding codes, vals, rowptr, cols
  void* mem = nullptr;
  uint64_t* codes = nullptr;
  uint32_t* rowptr = nullptr;
  uint32_t* cols = nullptr;
  double* vals = nullptr;
  uint32_t n_boxes = 0;
  uint64_t nnz = 0;
  std::string error;
};

struct Server;

struct Engine {
  Server* srv = nullptr;
  b12g_job key{};                  // family description (params and depth ignored)
  cudaStream_t stream = nullptr;
  std::thread thread;
  std::deque<Job*> waiting;        // guarded by Server::mu
  std::vector<Job*> slots;         // running jobs in slot order (engine thread only)
  Domain dom{};
  MapParams mp{};
  GridParams gp{};
  uint64_t P = 0;
  Tuning tuning{};
  // device state: parents in slot order, their children's survivors, the hit mask
  Buf<uint64_t> parents, children;
  Buf<uint8_t> flags_a, flags_b, hit;
  Buf<uint32_t> off, new_off, cnt, ctr, tiles_a, tiles_b, keep_off, fin_off, fin_slot, fin_rank, row0;
  Buf<double> params, fin_params;
  Buf<uint8_t> depth_child, fin_depth;
  Buf<ulonglong2> hash;
  uint32_t hash_log2 = 0, tag = 0;
  Buf<uint64_t> arena;               // finished jobs' leaves, contiguous
  Buf<uint32_t> stage_col, stage_cnt, row_count, rowptr, cols_all;
  Buf<double> vals_all;
  // the finishing jobs' last-step image targets and that step's compaction ranks
  Buf<uint32_t> targets, rank, fin_child;       // fin_child: child offsets (nf + 1), child bases (nf)
  Buf<uint64_t> tgt_base;                        // per slot: targets offset, ~0 when not finishing
  double* table = nullptr;           // forcing table (forced Duffing)
  // pinned host mirrors
  uint32_t* h = nullptr;             // counts, counters, ranks
  double* hp = nullptr;              // parameters
  uint8_t* hd = nullptr;             // depths and finishing marks
  uint64_t* ht = nullptr;            // targets offsets
  uint64_t boxes = 0;                // parents after the last tick
  // counters written by the engine thread
  std::atomic<uint64_t> ticks{0}, jobs_done{0};
  std::atomic<double> tick_seconds{0.0}, finish_seconds{0.0};
};

struct Server {
  cudaMemPool_t pool = nullptr;    // results (kept across synchronisations)
  cudaStream_t release_stream = nullptr;
  std::mutex mu;
  std::condition_variable cv;
  bool stop = false;
  uint64_t cap_bytes = 0;
  uint64_t in_use = 0;
  uint64_t next_id = 1;
  int device = 0;
  std::map<uint64_t, std::unique_ptr<Job>> jobs;
  std::vector<std::unique_ptr<Engine>> engines;
  std::deque<uint64_t> done_queue;
  std::atomic<uint64_t> ticks{0};
  std::atomic<uint64_t> box_images{0};
};

bool same_family(const b12g_job& a, const b12g_job& b)
{
  return a.map.kind == b.map.kind && a.map.arith == b.map.arith && a.map.steps == b.map.steps && a.map.h == b.map.h &&
         a.grid.kind == b.grid.kind && a.grid.n == b.grid.n && a.grid.points == b.grid.points &&
         a.grid.eps == b.grid.eps && a.grid.seed == b.grid.seed &&
         std::memcmp(&a.domain, &b.domain, sizeof(b12g_domain)) == 0;
}

// engine counter words
enum : int { E_ERROR = 0, E_QUEUE = 1, E_TOTAL = 2, E_KEEP = 3, E_FIN = 4, E_COUNT = 32 };

// pinned mirror layout (u32 words)
constexpr size_t kHostCounts = 0;                    // A counts
constexpr size_t kHostCtr = 2 * kMaxSlots;           // E_COUNT counters
constexpr size_t kHostRank = 3 * kMaxSlots;          // A finish ranks
constexpr size_t kHostScratch = 5 * kMaxSlots;       // finish bookkeeping (2 x (kMaxSlots + 1))
constexpr size_t kHostFinChildren = 8 * kMaxSlots;  // finishing jobs' children this tick
constexpr size_t kHostFinStage = 9 * kMaxSlots;     // their child offsets and bases (2 nf + 1)
constexpr size_t kHostWords = 11 * kMaxSlots + 16;

// ---------------------------------------------------------------------------- kernels
// append n_new surrounding boxes (code 0, flags SD) after the A current slots
__global__ void append_roots_kernel(uint32_t* off, uint32_t A, uint32_t n_new, uint64_t* codes, uint8_t* flags)
{
  const uint32_t base = off[A];
  for (uint32_t j = threadIdx.x; j < n_new; j += blockDim.x) {
    codes[base + j] = 0;
    flags[base + j] = B12G_SD;
    off[A + j + 1] = base + j + 1;
  }
}

// exclusive scan over one block of kSplitThreads threads of four counters at once
constexpr uint32_t kSplitThreads = kMaxSlots / 2;

__device__ uint4 block_exclusive_scan4(uint4 v, uint4* total)
{
  __shared__ uint4 warp_sums[kSplitThreads / 32];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint4 inc = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t x = __shfl_up_sync(0xFFFFFFFFu, inc.x, d), y = __shfl_up_sync(0xFFFFFFFFu, inc.y, d);
    const uint32_t z = __shfl_up_sync(0xFFFFFFFFu, inc.z, d), q = __shfl_up_sync(0xFFFFFFFFu, inc.w, d);
    if (lane >= uint32_t(d)) { inc.x += x; inc.y += y; inc.z += z; inc.w += q; }
  }
  if (lane == 31) warp_sums[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint4 s = lane < kSplitThreads / 32 ? warp_sums[lane] : make_uint4(0, 0, 0, 0);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t x = __shfl_up_sync(0xFFFFFFFFu, s.x, d), y = __shfl_up_sync(0xFFFFFFFFu, s.y, d);
      const uint32_t z = __shfl_up_sync(0xFFFFFFFFu, s.z, d), q = __shfl_up_sync(0xFFFFFFFFu, s.w, d);
      if (lane >= uint32_t(d)) { s.x += x; s.y += y; s.z += z; s.w += q; }
    }
    if (lane < kSplitThreads / 32) warp_sums[lane] = s;   // inclusive warp prefixes
  }
  __syncthreads();
  const uint4 before = w ? warp_sums[w - 1] : make_uint4(0, 0, 0, 0);
  *total = warp_sums[kSplitThreads / 32 - 1];
  return make_uint4(before.x + inc.x - v.x, before.y + inc.y - v.y, before.z + inc.z - v.z, before.w + inc.w - v.w);
}

// one block of kSplitThreads threads, two slots each: the survivors' offsets for all
// slots (new_off), for the continuing slots (keep_off, and packed into `off` as the
// parent offsets of the next tick) and for the finished slots (fin_off, in finish order)
__global__ void __launch_bounds__(kSplitThreads) split_offsets_kernel(const uint32_t* cnt, const uint8_t* finishing,
                                                                      uint32_t A, uint32_t* new_off,
                                                                      uint32_t* keep_off, uint32_t* fin_off,
                                                                      uint32_t* off, uint32_t* ctr)
{
  uint32_t c[2] = {0, 0}, f[2] = {0, 0};
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const uint32_t i = 2 * threadIdx.x + k;
    if (i < A) { c[k] = cnt[i]; f[k] = finishing[i] ? 1u : 0u; }
  }
  // (all survivors, continuing survivors, finished survivors, finished slots)
  const uint4 mine = make_uint4(c[0] + c[1], (1 - f[0]) * c[0] + (1 - f[1]) * c[1], f[0] * c[0] + f[1] * c[1],
                                f[0] + f[1]);
  uint4 total;
  uint4 p = block_exclusive_scan4(mine, &total);
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const uint32_t i = 2 * threadIdx.x + k;
    if (i >= A) break;
    new_off[i] = p.x;
    if (f[k]) {
      fin_off[p.w] = p.z;
    } else {
      keep_off[i] = p.y;
      off[i - p.w] = p.y;            // rank among the continuing slots
    }
    p.x += c[k];
    p.y += (1 - f[k]) * c[k];
    p.z += f[k] * c[k];
    p.w += f[k];
  }
  if (threadIdx.x == 0) {
    new_off[A] = total.x;
    fin_off[total.w] = total.z;
    off[A - total.w] = total.y;
    ctr[E_KEEP] = total.y;
    ctr[E_FIN] = total.z;
  }
}

// move every survivor to the packed parents of the continuing slots or to the arena
__global__ void split_copy_kernel(const uint64_t* survivors, const uint8_t* surv_flags, const uint32_t* new_off,
                                  uint32_t A, const uint8_t* finishing, const uint32_t* keep_off,
                                  const uint32_t* fin_off, const uint32_t* fin_rank, uint64_t* parents,
                                  uint8_t* parent_flags, uint64_t* arena, uint32_t cap, uint32_t arena_cap,
                                  uint32_t* error)
{
  __shared__ uint32_t off_s[kMaxSlots + 1];
  for (uint32_t i = threadIdx.x; i <= A; i += blockDim.x) off_s[i] = new_off[i];
  __syncthreads();
  const uint32_t total = off_s[A];
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    // largest slot with off_s[slot] <= g
    uint32_t lo = 0, len = A;
    while (len > 1) {
      const uint32_t half = len >> 1;
      lo = off_s[lo + half] <= g ? lo + half : lo;
      len -= half;
    }
    const uint32_t r = g - off_s[lo];
    if (finishing[lo]) {
      const uint32_t d = fin_off[fin_rank[lo]] + r;
      if (d < arena_cap) arena[d] = survivors[g];
      else atomicOr(error, 1u);
    } else {
      const uint32_t d = keep_off[lo] + r;
      if (d < cap) { parents[d] = survivors[g]; parent_flags[d] = surv_flags[g]; }
      else atomicOr(error, 1u);
    }
  }
}

// first nonzero of each finished job's rows: row0[q] = rowptr[fin_off[q]], q <= nf
__global__ void row_starts_kernel(const uint32_t* rowptr, const uint32_t* fin_off, uint32_t nf, uint32_t* row0)
{
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q <= nf; q += gridDim.x * blockDim.x)
    row0[q] = rowptr[fin_off[q]];
}

// one finished job's rows of the CSR rebased to 0, and its leaves, into its own memory
__global__ void extract_kernel(const uint32_t* rowptr, const uint32_t* cols, const double* vals, const uint64_t* arena,
                               uint32_t first_row, uint32_t rows, uint32_t* out_rowptr, uint32_t* out_cols,
                               double* out_vals, uint64_t* out_codes)
{
  const uint32_t e0 = rowptr[first_row], e1 = rowptr[first_row + rows];
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  for (uint32_t r = t; r <= rows; r += stride) out_rowptr[r] = rowptr[first_row + r] - e0;
  for (uint32_t r = t; r < rows; r += stride) out_codes[r] = arena[first_row + r];
  for (uint32_t e = e0 + t; e < e1; e += stride) {
    out_cols[e - e0] = cols[e];
    out_vals[e - e0] = vals[e];
  }
}

// ---------------------------------------------------------------------------- engine
b12g_status engine_reserve(Engine* e, uint64_t parents);

b12g_status engine_init(Engine* e, const b12g_job& key)
{
  e->key = key;
  b12g_tree* probe = nullptr;
  ST(b12g_tree_create(&key.domain, &probe));
  b12g_scheme sc{};
  sc.map = key.map;
  sc.grid = key.grid;
  sc.depth = B12G_LEAF_DEPTH;
  Prepared pr;
  b12g_status st = prepare(probe, &sc, pr);
  if (st == B12G_OK) {
    e->dom = probe->dom;
    e->mp = pr.a.map;
    e->gp = pr.a.grid;
    e->P = pr.P;
    if (key.map.kind == B12G_MAP_FORCED_DUFFING) {
      // the engine keeps its own copy of the forcing table
      const size_t n = 2 * size_t(key.map.steps) + 1;
      if (cudaMalloc(&e->table, n * sizeof(double)) != cudaSuccess ||
          cudaMemcpy(e->table, probe->table.p, n * sizeof(double), cudaMemcpyDeviceToDevice) != cudaSuccess)
        st = cuda_fail(cudaGetLastError(), "forcing table");
      e->mp.table = e->table;
    }
  }
  b12g_tree_destroy(probe);
  if (st != B12G_OK) return st;
  if (e->P > kMaxRowPoints)
    return fail(B12G_ERR_CAPACITY, "served jobs take up to %u grid points per box", kMaxRowPoints);
  e->tuning = batch_tuning(e->srv->device, key.map.kind, key.map.arith, key.grid.kind, key.domain.dim);
  CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
  CK(cudaMallocHost(&e->h, kHostWords * 4));
  CK(cudaMallocHost(&e->hp, size_t(kMaxSlots) * 6 * 8));
  CK(cudaMallocHost(&e->hd, 2 * size_t(kMaxSlots)));
  CK(cudaMallocHost(&e->ht, size_t(kMaxSlots) * 8));
  ST(e->tgt_base.ensure(kMaxSlots, "engine targets offsets"));
  ST(e->fin_child.ensure(2 * kMaxSlots + 1, "engine finishing children"));
  ST(e->off.ensure(kMaxSlots + 1, "engine offsets"));
  ST(e->new_off.ensure(kMaxSlots + 1, "engine offsets"));
  ST(e->keep_off.ensure(kMaxSlots + 1, "engine offsets"));
  ST(e->fin_off.ensure(kMaxSlots + 1, "engine offsets"));
  ST(e->fin_slot.ensure(kMaxSlots + 1, "engine offsets"));
  ST(e->fin_rank.ensure(kMaxSlots, "engine offsets"));
  ST(e->row0.ensure(kMaxSlots + 1, "engine offsets"));
  ST(e->cnt.ensure(kMaxSlots, "engine counts"));
  ST(e->ctr.ensure(E_COUNT, "engine counters"));
  ST(e->params.ensure(size_t(kMaxSlots) * 6, "engine params"));
  ST(e->fin_params.ensure(size_t(kMaxSlots) * 6, "engine params"));
  ST(e->depth_child.ensure(2 * kMaxSlots, "engine depths"));
  ST(e->fin_depth.ensure(kMaxSlots, "engine depths"));
  CK(cudaMemsetAsync(e->off.p, 0, (kMaxSlots + 1) * 4, e->stream));
  CK(cudaMemsetAsync(e->ctr.p, 0, E_COUNT * 4, e->stream));
  // working set for half a million leaves in flight before the first growth
  ST(engine_reserve(e, kInitialLeaves));
  ST(e->stage_col.ensure(kInitialLeaves * e->P, "row staging"));
  ST(e->stage_cnt.ensure(kInitialLeaves * e->P, "row staging"));
  CK(cudaStreamSynchronize(e->stream));
  return B12G_OK;
}

// grow-only buffers of an engine double when they grow: every reallocation frees the old
// buffer, which waits for the whole device
size_t grow(size_t have, size_t need) { return need <= have ? need : std::max(need, 2 * have); }

b12g_status engine_hash_capacity(Engine* e, uint64_t keys)
{
  uint32_t l = 6;
  while ((1ull << l) < 2ull * std::max<uint64_t>(keys, 1)) ++l;
  if (e->hash.p && l <= e->hash_log2) return B12G_OK;
  e->hash.release();
  ST(e->hash.ensure(size_t(1) << l, "engine lookup table"));
  CK(cudaMemsetAsync(e->hash.p, 0, e->hash.n * sizeof(ulonglong2), e->stream));
  e->hash_log2 = l;
  e->tag = 0;
  return B12G_OK;
}

// make room for a tick over `parents` leaves: their children, and the survivors (at
// most twice the parents) packed back into the parents buffer or moved to the arena
b12g_status engine_reserve(Engine* e, uint64_t parents)
{
  const uint64_t need = std::max<uint64_t>(parents, 1024);
  if (need > 0x3FFFFFF0ull) return fail(B12G_ERR_CAPACITY, "engine above 2^30 leaves");
  // the live parents (and their flags) survive a reallocation
  ST(e->parents.grow_keep(grow(e->parents.n, 2 * need), e->boxes, e->stream, "engine parents"));
  ST(e->flags_a.grow_keep(grow(e->flags_a.n, 2 * need), e->boxes, e->stream, "engine flags"));
  ST(e->children.ensure(grow(e->children.n, 2 * need), "engine survivors"));
  ST(e->flags_b.ensure(grow(e->flags_b.n, 2 * need), "engine survivor flags"));
  if (e->hit.n < 2 * need) {
    ST(e->hit.ensure(grow(e->hit.n, 2 * need), "engine hit mask"));
    CK(cudaMemsetAsync(e->hit.p, 0, e->hit.n, e->stream));
  }
  ST(e->arena.ensure(grow(e->arena.n, 2 * need), "engine arena"));
  const size_t most = std::max<size_t>(e->hit.n, 2 * need) + 1;
  ST(e->tiles_a.ensure(compact_tiles(most) + 2, "engine tiles"));
  ST(e->tiles_b.ensure(compact_tiles(most) + 2, "engine tiles"));
  return engine_hash_capacity(e, need);
}

// next build tag of the lookup table (cleared when the 8-bit tag would wrap)
b12g_status engine_next_tag(Engine* e, uint32_t* tag)
{
  if (e->tag >= 255) {
    CK(cudaMemsetAsync(e->hash.p, 0, e->hash.n * sizeof(ulonglong2), e->stream));
    e->tag = 0;
  }
  *tag = ++e->tag;
  return B12G_OK;
}

void fail_job_locked(Server* s, Job* j, const std::string& why)
{
  j->state = B12G_JOB_FAILED;
  j->error = why;
  j->t_done = now_s();
  s->done_queue.push_back(j->id);
}

// the finished slots of this tick: transition matrices and resident results
// stored: the tick kept the finishing jobs' image targets and compaction ranks
b12g_status engine_finish(Engine* e, const std::vector<uint32_t>& fin, uint32_t rows, bool stored)
{
  Server* s = e->srv;
  const double t_begin = now_s();
  const uint32_t nf = uint32_t(fin.size());
  if (nf == 0) return B12G_OK;
  // the finished jobs' parameters and depths, in finish order
  for (uint32_t q = 0; q < nf; ++q) {
    const Job* j = e->slots[fin[q]];
    for (int k = 0; k < 6; ++k) e->hp[size_t(q) * 6 + k] = j->spec.map.p[k];
    e->hd[q] = uint8_t(j->spec.depth);
    e->h[kHostScratch + q] = q;
  }
  if (!stored) {
    CK(cudaMemcpyAsync(e->fin_params.p, e->hp, size_t(nf) * 6 * 8, cudaMemcpyHostToDevice, e->stream));
    CK(cudaMemcpyAsync(e->fin_depth.p, e->hd, nf, cudaMemcpyHostToDevice, e->stream));
    CK(cudaMemcpyAsync(e->fin_slot.p, e->h + kHostScratch, nf * 4, cudaMemcpyHostToDevice, e->stream));
  }
  const uint64_t stage = std::max<uint64_t>(uint64_t(rows) * e->P, 1);
  ST(e->stage_col.ensure(grow(e->stage_col.n, stage), "row staging"));
  ST(e->stage_cnt.ensure(grow(e->stage_cnt.n, stage), "row staging"));
  ST(e->row_count.ensure(rows + 1, "row counts"));
  ST(e->rowptr.ensure(rows + 1, "row pointers"));
  ST(e->tiles_a.ensure(compact_tiles(rows + 1) + 2, "tiles"));
  if (stored) {
    // rows from the targets the last step kept: no map evaluation
    TargetRowArgs ta{};
    ta.n_inst = nf;
    ta.child_off = e->fin_child.p;
    ta.child_base = e->fin_child.p + (nf + 1);
    ta.row_off = e->fin_off.p;
    ta.rank = e->rank.p;
    ta.targets = e->targets.p;
    ta.arena = e->arena.p;
    ta.points = uint32_t(e->P);
    ta.keep_lost = 0;
    ta.stage_col = e->stage_col.p;
    ta.stage_cnt = e->stage_cnt.p;
    ta.row_count = e->row_count.p;
    CK(launch_target_rows(ta, e->h[kHostFinChildren], e->stream));
  } else {
  // lookup over the finished leaves keyed by (finish rank, code)
  ST(engine_hash_capacity(e, rows));
  uint32_t tag = 0;
  ST(engine_next_tag(e, &tag));
  const LeafHash h{e->hash.p, tag, e->hash_log2};
  CK(launch_batch_hash(e->arena.p, e->fin_off.p, nf, h, uint32_t(std::min<size_t>(e->arena.n, 0xFFFFFFFFu)),
                       e->ctr.p + E_ERROR, e->stream));
  BatchRowArgs ra{};
  ra.dom = e->dom;
  ra.map = e->mp;
  ra.grid = e->gp;
  ra.points = e->P;
  ra.params = e->fin_params.p;
  ra.depths = e->fin_depth.p;
  ra.n_inst = nf;
  ra.off = e->fin_off.p;
  ra.inst_of = e->fin_slot.p;
  ra.codes = e->arena.p;
  ra.hash = h;
  ra.keep_lost = 0;
  ra.stage_col = e->stage_col.p;
  ra.stage_cnt = e->stage_cnt.p;
  ra.row_count = e->row_count.p;
  CK(launch_batch_rows(e->key.map.kind, e->key.map.arith, e->key.grid.kind, ra, rows, e->stream));
  }
  CK(exclusive_scan_u32(e->row_count.p, e->rowptr.p, e->fin_off.p + nf, e->tiles_a.p, rows, e->stream));
  uint32_t* h_nnz = e->h + kHostScratch;
  CK(cudaMemcpyAsync(h_nnz, e->rowptr.p + rows, 4, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  const uint32_t nnz = *h_nnz;
  ST(e->cols_all.ensure(grow(e->cols_all.n, std::max<uint32_t>(nnz, 1)), "columns"));
  ST(e->vals_all.ensure(grow(e->vals_all.n, std::max<uint32_t>(nnz, 1)), "values"));
  CK(gather_rows(e->stage_col.p, e->stage_cnt.p, uint32_t(e->P), e->row_count.p, e->rowptr.p, e->fin_off.p + nf,
                 e->cols_all.p, e->vals_all.p, 0, double(e->P), rows, e->stream));
  row_starts_kernel<<<(nf + 256) / 256, 256, 0, e->stream>>>(e->rowptr.p, e->fin_off.p, nf, e->row0.p);
  count_launches(stored ? 6 : 7);
  // per finished job: its first row and first nonzero
  uint32_t* h_foff = e->h + kHostScratch;
  uint32_t* h_e0 = e->h + kHostScratch + (kMaxSlots + 1);
  CK(cudaMemcpyAsync(h_foff, e->fin_off.p, (nf + 1) * 4, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaMemcpyAsync(h_e0, e->row0.p, (nf + 1) * 4, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  std::vector<std::string> failed(nf);
  for (uint32_t q = 0; q < nf; ++q) {
    Job* j = e->slots[fin[q]];
    const uint32_t n = h_foff[q + 1] - h_foff[q];
    const uint64_t z = h_e0[q + 1] - h_e0[q];
    j->n_boxes = n;
    j->nnz = z;
    if (n == 0) continue;  // every box was removed: the result is the surrounding box
    const size_t b_codes = size_t(n) * 8, b_vals = z * 8, b_rowptr = size_t(n + 1) * 4;
    const size_t bytes = b_codes + b_vals + b_rowptr + z * 4;
    const cudaError_t ce = cudaMallocFromPoolAsync(&j->mem, bytes, s->pool, e->stream);
    if (ce == cudaSuccess) {
      uint8_t* m = static_cast<uint8_t*>(j->mem);
      j->codes = reinterpret_cast<uint64_t*>(m);
      j->vals = reinterpret_cast<double*>(m + b_codes);
      j->rowptr = reinterpret_cast<uint32_t*>(m + b_codes + b_vals);
      j->cols = reinterpret_cast<uint32_t*>(m + b_codes + b_vals + b_rowptr);
    } else {
      cudaGetLastError();
      failed[q] = "out of device memory for the job's result";
      continue;
    }
    const uint32_t work = std::max<uint32_t>(n + 1, uint32_t(std::min<uint64_t>(z, 0xFFFFFFFFu)));
    extract_kernel<<<std::min<uint32_t>(1024, (work + 255) / 256), 256, 0, e->stream>>>(
        e->rowptr.p, e->cols_all.p, e->vals_all.p, e->arena.p, h_foff[q], n, j->rowptr, j->cols, j->vals, j->codes);
    count_launches(1);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(e->stream));
  const double t = now_s();
  e->finish_seconds = e->finish_seconds + (t - t_begin);
  e->jobs_done += nf;
  std::lock_guard<std::mutex> lock(s->mu);
  for (uint32_t q = 0; q < nf; ++q) {
    Job* j = e->slots[fin[q]];
    if (!failed[q].empty()) {
      fail_job_locked(s, j, failed[q]);
      continue;
    }
    j->state = B12G_JOB_DONE;
    j->t_done = t;
    s->done_queue.push_back(j->id);
  }
  s->cv.notify_all();
  return B12G_OK;
}

// one subdivision step of every job of the engine, with `joining` added as new slots
b12g_status engine_tick(Engine* e, const std::vector<Job*>& joining)
{
  Server* s = e->srv;
  const uint32_t A0 = uint32_t(e->slots.size());
  const uint32_t J = uint32_t(joining.size());
  const uint32_t A = A0 + J;
  if (A == 0) return B12G_OK;
  const double t_begin = now_s();
  const uint64_t parents = e->boxes + J;
  ST(engine_reserve(e, parents));
  if (J) {
    append_roots_kernel<<<1, 256, 0, e->stream>>>(e->off.p, A0, J, e->parents.p, e->flags_a.p);
    count_launches(1);
    const double t = now_s();
    for (Job* j : joining) {
      j->t_start = t;
      e->slots.push_back(j);
    }
  }
  // per-slot parameters, children depths and finishing marks
  std::vector<uint32_t> fin;
  for (uint32_t i = 0; i < A; ++i) {
    const Job* j = e->slots[i];
    for (int k = 0; k < 6; ++k) e->hp[size_t(i) * 6 + k] = j->spec.map.p[k];
    e->hd[i] = uint8_t(j->depth_done + 1);
    const bool finishing = j->depth_done + 1 == j->spec.depth;
    e->hd[kMaxSlots + i] = finishing ? 1 : 0;
    e->h[kHostRank + i] = finishing ? uint32_t(fin.size()) : 0u;
    if (finishing) fin.push_back(i);
  }
  CK(cudaMemcpyAsync(e->params.p, e->hp, size_t(A) * 6 * 8, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(e->depth_child.p, e->hd, A, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(e->depth_child.p + kMaxSlots, e->hd + kMaxSlots, A, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(e->fin_rank.p, e->h + kHostRank, size_t(A) * 4, cudaMemcpyHostToDevice, e->stream));
  // the finishing jobs keep every image target of this step and the compaction's ranks,
  // from which their transition matrices follow without evaluating the map again.
  // Slot i's children start at twice the parents of the slots before it.
  const uint32_t nf = uint32_t(fin.size());
  bool store = nf > 0;
  uint64_t fin_children = 0;
  if (store) {
    uint32_t* child_off = e->h + kHostFinStage;
    uint32_t* child_base = child_off + (nf + 1);
    uint64_t before = 0;
    uint32_t q = 0;
    for (uint32_t i = 0; i < A; ++i) {
      const Job* j = e->slots[i];
      const uint64_t p = j->counts.empty() ? 1u : j->counts.back();
      if (e->hd[kMaxSlots + i]) {
        child_off[q] = uint32_t(fin_children);
        child_base[q] = uint32_t(2 * before);
        e->ht[i] = fin_children * e->P;
        fin_children += 2 * p;
        ++q;
      } else {
        e->ht[i] = ~0ull;
      }
      before += p;
    }
    child_off[nf] = uint32_t(fin_children);
    // the host's view of the layout must be the device's; else recompute the rows
    store = before == parents && fin_children < 0x7FFFFFFFull &&
            e->targets.ensure(grow(e->targets.n, std::max<uint64_t>(fin_children * e->P, 1)), "targets") ==
                B12G_OK &&
            e->rank.ensure(grow(e->rank.n, 2 * parents + 1), "ranks") == B12G_OK;
    if (store) {
      CK(cudaMemcpyAsync(e->tgt_base.p, e->ht, size_t(A) * 8, cudaMemcpyHostToDevice, e->stream));
      CK(cudaMemcpyAsync(e->fin_child.p, child_off, size_t(2 * nf + 1) * 4, cudaMemcpyHostToDevice, e->stream));
    }
  }
  e->h[kHostFinChildren] = uint32_t(fin_children);
  const uint32_t capu = uint32_t(std::min<size_t>(e->parents.n, 0xFFFFFFFFu));
  // 1. lookup table over (slot, parent code)
  uint32_t tag = 0;
  ST(engine_next_tag(e, &tag));
  const LeafHash h{e->hash.p, tag, e->hash_log2};
  CK(launch_batch_hash(e->parents.p, e->off.p, A, h, capu, e->ctr.p + E_ERROR, e->stream));
  // 2. images of every grid point of every child of every job
  CK(cudaMemsetAsync(e->ctr.p + E_QUEUE, 0, 4, e->stream));
  BatchArgs a{};
  a.dom = e->dom;
  a.map = e->mp;
  a.grid = e->gp;
  a.points = e->P;
  a.params = e->params.p;
  a.n_inst = A;
  a.off = e->off.p;
  a.codes = e->parents.p;
  a.inst_depth = e->depth_child.p;
  a.hash = h;
  a.hit = e->hit.p;
  a.hit_cap = uint32_t(std::min<size_t>(e->hit.n, 0xFFFFFFFFu));
  a.queue = e->ctr.p + E_QUEUE;
  a.chunk = e->tuning.chunk;
  a.error = e->ctr.p + E_ERROR;
  a.targets = store ? e->targets.p : nullptr;
  a.tgt_base = store ? e->tgt_base.p : nullptr;
  CK(launch_batch_image(e->key.map.kind, e->key.map.arith, e->key.grid.kind, e->tuning, a, e->stream));
  // 3. survivors per job, then one ordered compaction of all children
  CK(launch_inst_count(e->hit.p, e->off.p, A, e->cnt.p, e->hit.n, e->ctr.p + E_ERROR, e->stream));
  CompactArgs ca{};
  ca.code = e->parents.p;
  ca.flags = e->flags_a.p;
  ca.n = e->off.p + A;
  ca.hit = e->hit.p;
  ca.children = 1;
  ca.hit_cap = a.hit_cap;
  ca.out_code = e->children.p;
  ca.out_flags = e->flags_b.p;
  ca.n_out = e->ctr.p + E_TOTAL;
  ca.out_cap = uint32_t(std::min<size_t>(e->children.n, 0xFFFFFFFFu));
  ca.error = e->ctr.p + E_ERROR;
  ca.out_rank = store ? e->rank.p : nullptr;
  CK(compact(ca, {e->tiles_a.p, e->tiles_b.p}, uint32_t(parents), e->stream));
  // 4. continuing jobs packed back into the parents, finished ones into the arena
  split_offsets_kernel<<<1, kSplitThreads, 0, e->stream>>>(e->cnt.p, e->depth_child.p + kMaxSlots, A, e->new_off.p,
                                                           e->keep_off.p, e->fin_off.p, e->off.p, e->ctr.p);
  split_copy_kernel<<<device_sm_count() * 2, 256, 0, e->stream>>>(
      e->children.p, e->flags_b.p, e->new_off.p, A, e->depth_child.p + kMaxSlots, e->keep_off.p, e->fin_off.p,
      e->fin_rank.p, e->parents.p, e->flags_a.p, e->arena.p, capu,
      uint32_t(std::min<size_t>(e->arena.n, 0xFFFFFFFFu)), e->ctr.p + E_ERROR);
  count_launches(5 + compact_launches(true, uint32_t(parents)));   // hash, image, counts, compaction, split
  CK(cudaGetLastError());
  // this step's counts and the counters
  CK(cudaMemcpyAsync(e->h + kHostCounts, e->cnt.p, size_t(A) * 4, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaMemcpyAsync(e->h + kHostCtr, e->ctr.p, E_COUNT * 4, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  const uint32_t* hctr = e->h + kHostCtr;
  if (hctr[E_ERROR]) return fail(B12G_ERR_CAPACITY, "engine tick: capacity exceeded");
  const uint32_t keep_total = hctr[E_KEEP], fin_total = hctr[E_FIN];
  uint64_t images = 0;
  std::vector<Job*> rest;
  for (uint32_t i = 0; i < A; ++i) {
    Job* j = e->slots[i];
    images += 2ull * (j->counts.empty() ? 1u : j->counts.back());
    j->counts.push_back(e->h[kHostCounts + i]);
    j->depth_done += 1;
    if (!e->hd[kMaxSlots + i]) rest.push_back(j);
  }
  s->box_images += images;
  ST(engine_finish(e, fin, fin_total, store));
  e->slots.swap(rest);
  e->boxes = keep_total;
  s->ticks += 1;
  e->ticks += 1;
  e->tick_seconds = e->tick_seconds + (now_s() - t_begin);
  return B12G_OK;
}

void engine_loop(Engine* e)
{
  Server* s = e->srv;
  cudaSetDevice(s->device);
  for (;;) {
    std::vector<Job*> joining;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      s->cv.wait(lock, [&] { return s->stop || !e->slots.empty() || !e->waiting.empty(); });
      if (s->stop) break;
      // admission in submission order while the projected footprint fits the cap (a
      // job is always admitted into an otherwise idle server)
      while (!e->waiting.empty() && e->slots.size() + joining.size() < kMaxSlots) {
        Job* j = e->waiting.front();
        const uint64_t need = projected_bytes(j->spec);
        const bool idle = e->slots.empty() && joining.empty() && s->in_use == 0;
        if (s->in_use + need > s->cap_bytes && !idle) break;
        s->in_use += need;
        j->reserved = need;
        j->state = B12G_JOB_RUNNING;
        joining.push_back(j);
        e->waiting.pop_front();
      }
      if (e->slots.empty() && joining.empty()) {
        // nothing admissible until memory is released
        s->cv.wait_for(lock, std::chrono::milliseconds(2));
        continue;
      }
    }
    if (engine_tick(e, joining) != B12G_OK) {
      const std::string why = b12g_last_error();
      {
        std::lock_guard<std::mutex> lock(s->mu);
        for (Job* j : e->slots) fail_job_locked(s, j, why);
        s->cv.notify_all();
      }
      e->slots.clear();
      e->boxes = 0;
      cudaGetLastError();
      cudaMemsetAsync(e->off.p, 0, (kMaxSlots + 1) * 4, e->stream);
      cudaMemsetAsync(e->ctr.p, 0, E_COUNT * 4, e->stream);
      if (e->hit.p) cudaMemsetAsync(e->hit.p, 0, e->hit.n, e->stream);
      cudaStreamSynchronize(e->stream);
    }
  }
}

void free_job_memory(Server* s, Job* j)
{
  if (j->mem) cudaFreeAsync(j->mem, s->release_stream);
  j->mem = nullptr;
  j->codes = nullptr;
  j->rowptr = nullptr;
  j->cols = nullptr;
  j->vals = nullptr;
}

void engine_release(Engine* e)
{
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->table) cudaFree(e->table);
  if (e->h) cudaFreeHost(e->h);
  if (e->hp) cudaFreeHost(e->hp);
  if (e->hd) cudaFreeHost(e->hd);
  if (e->ht) cudaFreeHost(e->ht);
  e->targets.release(); e->rank.release(); e->fin_child.release(); e->tgt_base.release();
  e->parents.release(); e->children.release(); e->flags_a.release(); e->flags_b.release(); e->hit.release();
  e->off.release(); e->new_off.release(); e->cnt.release(); e->ctr.release(); e->tiles_a.release();
  e->tiles_b.release(); e->keep_off.release(); e->fin_off.release(); e->fin_slot.release(); e->fin_rank.release();
  e->row0.release(); e->params.release(); e->fin_params.release(); e->depth_child.release();
  e->fin_depth.release(); e->hash.release(); e->arena.release(); e->stage_col.release(); e->stage_cnt.release();
  e->row_count.release(); e->rowptr.release(); e->cols_all.release(); e->vals_all.release();
  if (e->stream) cudaStreamDestroy(e->stream);
  e->stream = nullptr;
}

}  // namespace

struct b12g_server {
  Server s;
};

extern "C" {

b12g_status b12g_server_create(uint64_t hbm_cap_bytes, b12g_server** out)
{
  if (!out) return fail(B12G_ERR_INVALID, "NULL argument");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(B12G_ERR_NO_DEVICE, "no CUDA device");
  }
  b12g_server* sv = new b12g_server();
  cudaGetDevice(&sv->s.device);
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  sv->s.cap_bytes = hbm_cap_bytes ? hbm_cap_bytes : uint64_t(double(free_b) * 0.8);
  // results come from a pool of the server's own that keeps freed memory for reuse
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = sv->s.device;
  cudaError_t ce = cudaMemPoolCreate(&sv->s.pool, &props);
  uint64_t keep = ~0ull;
  if (ce == cudaSuccess) ce = cudaMemPoolSetAttribute(sv->s.pool, cudaMemPoolAttrReleaseThreshold, &keep);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&sv->s.release_stream, cudaStreamNonBlocking);
  if (ce != cudaSuccess) {
    b12g_server_destroy(sv);
    return cuda_fail(ce, "server memory pool");
  }
  *out = sv;
  return B12G_OK;
}

b12g_status b12g_server_submit(b12g_server* sv, const b12g_job* job, uint64_t* id)
{
  if (!sv || !job || !id) return fail(B12G_ERR_INVALID, "NULL argument");
  if (job->depth < 1 || job->depth > 32) return fail(B12G_ERR_INVALID, "job depth must be 1..32");
  if (job->domain.dim < 1 || job->domain.dim > B12G_MAX_DIM) return fail(B12G_ERR_INVALID, "bad domain dimension");
  if (!batch_supported(job->map.kind, job->map.arith, job->grid.kind) ||
      !image_supported(job->map.kind, job->map.arith, job->grid.kind, job->domain.dim))
    return fail(B12G_ERR_INVALID, "map/arithmetic/grid not served (inner and full grids of Henon, Lorenz and "
                                  "forced Duffing)");
  Server& s = sv->s;
  Engine* e = nullptr;
  {
    std::lock_guard<std::mutex> lock(s.mu);
    for (auto& x : s.engines)
      if (same_family(x->key, *job)) e = x.get();
  }
  if (!e) {
    auto ne = std::make_unique<Engine>();
    ne->srv = &s;
    const b12g_status st = engine_init(ne.get(), *job);
    if (st != B12G_OK) {
      engine_release(ne.get());
      return st;
    }
    e = ne.get();
    std::lock_guard<std::mutex> lock(s.mu);
    s.engines.push_back(std::move(ne));
    e->thread = std::thread(engine_loop, e);
  }
  auto j = std::make_unique<Job>();
  j->spec = *job;
  j->t_submit = now_s();
  std::lock_guard<std::mutex> lock(s.mu);
  j->id = s.next_id++;
  *id = j->id;
  e->waiting.push_back(j.get());
  s.jobs[j->id] = std::move(j);
  s.cv.notify_all();
  return B12G_OK;
}

b12g_status b12g_server_poll(b12g_server* sv, uint64_t* ids, uint32_t max, uint32_t* n, double wait_seconds)
{
  if (!sv || !n) return fail(B12G_ERR_INVALID, "NULL argument");
  Server& s = sv->s;
  std::unique_lock<std::mutex> lock(s.mu);
  if (s.done_queue.empty() && wait_seconds > 0)
    s.cv.wait_for(lock, std::chrono::duration<double>(wait_seconds), [&] { return !s.done_queue.empty(); });
  uint32_t k = 0;
  while (k < max && !s.done_queue.empty()) {
    if (ids) ids[k] = s.done_queue.front();
    s.done_queue.pop_front();
    ++k;
  }
  *n = k;
  return B12G_OK;
}

b12g_status b12g_server_job(b12g_server* sv, uint64_t id, b12g_job_info* info)
{
  if (!sv || !info) return fail(B12G_ERR_INVALID, "NULL argument");
  Server& s = sv->s;
  std::lock_guard<std::mutex> lock(s.mu);
  auto it = s.jobs.find(id);
  if (it == s.jobs.end()) return fail(B12G_ERR_INVALID, "unknown job %llu", (unsigned long long)id);
  const Job* j = it->second.get();
  info->state = uint32_t(j->state);
  info->depth = j->spec.depth;
  info->n_boxes = j->state == B12G_JOB_DONE ? std::max<uint32_t>(j->n_boxes, 1) : 0;
  info->pad = 0;
  info->nnz = j->state == B12G_JOB_DONE ? j->nnz : 0;
  info->t_submit = j->t_submit;
  info->t_start = j->t_start;
  info->t_done = j->t_done;
  return B12G_OK;
}

b12g_status b12g_server_result(b12g_server* sv, uint64_t id, uint64_t* codes, uint32_t* counts, uint32_t* rowptr,
                               uint32_t* cols, double* vals)
{
  if (!sv) return fail(B12G_ERR_INVALID, "NULL server");
  Server& s = sv->s;
  Job* j = nullptr;
  {
    std::lock_guard<std::mutex> lock(s.mu);
    auto it = s.jobs.find(id);
    if (it == s.jobs.end()) return fail(B12G_ERR_INVALID, "unknown job %llu", (unsigned long long)id);
    j = it->second.get();
    if (j->state == B12G_JOB_FAILED) return fail(B12G_ERR_CUDA, "job failed: %s", j->error.c_str());
    if (j->state != B12G_JOB_DONE) return fail(B12G_ERR_INVALID, "job not finished");
  }
  if (counts) {
    // a step that removed every box leaves the surrounding box (insertSurroundingBoxIfEmpty)
    bool empty = false;
    for (size_t k = 0; k < j->counts.size(); ++k) {
      if (j->counts[k] == 0) empty = true;
      counts[k] = empty ? 1u : j->counts[k];
    }
  }
  if (j->n_boxes == 0) {
    if (codes) codes[0] = 0;
    if (rowptr) rowptr[0] = rowptr[1] = 0;
    return B12G_OK;
  }
  if (codes) CK(cudaMemcpy(codes, j->codes, size_t(j->n_boxes) * 8, cudaMemcpyDeviceToHost));
  if (rowptr) CK(cudaMemcpy(rowptr, j->rowptr, size_t(j->n_boxes + 1) * 4, cudaMemcpyDeviceToHost));
  if (cols && j->nnz) CK(cudaMemcpy(cols, j->cols, j->nnz * 4, cudaMemcpyDeviceToHost));
  if (vals && j->nnz) CK(cudaMemcpy(vals, j->vals, j->nnz * 8, cudaMemcpyDeviceToHost));
  return B12G_OK;
}

b12g_status b12g_server_release(b12g_server* sv, uint64_t id)
{
  if (!sv) return fail(B12G_ERR_INVALID, "NULL server");
  Server& s = sv->s;
  std::unique_ptr<Job> j;
  {
    std::lock_guard<std::mutex> lock(s.mu);
    auto it = s.jobs.find(id);
    if (it == s.jobs.end()) return fail(B12G_ERR_INVALID, "unknown job %llu", (unsigned long long)id);
    if (it->second->state < B12G_JOB_DONE) return fail(B12G_ERR_INVALID, "job still waiting or running");
    j = std::move(it->second);
    s.jobs.erase(it);
    s.in_use -= std::min(s.in_use, j->reserved);
    s.cv.notify_all();
  }
  free_job_memory(&s, j.get());
  return B12G_OK;
}

b12g_status b12g_server_stats(b12g_server* sv, uint64_t* ticks, uint64_t* box_images, uint64_t* in_use_bytes,
                              uint64_t* cap_bytes, uint32_t* waiting, uint32_t* running)
{
  if (!sv) return fail(B12G_ERR_INVALID, "NULL server");
  Server& s = sv->s;
  std::lock_guard<std::mutex> lock(s.mu);
  if (ticks) *ticks = s.ticks;
  if (box_images) *box_images = s.box_images;
  if (in_use_bytes) *in_use_bytes = s.in_use;
  if (cap_bytes) *cap_bytes = s.cap_bytes;
  uint32_t w = 0, r = 0;
  for (auto& kv : s.jobs) {
    w += kv.second->state == B12G_JOB_WAITING ? 1u : 0u;
    r += kv.second->state == B12G_JOB_RUNNING ? 1u : 0u;
  }
  if (waiting) *waiting = w;
  if (running) *running = r;
  return B12G_OK;
}

b12g_status b12g_server_engine_stats(b12g_server* sv, uint32_t i, uint32_t* map_kind, uint64_t* ticks,
                                     uint64_t* jobs_done, double* tick_seconds, double* finish_seconds)
{
  if (!sv) return fail(B12G_ERR_INVALID, "NULL server");
  Server& s = sv->s;
  std::lock_guard<std::mutex> lock(s.mu);
  if (i >= s.engines.size()) return fail(B12G_ERR_INVALID, "engine %u of %zu", i, s.engines.size());
  const Engine* e = s.engines[i].get();
  if (map_kind) *map_kind = e->key.map.kind;
  if (ticks) *ticks = e->ticks;
  if (jobs_done) *jobs_done = e->jobs_done;
  if (tick_seconds) *tick_seconds = e->tick_seconds;
  if (finish_seconds) *finish_seconds = e->finish_seconds;
  return B12G_OK;
}

b12g_status b12g_server_destroy(b12g_server* sv)
{
  if (!sv) return B12G_OK;
  Server& s = sv->s;
  {
    std::lock_guard<std::mutex> lock(s.mu);
    s.stop = true;
    s.cv.notify_all();
  }
  for (auto& e : s.engines)
    if (e->thread.joinable()) e->thread.join();
  for (auto& e : s.engines) engine_release(e.get());
  for (auto& kv : s.jobs) free_job_memory(&s, kv.second.get());
  if (s.release_stream) {
    cudaStreamSynchronize(s.release_stream);
    cudaStreamDestroy(s.release_stream);
  }
  if (s.pool) cudaMemPoolDestroy(s.pool);
  delete sv;
  return B12G_OK;
}

}  // extern "C"
