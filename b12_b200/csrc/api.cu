// Host side of libb12g: the tree object that owns device memory and a stream, and
// the C ABI declared in include/b12g.h.  Each entry point restates the reference
// member function named in the header on top of the device kernels.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "csr.h"
#include "kernels.h"
#include "tree.h"

using namespace b12g;
using namespace b12g::host;

namespace {

thread_local std::string g_last_error;

uint64_t ipow(uint64_t b, uint32_t e)
{
  uint64_t r = 1;
  while (e--) r *= b;
  return r;
}


}  // namespace

namespace b12g {
namespace host {

b12g_status fail(b12g_status s, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

b12g_status cuda_fail(cudaError_t e, const char* where)
{
  return fail(e == cudaErrorMemoryAllocation ? B12G_ERR_OOM : B12G_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

b12g_status sync(b12g_tree* t, const char* where)
{
  cudaError_t e = cudaStreamSynchronize(t->stream);
  if (e != cudaSuccess) return cuda_fail(e, where);
  return B12G_OK;
}

b12g_status read_ctr(b12g_tree* t, int first, int count)
{
  CK(cudaMemcpyAsync(t->h_ctr + first, t->ctr.p + first, count * sizeof(uint32_t), cudaMemcpyDeviceToHost, t->stream));
  return sync(t, "read counters");
}

// A counter is set without staging the value in host memory: zero by a memset, any
// other value by a one-thread kernel that takes it as a launch parameter.  A copy from
// the pinned counter block would read that slot whenever the stream reaches it, so a
// later host write of the slot (before a synchronisation) could change the value copied.
__global__ void set_word_kernel(uint32_t* p, uint32_t v) { *p = v; }

b12g_status set_ctr(b12g_tree* t, int slot, uint32_t v)
{
  t->h_ctr[slot] = v;
  if (v == 0) {
    CK(cudaMemsetAsync(t->ctr.p + slot, 0, sizeof(uint32_t), t->stream));
  } else {
    set_word_kernel<<<1, 1, 0, t->stream>>>(t->ctr.p + slot, v);
    CK(cudaGetLastError());
    count_launches(1);
  }
  return B12G_OK;
}

b12g_status reserve_exact(b12g_tree* t, uint64_t n_boxes);

// Room for n_boxes leaves.  A tree that has to grow gets room for twice as many (or, if
// that much memory is not free, the exact need): trees grow step by step, and every
// reallocation frees the old buffers (cudaFree synchronises the device).
b12g_status reserve(b12g_tree* t, uint64_t n_boxes)
{
  if (n_boxes > 0xFFFFFFF0ull) return fail(B12G_ERR_CAPACITY, "at most 2^32-16 boxes per tree");
  if (n_boxes <= t->code[0].n && n_boxes <= t->code[1].n && n_boxes <= t->hit.n) return reserve_exact(t, n_boxes);
  const uint64_t ample = std::min<uint64_t>(2 * n_boxes, 0xFFFFFFF0ull);
  if (reserve_exact(t, ample) == B12G_OK) return B12G_OK;
  return reserve_exact(t, n_boxes);
}

b12g_status reserve_exact(b12g_tree* t, uint64_t n_boxes)
{
  const size_t keep = t->n;
  for (int b = 0; b < 2; ++b) {
    ST(t->code[b].grow_keep(n_boxes, b == t->cur ? keep : 0, t->stream, "leaf codes"));
    ST(t->flags[b].grow_keep(n_boxes, b == t->cur ? keep : 0, t->stream, "leaf flags"));
    if (t->mixed) ST(t->dep[b].grow_keep(n_boxes, b == t->cur ? keep : 0, t->stream, "leaf depths"));
  }
  if (t->hit.n < n_boxes) {
    ST(t->hit.ensure(n_boxes, "hit mask"));
    CK(cudaMemsetAsync(t->hit.p, 0, t->hit.n, t->stream));
  }
  // tiles cover the largest array a compaction or scan can run over
  const size_t most = std::max({size_t(n_boxes), t->hit.n, t->code[0].n, t->code[1].n}) + 1;
  ST(t->tiles_a.ensure(compact_tiles(most) + 2, "tile counts"));
  ST(t->tiles_b.ensure(compact_tiles(most) + 2, "tile offsets"));
  return B12G_OK;
}

// two schemes map and sample alike: field by field (the padding is not compared), the
// doubles by their bits
bool same_bits(double a, double b) { return std::memcmp(&a, &b, sizeof(double)) == 0; }

bool same_scheme(const b12g_scheme& a, const b12g_scheme& b)
{
  if (a.map.kind != b.map.kind || a.map.arith != b.map.arith || a.map.steps != b.map.steps ||
      !same_bits(a.map.h, b.map.h))
    return false;
  for (int i = 0; i < 6; ++i)
    if (!same_bits(a.map.p[i], b.map.p[i])) return false;
  return a.grid.kind == b.grid.kind && a.grid.n == b.grid.n && a.grid.points == b.grid.points &&
         a.grid.seed == b.grid.seed && same_bits(a.grid.eps, b.grid.eps) && a.depth == b.depth &&
         a.flags_to_check == b.flags_to_check;
}

// the stored targets of the last subdivision step describe the current leaves under
// this scheme: no change of the leaf set since they were stored (generation), and the
// same scheme field by field
bool stored_rows_fit(b12g_tree* t, const b12g_scheme* sc, const Prepared& pr)
{
  if (!t->tgt_ok || t->mixed || t->leaf_gen != t->tgt_gen || t->n != t->tgt_n || t->depth != t->tgt_depth ||
      pr.P != t->tgt_points)
    return false;
  return same_scheme(*sc, t->tgt_scheme);
}

b12g_status prepare(b12g_tree* t, const b12g_scheme* sc, Prepared& pr)
{
  if (!sc) return fail(B12G_ERR_INVALID, "scheme is NULL");
  const b12g_map& m = sc->map;
  const b12g_grid& g = sc->grid;
  const uint32_t D = t->domain.dim;
  if (!image_supported(m.kind, m.arith, g.kind, D))
    return fail(B12G_ERR_INVALID, "unsupported map/arith/grid/dimension combination (%u,%u,%u,%u)", m.kind, m.arith,
                g.kind, D);
  ImageArgs& a = pr.a;
  a.dom = t->dom;
  MapParams& mp = a.map;
  mp.h = m.h;
  mp.h2 = m.h / 2.0;
  mp.h3 = m.h / 3.0;
  mp.h6 = m.h / 6.0;
  for (int i = 0; i < 6; ++i) mp.p[i] = m.p[i];
  mp.steps = m.steps;
  mp.table = nullptr;
  if (m.kind == B12G_MAP_FORCED_DUFFING) {
    // cos at the stage times t = j * h / 2 (period = steps * h)
    std::vector<double> tab(2 * size_t(m.steps) + 1);
    const double period = m.h * double(m.steps);
    for (size_t j = 0; j < tab.size(); ++j) tab[j] = std::cos(double(j) * (period / double(2 * m.steps)));
    ST(t->table.ensure(tab.size(), "forcing table"));
    CK(cudaMemcpyAsync(t->table.p, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, t->stream));
    CK(cudaStreamSynchronize(t->stream));
    mp.table = t->table.p;
  }
  GridParams& gp = a.grid;
  if (g.kind == B12G_GRID_INNER || g.kind == B12G_GRID_FULL) {
    if (g.n < 1 || g.n > 64) return fail(B12G_ERR_INVALID, "grid points per dimension must be 1..64");
    if (g.kind == B12G_GRID_FULL && g.n < 2) return fail(B12G_ERR_INVALID, "full grid needs n >= 2");
    gp.n = g.n;
    pr.P = ipow(g.n, D);
    const double nn = double(g.n);
    for (uint32_t d = 0; d < 64; ++d) {
      if (g.kind == B12G_GRID_INNER) gp.coord[d] = ((double(d) * 2.0 + 1.0) - nn) / nn;   // Grids.hpp:113-116
      else gp.coord[d] = (double(d) * 2.0) / double(uint64_t(g.n) - 1) - 1.0;           // Grids.hpp:75-78
    }
    gp.eps1 = 1.0 + g.eps;
  } else {
    if (g.points < 1) return fail(B12G_ERR_INVALID, "philox grid needs points >= 1");
    gp.n = 1;
    pr.P = g.points;
    for (double& c : gp.coord) c = 0.0;
  }
  gp.points = pr.P;
  gp.seed = g.seed;
  a.points = pr.P;
  a.codes = t->codes();
  a.n_leaves = t->dn();
  a.depth = t->depth;
  a.children = 0;
  a.src = nullptr;
  a.n_src = nullptr;
  a.hit = t->hit.p;
  a.hit_cap = uint32_t(std::min<size_t>(t->hit.n, 0xFFFFFFFFu));
  a.error = t->ctr.p + C_ERROR;
  a.cand_count = t->ctr.p + C_CAND;
  a.work = reinterpret_cast<unsigned long long*>(t->ctr.p + C_WORK);
  return B12G_OK;
}

b12g_status check_depth(b12g_tree* t, uint8_t depth)
{
  if (depth == B12G_LEAF_DEPTH || depth == t->depth) return B12G_OK;
  return fail(B12G_ERR_UNSUPPORTED_MIXED_DEPTH, "depth %u is neither the leaf depth (%u) nor 255", depth, t->depth);
}

// source boxes of a scheme: all leaves, or the leaves with all flags_to_check set
b12g_status select_sources(b12g_tree* t, const b12g_scheme* sc, Prepared& pr, uint32_t& n_src)
{
  if (sc->depth != B12G_LEAF_DEPTH && sc->depth != t->depth)
    return fail(B12G_ERR_UNSUPPORTED_MIXED_DEPTH, "scheme depth %u is not the leaf depth %u", sc->depth, t->depth);
  if (sc->flags_to_check == 0) {
    n_src = t->n;
    return B12G_OK;
  }
  ST(t->src.ensure(std::max<uint32_t>(t->n, 1), "source list"));
  CompactArgs ca{};
  ca.code = t->codes();
  ca.flags = t->flg();
  ca.n = t->dn();
  ca.keep_flags = sc->flags_to_check;
  ca.out_index = t->src.p;
  ca.n_out = t->ctr.p + C_NSRC;
  ca.out_cap = uint32_t(t->src.n);
  ca.error = t->ctr.p + C_ERROR;
  CK(compact(ca, {t->tiles_a.p, t->tiles_b.p}, t->n, t->stream));
  count_launches(compact_launches(false, t->n));
  ST(read_ctr(t, C_NSRC, 1));
  n_src = t->h_ctr[C_NSRC];
  pr.a.src = t->src.p;
  pr.a.n_src = t->ctr.p + C_NSRC;
  return B12G_OK;
}

b12g_status check_error(b12g_tree* t, const char* where)
{
  ST(read_ctr(t, C_ERROR, 1));
  if (t->h_ctr[C_ERROR]) {
    const uint32_t e = t->h_ctr[C_ERROR];
    set_ctr(t, C_ERROR, 0);
    if (e & 2u) return fail(B12G_ERR_TIMEOUT, "%s: a bounded device wait gave up", where);
    return fail(B12G_ERR_CAPACITY, "%s: device buffer capacity exceeded", where);
  }
  return B12G_OK;
}

// make the tree the single surrounding box (insertSurroundingBoxIfEmpty)
b12g_status set_root(b12g_tree* t, uint8_t flags)
{
  const uint64_t zero = 0;
  CK(cudaMemcpyAsync(t->codes(), &zero, 8, cudaMemcpyHostToDevice, t->stream));
  CK(cudaMemsetAsync(t->flg(), flags, 1, t->stream));
  t->n = 1;
  ++t->leaf_gen;
  t->depth = 0;
  t->mixed = false;
  ST(set_ctr(t, t->ncur, 1));
  return sync(t, "set root");
}

b12g_status flag_call(b12g_tree* t, int op, uint8_t u, uint8_t f, uint8_t depth, uint32_t* n_changed)
{
  if (!t) return fail(B12G_ERR_INVALID, "NULL tree");
  if (depth != 0 && depth != B12G_LEAF_DEPTH && (t->mixed || depth != t->depth)) {
    // the boxes at a depth that is not every leaf's own: all leaves of each box change
    if (depth == 254) return fail(B12G_ERR_UNSUPPORTED_MIXED_DEPTH, "flags at the unsubdividable depth 254");
    if (depth > 64) return fail(B12G_ERR_INVALID, "depth %u above the maximal depth 64", depth);
    return mixed_flags_at_depth(t, op, u, f, depth, n_changed);
  }
  ST(set_ctr(t, C_CHANGED, 0));
  CK(flag_op(t->flg(), t->dn(), op, u, f, t->ctr.p + C_CHANGED, t->n, t->stream));
  count_launches(1);
  if (!n_changed) return B12G_OK;   // nobody reads the count: no round trip (the stream keeps the order)
  ST(read_ctr(t, C_CHANGED, 1));
  uint32_t c = t->h_ctr[C_CHANGED];
  if (depth == 0 && t->depth != 0) {
    // depth 0 is the surrounding box, whose flags combine its leaves' flags
    // (countIfFlags depth-0 branch, ImplicitBoxTree.hpp:1119-1127): one box, changed
    // if the combination matched before the update.  The combination is recomputed
    // from the per-leaf counts: AND-combination for set/change, OR for unset.
    if (op == 0) c = c > 0 ? 1u : 0u;            // not all leaves had f  <=> AND lacks f
    else if (op == 1) c = c > 0 ? 1u : 0u;       // some leaf had any of f <=> OR has one
    else c = (c == t->n) ? 1u : 0u;              // all leaves had u      <=> AND has u
  }
  if (n_changed) *n_changed = c;
  return B12G_OK;
}

uint32_t host_hash_log2(uint64_t n)
{
  uint32_t l = 6;
  while ((1ull << l) < 2ull * n) ++l;
  return l;
}

b12g_status ensure_hash(b12g_tree* t, uint64_t max_n)
{
  const uint32_t l = host_hash_log2(std::max<uint64_t>(max_n, 1));
  ST(t->pk.ensure(std::max<uint64_t>(max_n, 1), "packed leaf keys"));
  if (t->hash.p && l <= t->hash_log2) return B12G_OK;
  t->hash.release();
  ST(t->hash.ensure(size_t(1) << l, "leaf lookup table"));
  CK(cudaMemsetAsync(t->hash.p, 0, t->hash.n * sizeof(ulonglong2), t->stream));
  t->hash_log2 = l;
  t->hash_tag = 0;
  return B12G_OK;
}

b12g_status next_hash_tag(b12g_tree* t, uint32_t* tag)
{
  if (t->hash_tag >= 255) {
    CK(cudaMemsetAsync(t->hash.p, 0, t->hash.n * sizeof(ulonglong2), t->stream));
    t->hash_tag = 0;
  }
  *tag = ++t->hash_tag;
  return B12G_OK;
}

b12g_status build_current_hash(b12g_tree* t, Prepared& pr)
{
  pr.a.hash = LeafHash{nullptr, 0, 0, nullptr};
  if (t->depth > kHashMaxDepth || t->n == 0 || t->domain.dim < 2) return B12G_OK;
  ST(ensure_hash(t, t->n));
  uint32_t tag = 0;
  ST(next_hash_tag(t, &tag));
  const LeafHash h{t->hash.p, tag, t->hash_log2, t->pk.p};
  CK(build_leaf_hash(t->codes(), t->dn(), int(t->depth), int(t->domain.dim), h, t->ctr.p + C_ERROR, t->n, t->stream));
  count_launches(1);
  pr.a.hash = h;
  return B12G_OK;
}

void prof_mark(b12g_tree* t, int kind)
{
  if (!t->profile) return;
  auto& v = t->prof_events[kind];
  if (t->prof_used[kind] == v.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    v.push_back(e);
  }
  // during capture an external record becomes a real event node of the graph
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(t->stream, &cs);
  cudaEvent_t e = v[t->prof_used[kind]++];
  if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(e, t->stream, cudaEventRecordExternal);
  else cudaEventRecord(e, t->stream);
}

static void sum_pairs(const std::vector<cudaEvent_t>& v, size_t used, double& ms, uint64_t& launches)
{
  for (size_t i = 0; i + 1 < used; i += 2) {
    float x = 0.f;
    if (cudaEventElapsedTime(&x, v[i], v[i + 1]) == cudaSuccess) { ms += x; ++launches; }
  }
  cudaGetLastError();
}

// after a stream sync: fold recorded event pairs into the per-kind totals
b12g_status prof_collect(b12g_tree* t)
{
  if (!t->profile) return B12G_OK;
  for (int k = 0; k < 2; ++k) {
    sum_pairs(t->prof_events[k], t->prof_used[k], t->prof_ms[k], t->prof_launches[k]);
    t->prof_used[k] = 0;
  }
  return B12G_OK;
}

}  // namespace host
}  // namespace b12g

// =====================================================================================
extern "C" {

const char* b12g_last_error(void) { return g_last_error.c_str(); }

const char* b12g_version(void) { return "b12g 0.1 (sm_100a)"; }

b12g_status b12g_tree_create(const b12g_domain* domain, b12g_tree** out)
{
  if (!domain || !out) return fail(B12G_ERR_INVALID, "NULL argument");
  if (domain->dim < 1 || domain->dim > B12G_MAX_DIM) return fail(B12G_ERR_INVALID, "dim must be 1..4");
  for (uint32_t j = 0; j < domain->dim; ++j)
    if (!(domain->radius[j] > 0.0)) return fail(B12G_ERR_INVALID, "radius must be positive");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(B12G_ERR_NO_DEVICE, "no CUDA device");
  }
  b12g_tree* t = new b12g_tree();
  cudaGetDevice(&t->device);
  t->domain = *domain;
  for (uint32_t j = 0; j < B12G_MAX_DIM; ++j) {
    const double c = j < domain->dim ? domain->center[j] : 0.0, r = j < domain->dim ? domain->radius[j] : 1.0;
    t->dom.c[j] = c;
    t->dom.r[j] = r;
    t->dom.lo[j] = c - r;
    t->dom.hi[j] = c + r;
    // the point-code fast path multiplies by RN(1/r) (checked against the IEEE quotient
    // per point); radii far from 1 keep the division alone
    t->dom.inv_r[j] = (r >= 0x1p-500 && r <= 0x1p500) ? 1.0 / r : 0.0;
  }
  b12g_status st = B12G_OK;
  if (cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking) != cudaSuccess) st = cuda_fail(cudaGetLastError(), "stream");
  if (st == B12G_OK && cudaMallocHost(&t->h_ctr, C_COUNT * sizeof(uint32_t)) != cudaSuccess)
    st = cuda_fail(cudaGetLastError(), "pinned counters");
  if (st == B12G_OK) st = t->ctr.ensure(C_COUNT, "counters");
  if (st == B12G_OK && cudaMemsetAsync(t->ctr.p, 0, C_COUNT * sizeof(uint32_t), t->stream) != cudaSuccess)
    st = cuda_fail(cudaGetLastError(), "memset");
  if (st == B12G_OK) st = reserve(t, 1024);
  if (st == B12G_OK) st = set_root(t, B12G_NONE);
  if (st != B12G_OK) {
    b12g_tree_destroy(t);
    return st;
  }
  *out = t;
  return B12G_OK;
}

b12g_status b12g_tree_destroy(b12g_tree* t)
{
  if (!t) return B12G_OK;
  if (t->stream) cudaStreamSynchronize(t->stream);
  if (t->sub_graph) cudaGraphExecDestroy(t->sub_graph);
  for (int k = 0; k < 2; ++k) {
    for (cudaEvent_t e : t->prof_events[k]) cudaEventDestroy(e);
    for (cudaEvent_t e : t->graph_prof[k]) cudaEventDestroy(e);
  }
  for (int b = 0; b < 2; ++b) { t->code[b].release(); t->flags[b].release(); t->dep[b].release(); }
  t->cmp.release(); t->cmp_tab.release(); t->hash.release(); t->points.release();
  t->pvalid.release(); t->ins_dep.release(); t->ins_dep2.release(); t->scan_dep.release(); t->scan_flags.release();
  t->ins_code.release(); t->scan_code.release(); t->ins_pos.release(); t->ins_head.release();
  for (int b = 0; b < 2; ++b) { t->ins_key[b].release(); t->ins_idx[b].release(); }
  t->isrc_head.release(); t->isrc_pos.release(); t->isrc_and.release(); t->isrc.release();
  t->hit.release(); t->ctr.release(); t->tiles_a.release(); t->tiles_b.release();
  t->src.release(); t->out.release(); t->stage_col.release(); t->stage_cnt.release();
  t->row_count.release(); t->rowptr.release(); t->cand.release(); t->cand2.release();
  t->sort_idx.release(); t->table.release(); t->step_counts.release(); t->sort_tmp.release();
  t->last_tgt.release(); t->last_rank.release();
  if (t->h_ctr) cudaFreeHost(t->h_ctr);
  if (t->stream) cudaStreamDestroy(t->stream);
  delete t;
  return B12G_OK;
}

b12g_status b12g_tree_reserve(b12g_tree* t, uint64_t n_boxes)
{
  if (!t) return fail(B12G_ERR_INVALID, "NULL tree");
  ST(reserve(t, n_boxes));
  return sync(t, "reserve");
}

b12g_status b12g_count(b12g_tree* t, uint8_t depth, uint32_t* count)
{
  if (!t || !count) return fail(B12G_ERR_INVALID, "NULL argument");
  if (t->mixed) return mixed_count(t, depth, count);
  // count(depth) (ImplicitBoxTree.hpp:1061-1095) for a uniform-depth tree
  if (depth == 0) *count = 1;
  else if (depth == B12G_LEAF_DEPTH || depth == t->depth) *count = t->n;
  else if (depth > t->depth) *count = 0;
  else return fail(B12G_ERR_UNSUPPORTED_MIXED_DEPTH, "count of inner depth %u", depth);
  return B12G_OK;
}

b12g_status b12g_depth(b12g_tree* t, uint8_t* depth)
{
  if (!t || !depth) return fail(B12G_ERR_INVALID, "NULL argument");
  *depth = t->depth;
  return B12G_OK;
}

b12g_status b12g_leaves(b12g_tree* t, uint64_t* codes, uint8_t* depths, uint8_t* flags)
{
  if (!t) return fail(B12G_ERR_INVALID, "NULL tree");
  if (t->mixed) return mixed_leaves(t, codes, depths, flags);
  // host or device buffers (unified addressing tells the copies which)
  if (codes) CK(cudaMemcpyAsync(codes, t->codes(), size_t(t->n) * 8, cudaMemcpyDefault, t->stream));
  if (flags) CK(cudaMemcpyAsync(flags, t->flg(), t->n, cudaMemcpyDefault, t->stream));
  cudaPointerAttributes pa{};
  bool dev_depths = false;
  if (depths) {
    if (cudaPointerGetAttributes(&pa, depths) == cudaSuccess) dev_depths = pa.type == cudaMemoryTypeDevice;
    else cudaGetLastError();  // a pointer CUDA does not know is host memory
  }
  if (dev_depths) CK(cudaMemsetAsync(depths, t->depth, t->n, t->stream));
  ST(sync(t, "leaves"));
  if (depths && !dev_depths) std::memset(depths, t->depth, t->n);
  return B12G_OK;
}

b12g_status b12g_load_leaves(b12g_tree* t, const uint64_t* codes, const uint8_t* depths, const uint8_t* flags,
                             uint32_t n)
{
  if (!t || !codes || !depths || !flags) return fail(B12G_ERR_INVALID, "NULL argument");
  if (n == 0) return set_root(t, B12G_NONE);
  const uint8_t d = depths[0];
  if (d > 64) return fail(B12G_ERR_INVALID, "depth %u above the maximal depth 64", d);
  for (uint32_t i = 1; i < n; ++i)
    if (depths[i] != d) return mixed_load(t, codes, depths, flags, n);
  for (uint32_t i = 0; i < n; ++i) {
    if (d < 64 && (codes[i] >> d) != 0) return fail(B12G_ERR_INVALID, "code %u has bits above its depth", i);
    if (i && codes[i] <= codes[i - 1]) return fail(B12G_ERR_INVALID, "codes must be sorted and unique");
  }
  ST(reserve(t, n));
  CK(cudaMemcpyAsync(t->codes(), codes, size_t(n) * 8, cudaMemcpyHostToDevice, t->stream));
  CK(cudaMemcpyAsync(t->flg(), flags, n, cudaMemcpyHostToDevice, t->stream));
  t->n = n;
  ++t->leaf_gen;
  t->depth = d;
  t->mixed = false;
  ST(set_ctr(t, t->ncur, n));
  return sync(t, "load leaves");
}

// ---- flags ----
b12g_status b12g_set_flags(b12g_tree* t, uint8_t flags, uint8_t depth, uint32_t* n_changed)
{
  return flag_call(t, 0, 0, flags, depth, n_changed);
}

b12g_status b12g_unset_flags(b12g_tree* t, uint8_t flags, uint8_t depth, uint32_t* n_changed)
{
  return flag_call(t, 1, 0, flags, depth, n_changed);
}

b12g_status b12g_change_flags(b12g_tree* t, uint8_t to_unset, uint8_t to_set, uint8_t depth, uint32_t* n_changed)
{
  return flag_call(t, 2, to_unset, to_set, depth, n_changed);
}

// ---- structure ------------------------------------------------------------------------
b12g_status b12g_subdivide(b12g_tree* t, uint8_t flags, uint32_t* n_subdivided)
{
  if (!t) return fail(B12G_ERR_INVALID, "NULL tree");
  if (t->mixed) return mixed_subdivide(t, flags, n_subdivided);
  // subdivide (ImplicitBoxTree.hpp:2884-2929) returns the number of leaves with all
  // flags set; IsSubdividableFunctor (Functors.hpp:332-335) splits those below depth 64
  uint32_t m = 0;
  ST(set_ctr(t, C_TMP, 0));
  CK(count_flags(t->flg(), t->dn(), flags, t->ctr.p + C_TMP, t->n, t->stream));
  count_launches(1);
  ST(read_ctr(t, C_TMP, 1));
  m = t->h_ctr[C_TMP];
  if (m != 0 && m != t->n && t->depth < 64) {
    // some leaves split: the tree's leaves get two depths
    ST(mixed_enter(t));
    return mixed_subdivide(t, flags, n_subdivided);
  }
  if (m == t->n && t->depth < 64) {
    ST(reserve(t, 2ull * t->n));
    const int o = 1 - t->cur, no = 1 - t->ncur;
    CK(split_codes(t->codes(), t->flg(), t->dn(), t->code[o].p, t->flags[o].p, t->ctr.p + no, t->n, t->stream));
    count_launches(1);
    ST(sync(t, "subdivide"));
    t->cur = o;
    ++t->leaf_gen;
    t->ncur = no;
    t->n *= 2;
    t->depth += 1;
  }
  if (n_subdivided) *n_subdivided = m;
  return B12G_OK;
}

b12g_status b12g_remove(b12g_tree* t, uint8_t flags, uint32_t* n_removed)
{
  if (!t) return fail(B12G_ERR_INVALID, "NULL tree");
  if (t->mixed) return mixed_remove(t, flags, n_removed);
  const int o = 1 - t->cur, no = 1 - t->ncur;
  CompactArgs ca{};
  ca.code = t->codes();
  ca.flags = t->flg();
  ca.n = t->dn();
  ca.keep_flags = flags;
  ca.out_code = t->code[o].p;
  ca.out_flags = t->flags[o].p;
  ca.n_out = t->ctr.p + no;
  ca.out_cap = uint32_t(std::min<size_t>(t->code[o].n, t->flags[o].n));
  ca.error = t->ctr.p + C_ERROR;
  CK(compact(ca, {t->tiles_a.p, t->tiles_b.p}, t->n, t->stream));
  count_launches(compact_launches(false, t->n));
  ST(read_ctr(t, no, 1));
  ST(check_error(t, "remove"));
  const uint32_t kept = t->h_ctr[no];
  const uint32_t removed = t->n - kept;
  t->cur = o;
  ++t->leaf_gen;
  t->ncur = no;
  t->n = kept;
  ++t->leaf_gen;
  if (kept == 0) ST(set_root(t, B12G_NONE));  // insertSurroundingBoxIfEmpty
  if (n_removed) *n_removed = removed;
  return B12G_OK;
}

b12g_status b12g_unsubdivide(b12g_tree* t, uint8_t flags, uint32_t* n_parents)
{
  if (!t) return fail(B12G_ERR_INVALID, "NULL tree");
  return mixed_unsubdivide(t, flags, n_parents);
}

b12g_status b12g_delete_depth(b12g_tree* t, uint8_t depth, uint32_t* n_deleted)
{
  if (!t) return fail(B12G_ERR_INVALID, "NULL tree");
  uint32_t c = 0;
  if (depth == 0) {
    ST(set_root(t, B12G_NONE));
    c = 1;
  } else if (depth == B12G_LEAF_DEPTH || depth > t->depth) {
    c = 0;
  } else {
    return fail(B12G_ERR_UNSUPPORTED_MIXED_DEPTH, "deleteDepth(%u) of a tree of depth %u", depth, t->depth);
  }
  if (n_deleted) *n_deleted = c;
  return B12G_OK;
}

// ---- box images -------------------------------------------------------------------------
b12g_status b12g_set_flags_by_image(b12g_tree* t, const b12g_scheme* sc, uint8_t flags, uint8_t depth,
                                    uint32_t* n_changed)
{
  if (!t) return fail(B12G_ERR_INVALID, "NULL tree");
  if (t->mixed || (depth != B12G_LEAF_DEPTH && depth != t->depth) ||
      (sc && sc->depth != B12G_LEAF_DEPTH && sc->depth != t->depth))
    return mixed_set_flags_by_image(t, sc, flags, depth, n_changed);
  ST(check_depth(t, depth));
  Prepared pr;
  ST(prepare(t, sc, pr));
  uint32_t n_src = 0;
  ST(select_sources(t, sc, pr, n_src));
  ST(build_current_hash(t, pr));
  ST(set_ctr(t, C_CHANGED, 0));
  pr.a.hit_cap = uint32_t(std::min<size_t>(t->hit.n, 0xFFFFFFFFu));
  prof_mark(t, 0);
  CK(launch_image(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, ImageMode::Hit, pr.a,
                  uint64_t(n_src) * pr.P, t->stream));
  prof_mark(t, 0);
  CK(apply_hits(t->flg(), t->hit.p, t->dn(), flags, t->ctr.p + C_CHANGED, t->n, t->stream));
  count_launches(2);
  ST(read_ctr(t, C_CHANGED, 1));
  ST(prof_collect(t));
  ST(check_error(t, "set_flags_by_image"));
  if (n_changed) *n_changed = t->h_ctr[C_CHANGED];
  return B12G_OK;
}

b12g_status b12g_search_by_image(b12g_tree* t, const b12g_scheme* sc, uint8_t depth, uint32_t* out, uint64_t capacity,
                                 uint64_t* n_points)
{
  if (!t) return fail(B12G_ERR_INVALID, "NULL tree");
  if (t->mixed || (depth != B12G_LEAF_DEPTH && depth != t->depth) ||
      (sc && sc->depth != B12G_LEAF_DEPTH && sc->depth != t->depth)) {
    // leaves of several depths, or a depth inside the tree (of the sources or the
    // targets): the index of each point's leaf, or of its box at that depth
    uint64_t np = 0;
    if (depth == B12G_LEAF_DEPTH) ST(mixed_search(t, sc, &np));
    else ST(mixed_image_at_depth(t, sc, depth, 0, true, &np, nullptr));
    if (n_points) *n_points = np;
    if (out && capacity < np)
      return fail(B12G_ERR_CAPACITY, "output holds %llu of %llu points", (unsigned long long)capacity,
                  (unsigned long long)np);
    if (out) CK(cudaMemcpyAsync(out, t->out.p, np * 4, cudaMemcpyDeviceToHost, t->stream));
    ST(sync(t, "search_by_image"));
    return mixed_settle(t);
  }
  ST(check_depth(t, depth));
  Prepared pr;
  ST(prepare(t, sc, pr));
  uint32_t n_src = 0;
  ST(select_sources(t, sc, pr, n_src));
  const uint64_t np = uint64_t(n_src) * pr.P;
  if (n_points) *n_points = np;
  if (!out) return B12G_OK;
  if (capacity < np) return fail(B12G_ERR_CAPACITY, "output holds %llu of %llu points", (unsigned long long)capacity,
                                 (unsigned long long)np);
  ST(t->out.ensure(std::max<uint64_t>(np, 1), "search output"));
  ST(build_current_hash(t, pr));
  pr.a.out = t->out.p;
  CK(launch_image(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, ImageMode::Search, pr.a, np, t->stream));
  count_launches(1);
  CK(cudaMemcpyAsync(out, t->out.p, np * 4, cudaMemcpyDeviceToHost, t->stream));
  return sync(t, "search_by_image");
}

// ---- transition matrix -----------------------------------------------------------------
b12g_status b12g_transition_matrix(b12g_tree* t, const b12g_scheme* sc, int absolute, int invalid_column,
                                   b12g_csr** out)
{
  if (!t || !out) return fail(B12G_ERR_INVALID, "NULL argument");
  Prepared pr;
  ST(prepare(t, sc, pr));
  if (pr.P > kMaxRowPoints) return fail(B12G_ERR_CAPACITY, "transition rows support up to %u points per box",
                                        kMaxRowPoints);
  if (sc->flags_to_check != 0 || (sc->depth != B12G_LEAF_DEPTH && sc->depth != t->depth))
    return fail(B12G_ERR_INVALID, "transitionMatrixForLeaves maps every leaf");
  const uint32_t n = t->n;
  const uint64_t stage = uint64_t(n) * pr.P;
  ST(t->stage_col.ensure(stage, "row staging"));
  ST(t->stage_cnt.ensure(stage, "row staging"));
  ST(t->row_count.ensure(n + 1, "row counts"));
  ST(t->rowptr.ensure(n + 1, "row pointers"));
  if (t->mixed) {
    prof_mark(t, 1);
    ST(mixed_rows(t, sc, invalid_column));
    prof_mark(t, 1);
  } else if (stored_rows_fit(t, sc, pr)) {
    // the targets the last subdivision step stored, for these very leaves and scheme
    StoredRowArgs ra{};
    ra.targets = t->last_tgt.p;
    ra.rank = t->last_rank.p;
    ra.codes = t->codes();
    ra.n_children = t->tgt_children;
    ra.n_leaves = n;
    ra.points = uint32_t(pr.P);
    ra.stage_col = t->stage_col.p;
    ra.stage_cnt = t->stage_cnt.p;
    ra.row_count = t->row_count.p;
    ra.keep_lost = invalid_column ? 1 : 0;
    prof_mark(t, 1);
    CK(launch_stored_rows(ra, t->stream));
    prof_mark(t, 1);
  } else {
    ST(build_current_hash(t, pr));
    RowArgs ra{};
    ra.img = pr.a;
    ra.stage_col = t->stage_col.p;
    ra.stage_cnt = t->stage_cnt.p;
    ra.row_count = t->row_count.p;
    ra.keep_lost = invalid_column ? 1 : 0;
    ra.lost_col = n + 1;  // ImplicitBoxTree.hpp:3075-3090: nColumns += 1, lost entries get index nColumns
    prof_mark(t, 1);
    CK(launch_rows(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, ra, n, t->stream));
    prof_mark(t, 1);
  }
  if (!t->mixed) count_launches(1);    // mixed_rows counts its own launches
  ST(finish_rows(t, uint32_t(pr.P), n, absolute, invalid_column, out));
  return prof_collect(t);
}

}  // extern "C"

namespace b12g {
namespace host {

// The CSR of the rows staged for the tree's n leaves (stage_col / stage_cnt / row_count,
// P slots a row): row pointers by a scan, then every row's runs gathered.  Columns index
// n_cols boxes; lost points, kept in column n_cols + 1, make nColumns n_cols + 1 only when
// some row has one (ImplicitBoxTree.hpp:3075-3090).  An existing matrix in *out is
// refilled in place (its buffers only grow).
b12g_status finish_rows(b12g_tree* t, uint32_t P, uint32_t n_cols, int absolute, int invalid_column, b12g_csr** out)
{
  const uint32_t n = t->n;
  CK(exclusive_scan_u32(t->row_count.p, t->rowptr.p, t->dn(), t->tiles_a.p, n, t->stream));
  CK(cudaMemcpyAsync(t->h_ctr + C_NNZ, t->rowptr.p + n, 4, cudaMemcpyDeviceToHost, t->stream));
  count_launches(3);
  ST(sync(t, "transition rows"));
  const uint32_t nnz32 = t->h_ctr[C_NNZ];
  const bool fresh = *out == nullptr;
  b12g_csr* m = fresh ? new b12g_csr() : *out;
  m->device = t->device;
  m->n_rows = n;
  m->n_cols = n_cols;
  m->nnz = nnz32;
  m->has_transpose = false;
  b12g_status st = B12G_OK;
  if (!m->stream && cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess)
    st = cuda_fail(cudaGetLastError(), "stream");
  if (st == B12G_OK) st = m->rowptr.ensure(n + 1, "rowptr");
  if (st == B12G_OK) st = m->cols.ensure(std::max<uint64_t>(m->nnz, 1), "cols");
  if (st == B12G_OK) st = m->vals.ensure(std::max<uint64_t>(m->nnz, 1), "vals");
  if (st == B12G_OK) st = m->ctr.ensure(256, "csr counters");
  const bool find_lost = invalid_column && nnz32 != 0;
  if (st == B12G_OK && find_lost) st = set_ctr(t, C_TMP, 0);
  if (st == B12G_OK) {
    cudaMemcpyAsync(m->rowptr.p, t->rowptr.p, size_t(n + 1) * 4, cudaMemcpyDeviceToDevice, t->stream);
    gather_rows(t->stage_col.p, t->stage_cnt.p, P, t->row_count.p, t->rowptr.p, t->dn(), m->cols.p, m->vals.p,
                absolute, double(P), n, t->stream);
    count_launches(1);
    if (find_lost) {
      value_present(m->cols.p, nnz32, n_cols + 1, t->ctr.p + C_TMP, t->stream);
      count_launches(1);
    }
    st = sync(t, "gather rows");
  }
  if (st == B12G_OK && find_lost) {
    st = read_ctr(t, C_TMP, 1);
    if (st == B12G_OK && t->h_ctr[C_TMP] != 0) m->n_cols = n_cols + 1;
  }
  if (st != B12G_OK) {
    if (fresh) b12g_csr_destroy(m);
    return st;
  }
  *out = m;
  return B12G_OK;
}

}  // namespace host
}  // namespace b12g

extern "C" {

b12g_status b12g_csr_shape(const b12g_csr* m, uint32_t* n_rows, uint32_t* n_cols, uint64_t* nnz)
{
  if (!m) return fail(B12G_ERR_INVALID, "NULL matrix");
  if (n_rows) *n_rows = m->n_rows;
  if (n_cols) *n_cols = m->n_cols;
  if (nnz) *nnz = m->nnz;
  return B12G_OK;
}

b12g_status b12g_csr_copy(const b12g_csr* m, uint32_t* rowptr, uint32_t* cols, double* vals)
{
  if (!m) return fail(B12G_ERR_INVALID, "NULL matrix");
  if (rowptr) CK(cudaMemcpyAsync(rowptr, m->rowptr.p, size_t(m->n_rows + 1) * 4, cudaMemcpyDeviceToHost, m->stream));
  if (cols && m->nnz) CK(cudaMemcpyAsync(cols, m->cols.p, m->nnz * 4, cudaMemcpyDeviceToHost, m->stream));
  if (vals && m->nnz) CK(cudaMemcpyAsync(vals, m->vals.p, m->nnz * 8, cudaMemcpyDeviceToHost, m->stream));
  CK(cudaStreamSynchronize(m->stream));
  return B12G_OK;
}

b12g_status b12g_csr_destroy(b12g_csr* m)
{
  if (!m) return B12G_OK;
  if (m->stream) cudaStreamSynchronize(m->stream);
  m->rowptr.release(); m->cols.release(); m->vals.release(); m->tptr.release(); m->trows.release();
  m->work.release(); m->tiles.release(); m->tvals.release(); m->w0.release(); m->w1.release();
  m->partial.release(); m->vout.release(); m->ctr.release(); m->vstart.release(); m->change.release();
  m->long_flag.release(); m->long_pos.release(); m->long_list.release(); m->mid_list.release();
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return B12G_OK;
}

}  // extern "C"

namespace b12g {
namespace host {

// P^T of a matrix (rows ascending per column, the lost column dropped) and its rows
// split by length class, built once per matrix
b12g_status ensure_transpose(b12g_csr* m)
{
  const uint32_t n = m->n_rows;
  cudaStream_t s = m->stream;
  if (n == 0) return B12G_OK;
  if (!m->has_transpose) {
    ST(m->tptr.ensure(n + 1, "transpose"));
    ST(m->trows.ensure(std::max<uint64_t>(m->nnz, 1), "transpose"));
    ST(m->tvals.ensure(std::max<uint64_t>(m->nnz, 1), "transpose"));
    ST(m->work.ensure(n + 1, "transpose"));
    ST(m->tiles.ensure(compact_tiles(n + 1) + 2, "transpose"));
    uint32_t h[3] = {n, uint32_t(m->nnz), n};
    CK(cudaMemcpyAsync(m->ctr.p, h, sizeof h, cudaMemcpyHostToDevice, s));
    CK(transpose_csr(m->rowptr.p, m->cols.p, m->vals.p, m->ctr.p, m->ctr.p + 1, n, m->nnz, n, m->tptr.p,
                     m->trows.p, m->tvals.p, m->work.p, m->tiles.p, m->ctr.p + 2, s));
    ST(m->long_flag.ensure(n + 1, "row classes"));
    ST(m->long_pos.ensure(n + 1, "row classes"));
    ST(m->long_list.ensure(n + 1, "row classes"));
    ST(m->mid_list.ensure(n + 1, "row classes"));
    CK(max_row_length(m->tptr.p, n, m->ctr.p + 6, s));
    count_launches(7);
    uint32_t max_row = 0;
    CK(cudaMemcpyAsync(&max_row, m->ctr.p + 6, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (measure_on_chip(m->nnz, max_row, uint32_t(measure_partial_slots()))) {
      // the power iteration keeps the matrix on chip and reads no row-class lists
      m->n_mid = 0;
      m->n_long = 0;
    } else {
      // both classes' counts (each at long_pos[n] after its pass) gathered in two counter
      // words and read back together
      uint32_t counts[2] = {0, 0};
      CK(class_rows(m->tptr.p, n, 1, m->long_flag.p, m->long_pos.p, m->mid_list.p, m->ctr.p, m->tiles.p, s));
      CK(cudaMemcpyAsync(m->ctr.p + 4, m->long_pos.p + n, 4, cudaMemcpyDeviceToDevice, s));
      CK(class_rows(m->tptr.p, n, 2, m->long_flag.p, m->long_pos.p, m->long_list.p, m->ctr.p, m->tiles.p, s));
      CK(cudaMemcpyAsync(m->ctr.p + 5, m->long_pos.p + n, 4, cudaMemcpyDeviceToDevice, s));
      CK(cudaMemcpyAsync(counts, m->ctr.p + 4, sizeof counts, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      m->n_mid = counts[0];
      m->n_long = counts[1];
      count_launches(10);
    }
    m->has_transpose = true;
  }
  return B12G_OK;
}

}  // namespace host
}  // namespace b12g

extern "C" {

b12g_status b12g_invariant_measure(b12g_csr* m, uint32_t iters, double* v)
{
  if (!m) return fail(B12G_ERR_INVALID, "NULL matrix");
  const uint32_t n = m->n_rows;
  if (n == 0) return B12G_OK;
  cudaStream_t s = m->stream;
  ST(ensure_transpose(m));
  ST(m->w0.ensure(n, "measure"));
  ST(m->w1.ensure(n, "measure"));
  ST(m->vout.ensure(n, "measure"));
  const int slots = measure_partial_slots();
  ST(m->partial.ensure(slots, "measure"));
  CK(invariant_measure(m->tptr.p, m->trows.p, m->tvals.p, m->mid_list.p, m->n_mid, m->long_list.p, m->n_long, n,
                       iters, m->w0.p, m->w1.p, m->partial.p, uint32_t(slots), m->vout.p, m->ctr.p + 64, s,
                       m->nnz));
  count_launches(1);
  if (v) CK(cudaMemcpyAsync(v, m->vout.p, size_t(n) * 8, cudaMemcpyDeviceToHost, s));
  uint32_t err = 0;
  CK(cudaMemcpyAsync(&err, m->ctr.p + 64 + 64, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (err & 2u) return fail(B12G_ERR_TIMEOUT, "invariant measure: grid barrier gave up");
  if (err & 4u) return fail(B12G_ERR_CAPACITY, "invariant measure: a block's rows exceed its shared memory");
  return B12G_OK;
}

b12g_status b12g_invariant_measure_tol(b12g_csr* m, double tol, uint32_t max_iters, uint32_t check_every, double* v,
                                       uint32_t* iters_done, double* last_change)
{
  if (!m) return fail(B12G_ERR_INVALID, "NULL matrix");
  if (!(tol >= 0.0) || check_every == 0 || max_iters == 0)
    return fail(B12G_ERR_INVALID, "tolerance >= 0, check_every >= 1 and max_iters >= 1 required");
  const uint32_t n = m->n_rows;
  if (iters_done) *iters_done = 0;
  if (last_change) *last_change = 0.0;
  if (n == 0) return B12G_OK;
  cudaStream_t s = m->stream;
  ST(ensure_transpose(m));
  ST(m->w0.ensure(n, "measure"));
  ST(m->w1.ensure(n, "measure"));
  ST(m->vout.ensure(n, "measure"));
  ST(m->vstart.ensure(n, "measure"));
  const int slots = measure_partial_slots();
  const int nchg = slots / 2;          // at least the largest grid of a launch
  ST(m->partial.ensure(slots, "measure"));
  ST(m->change.ensure(nchg, "measure"));
  std::vector<double> chg(nchg);
  uint32_t done = 0;
  double change = 0.0;
  const double* start = nullptr;
  for (;;) {
    const uint32_t k = std::min(check_every, max_iters - done);
    CK(cudaMemsetAsync(m->change.p, 0, size_t(nchg) * 8, s));
    CK(invariant_measure(m->tptr.p, m->trows.p, m->tvals.p, m->mid_list.p, m->n_mid, m->long_list.p, m->n_long, n,
                         k, m->w0.p, m->w1.p, m->partial.p, uint32_t(slots), m->vout.p, m->ctr.p + 64, s, m->nnz,
                         start, m->change.p));
    count_launches(1);
    uint32_t err = 0;
    CK(cudaMemcpyAsync(chg.data(), m->change.p, size_t(nchg) * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&err, m->ctr.p + 64 + 64, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (err & 2u) return fail(B12G_ERR_TIMEOUT, "invariant measure: grid barrier gave up");
    if (err & 4u) return fail(B12G_ERR_CAPACITY, "invariant measure: a block's rows exceed its shared memory");
    change = 0.0;
    for (double c : chg) change += c;          // fixed order: the same sum every run
    done += k;
    if (change <= tol || done >= max_iters) break;
    CK(cudaMemcpyAsync(m->vstart.p, m->vout.p, size_t(n) * 8, cudaMemcpyDeviceToDevice, s));
    start = m->vstart.p;
  }
  if (v) CK(cudaMemcpyAsync(v, m->vout.p, size_t(n) * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (iters_done) *iters_done = done;
  if (last_change) *last_change = change;
  return B12G_OK;
}

b12g_status b12g_csr_measure(const b12g_csr* m, double* v)
{
  if (!m || !v) return fail(B12G_ERR_INVALID, "NULL argument");
  if (m->vout.n < m->n_rows) return fail(B12G_ERR_INVALID, "no invariant measure computed yet");
  CK(cudaMemcpyAsync(v, m->vout.p, size_t(m->n_rows) * 8, cudaMemcpyDeviceToHost, m->stream));
  CK(cudaStreamSynchronize(m->stream));
  return B12G_OK;
}

// ---- fused subdivision loop --------------------------------------------------------------
b12g_status b12g_subdivision_run(b12g_tree* t, const b12g_scheme* sc, uint32_t steps, uint32_t* counts)
{
  if (!t || !sc) return fail(B12G_ERR_INVALID, "NULL argument");
  if (steps == 0) return B12G_OK;
  if (sc->flags_to_check != 0 || sc->depth != B12G_LEAF_DEPTH)
    return fail(B12G_ERR_INVALID, "the subdivision loop maps every leaf (depth 255, no flag filter)");
  if (int(t->depth) + int(steps) > 64) return fail(B12G_ERR_INVALID, "depth would exceed 64");
  // setFlags(SD) on every leaf (subdivision.m:16, B12_doc.tex:266)
  ST(flag_call(t, 0, 0, B12G_SD, B12G_LEAF_DEPTH, nullptr));
  if (t->mixed) {
    // leaves of several depths: the steps of subdivision.m:18-45 one call at a time
    uint32_t k = 0;
    for (uint32_t s = 0; s < steps; ++s) {
      ST(b12g_subdivide(t, B12G_SD, &k));
      ST(b12g_set_flags_by_image(t, sc, B12G_HIT, B12G_LEAF_DEPTH, &k));
      ST(b12g_remove(t, B12G_HIT, &k));
      ST(b12g_unset_flags(t, B12G_HIT, B12G_LEAF_DEPTH, &k));
      if (counts) counts[s] = t->n;
    }
    return B12G_OK;
  }

  // keep the initial state so that a capacity overflow can be retried with more room
  const uint32_t n0 = t->n;
  const uint8_t d0 = t->depth;
  std::vector<uint64_t> c0(n0);
  std::vector<uint8_t> f0(n0);
  CK(cudaMemcpyAsync(c0.data(), t->codes(), size_t(n0) * 8, cudaMemcpyDeviceToHost, t->stream));
  CK(cudaMemcpyAsync(f0.data(), t->flg(), n0, cudaMemcpyDeviceToHost, t->stream));
  ST(sync(t, "snapshot"));
  ST(t->step_counts.ensure(steps + 1, "step counts"));

  uint64_t cap = std::max<uint64_t>(t->code[0].n, std::max<uint64_t>(4ull * n0, 1ull << 16));
  t->tgt_ok = false;
  for (int attempt = 0; attempt < 12; ++attempt) {
    ST(reserve(t, cap));
    const bool use_hash = int(d0) + int(steps) - 1 <= kHashMaxDepth && t->domain.dim >= 2;
    if (use_hash) ST(ensure_hash(t, cap));
    Prepared pr;
    ST(prepare(t, sc, pr));
    // The last step keeps every point's target and the compaction ranks for the
    // transition matrix of the result.  The buffer is sized by the previous run of this
    // tree (a tree's first run stores nothing and allocates nothing); a last step with
    // more points than it holds only marks the stored targets unusable.
    const uint64_t tgt_entries = t->tgt_want;
    const bool store = tgt_entries > 0 && pr.P <= kMaxRowPoints && tgt_entries * 4 <= (8ull << 30);
    if (store) {
      ST(t->last_tgt.ensure(tgt_entries, "stored targets"));
      ST(t->last_rank.ensure(2ull * cap + 1, "stored ranks"));
    }
    uint32_t* const store_tgt = store ? t->last_tgt.p : nullptr;
    uint32_t* const store_rank = store ? t->last_rank.p : nullptr;
    const uint64_t store_cap = store ? t->last_tgt.n : 0;
    // key of the captured graph: every pointer and parameter the launches bake in
    std::vector<uint8_t> key(sizeof(b12g_scheme) + 88);
    std::memcpy(key.data(), sc, sizeof(b12g_scheme));
    uint64_t extra[11] = {uint64_t(uintptr_t(t->pk.p)), steps, cap, uint64_t(t->cur) | uint64_t(t->ncur) << 1 | uint64_t(t->profile) << 2, uint64_t(d0),
                          uint64_t(uintptr_t(t->code[0].p)), uint64_t(uintptr_t(t->hit.p)), uint64_t(uintptr_t(t->table.p)),
                          uint64_t(uintptr_t(t->code[1].p)) ^ (uint64_t(uintptr_t(t->hash.p)) << 1),
                          uint64_t(uintptr_t(store_tgt)) ^ (store_cap << 1), uint64_t(uintptr_t(store_rank))};
    std::memcpy(key.data() + sizeof(b12g_scheme), extra, sizeof extra);

    if (!t->sub_graph || key != t->sub_key) {
      if (t->sub_graph) { cudaGraphExecDestroy(t->sub_graph); t->sub_graph = nullptr; }
      cudaGraph_t g = nullptr;
      for (int k = 0; k < 2; ++k) {
        for (cudaEvent_t e : t->graph_prof[k]) cudaEventDestroy(e);
        t->graph_prof[k].clear();
      }
      t->prof_used[0] = t->prof_used[1] = 0;
      CK(cudaStreamBeginCapture(t->stream, cudaStreamCaptureModeThreadLocal));
      int cur = t->cur, ncur = t->ncur;
      cudaError_t err = cudaSuccess;
      // the lookup table starts clean at every replay; step s builds with tag s + 1
      if (use_hash) err = cudaMemsetAsync(t->hash.p, 0, t->hash.n * sizeof(ulonglong2), t->stream);
      for (uint32_t s = 0; s < steps && err == cudaSuccess; ++s) {
        const int o = 1 - cur, no = 1 - ncur;
        ImageArgs a = pr.a;
        a.hash = LeafHash{nullptr, 0, 0, nullptr};
        if (use_hash) {
          a.hash = LeafHash{t->hash.p, s + 1, t->hash_log2, t->pk.p};
          err = build_leaf_hash(t->code[cur].p, t->ctr.p + ncur, int(d0) + int(s), int(t->domain.dim), a.hash,
                                t->ctr.p + C_ERROR, uint32_t(std::min<uint64_t>(cap, 0xFFFFFFFFu)), t->stream);
          if (err != cudaSuccess) break;
        }
        a.codes = t->code[cur].p;
        a.n_leaves = t->ctr.p + ncur;
        a.depth = int(d0) + int(s) + 1;
        a.children = 1;
        a.hit_cap = uint32_t(std::min<size_t>(t->hit.n, 0xFFFFFFFFu));
        const bool last = s + 1 == steps;
        a.targets = last ? store_tgt : nullptr;
        a.targets_cap = store_cap;
        a.targets_over = t->ctr.p + C_TGT;
        prof_mark(t, 0);
        err = launch_image(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, ImageMode::Hit, a,
                           2ull * cap * pr.P, t->stream);
        prof_mark(t, 0);
        if (err != cudaSuccess) break;
        CompactArgs ca{};
        ca.code = t->code[cur].p;
        ca.flags = t->flags[cur].p;
        ca.n = t->ctr.p + ncur;
        ca.hit = t->hit.p;
        ca.children = 1;
        ca.hit_cap = a.hit_cap;
        ca.out_code = t->code[o].p;
        ca.out_flags = t->flags[o].p;
        ca.n_out = t->ctr.p + no;
        ca.n_out2 = t->step_counts.p + s;
        ca.out_cap = uint32_t(std::min<size_t>(t->code[o].n, 0xFFFFFFFFu));
        ca.error = t->ctr.p + C_ERROR;
        ca.out_rank = last ? store_rank : nullptr;
        err = compact(ca, {t->tiles_a.p, t->tiles_b.p}, uint32_t(std::min<uint64_t>(cap, 0xFFFFFFFFu)), t->stream);
        cur = o;
        ncur = no;
      }
      cudaError_t e2 = cudaStreamEndCapture(t->stream, &g);
      if (err != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(err, "capture subdivision"); }
      if (e2 != cudaSuccess) return cuda_fail(e2, "end capture");
      cudaError_t e3 = cudaGraphInstantiate(&t->sub_graph, g, 0);
      cudaGraphDestroy(g);
      if (e3 != cudaSuccess) { t->sub_graph = nullptr; return cuda_fail(e3, "instantiate"); }
      t->sub_key = key;
      t->sub_graph_kernels =
          uint64_t((use_hash ? 2 : 1) + compact_launches(true, uint32_t(std::min<uint64_t>(cap, 0xFFFFFFFFu)))) * steps;
      // the events recorded during capture belong to the graph from now on
      for (int k = 0; k < 2; ++k) {
        t->graph_prof[k].assign(t->prof_events[k].begin(), t->prof_events[k].begin() + t->prof_used[k]);
        t->prof_events[k].erase(t->prof_events[k].begin(), t->prof_events[k].begin() + t->prof_used[k]);
        t->prof_used[k] = 0;
      }
    }
    ST(set_ctr(t, C_TGT, 0));
    CK(cudaGraphLaunch(t->sub_graph, t->stream));
    count_launches(t->sub_graph_kernels);
    if (use_hash) t->hash_tag = steps;
    std::vector<uint32_t> hc(steps);
    CK(cudaMemcpyAsync(hc.data(), t->step_counts.p, steps * 4, cudaMemcpyDeviceToHost, t->stream));
    CK(cudaMemcpyAsync(t->h_ctr + C_ERROR, t->ctr.p + C_ERROR, 4, cudaMemcpyDeviceToHost, t->stream));
    CK(cudaMemcpyAsync(t->h_ctr + C_TGT, t->ctr.p + C_TGT, 4, cudaMemcpyDeviceToHost, t->stream));
    ST(sync(t, "subdivision run"));
    if (t->profile)
      for (int k = 0; k < 2; ++k)
        sum_pairs(t->graph_prof[k], t->graph_prof[k].size(), t->prof_ms[k], t->prof_launches[k]);
    if (t->h_ctr[C_ERROR] & 1u) {
      // capacity exceeded: restore the initial leaves and retry with 4x the room
      ST(set_ctr(t, C_ERROR, 0));
      cap *= 4;
      ST(reserve(t, cap));
      CK(cudaMemsetAsync(t->hit.p, 0, t->hit.n, t->stream));
      CK(cudaMemcpyAsync(t->codes(), c0.data(), size_t(n0) * 8, cudaMemcpyHostToDevice, t->stream));
      CK(cudaMemcpyAsync(t->flg(), f0.data(), n0, cudaMemcpyHostToDevice, t->stream));
      ST(set_ctr(t, t->ncur, n0));
      ST(sync(t, "restore"));
      t->n = n0;
      ++t->leaf_gen;
      t->depth = d0;
      continue;
    }
    // steps alternate the buffers: after an odd number of steps the other one is current
    if (steps & 1u) { t->cur = 1 - t->cur; t->ncur = 1 - t->ncur; }
    uint32_t final_n = hc[steps - 1];
    uint32_t done = steps;
    for (uint32_t s = 0; s < steps; ++s)
      if (hc[s] == 0) { done = s; break; }
    if (done < steps) {
      // a step removed every box: the reference re-inserts the surrounding box, which
      // has no SD flag and so stays the only leaf
      for (uint32_t s = done; s < steps; ++s) hc[s] = 1;
      ST(set_root(t, B12G_NONE));
      final_n = 1;
    } else {
      t->n = final_n;
      ++t->leaf_gen;
      t->depth = uint8_t(d0 + steps);
      const uint64_t children = 2ull * (steps >= 2 ? hc[steps - 2] : n0);
      t->tgt_want = std::max<uint64_t>(t->tgt_want, (children + children / 8 + 1) * pr.P);
      if (store && t->h_ctr[C_TGT] == 0) {
        t->tgt_children = uint32_t(children);
        t->tgt_n = final_n;
        t->tgt_depth = t->depth;
        t->tgt_points = uint32_t(pr.P);
        t->tgt_scheme = *sc;
        t->tgt_gen = t->leaf_gen;
        t->tgt_ok = true;
      }
    }
    if (counts) std::memcpy(counts, hc.data(), steps * 4);
    return B12G_OK;
  }
  return fail(B12G_ERR_CAPACITY, "subdivision run: capacity retries exhausted");
}

// ---- measurement hooks --------------------------------------------------------------------
b12g_status b12g_tree_stream(b12g_tree* t, void** stream)
{
  if (!t || !stream) return fail(B12G_ERR_INVALID, "NULL argument");
  *stream = (void*)t->stream;
  return B12G_OK;
}

b12g_status b12g_profile_enable(b12g_tree* t, int enable)
{
  if (!t) return fail(B12G_ERR_INVALID, "NULL tree");
  t->profile = enable != 0;
  return B12G_OK;
}

b12g_status b12g_profile_read(b12g_tree* t, uint32_t kind, double* ms_total, uint64_t* launches, int reset)
{
  if (!t || kind > 1) return fail(B12G_ERR_INVALID, "bad argument");
  if (ms_total) *ms_total = t->prof_ms[kind];
  if (launches) *launches = t->prof_launches[kind];
  if (reset) { t->prof_ms[kind] = 0.0; t->prof_launches[kind] = 0; }
  return B12G_OK;
}

}  // extern "C"
