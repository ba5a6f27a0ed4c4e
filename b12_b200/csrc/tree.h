// Host-side objects of libb12g shared by the C ABI translation units.
#pragma once

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "kernels.h"

namespace b12g {
namespace host {

b12g_status fail(b12g_status s, const char* fmt, ...);
b12g_status cuda_fail(cudaError_t e, const char* where);

#define CK(call)                                                   \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return ::b12g::host::cuda_fail(e_, #call); \
  } while (0)

// the launch just queued (or an earlier one) failed: report it with `where`
#define LAUNCHED(where)                                            \
  do {                                                             \
    cudaError_t e_ = cudaGetLastError();                           \
    if (e_ != cudaSuccess) return ::b12g::host::cuda_fail(e_, where); \
  } while (0)

#define ST(call)                                                   \
  do {                                                             \
    b12g_status s_ = (call);                                       \
    if (s_ != B12G_OK) return s_;                                  \
  } while (0)

// grow-only device buffer
template<class T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  b12g_status ensure(size_t count, const char* what)
  {
    if (count <= n) return B12G_OK;
    size_t want = std::max<size_t>(count, n + n / 2);
    want = std::max<size_t>(want, 256);
    T* q = nullptr;
    cudaError_t e = cudaMalloc(&q, want * sizeof(T));
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(B12G_ERR_OOM, "cannot allocate %zu bytes for %s", want * sizeof(T), what);
    }
    if (p) cudaFree(p);
    p = q;
    n = want;
    return B12G_OK;
  }
  // grow keeping the first `keep` elements
  b12g_status grow_keep(size_t count, size_t keep, cudaStream_t s, const char* what)
  {
    if (count <= n) return B12G_OK;
    T* old = p;
    size_t oldn = n;
    p = nullptr;
    n = 0;
    b12g_status st = ensure(count, what);
    if (st != B12G_OK) { p = old; n = oldn; return st; }
    if (old) {
      // the old buffer holds oldn elements, whatever the caller counts as kept
      keep = std::min(keep, oldn);
      cudaError_t e = keep ? cudaMemcpyAsync(p, old, keep * sizeof(T), cudaMemcpyDeviceToDevice, s) : cudaSuccess;
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      cudaFree(old);
      if (e != cudaSuccess) return ::b12g::host::cuda_fail(e, what);
    }
    return B12G_OK;
  }
  // ensure room for `count`, and when that means a new buffer, for `factor` times as
  // many: for buffers that grow step by step (cudaFree synchronises the device)
  b12g_status ensure_room(size_t count, const char* what, size_t factor = 2)
  {
    return ensure(count <= n ? count : factor * count, what);
  }
  void release()
  {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// device counter slots
enum : int {
  C_N0 = 0,        // leaf count (ping)
  C_N1 = 1,        // leaf count (pong)
  C_CHANGED = 2,
  C_ERROR = 3,
  C_CAND = 4,
  C_NSRC = 5,
  C_TMP = 6,
  C_NNZ = 7,
  C_NCOLS = 8,
  C_SYNC = 9,      // 3 words for the grid barrier
  C_NNEW = 12,
  C_TGT = 13,      // the stored image targets overflowed their buffer
  C_WORK = 14,     // 2 words (8-byte aligned): the image kernel's work-queue counter
  C_DEFER = 16,    // error bits of launches whose status is read with a later read-back
  C_COUNT = 18
};

}  // namespace host
}  // namespace b12g

struct b12g_tree {
  template<class T> using Buf = b12g::host::Buf<T>;
  int device = 0;
  cudaStream_t stream = nullptr;
  b12g_domain domain{};
  b12g::Domain dom{};
  uint32_t n = 1;
  uint8_t depth = 0;
  int cur = 0;     // current code/flags buffer
  int ncur = 0;    // current count slot (C_N0 / C_N1)
  Buf<uint64_t> code[2];
  Buf<uint8_t> flags[2];
  Buf<uint8_t> hit;
  Buf<uint32_t> ctr;
  Buf<uint32_t> tiles_a, tiles_b;
  Buf<uint32_t> src, out, stage_col, stage_cnt, row_count, rowptr;
  Buf<uint64_t> cand, cand2;
  Buf<double> srcc;            // centres of an image launch's source boxes (kSrcStride a source)
  Buf<uint32_t> bits;          // continuation: a bit for every box of the depth
  Buf<uint32_t> sort_idx;
  Buf<double> table;
  Buf<double> points;
  Buf<uint32_t> step_counts;
  Buf<uint8_t> sort_tmp;
  // leaves of different depths: per-leaf depths (with code/flags) and comparable patterns
  bool mixed = false;
  Buf<uint8_t> dep[2];
  Buf<uint64_t> cmp;
  Buf<uint32_t> cmp_tab;       // prefix table over cmp: first leaf per top-bits value
  uint32_t cmp_bits = 1;
  // insertion into such trees: point-box validity, new boxes, their sort, the merge scans
  Buf<uint8_t> pvalid, ins_dep, ins_dep2, scan_dep, scan_flags;
  Buf<uint64_t> ins_code, ins_key[2], scan_code;
  Buf<uint32_t> ins_idx[2], ins_pos, ins_head;
  Buf<uint32_t> isrc_head, isrc_pos, isrc_and, isrc;   // scheme sources at an inner depth
  Buf<uint32_t> route_runs, route_cnt;   // routing of point boxes to ranks: run starts and ranks, counts
  Buf<ulonglong2> hash;        // leaf lookup table
  Buf<uint64_t> pk;            // the leaves' packed per-dimension indices (the table's keys)
  uint32_t hash_tag = 0;       // tag of the last build (1..255; 0 = cleared)
  uint32_t hash_log2 = 0;      // log2 of the table's slots
  uint32_t* h_ctr = nullptr;   // pinned mirror of ctr
  // graph cache of the fused subdivision loop
  cudaGraphExec_t sub_graph = nullptr;
  std::vector<uint8_t> sub_key;
  uint64_t sub_graph_kernels = 0;
  // optional per-kernel timing: event pairs around image / transition-row launches
  bool profile = false;
  std::vector<cudaEvent_t> prof_events[2];   // [kind] start/stop pairs, reused
  size_t prof_used[2] = {0, 0};
  double prof_ms[2] = {0.0, 0.0};
  uint64_t prof_launches[2] = {0, 0};
  std::vector<cudaEvent_t> graph_prof[2];    // events baked into the captured loop
  // the last step of the fused loop stores its image targets and compaction ranks; the
  // transition matrix of the same leaves and scheme is assembled from them
  // (valid while leaf_gen is the generation they were stored at: every change of the
  // leaf set - count, codes, order, depths - increments leaf_gen)
  Buf<uint32_t> last_tgt, last_rank;
  uint64_t leaf_gen = 0;
  bool tgt_ok = false;
  uint64_t tgt_want = 0;       // entries the next run's last step needs (from this run)
  uint32_t tgt_children = 0, tgt_n = 0, tgt_points = 0;
  uint8_t tgt_depth = 0;
  b12g_scheme tgt_scheme{};
  uint64_t tgt_gen = 0;

  uint64_t* codes() { return code[cur].p; }
  uint8_t* flg() { return flags[cur].p; }
  uint32_t* dn() { return ctr.p + ncur; }
};

struct b12g_csr {
  template<class T> using Buf = b12g::host::Buf<T>;
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t n_rows = 0, n_cols = 0;
  uint64_t nnz = 0;
  Buf<uint32_t> rowptr, cols;
  Buf<double> vals;
  // P^T, built on first use by the invariant measure
  Buf<uint32_t> tptr, trows, work, tiles, long_flag, long_pos, long_list, mid_list;
  uint32_t n_long = 0, n_mid = 0;
  Buf<double> tvals, w0, w1, partial, vout;
  Buf<double> vstart, change;   // tolerance-driven runs: the iterate carried between launches, change partials
  Buf<uint32_t> ctr;
  bool has_transpose = false;
};

namespace b12g {
void count_launches(unsigned long long k);
namespace host {

// host-side validation and kernel argument set-up for a scheme
struct Prepared {
  ImageArgs a{};
  uint64_t P = 0;
};

b12g_status sync(b12g_tree* t, const char* where);
b12g_status read_ctr(b12g_tree* t, int first, int count);
b12g_status set_ctr(b12g_tree* t, int slot, uint32_t v);
b12g_status reserve(b12g_tree* t, uint64_t n_boxes);
b12g_status prepare(b12g_tree* t, const b12g_scheme* sc, Prepared& pr);
bool stored_rows_fit(b12g_tree* t, const b12g_scheme* sc, const Prepared& pr);
b12g_status check_depth(b12g_tree* t, uint8_t depth);
b12g_status select_sources(b12g_tree* t, const b12g_scheme* sc, Prepared& pr, uint32_t& n_src);
b12g_status check_error(b12g_tree* t, const char* where);
// log2 of the lookup-table slots n leaves use (the device's hash_log2)
uint32_t host_hash_log2(uint64_t n);
b12g_status set_root(b12g_tree* t, uint8_t flags);
b12g_status flag_call(b12g_tree* t, int op, uint8_t u, uint8_t f, uint8_t depth, uint32_t* n_changed);
// make the lookup table hold up to max_n codes (clears it when it grows)
b12g_status ensure_hash(b12g_tree* t, uint64_t max_n);
// next build tag (clears the table when the 8-bit tag would wrap)
b12g_status next_hash_tag(b12g_tree* t, uint32_t* tag);
// build the table for the current leaves and point pr.a.hash at it (no-op above depth 56)
b12g_status build_current_hash(b12g_tree* t, Prepared& pr);
// record a timing event of `kind` (0: box-image kernel, 1: transition rows) on the tree stream
void prof_mark(b12g_tree* t, int kind);
b12g_status prof_collect(b12g_tree* t);
// P^T of a matrix and its row classes, built on first use (api.cu)
b12g_status ensure_transpose(b12g_csr* m);
// the CSR of the rows staged in stage_col / stage_cnt / row_count for the tree's leaves (api.cu)
b12g_status finish_rows(b12g_tree* t, uint32_t P, uint32_t n_cols, int absolute, int invalid_column, b12g_csr** out);

// trees of mixed leaf depths (mixed.cu); t->mixed selects them, t->depth is the deepest leaf
b12g_status mixed_enter(b12g_tree* t);
b12g_status mixed_settle(b12g_tree* t);
b12g_status mixed_load(b12g_tree* t, const uint64_t* codes, const uint8_t* depths, const uint8_t* flags, uint32_t n);
b12g_status mixed_count(b12g_tree* t, uint8_t depth, uint32_t* count);
// set / unset / change (op 0 / 1 / 2) flags of the boxes at a depth inside the tree
b12g_status mixed_flags_at_depth(b12g_tree* t, int op, uint8_t u, uint8_t f, uint8_t depth, uint32_t* n_changed);
// images of the scheme's source leaves located at an inner depth: flags on the boxes hit,
// or (search) each point's box index at that depth into t->out; settles the tree's
// layout unless searching (the caller reads t->out first, then settles)
b12g_status mixed_image_at_depth(b12g_tree* t, const b12g_scheme* sc, uint8_t depth, uint8_t flags, bool search,
                                 uint64_t* n_points, uint32_t* n_changed);
b12g_status mixed_leaves(b12g_tree* t, uint64_t* codes, uint8_t* depths, uint8_t* flags);
b12g_status mixed_subdivide(b12g_tree* t, uint8_t flags, uint32_t* n_subdivided);
b12g_status mixed_remove(b12g_tree* t, uint8_t flags, uint32_t* n_removed);
b12g_status mixed_set_flags_by_image(b12g_tree* t, const b12g_scheme* sc, uint8_t flags, uint8_t depth,
                                     uint32_t* n_changed);
// target leaf of every point of the scheme's source leaves into t->out; *n_points of them
b12g_status mixed_search(b12g_tree* t, const b12g_scheme* sc, uint64_t* n_points);
// transition rows of every leaf into t->stage_col / stage_cnt / row_count
b12g_status mixed_rows(b12g_tree* t, const b12g_scheme* sc, int invalid_column);
// unsubdivide(flags); *n_parents = the parents made
b12g_status mixed_unsubdivide(b12g_tree* t, uint8_t flags, uint32_t* n_parents);
// the general insert of the point boxes in t->cand / t->pvalid (np of them) at depth
// (255: leaf depth; not 0); *n_inserted = distinct new boxes
b12g_status mixed_insert_boxes(b12g_tree* t, uint64_t np, uint8_t depth, uint8_t ins, uint8_t hit,
                               uint32_t* n_inserted);
// point boxes of host points, or of the images of a scheme's source leaves
b12g_status mixed_point_boxes(b12g_tree* t, const double* points, uint64_t n_points);
b12g_status mixed_image_boxes(b12g_tree* t, const b12g_scheme* sc, uint64_t* n_points);
// point boxes in the caller's device buffers (range-partitioned trees): the images of the
// scheme's sources (every point, or each warp's distinct point boxes once, cut to their
// first keep_depth bisections), the leaf of each given point box, or flags set on the
// leaves hit
b12g_status mixed_image_point_boxes(b12g_tree* t, const b12g_scheme* sc, uint64_t* codes, uint8_t* valid,
                                    uint64_t capacity, uint64_t* n_points, bool distinct = false,
                                    uint8_t keep_depth = 64);
b12g_status mixed_point_box_search(b12g_tree* t, const uint64_t* codes, const uint8_t* valid, uint64_t n,
                                   uint32_t* index, uint8_t flags, uint32_t* n_changed);
// leaves from device memory, checked for order and nesting on the device
b12g_status mixed_load_device(b12g_tree* t, const uint64_t* codes, const uint8_t* depths, const uint8_t* flags,
                              uint32_t n);

}  // namespace host
}  // namespace b12g
