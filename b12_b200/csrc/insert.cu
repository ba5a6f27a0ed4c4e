// Insertion of new boxes and the continuation driver.
//
// insertByPoints / insertByIterators (ImplicitBoxTree.hpp:1615-1946) at one depth d
// equal to the tree's: every point (or mapped grid point) is located among the leaves;
// a hit leaf gets flagsForHit, a point in no leaf contributes its depth-d code as a
// candidate.  Candidates are radix-sorted, made unique and merged into the sorted
// leaf array with flagsForInserted.  The reference's whole-tree re-sort and its two
// HasSamePath scans (1875-1897) reduce to this merge because all leaves share a depth
// and no candidate equals a leaf.
#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "sort.h"
#include "tree.h"

using namespace b12g;
using namespace b12g::host;

namespace {

constexpr int kThreads = 256;

// locate given points among the leaves: hit mask for found leaves, candidate codes for
// points inside the domain but in no leaf
template<int D>
__global__ void locate_points_kernel(const double* pts, uint32_t n_pts, Domain dom, int depth,
                                     const uint64_t* codes, const uint32_t* n_leaves, LeafHash hash, bool root_only,
                                     uint8_t* hit, uint64_t* cand, uint32_t* cand_count, uint32_t cand_cap,
                                     uint32_t* error)
{
  const uint32_t n = *n_leaves;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_pts; i += gridDim.x * blockDim.x) {
    double p[D];
#pragma unroll
    for (int j = 0; j < D; ++j) p[j] = pts[size_t(i) * D + j];
    uint32_t bits[D];
    if (!point_bits<D>(dom, p, depth, bits)) continue;
    const uint32_t t = root_only ? kInvalidIndex : find_leaf_bits<D>(hash, codes, n, true, bits, depth);
    if (t != kInvalidIndex) {
      if (hit) hit[t] = 1;
    } else {
      int k[D];
#pragma unroll
      for (int j = 0; j < D; ++j) k[j] = bisections<D>(depth, j);
      const uint32_t pos = atomicAdd(cand_count, 1u);
      if (pos < cand_cap) cand[pos] = interleave<D>(bits, k, depth);
      else atomicOr(error, 1u);
    }
  }
}

cudaError_t launch_locate_points(uint32_t dim, const double* pts, uint32_t n_pts, const Domain& dom, int depth,
                                 const uint64_t* codes, const uint32_t* n_leaves, LeafHash hash, bool root_only,
                                 uint8_t* hit, uint64_t* cand, uint32_t* cand_count, uint32_t cand_cap,
                                 uint32_t* error, cudaStream_t s)
{
  const int grid = int(std::min<uint64_t>(std::max<uint64_t>((n_pts + kThreads - 1) / kThreads, 1), 1024));
  switch (dim) {
    case 1: locate_points_kernel<1><<<grid, kThreads, 0, s>>>(pts, n_pts, dom, depth, codes, n_leaves, hash, root_only, hit, cand, cand_count, cand_cap, error); break;
    case 2: locate_points_kernel<2><<<grid, kThreads, 0, s>>>(pts, n_pts, dom, depth, codes, n_leaves, hash, root_only, hit, cand, cand_count, cand_cap, error); break;
    case 3: locate_points_kernel<3><<<grid, kThreads, 0, s>>>(pts, n_pts, dom, depth, codes, n_leaves, hash, root_only, hit, cand, cand_count, cand_cap, error); break;
    case 4: locate_points_kernel<4><<<grid, kThreads, 0, s>>>(pts, n_pts, dom, depth, codes, n_leaves, hash, root_only, hit, cand, cand_count, cand_cap, error); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// the centre of every source box by rank (kSrcStride doubles a source), for the image
// kernel: its points then read the centre instead of decoding the code and rebuilding
// the box for each point
template<int D>
__global__ void source_centres_kernel(const uint64_t* __restrict__ codes, const uint32_t* __restrict__ src,
                                      const uint32_t* n_src, uint32_t n_all, Domain dom, DepthConst dc, int depth,
                                      double* __restrict__ out)
{
  const uint32_t n = n_src ? *n_src : n_all;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const uint64_t code = __ldg(codes + (src ? __ldg(src + r) : r));
    double c[kSrcStride] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int j = 0; j < D; ++j) {
      double rr;
      box_axis(dom, dc.ax[j], j, deinterleave<D>(code, depth, j), c[j], rr);
    }
    double2* o = reinterpret_cast<double2*>(out + size_t(kSrcStride) * r);
    o[0] = make_double2(c[0], c[1]);
    o[1] = make_double2(c[2], c[3]);
  }
}

// packed keys (pack_bits at `depth`) -> depth-d codes, in place
template<int D>
__global__ void packed_to_codes_kernel(uint64_t* keys, const uint32_t* n_ptr, DepthConst dc, int depth)
{
  const uint32_t n = *n_ptr;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t bits[D];
    unpack_bits_k<D>(keys[i], dc.k, bits);
    int k[D];
#pragma unroll
    for (int j = 0; j < D; ++j) k[j] = dc.k[j];
    keys[i] = interleave<D>(bits, k, depth);
  }
}

template<class F>
cudaError_t by_dim(uint32_t dim, F&& f)
{
  switch (dim) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    default: return cudaErrorInvalidValue;
  }
}

int grid_over(uint64_t n, int per_sm = 8)
{
  const uint64_t want = std::max<uint64_t>((n + kThreads - 1) / kThreads, 1);
  return int(std::min<uint64_t>(want, uint64_t(device_sm_count()) * per_sm));
}

// centres of the boxes codes[src[r]] (codes[r] without a list), r < *n_src (at most
// max_src), at the tree's depth, into t->srcc
b12g_status centres_of(b12g_tree* t, const uint64_t* codes, const uint32_t* src, const uint32_t* n_src,
                       uint32_t max_src)
{
  ST(t->srcc.ensure_room(uint64_t(std::max<uint32_t>(max_src, 1)) * kSrcStride, "source centres", 2));
  DepthConst dc;
  fill_depth_const(t->dom, int(t->domain.dim), t->depth, dc);
  const int g = grid_over(max_src);
  CK(by_dim(t->domain.dim, [&](auto d) {
    source_centres_kernel<decltype(d)::value><<<g, kThreads, 0, t->stream>>>(codes, src, n_src, max_src, t->dom, dc,
                                                                             int(t->depth), t->srcc.p);
    return cudaGetLastError();
  }));
  count_launches(1);
  return B12G_OK;
}

// the source centres of an image launch over n_src sources
b12g_status source_centres(b12g_tree* t, Prepared& pr, uint32_t n_src)
{
  ST(centres_of(t, t->codes(), pr.a.src, pr.a.n_src, n_src));
  pr.a.src_c = t->srcc.p;
  return B12G_OK;
}

// candidates (count in C_CAND) -> sorted unique codes in t->cand2 (count in C_NNEW)
b12g_status sort_unique_candidates(b12g_tree* t, uint32_t m, uint8_t depth, uint32_t* u, bool distinct = false)
{
  *u = 0;
  if (m == 0) return set_ctr(t, C_NNEW, 0);
  if (distinct) {
    // candidates that are distinct already (claimed in the lookup table): the sort alone
    const uint64_t cells = sort_scratch_u32(m);
    ST(t->cand2.ensure(m, "candidate sort"));
    ST(t->sort_idx.ensure(cells + 8, "candidate sort scratch"));
    uint64_t* sorted = nullptr;
    const int bits = std::max(8, ((int(depth) + 7) / 8) * 8);
    // (its error bits go to C_DEFER, read with the next counter read-back)
    CK(radix_sort_u64(t->cand.p, t->cand2.p, t->ctr.p + C_CAND, m, bits, t->sort_idx.p, t->ctr.p + C_DEFER, &sorted,
                      t->stream));
    count_launches(uint64_t(sort_launches(bits)));
    if (sorted == t->cand.p) {     // merge_new reads t->cand2
      std::swap(t->cand.p, t->cand2.p);
      std::swap(t->cand.n, t->cand2.n);
    }
    CK(cudaMemcpyAsync(t->ctr.p + C_NNEW, t->ctr.p + C_CAND, sizeof(uint32_t), cudaMemcpyDeviceToDevice, t->stream));
    *u = m;
    return B12G_OK;
  }
  const uint64_t cells = sort_scratch_u32(m);
  ST(t->cand2.ensure(m, "candidate sort"));
  ST(t->sort_idx.ensure(cells + 2 * (size_t(m) + 1) + compact_tiles(uint64_t(m) + 1) + 8, "candidate sort scratch"));
  uint32_t* scratch = t->sort_idx.p;
  uint32_t* flag = scratch + cells;
  uint32_t* pos = flag + (m + 1);
  uint32_t* tiles = pos + (m + 1);
  uint64_t* sorted = nullptr;
  const int bits = std::max(8, ((int(depth) + 7) / 8) * 8);
  CK(radix_sort_u64(t->cand.p, t->cand2.p, t->ctr.p + C_CAND, m, bits, scratch, t->ctr.p + C_ERROR, &sorted,
                    t->stream));
  uint64_t* other = sorted == t->cand.p ? t->cand2.p : t->cand.p;
  CK(unique_sorted_u64(sorted, t->ctr.p + C_CAND, m, other, t->ctr.p + C_NNEW, flag, pos, tiles, t->stream));
  count_launches(uint64_t(sort_launches(bits)) + 5);
  ST(check_error(t, "candidate sort"));
  ST(read_ctr(t, C_NNEW, 1));
  *u = t->h_ctr[C_NNEW];
  // the unique codes must end up in t->cand2 for merge_new
  if (other != t->cand2.p)
    CK(cudaMemcpyAsync(t->cand2.p, other, size_t(*u) * 8, cudaMemcpyDeviceToDevice, t->stream));
  return B12G_OK;
}

// merge the u unique new codes of t->cand2 into the leaves with flags `ins`; the old
// leaves' flags are ANDed with `a_keep`
b12g_status merge_new(b12g_tree* t, uint32_t u, uint8_t ins, uint8_t a_keep = 0xFF, bool wait = true)
{
  if (u == 0) return B12G_OK;
  const uint64_t total = uint64_t(t->n) + u;
  ST(reserve(t, total));
  const int o = 1 - t->cur, no = 1 - t->ncur;
  CK(merge_sorted(t->codes(), t->flg(), t->dn(), a_keep, t->cand2.p, ins, t->ctr.p + C_NNEW, uint32_t(total),
                  t->code[o].p, t->flags[o].p, t->ctr.p + no, t->stream));
  count_launches(1);
  if (wait) ST(sync(t, "merge"));
  t->cur = o;
  ++t->leaf_gen;
  t->ncur = no;
  t->n = uint32_t(total);
  ++t->leaf_gen;
  return B12G_OK;
}

b12g_status ensure_candidates(b12g_tree* t, uint64_t m)
{
  if (m > 0xFFFFFFF0ull) return fail(B12G_ERR_CAPACITY, "more than 2^32 candidate boxes in one insert");
  ST(t->cand.ensure(std::max<uint64_t>(m, 256), "insert candidates"));
  return B12G_OK;
}

// hit flags of leaves that were hit (and not newly inserted)
b12g_status apply_hit_flags(b12g_tree* t, uint8_t hit_flags)
{
  if (!hit_flags) return B12G_OK;
  CK(apply_hits(t->flg(), t->hit.p, t->dn(), hit_flags, t->ctr.p + C_CHANGED, t->n, t->stream));
  count_launches(1);
  return B12G_OK;
}

b12g_status insert_points_impl(b12g_tree* t, const double* points, uint64_t n_points, uint8_t depth, uint8_t ins,
                               uint8_t hit_flags, uint32_t* n_inserted)
{
  if (!t || (!points && n_points)) return fail(B12G_ERR_INVALID, "NULL argument");
  if (n_points > 0xFFFFFFF0ull) return fail(B12G_ERR_CAPACITY, "too many points");
  if (depth > 64 && depth != B12G_LEAF_DEPTH) return fail(B12G_ERR_INVALID, "depth above 64");
  if (depth == 0) {
    // the surrounding box always exists: only flagsForHit (ImplicitBoxTree.hpp:1625-1640)
    if (hit_flags && n_points) {
      // any point inside the domain hits the root
      ST(ensure_candidates(t, n_points));
      ST(set_ctr(t, C_CAND, 0));
      ST(t->points.ensure(n_points * t->domain.dim, "points"));
      CK(cudaMemcpyAsync(t->points.p, points, n_points * t->domain.dim * 8, cudaMemcpyHostToDevice, t->stream));
      CK(launch_locate_points(t->domain.dim, t->points.p, uint32_t(n_points), t->dom, 0, t->codes(), t->dn(),
                              LeafHash{nullptr, 0, 0}, true, nullptr, t->cand.p, t->ctr.p + C_CAND,
                              uint32_t(t->cand.n), t->ctr.p + C_ERROR, t->stream));
      ST(read_ctr(t, C_CAND, 1));
      if (t->h_ctr[C_CAND] > 0) ST(flag_call(t, 0, 0, hit_flags, 0, nullptr));
    }
    if (n_inserted) *n_inserted = 0;
    return B12G_OK;
  }
  const bool root_only = t->n == 1 && t->depth == 0;
  if (t->mixed || depth == B12G_LEAF_DEPTH || (root_only && t->domain.dim >= 2) || (!root_only && depth != t->depth)) {
    // new boxes may nest in or around leaves: the reference's general insert
    ST(mixed_point_boxes(t, points, n_points));
    return mixed_insert_boxes(t, n_points, depth, ins, hit_flags, n_inserted);
  }
  uint32_t u = 0;
  if (n_points) {
    ST(ensure_candidates(t, n_points));
    ST(set_ctr(t, C_CAND, 0));
    ST(t->points.ensure(n_points * t->domain.dim, "points"));
    CK(cudaMemcpyAsync(t->points.p, points, n_points * t->domain.dim * 8, cudaMemcpyHostToDevice, t->stream));
    Prepared pr;
    pr.a.hash = LeafHash{nullptr, 0, 0};
    if (!root_only) ST(build_current_hash(t, pr));
    CK(launch_locate_points(t->domain.dim, t->points.p, uint32_t(n_points), t->dom, depth, t->codes(), t->dn(),
                            pr.a.hash, root_only, hit_flags ? t->hit.p : nullptr, t->cand.p, t->ctr.p + C_CAND,
                            uint32_t(t->cand.n), t->ctr.p + C_ERROR, t->stream));
    count_launches(1);
    ST(read_ctr(t, C_CAND, 1));
    ST(check_error(t, "insert_points"));
    const uint32_t m = t->h_ctr[C_CAND];
    if (!root_only) ST(apply_hit_flags(t, hit_flags));
    ST(sort_unique_candidates(t, m, depth, &u));
  }
  if (root_only) {
    // the surrounding box shares its path with every box and merges into the one new
    // box, which keeps the union of both flags (ImplicitBoxTree.hpp:1878-1897)
    if (u == 0) {
      if (n_inserted) *n_inserted = 0;
      return B12G_OK;
    }
    if (u > 1)
      return fail(B12G_ERR_UNSUPPORTED_MIXED_DEPTH,
                  "inserting %u distinct boxes into the surrounding box alone (the reference merges them)", u);
    uint8_t root_flags = 0;
    CK(cudaMemcpyAsync(&root_flags, t->flg(), 1, cudaMemcpyDeviceToHost, t->stream));
    ST(sync(t, "root flags"));
    CK(cudaMemcpyAsync(t->codes(), t->cand2.p, 8, cudaMemcpyDeviceToDevice, t->stream));
    CK(cudaMemsetAsync(t->flg(), uint8_t(ins | root_flags), 1, t->stream));
    t->depth = depth;
    ++t->leaf_gen;
    ST(set_ctr(t, t->ncur, 1));
    ST(sync(t, "insert into the surrounding box"));
    if (n_inserted) *n_inserted = 1;
    return B12G_OK;
  }
  ST(merge_new(t, u, ins));
  if (n_inserted) *n_inserted = u;
  return B12G_OK;
}

// A lookup table kept across the sweeps of a continuation: built for n leaves with
// 2^l >= 4n slots (at least 2^16), it takes each sweep's new boxes as the image kernel
// finds them (claimed: marked present only, since the insertion asks whether an image
// box is a leaf, not which one), so the candidates come out distinct; a sweep that at
// most doubles the count leaves it at most half full.  It is rebuilt when the leaf count
// asks for a larger one, or one size up when a claim found no free slot.
struct PresenceTable {
  LeafHash h{};
  uint32_t l = 0;       // log2 of the table's slots
  uint32_t extra = 0;   // sizes added after a full table
  bool ok = false;
};

uint32_t presence_log2(uint32_t n, uint32_t extra)
{
  return std::max<uint32_t>(host_hash_log2(2ull * std::max<uint32_t>(n, 1)), 16) + extra;
}

b12g_status build_presence_table(b12g_tree* t, PresenceTable* keep)
{
  const uint32_t l = presence_log2(t->n, keep->extra);
  ST(ensure_hash(t, uint64_t(1) << (l - 1)));      // >= 2^l slots
  uint32_t tag = 0;
  ST(next_hash_tag(t, &tag));
  keep->h = LeafHash{t->hash.p, tag, t->hash_log2, t->pk.p, l};
  CK(build_leaf_hash(t->codes(), t->dn(), int(t->depth), int(t->domain.dim), keep->h, t->ctr.p + C_ERROR, t->n,
                     t->stream));
  count_launches(1);
  keep->h.pk = nullptr;      // leaf indices move with every merge
  keep->l = l;
  keep->ok = true;
  return B12G_OK;
}

// the error bits C_DEFER collected (host copy read): a timeout or capacity failure of the
// launch that set them
b12g_status deferred_errors(b12g_tree* t)
{
  const uint32_t e = t->h_ctr[C_DEFER];
  if (!e) return B12G_OK;
  set_ctr(t, C_DEFER, 0);
  if (e & 2u) return fail(B12G_ERR_TIMEOUT, "candidate sort: a bounded device wait gave up");
  return fail(B12G_ERR_CAPACITY, "candidate sort: inconsistent digit counts");
}

// The image kernel in Insert mode over `points` points of the prepared sources (their
// centres at pr.a.src_c), run again with more room when a buffer overflows; the
// candidates end as depth-d codes in t->cand, *m of them (also at C_CAND).  With `keep`
// (pr.a.claim set) they are distinct new boxes, claimed in its table.
b12g_status image_candidates(b12g_tree* t, const b12g_scheme* sc, Prepared& pr, uint64_t points, uint8_t depth,
                             uint8_t hit_flags, PresenceTable* keep, uint32_t* m_out)
{
  // room for every point to be a new box; grows (and the images are recomputed) on overflow
  uint64_t cap = std::min<uint64_t>(points, std::max<uint64_t>(uint64_t(t->cand.n), uint64_t(1) << 20));
  for (int attempt = 0; attempt < 8; ++attempt) {
    ST(ensure_candidates(t, cap));
    ST(set_ctr(t, C_CAND, 0));
    pr.a.cand = t->cand.p;
    pr.a.cand_count = t->ctr.p + C_CAND;
    pr.a.cand_cap = uint32_t(std::min<size_t>(t->cand.n, 0xFFFFFFFFu));
    pr.a.hit = hit_flags ? t->hit.p : nullptr;
    prof_mark(t, 0);
    CK(launch_image(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, ImageMode::Insert, pr.a, points,
                    t->stream));
    prof_mark(t, 0);
    count_launches(1);
    // one read-back: the error word, the candidate count, and the deferred error bits of
    // the launches before
    ST(read_ctr(t, C_ERROR, C_DEFER - C_ERROR + 1));
    ST(prof_collect(t));
    ST(deferred_errors(t));
    const uint32_t m = t->h_ctr[C_CAND];
    if (t->h_ctr[C_ERROR] & 1u) {
      ST(set_ctr(t, C_ERROR, 0));
      if (keep) {
        // the failed launch claimed boxes it did not keep: a fresh table, one size up if
        // a claim found it full
        if (m <= pr.a.cand_cap) ++keep->extra;
        ST(build_presence_table(t, keep));
        pr.a.hash = keep->h;
      }
      cap = std::min<uint64_t>(points, std::max<uint64_t>(uint64_t(m), cap * 2));
      continue;
    }
    if (m > 0) {
      // the image kernel appends packed keys: codes for the sort and the merge
      DepthConst dc;
      fill_depth_const(t->dom, int(t->domain.dim), int(depth), dc);
      const int g = grid_over(m);
      CK(by_dim(t->domain.dim, [&](auto d) {
        packed_to_codes_kernel<decltype(d)::value><<<g, kThreads, 0, t->stream>>>(t->cand.p, t->ctr.p + C_CAND, dc,
                                                                                 int(depth));
        return cudaGetLastError();
      }));
      count_launches(1);
    }
    ST(apply_hit_flags(t, hit_flags));
    *m_out = m;
    return B12G_OK;
  }
  return fail(B12G_ERR_CAPACITY, "insert_by_image: candidate buffer retries exhausted");
}

b12g_status insert_by_image_impl(b12g_tree* t, const b12g_scheme* sc, uint8_t depth, uint8_t ins, uint8_t hit_flags,
                                 uint32_t* n_inserted, PresenceTable* keep = nullptr)
{
  if (!t || !sc) return fail(B12G_ERR_INVALID, "NULL argument");
  if (depth == 0) return fail(B12G_ERR_UNSUPPORTED_MIXED_DEPTH, "insertion of images at depth 0");
  if (depth > 64 && depth != B12G_LEAF_DEPTH) return fail(B12G_ERR_INVALID, "depth above 64");
  if (t->mixed || depth == B12G_LEAF_DEPTH || depth != t->depth || t->depth == 0 ||
      (sc->depth != B12G_LEAF_DEPTH && sc->depth != t->depth)) {
    // new boxes may nest in or around leaves: the reference's general insert of the
    // images of the scheme's source leaves (sources at the leaf depth)
    b12g_scheme s = *sc;
    if (!t->mixed && s.depth == t->depth) s.depth = B12G_LEAF_DEPTH;
    uint64_t np = 0;
    ST(mixed_image_boxes(t, &s, &np));
    return mixed_insert_boxes(t, np, depth, ins, hit_flags, n_inserted);
  }
  Prepared pr;
  ST(prepare(t, sc, pr));
  uint32_t n_src = 0;
  ST(select_sources(t, sc, pr, n_src));
  const uint64_t points = uint64_t(n_src) * pr.P;
  if (points == 0) {
    if (n_inserted) *n_inserted = 0;
    return B12G_OK;
  }
  const bool claim = keep && !hit_flags && t->depth <= kHashMaxDepth && t->domain.dim >= 2 && t->n > 0;
  if (claim) {
    if (!keep->ok || keep->l != presence_log2(t->n, keep->extra)) ST(build_presence_table(t, keep));
    pr.a.hash = keep->h;
    pr.a.claim = 1;
  } else {
    ST(build_current_hash(t, pr));
  }
  ST(source_centres(t, pr, n_src));
  uint32_t m = 0, u = 0;
  ST(image_candidates(t, sc, pr, points, depth, hit_flags, claim ? keep : nullptr, &m));
  ST(sort_unique_candidates(t, m, depth, &u, claim));
  ST(merge_new(t, u, ins));          // (claimed boxes are in the table already)
  if (n_inserted) *n_inserted = u;
  return B12G_OK;
}

// One sweep of the continuation on a tree of one depth whose sources are given by their
// centres (t->srcc, n_src of them: the boxes the sweep before inserted, which carry INS
// and no other leaf does): the images of their points claim the new boxes in the kept
// presence table, the new boxes are sorted and merged in with INS while every old leaf
// loses INS and EXPD, and their centres become the next sweep's sources.  This is
// changeFlags(INS -> EXPD), insert(scheme of the EXPD boxes, INS) and unsetFlags(EXPD)
// with the flag passes folded into the merge; a sweep that inserts nothing leaves the
// flags to the caller.
b12g_status continuation_sweep(b12g_tree* t, const b12g_scheme* sc, uint8_t depth, PresenceTable* keep,
                               uint32_t n_src, uint32_t* u_out)
{
  *u_out = 0;
  Prepared pr;
  ST(prepare(t, sc, pr));
  const uint64_t points = uint64_t(n_src) * pr.P;
  if (points == 0) return B12G_OK;
  ST(set_ctr(t, C_NSRC, n_src));
  pr.a.src = nullptr;
  pr.a.n_src = t->ctr.p + C_NSRC;
  pr.a.src_c = t->srcc.p;
  if (!keep->ok || keep->l != presence_log2(t->n, keep->extra)) ST(build_presence_table(t, keep));
  pr.a.hash = keep->h;
  pr.a.claim = 1;
  uint32_t m = 0, u = 0;
  ST(image_candidates(t, sc, pr, points, depth, 0, keep, &m));
  ST(sort_unique_candidates(t, m, depth, &u, true));
  ST(merge_new(t, u, B12G_INS, uint8_t(~(B12G_INS | B12G_EXPD)), false));
  if (u > 0) ST(centres_of(t, t->cand2.p, nullptr, t->ctr.p + C_NNEW, u));
  *u_out = u;
  return B12G_OK;
}

// ---------------------------------------------------------------------------------
// Continuation over a bitmap of every box of the depth (depth <= kBitmapMaxDepth: at most
// 2^30 bits, 128 MB; 2 MB at depth 24, resident in L2): bit c is set when the box of
// code c is a leaf.  A sweep is one image launch in Mark mode over the boxes the sweep
// before added: an image box whose bit it sets first is new and is marked in a second
// bitmap too, whose set bits, read in code order, are the next sweep's sources (in leaf
// order, as the reference iterates them, which fixes each point's index in the grid).
// Nothing is sorted or merged while the sweeps run; the sorted leaves are the set bits
// in code order, written once at the end.
// ---------------------------------------------------------------------------------
constexpr int kBitmapMaxDepth = 30;

__global__ void set_bits_kernel(const uint64_t* __restrict__ codes, const uint32_t* n_ptr, uint32_t* bits)
{
  const uint32_t n = *n_ptr;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint64_t c = codes[i];
    atomicOr(bits + (c >> 5), 1u << uint32_t(c & 31u));
  }
}

// Bitmap compaction: a count of set bits per tile of kWordTile words; the tiles' first
// positions (each tile sums the counts before it when there are at most kLocalTiles
// tiles, else a scan of the counts); then every tile scans its words and writes the
// codes of its set bits in order, with flags when asked (f where a second bitmap has the
// bit, else 0), clearing its words when asked.
constexpr uint32_t kWordTile = 1024;
constexpr int kWordsPerThread = kWordTile / kThreads;   // 4
constexpr uint32_t kLocalTiles = 4096;

__device__ __forceinline__ uint32_t block_sum_u32(uint32_t v, uint32_t* red)
{
  for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, d);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  uint32_t t = 0;
  for (int w = 0; w < kThreads / 32; ++w) t += red[w];
  __syncthreads();
  return t;
}

__global__ void __launch_bounds__(kThreads) tile_count_kernel(const uint32_t* __restrict__ bits, uint32_t words,
                                                              uint32_t* __restrict__ tile_count)
{
  __shared__ uint32_t red[kThreads / 32];
  const uint32_t tiles = (words + kWordTile - 1) / kWordTile;
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    uint32_t c = 0;
    for (uint32_t w = t * kWordTile + threadIdx.x; w < min(words, (t + 1) * kWordTile); w += kThreads)
      c += __popc(bits[w]);
    c = block_sum_u32(c, red);
    if (threadIdx.x == 0) tile_count[t] = c;
  }
}

// tile_first: the tiles' first positions (a scan of the counts), or nullptr: summed here
__global__ void __launch_bounds__(kThreads) tile_scatter_kernel(uint32_t* __restrict__ bits, uint32_t words,
                                                                const uint32_t* __restrict__ tile_count,
                                                                const uint32_t* __restrict__ tile_first,
                                                                uint64_t* __restrict__ out, int clear,
                                                                const uint32_t* __restrict__ mark,
                                                                uint8_t* __restrict__ flags, uint8_t f)
{
  __shared__ uint32_t red[kThreads / 32];
  __shared__ uint32_t wsum[kThreads / 32];
  const uint32_t tiles = (words + kWordTile - 1) / kWordTile;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    uint32_t before = 0;
    if (tile_first) {
      before = tile_first[t];
    } else {
      for (uint32_t q = threadIdx.x; q < t; q += kThreads) before += tile_count[q];
      before = block_sum_u32(before, red);
    }
    // thread i holds words t*kWordTile + 4i .. 4i+3
    const uint32_t w0 = t * kWordTile + threadIdx.x * kWordsPerThread;
    uint32_t v[kWordsPerThread];
    uint32_t c = 0;
#pragma unroll
    for (int q = 0; q < kWordsPerThread; ++q) {
      v[q] = w0 + q < words ? bits[w0 + q] : 0u;
      c += __popc(v[q]);
    }
    uint32_t x = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
      if (lane >= d) x += y;
    }
    if (lane == 31) wsum[wp] = x;
    __syncthreads();
    uint32_t p = before + x - c;
    for (int q = 0; q < wp; ++q) p += wsum[q];
#pragma unroll
    for (int q = 0; q < kWordsPerThread; ++q) {
      uint32_t b = v[q];
      const uint32_t mk = (mark && b) ? mark[w0 + q] : 0u;
      while (b) {
        const int bit = __ffs(b) - 1;
        out[p] = (uint64_t(w0 + q) << 5) | uint64_t(bit);
        if (flags) flags[p] = ((mk >> bit) & 1u) ? f : uint8_t(0);
        ++p;
        b &= b - 1u;
      }
      if (clear && v[q]) bits[w0 + q] = 0u;
    }
    __syncthreads();
  }
}

// the codes of the set bits of `bits` (words u32) in increasing order into `out`, and
// flags into `flags` when not null (f where `mark` has the bit); clears the bitmap when
// asked
b12g_status bitmap_codes(b12g_tree* t, uint32_t* bits, uint32_t words, uint64_t* out, bool clear,
                         const uint32_t* mark = nullptr, uint8_t* flags = nullptr, uint8_t f = 0)
{
  const uint32_t tiles = (words + kWordTile - 1) / kWordTile;
  ST(t->sort_idx.ensure(2 * (size_t(tiles) + 1) + compact_tiles(uint64_t(tiles) + 1) + 8, "bitmap tile counts"));
  uint32_t* count = t->sort_idx.p;
  uint32_t* first = nullptr;
  const int g = int(std::min<uint64_t>(tiles, uint64_t(device_sm_count()) * 8));
  tile_count_kernel<<<g, kThreads, 0, t->stream>>>(bits, words, count);
  CK(cudaGetLastError());
  count_launches(1);
  if (tiles > kLocalTiles) {
    first = count + tiles + 1;
    ST(set_ctr(t, C_TMP, tiles));
    CK(exclusive_scan_u32(count, first, t->ctr.p + C_TMP, first + tiles + 1, tiles, t->stream));
    count_launches(3);
  }
  tile_scatter_kernel<<<g, kThreads, 0, t->stream>>>(bits, words, count, first, out, clear ? 1 : 0, mark, flags, f);
  CK(cudaGetLastError());
  count_launches(1);
  return B12G_OK;
}

// the sweeps of continuation.m:29-44 on a tree of one depth whose leaves all carry INS
// (the boxes of the start points); leaves the tree as the flag passes would: every
// leaf's flags 0, except INS on the last sweep's new boxes when max_sweeps ended the run
b12g_status continuation_bitmap(b12g_tree* t, const b12g_scheme* s, uint8_t depth, uint32_t max_sweeps,
                                uint32_t* counts, uint32_t* n_sweeps)
{
  const uint64_t boxes = uint64_t(1) << depth;
  const uint32_t words = uint32_t(std::max<uint64_t>(boxes >> 5, 1));
  ST(t->bits.ensure(2 * size_t(words), "box bitmaps"));
  uint32_t* bits = t->bits.p;            // every leaf
  uint32_t* fresh = t->bits.p + words;   // the boxes the running sweep adds
  CK(cudaMemsetAsync(t->bits.p, 0, 2 * size_t(words) * 4, t->stream));
  set_bits_kernel<<<grid_over(t->n), kThreads, 0, t->stream>>>(t->codes(), t->dn(), bits);
  CK(cudaGetLastError());
  count_launches(1);
  ST(centres_of(t, t->codes(), nullptr, t->dn(), t->n));   // the first sources: every leaf
  Prepared pr;
  ST(prepare(t, s, pr));
  pr.a.src = nullptr;
  pr.a.n_src = nullptr;
  pr.a.bits = bits;
  pr.a.fresh = fresh;
  pr.a.cand_count = t->ctr.p + C_CAND;
  uint64_t n = t->n;
  uint32_t n_src = t->n, u = 0, k = 0, nb0 = 0, nb1 = t->n;
  while (nb1 > nb0 && k < max_sweeps) {
    const uint64_t points = uint64_t(n_src) * pr.P;
    ST(set_ctr(t, C_CAND, 0));
    pr.a.n_src_value = n_src;
    pr.a.src_c = t->srcc.p;
    u = 0;
    if (points > 0) {
      prof_mark(t, 0);
      CK(launch_image(s->map.kind, s->map.arith, s->grid.kind, t->domain.dim, ImageMode::Mark, pr.a, points,
                      t->stream));
      prof_mark(t, 0);
      count_launches(1);
      ST(read_ctr(t, C_ERROR, C_DEFER - C_ERROR + 1));
      ST(prof_collect(t));
      if (t->h_ctr[C_ERROR]) {
        set_ctr(t, C_ERROR, 0);
        return fail(B12G_ERR_CAPACITY, "continuation: device error bits %u", t->h_ctr[C_ERROR]);
      }
      u = t->h_ctr[C_CAND];
      if (u > 0) {
        // the next sources: the new boxes in code order, their codes and centres
        // (the centres by a thread per box: inside the compaction's loop over a word's
        // bits they would serialise, 1.9 ms against 0.95 ms for the run's compactions and
        // centres apart)
        ST(t->cand.ensure_room(u, "new boxes", 2));
        ST(bitmap_codes(t, fresh, words, t->cand.p, true));
        ST(centres_of(t, t->cand.p, nullptr, t->ctr.p + C_CAND, u));
      }
    }
    n += u;
    n_src = u;
    nb0 = nb1;
    nb1 = uint32_t(n);
    if (counts) counts[k] = nb1;
    ++k;
  }
  *n_sweeps = k;
  if (k == 0) return B12G_OK;
  // the leaves: the set bits in code order; flags 0, INS on the last sweep's new boxes
  // when max_sweeps ended the run while boxes were still being added
  ST(reserve(t, n));
  const int o = 1 - t->cur, no = 1 - t->ncur;
  if (u > 0) {
    set_bits_kernel<<<grid_over(u), kThreads, 0, t->stream>>>(t->cand.p, t->ctr.p + C_CAND, fresh);
    CK(cudaGetLastError());
    count_launches(1);
  }
  ST(bitmap_codes(t, bits, words, t->code[o].p, false, u > 0 ? fresh : nullptr, t->flags[o].p, B12G_INS));
  ST(set_ctr(t, no, uint32_t(n)));
  ST(sync(t, "continuation leaves"));
  t->cur = o;
  t->ncur = no;
  t->n = uint32_t(n);
  ++t->leaf_gen;
  return B12G_OK;
}

}  // namespace

extern "C" {

b12g_status b12g_insert_points(b12g_tree* t, const double* points, uint64_t n_points, uint8_t depth,
                               uint8_t flags_for_inserted, uint8_t flags_for_hit, uint32_t* n_inserted)
{
  return insert_points_impl(t, points, n_points, depth, flags_for_inserted, flags_for_hit, n_inserted);
}

b12g_status b12g_insert_by_image(b12g_tree* t, const b12g_scheme* sc, uint8_t depth, uint8_t flags_for_inserted,
                                 uint8_t flags_for_hit, uint32_t* n_inserted)
{
  return insert_by_image_impl(t, sc, depth, flags_for_inserted, flags_for_hit, n_inserted);
}

// continuation.m:13-44 at one depth
b12g_status b12g_continuation_run(b12g_tree* t, const b12g_scheme* sc, const double* x0, uint64_t n_x0,
                                  uint8_t depth, uint32_t max_sweeps, uint32_t* counts, uint32_t* n_sweeps)
{
  if (!t || !sc || !x0) return fail(B12G_ERR_INVALID, "NULL argument");
  ST(set_root(t, B12G_NONE));                                               // deleteDepth(0)
  ST(insert_points_impl(t, x0, n_x0, depth, B12G_INS, B12G_NONE, nullptr));  // insert(points, d, INS)
  b12g_scheme s = *sc;
  s.depth = depth;
  s.flags_to_check = B12G_EXPD;                                             // {grid, map, d, EXPD}
  uint32_t nb0 = 0, nb1 = t->depth == depth ? t->n : 0;
  uint32_t k = 0;
  if (nb1 > 0 && !t->mixed && depth <= kBitmapMaxDepth && t->domain.dim >= 2) {
    ST(continuation_bitmap(t, &s, depth, max_sweeps, counts, &k));
    if (n_sweeps) *n_sweeps = k;
    return B12G_OK;
  }
  PresenceTable keep;
  // a tree of one depth (every leaf carries INS after the insertion): the sweeps take
  // their sources from the boxes the sweep before inserted
  const bool fast = nb1 > 0 && !t->mixed && depth <= kHashMaxDepth && t->domain.dim >= 2;
  uint32_t n_src = 0;
  if (fast) {
    ST(centres_of(t, t->codes(), nullptr, t->dn(), t->n));
    n_src = t->n;
  }
  while (nb1 > nb0 && k < max_sweeps) {
    if (fast) {
      uint32_t u = 0;
      ST(continuation_sweep(t, &s, depth, &keep, n_src, &u));
      // nothing new: the sources lose INS (and EXPD) as the flag passes would have it
      if (u == 0) ST(flag_call(t, 1, 0, uint8_t(B12G_INS | B12G_EXPD), B12G_LEAF_DEPTH, nullptr));
      n_src = u;
    } else {
      ST(flag_call(t, 2, B12G_INS, B12G_EXPD, depth, nullptr));              // changeFlags('all', INS, EXPD, d)
      ST(insert_by_image_impl(t, &s, depth, B12G_INS, B12G_NONE, nullptr, &keep));   // insert(scheme, d, INS, NONE)
      ST(flag_call(t, 1, 0, B12G_EXPD, B12G_LEAF_DEPTH, nullptr));           // unsetFlags('all', EXPD)
    }
    nb0 = nb1;
    nb1 = t->n;
    if (counts) counts[k] = nb1;
    ++k;
  }
  // the last sweep's sort and merge ran without a read-back
  ST(read_ctr(t, C_ERROR, C_DEFER - C_ERROR + 1));
  ST(deferred_errors(t));
  if (n_sweeps) *n_sweeps = k;
  return B12G_OK;
}

}  // extern "C"
