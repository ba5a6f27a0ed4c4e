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
#include "sort.h"
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

// The leaves' comparable patterns with a prefix table: tab[v] is the first leaf whose
// pattern is at least v << (64 - bits), tab[2^bits] = n, so the lower bound of a key lies
// between tab[v] and tab[v + 1] for v = key >> (64 - bits).
struct CmpIndex {
  const uint64_t* cmp;
  const uint32_t* tab;
  uint32_t n;
  uint32_t bits;               // 1..24
};

// first leaf whose comparable pattern is not below `key`
__device__ __forceinline__ uint32_t lower_bound_idx(const CmpIndex& ix, uint64_t key)
{
  const uint32_t v = uint32_t(key >> (64 - ix.bits));
  uint32_t lo = __ldg(ix.tab + v);
  uint32_t len = __ldg(ix.tab + v + 1) - lo;
  while (len > 0) {
    const uint32_t half = len >> 1;
    if (__ldg(ix.cmp + lo + half) < key) {
      lo += half + 1;
      len -= half + 1;
    } else {
      len = half;
    }
  }
  return lo;
}

// search of one point among the leaves (ImplicitBoxTree.hpp:2394-2432, leaf branch)
__device__ __forceinline__ uint32_t locate_mixed(const CmpIndex& ix, const uint64_t* __restrict__ code,
                                                 const uint8_t* __restrict__ dep, bool valid, uint64_t p64)
{
  const uint32_t n = ix.n;
  if (n == 0) return kInvalidIndex;
  if (!valid) {
    // the invalid box shares its path with a last leaf of code 0
    return __ldg(code + n - 1) == 0 ? n - 1 : kInvalidIndex;
  }
  // lower bound: first leaf that does not strictly precede the depth-64 point box
  const uint32_t lo = lower_bound_idx(ix, p64);
  const uint32_t a = lo > 0 ? lo - 1 : 0;
  const uint32_t b = lo < n - 1 ? lo : n - 1;
  if (on_path(p64, __ldg(code + a), __ldg(dep + a))) return lo > 0 ? lo - 1 : 0;
  if (on_path(p64, __ldg(code + b), __ldg(dep + b))) return lo;
  return kInvalidIndex;
}

// the prefix table of CmpIndex, 2^bits + 1 entries
__global__ void cmp_table_kernel(const uint64_t* cmp, uint32_t n, uint32_t bits, uint32_t* tab)
{
  const uint32_t entries = (1u << bits) + 1u;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < entries; v += gridDim.x * blockDim.x) {
    if (v == entries - 1) {
      tab[v] = n;
      continue;
    }
    const uint64_t key = uint64_t(v) << (64 - bits);
    uint32_t lo = 0, len = n;
    while (len > 0) {
      const uint32_t half = len >> 1;
      if (cmp[lo + half] < key) {
        lo += half + 1;
        len -= half + 1;
      } else {
        len = half;
      }
    }
    tab[v] = lo;
  }
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

// ---- flags of the boxes at an inner depth d: a box is a run of leaves at least d deep
// with one d-prefix; head[i] marks the run's first leaf, and after a scan pos[i + 1] - 1
// is the box of leaf i
__global__ void box_head_kernel(const uint64_t* code, const uint8_t* dep, uint32_t n, uint32_t d, uint32_t* head)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    bool fresh = false;
    if (dep[i] >= d) {
      fresh = i == 0 || dep[i - 1] < d;
      if (!fresh) fresh = (code[i - 1] >> (dep[i - 1] - d)) != (code[i] >> (dep[i] - d));
    }
    head[i] = fresh ? 1u : 0u;
  }
}

// every box's AND and OR of its leaves' flags (box_and starts all ones, box_or zero)
__global__ void box_combine_kernel(const uint8_t* flags, const uint8_t* dep, uint32_t n, uint32_t d,
                                   const uint32_t* pos, uint32_t* box_and, uint32_t* box_or)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (dep[i] < d) continue;
    const uint32_t b = pos[i + 1] - 1;
    atomicAnd(box_and + b, uint32_t(flags[i]));
    atomicOr(box_or + b, uint32_t(flags[i]));
  }
}

// op 0: setFlags (boxes whose AND lacked f), 1: unsetFlags (boxes whose OR had any of f),
// 2: changeFlags (boxes whose AND has all of u: their leaves change); counts those boxes
__device__ __forceinline__ bool box_selected(int op, uint32_t all, uint32_t any, uint8_t u, uint8_t f)
{
  if (op == 0) return (all & f) != f;
  if (op == 1) return (any & f) != 0;
  return (all & u) == u;
}

__global__ void box_apply_kernel(uint8_t* flags, const uint8_t* dep, uint32_t n, uint32_t d, const uint32_t* pos,
                                 const uint32_t* box_and, const uint32_t* box_or, uint32_t n_boxes, int op, uint8_t u,
                                 uint8_t f, uint32_t* count)
{
  uint32_t c = 0;
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < n_boxes; b += gridDim.x * blockDim.x)
    c += box_selected(op, box_and[b], box_or[b], u, f);
  if (c) atomicAdd(count, c);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (dep[i] < d) continue;
    const uint8_t x = flags[i];
    if (op == 0) flags[i] = x | f;
    else if (op == 1) flags[i] = x & uint8_t(~f);
    else {
      const uint32_t b = pos[i + 1] - 1;
      if (box_selected(2, box_and[b], box_or[b], u, f)) flags[i] = uint8_t(x & uint8_t(~u)) | f;
    }
  }
}

// flags f on every leaf of the boxes marked hit; counts the marked boxes whose leaves did
// not all have f (setFlagsBySearch below the leaves: a stencil over the boxes, then
// setFlagsByStencil, ImplicitBoxTree.hpp:2776-2800, 2805-2882)
__global__ void box_hit_apply_kernel(uint8_t* flags, const uint8_t* dep, uint32_t n, uint32_t d, const uint32_t* pos,
                                     const uint32_t* box_and, const uint8_t* box_hit, uint32_t n_boxes, uint8_t f,
                                     uint32_t* count)
{
  uint32_t c = 0;
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < n_boxes; b += gridDim.x * blockDim.x)
    c += box_hit[b] && (box_and[b] & f) != f;
  if (c) atomicAdd(count, c);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (dep[i] >= d && box_hit[pos[i + 1] - 1]) flags[i] |= f;
}

// every box's AND of its leaves' flags (box_and starts all ones)
__global__ void box_and_kernel(const uint8_t* flags, const uint8_t* dep, uint32_t n, uint32_t d, const uint32_t* pos,
                               uint32_t* box_and)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (dep[i] >= d) atomicAnd(box_and + (pos[i + 1] - 1), uint32_t(flags[i]));
}

// the sources of a scheme at an inner depth (initializeLeafIndicesFromDepth,
// ImplicitBoxTree.hpp:1476-1611): the first leaf of every box whose leaves all have f
__global__ void source_select_kernel(uint32_t* head, const uint32_t* pos, const uint32_t* box_and, uint32_t n, uint8_t f)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (head[i]) head[i] = (box_and[pos[i + 1] - 1] & f) == f ? 1u : 0u;
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

// ---------------------------------------------------------------------------- boxes
// A box as the reference's Box<N> (code, depth, flags); depth above 64 is the invalid box.
struct Bx {
  uint64_t c;
  uint32_t d;
  uint32_t f;
};

__device__ __forceinline__ uint64_t srs(uint64_t b, int i) { return i <= 0 ? b : (i >= 64 ? 0ull : b >> i); }
__device__ __forceinline__ uint64_t sls(uint64_t b, int i) { return i <= 0 ? b : (i >= 64 ? 0ull : b << i); }

__device__ __forceinline__ Bx load_box(const uint64_t* code, const uint8_t* dep, const uint8_t* flags, uint32_t i)
{
  return Bx{code[i], dep[i], flags ? flags[i] : 0u};
}

// hasSamePath (Box.hpp:75-83)
__device__ __forceinline__ bool same_path(const Bx& a, const Bx& b)
{
  const int diff = int(a.d) - int(b.d);
  return (a.d > 64 && b.d > 64) || srs(a.c, diff) == srs(b.c, -diff);
}

// isSameBox (Box.hpp:113-120)
__device__ __forceinline__ bool same_box(const Bx& a, const Bx& b)
{
  return (a.d > 64 && b.d > 64) || (a.c == b.c && a.d == b.d);
}

// isStrictlyPreceding (Box.hpp:124-135)
__device__ __forceinline__ bool precedes(const Bx& a, const Bx& b)
{
  if (a.d > 64) return false;
  if (b.d > 64) return true;
  const uint64_t ka = comparable(a.c, a.d), kb = comparable(b.c, b.d);
  return ka < kb || (ka == kb && b.d < a.d);
}

// ComputeMaxBitPatternMaxDepthOrFlagsFunctor (Functors.hpp:396-401)
__device__ __forceinline__ Bx combine(const Bx& a, const Bx& b)
{
  return Bx{a.c > b.c ? a.c : b.c, a.d > b.d ? a.d : b.d, a.f | b.f};
}

// decrementDepthBy(box, 1) (Box.hpp:151-158)
__device__ __forceinline__ Bx parent_of(Bx b)
{
  if (b.d > 0) {
    b.c = srs(b.c, 1);
    b.d -= 1;
  }
  return b;
}

// computeDepthOfMutualAncestor (Box.hpp:209-223)
__device__ __forceinline__ uint32_t mutual_ancestor(const Bx& a, const Bx& b)
{
  const uint64_t x = sls(a.c, 64 - int(a.d)) ^ sls(b.c, 64 - int(b.d));
  const uint32_t lz = uint32_t(__clzll(x));    // 64 for x == 0
  const uint32_t m = a.d < b.d ? a.d : b.d;
  return lz < m ? lz : m;
}

// changeDepthTo (Box.hpp:180-198) for target depths 0..64
__device__ __forceinline__ Bx change_depth_to(Bx b, uint32_t depth)
{
  if (depth < b.d) {
    b.c = srs(b.c, int(b.d - depth));
    b.d = depth;
  } else if (depth > b.d) {
    if (depth > 64) depth = 64;
    b.c = sls(b.c, int(depth - b.d));
    b.d = depth;
  }
  return b;
}

// unsubdivide, IsUnsubdividableFunctor (Functors.hpp:343-364): marks and their number
__global__ void unsub_mark_kernel(const uint64_t* code, const uint8_t* dep, const uint8_t* flags, uint32_t n, uint8_t f,
                                  uint32_t* mark, uint32_t* count)
{
  uint32_t c = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Bx b = load_box(code, dep, flags, i);
    bool res = uint8_t(b.f & f) == f && b.d > 0;
    if (res) {
      const uint32_t j = (b.c & 1ull) ? (i > 0 ? i - 1 : 0) : (i + 1 < n ? i + 1 : n - 1);
      const Bx nb = load_box(code, dep, flags, j);
      const Bx p = parent_of(b);
      res = same_box(p, parent_of(nb)) ? uint8_t(nb.f & f) == f : !same_path(p, nb);
    }
    mark[i] = res ? 1u : 0u;
    c += res;
  }
  if (c) atomicAdd(count, c);
}

// the marked leaves become their parents; two equal parents keep the first with the AND
// of both flags (the reverse inclusive_scan_by_key and unique of unsubdivide,
// ImplicitBoxTree.hpp:3430-3452; equal boxes come at most in pairs, as leaves are disjoint)
__global__ void unsub_apply_kernel(const uint64_t* code, const uint8_t* dep, const uint8_t* flags, uint32_t n,
                                   const uint32_t* mark, uint64_t* out_code, uint8_t* out_dep, uint8_t* out_flags,
                                   uint32_t* keep)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Bx b = load_box(code, dep, flags, i);
    if (mark[i]) b = parent_of(b);
    uint32_t f = b.f;
    if (i + 1 < n) {
      Bx nx = load_box(code, dep, flags, i + 1);
      if (mark[i + 1]) nx = parent_of(nx);
      if (same_box(nx, b)) f &= nx.f;
    }
    bool first = true;
    if (i > 0) {
      Bx pv = load_box(code, dep, nullptr, i - 1);
      if (mark[i - 1]) pv = parent_of(pv);
      first = !same_box(pv, b);
    }
    out_code[i] = b.c;
    out_dep[i] = uint8_t(b.d);
    out_flags[i] = uint8_t(f);
    keep[i] = first ? 1u : 0u;
  }
}

// the box at the inner depth d around a point (searchByIterators below the leaves,
// ImplicitBoxTree.hpp:2473-2566): it exists when the first leaf at or after the box's
// first address lies inside it; its index is that leaf's box (pos: scan of the box heads
// at d).  A point that left the domain is found in the last leaf's box when that leaf's
// d-prefix is 0, as hasSamePath of the invalid box makes it.
__device__ __forceinline__ uint32_t inner_box_of(const CmpIndex& ix, const uint64_t* __restrict__ code,
                                                 const uint8_t* __restrict__ dep, const uint32_t* __restrict__ pos,
                                                 uint32_t d, bool valid, uint64_t p64)
{
  const uint32_t n = ix.n;
  if (n == 0) return kInvalidIndex;
  uint32_t j;
  bool in;
  if (!valid) {
    j = n - 1;
    in = __ldg(dep + j) >= d && (__ldg(code + j) >> (__ldg(dep + j) - d)) == 0;
  } else {
    const int sh = 64 - int(d);
    const uint64_t q = srs(p64, sh);
    j = lower_bound_idx(ix, sls(q, sh));
    in = j < n && __ldg(dep + j) >= d && srs(__ldg(code + j), int(__ldg(dep + j)) - int(d)) == q;
  }
  return in ? __ldg(pos + j + 1) - 1 : kInvalidIndex;
}

// insertByIterators (ImplicitBoxTree.hpp:1615-1910): the new box of every point box
struct InsertArgs {
  const uint64_t* p64;         // depth-64 point codes
  const uint8_t* valid;        // 0: the point left the domain (the invalid box)
  uint64_t np;
  const uint64_t* code;        // leaves
  const uint8_t* dep;
  const uint64_t* cmp;
  const uint32_t* tab;         // prefix table of cmp (CmpIndex)
  uint32_t tab_bits;
  uint32_t n;
  uint32_t depth;              // insertion depth; 255: the leaf depth
  int mode;                    // 0: leaf depth, 2: below an existing depth, 3: deeper than every leaf
  uint8_t* hit;                // marks of leaves hit (leaf depth, when flags for hit are given)
  const uint32_t* box_pos;     // inner depth: scan of the box heads
  uint8_t* box_hit;            //              marks of the boxes hit (when flags for hit are given)
  uint64_t* out_code;          // new boxes (appended)
  uint8_t* out_dep;
  uint32_t* count;
  uint32_t cap;
  uint32_t* error;
};

__global__ void insert_boxes_kernel(const InsertArgs a)
{
  for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < a.np; k += uint64_t(gridDim.x) * blockDim.x) {
    const bool valid = a.valid[k] != 0;
    const Bx p = valid ? Bx{a.p64[k], 64u, 0u} : Bx{~0ull, 255u, 0u};
    bool to_insert;
    uint32_t lo = 0;
    if (a.mode == 0) {
      // searchByIterators at the leaf depth, then the leaf-depth rule (1672-1702):
      // a point in no leaf is inserted if valid, one in a leaf if that leaf is above depth 64
      lo = valid ? lower_bound_idx(CmpIndex{a.cmp, a.tab, a.n, a.tab_bits}, p.c) : a.n;
      const uint32_t ia = lo > 0 ? lo - 1 : 0, ib = lo < a.n - 1 ? lo : a.n - 1;
      uint32_t s = kInvalidIndex;
      if (same_path(p, load_box(a.code, a.dep, nullptr, ia))) s = lo > 0 ? lo - 1 : 0;
      else if (same_path(p, load_box(a.code, a.dep, nullptr, ib))) s = lo;
      to_insert = s == kInvalidIndex ? valid : a.dep[s] < 64;
      if (!to_insert && s != kInvalidIndex && a.hit) a.hit[s] = 1;
    } else if (a.mode == 2) {
      // the box at the inner depth around the point; its leaves get the flags for hit
      const uint32_t b = inner_box_of(CmpIndex{a.cmp, a.tab, a.n, a.tab_bits}, a.code, a.dep, a.box_pos, a.depth,
                                      valid, p.c);
      if (b != kInvalidIndex && a.box_hit) a.box_hit[b] = 1;
      to_insert = valid && b == kInvalidIndex;
    } else {
      to_insert = valid;
    }
    if (!to_insert) continue;
    Bx b;
    if (a.mode == 0) {
      // AdaptDepthOfFirstBoxFunctor (Functors.hpp:381-389): one below the deepest common
      // ancestor with the two neighbours at the lower bound
      const uint32_t ia = lo > 0 ? lo - 1 : 0, ib = lo < a.n - 1 ? lo : a.n - 1;
      const uint32_t x = mutual_ancestor(p, load_box(a.code, a.dep, nullptr, ia));
      const uint32_t y = mutual_ancestor(p, load_box(a.code, a.dep, nullptr, ib));
      b = change_depth_to(p, (x > y ? x : y) + 1);
    } else {
      b = change_depth_to(p, a.depth);     // decrementDepthTo(depth)
    }
    const uint32_t slot = atomicAdd(a.count, 1u);
    if (slot < a.cap) {
      a.out_code[slot] = b.c;
      a.out_dep[slot] = uint8_t(b.d);
    } else {
      atomicOr(a.error, 1u);
    }
  }
}

// sort keys of the new boxes: deeper first (pass 1), then the comparable pattern
__global__ void depth_key_kernel(const uint8_t* dep, uint32_t m, uint64_t* key, uint32_t* idx)
{
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    key[j] = 255u - dep[j];
    idx[j] = j;
  }
}

__global__ void pattern_key_kernel(const uint64_t* code, const uint8_t* dep, const uint32_t* idx, uint32_t m,
                                   uint64_t* key)
{
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x)
    key[j] = comparable(code[idx[j]], dep[idx[j]]);
}

// distinct new boxes in order: heads of runs of equal boxes (unique with IsSameBoxFunctor)
__global__ void new_heads_kernel(const uint64_t* code, const uint8_t* dep, const uint32_t* idx, uint32_t m,
                                 uint32_t* head)
{
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x)
    head[j] = (j == 0 || code[idx[j]] != code[idx[j - 1]] || dep[idx[j]] != dep[idx[j - 1]]) ? 1u : 0u;
}

__global__ void new_scatter_kernel(const uint64_t* code, const uint8_t* dep, const uint32_t* idx, uint32_t m,
                                   const uint32_t* pos, uint64_t* ucode, uint8_t* udep)
{
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x)
    if (pos[j + 1] != pos[j]) {
      ucode[pos[j]] = code[idx[j]];
      udep[pos[j]] = dep[idx[j]];
    }
}

// sortBoxes of the leaves and the new boxes together (stable: a leaf before an equal
// new box): the merge of two sorted lists by rank
__global__ void merge_boxes_kernel(const uint64_t* code, const uint8_t* dep, const uint8_t* flags, uint32_t n,
                                   const uint64_t* ucode, const uint8_t* udep, uint8_t ins, uint32_t u,
                                   uint64_t* out_code, uint8_t* out_dep, uint8_t* out_flags)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n + u; i += gridDim.x * blockDim.x) {
    if (i < n) {
      const Bx b = load_box(code, dep, flags, i);
      // new boxes strictly before the leaf
      uint32_t lo = 0, len = u;
      while (len > 0) {
        const uint32_t half = len >> 1;
        if (precedes(Bx{ucode[lo + half], udep[lo + half], 0u}, b)) { lo += half + 1; len -= half + 1; }
        else len = half;
      }
      out_code[i + lo] = b.c;
      out_dep[i + lo] = uint8_t(b.d);
      out_flags[i + lo] = uint8_t(b.f);
    } else {
      const uint32_t j = i - n;
      const Bx b{ucode[j], udep[j], ins};
      // leaves not strictly after the new box
      uint32_t lo = 0, len = n;
      while (len > 0) {
        const uint32_t half = len >> 1;
        if (!precedes(b, load_box(code, dep, nullptr, lo + half))) { lo += half + 1; len -= half + 1; }
        else len = half;
      }
      out_code[j + lo] = b.c;
      out_dep[j + lo] = uint8_t(b.d);
      out_flags[j + lo] = ins;
    }
  }
}

// forward inclusive_scan_by_key (ImplicitBoxTree.hpp:1878-1884): runs of adjacent boxes
// on one path, each run walked by the thread of its first box
__global__ void forward_scan_kernel(const uint64_t* code, const uint8_t* dep, const uint8_t* flags, uint32_t total,
                                    uint64_t* fc, uint8_t* fd, uint8_t* ff)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    Bx acc = load_box(code, dep, flags, i);
    if (i > 0 && same_path(load_box(code, dep, nullptr, i - 1), acc)) continue;
    fc[i] = acc.c; fd[i] = uint8_t(acc.d); ff[i] = uint8_t(acc.f);
    Bx prev = acc;
    for (uint32_t j = i + 1; j < total; ++j) {
      const Bx b = load_box(code, dep, flags, j);
      if (!same_path(prev, b)) break;
      acc = combine(acc, b);
      fc[j] = acc.c; fd[j] = uint8_t(acc.d); ff[j] = uint8_t(acc.f);
      prev = b;
    }
  }
}

// reverse scan keyed by the forward scan's output (1886-1892), from each run's last box
__global__ void reverse_scan_kernel(const uint64_t* fc, const uint8_t* fd, const uint8_t* ff, uint32_t total,
                                    uint64_t* rc, uint8_t* rd, uint8_t* rf)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    Bx acc = load_box(fc, fd, ff, i);
    if (i + 1 < total && same_path(load_box(fc, fd, nullptr, i + 1), acc)) continue;
    rc[i] = acc.c; rd[i] = uint8_t(acc.d); rf[i] = uint8_t(acc.f);
    Bx prev = acc;
    for (uint32_t j = i; j-- > 0;) {
      const Bx b = load_box(fc, fd, ff, j);
      if (!same_path(prev, b)) break;
      acc = combine(acc, b);
      rc[j] = acc.c; rd[j] = uint8_t(acc.d); rf[j] = uint8_t(acc.f);
      prev = b;
    }
  }
}

// unique(HasSamePathFunctor) (1894-1897): a box stays unless it shares a path with the one before
__global__ void path_heads_kernel(const uint64_t* code, const uint8_t* dep, uint32_t total, uint32_t* keep)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
    keep[i] = (i == 0 || !same_path(load_box(code, dep, nullptr, i - 1), load_box(code, dep, nullptr, i))) ? 1u : 0u;
}

template<int D>
__global__ void point_codes_kernel(const double* pts, uint64_t np, Domain dom, uint64_t* p64, uint8_t* valid)
{
  for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < np; k += uint64_t(gridDim.x) * blockDim.x) {
    double p[D];
#pragma unroll
    for (int j = 0; j < D; ++j) p[j] = pts[k * D + j];
    uint64_t c = 0;
    valid[k] = point_code<D>(dom, p, 64, c) ? 1 : 0;
    p64[k] = c;
  }
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
  const uint32_t* tab;         // prefix table of cmp (CmpIndex)
  uint32_t tab_bits;
  uint32_t n;                  // leaves
  const uint32_t* src;         // source leaves (nullptr: every leaf)
  uint32_t n_src;
  uint32_t src_depth;          // 0: each source is its leaf; d: the leaf's box at depth d
  uint8_t* hit;                // Hit: marks of the leaves hit
  uint32_t* out;               // Search: leaf index of every point
  uint64_t* p64_out;           // Codes: depth-64 code of every image point
  uint8_t* valid_out;          //        1 if it lies in the domain
  uint32_t* n_out;             // Distinct codes: how many were written (at most p64_cap)
  uint64_t p64_cap;
  uint64_t p64_keep;           //        the bits of a code kept: its first bisections
  const uint32_t* box_pos;     // inner depth: scan of the box heads (box of leaf j: box_pos[j + 1] - 1)
  uint32_t inner_depth;
  uint8_t* box_hit;            //              hit marks of the boxes
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

// the depth-64 code of the image of point k of source leaf `leaf` (point index g);
// false if the image left the domain
template<class Map, class Grid>
__device__ __forceinline__ bool image_code(const MixedArgs& a, const double* pts, bool table, uint32_t leaf,
                                           uint32_t k, uint64_t g, uint64_t& p64)
{
  constexpr int D = Map::D;
  double c[D], r[D], gp[D], x[D], y[D];
  uint64_t code = __ldg(a.code + leaf);
  int depth = int(__ldg(a.dep + leaf));
  if (a.src_depth) {
    // a box of an inner depth, by its first leaf
    code >>= depth - int(a.src_depth);
    depth = int(a.src_depth);
  }
  box_coordinates<D>(a.dom, code, depth, c, r);
  if (Grid::kTable && table) {
#pragma unroll
    for (int j = 0; j < D; ++j) gp[j] = pts[j * uint32_t(a.points) + k];
  } else {
    Grid::template point<D>(a.grid, pts, g, k, gp);
  }
#pragma unroll
  for (int j = 0; j < D; ++j) x[j] = __dadd_rn(c[j], __dmul_rn(gp[j], r[j]));
  Map::apply(a.map, x, y);
  p64 = 0;
  return point_code<D>(a.dom, y, 64, p64);
}

// the leaf the image of point k of source leaf `leaf` lands in (point index g)
template<class Map, class Grid>
__device__ __forceinline__ uint32_t image_of(const MixedArgs& a, const double* pts, bool table, uint32_t leaf,
                                             uint32_t k, uint64_t g)
{
  uint64_t p64;
  const bool valid = image_code<Map, Grid>(a, pts, table, leaf, k, g, p64);
  return locate_mixed(CmpIndex{a.cmp, a.tab, a.n, a.tab_bits}, a.code, a.dep, valid, p64);
}

// kMode 0: hit marks of the leaves hit; 1: leaf index of every point; 2: the points'
// depth-64 codes and validity (the point boxes of an insertion); 3: hit marks of the
// boxes at the inner depth a.inner_depth; 4: box index at that depth of every point;
// 5: the point boxes of mode 2 cut to their first bisections (a.p64_keep), each distinct
// (code, validity) pair of a warp's 32 points once, appended in no fixed order (the set
// the flags of a step need)
template<class Map, class Grid, int kMode>
__global__ void __launch_bounds__(kThreads) mixed_image_kernel(const MixedArgs a)
{
  __shared__ double pts[kTable];
  const bool table = load_table<Grid, Map::D>(a.grid, a.points, pts);
  const uint64_t P = a.points;
  const uint64_t total = uint64_t(a.n_src) * P;
  if constexpr (kMode == 5) {
    // whole warps take the loop's trips together (the warp collectives stay converged)
    const int lane = threadIdx.x & 31;
    for (uint64_t g0 = uint64_t(blockIdx.x) * blockDim.x + (threadIdx.x & ~31u); g0 < total;
         g0 += uint64_t(gridDim.x) * blockDim.x) {
      const uint64_t g = g0 + uint64_t(lane);
      const bool active = g < total;
      uint64_t key = 0;
      bool valid = false;
      if (active) {
        const uint64_t rank = g / P;
        const uint32_t k = uint32_t(g - rank * P);
        const uint32_t leaf = a.src ? __ldg(a.src + rank) : uint32_t(rank);
        uint64_t p64;
        valid = image_code<Map, Grid>(a, pts, table, leaf, k, g, p64);
        key = valid ? (p64 & a.p64_keep) : ~0ull;   // the invalid box (~0, 255) of PointToBox
      }
      // a valid box of code ~0 and the invalid box differ in validity: keys of both kinds
      // lead separately
      const unsigned act = __ballot_sync(0xFFFFFFFFu, active);
      const unsigned vmask = __ballot_sync(0xFFFFFFFFu, active && valid);
      const unsigned same = __match_any_sync(0xFFFFFFFFu, key) & act & (valid ? vmask : ~vmask);
      const bool leader = active && lane == __ffs(same) - 1;
      const unsigned lead = __ballot_sync(0xFFFFFFFFu, leader);
      uint32_t slot = 0;
      if (lane == 0 && lead) slot = atomicAdd(a.n_out, uint32_t(__popc(lead)));
      slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
      if (leader) {
        const uint64_t pos = uint64_t(slot) + __popc(lead & ((1u << lane) - 1u));
        if (pos < a.p64_cap) {
          a.p64_out[pos] = key;
          a.valid_out[pos] = valid ? 1 : 0;
        }
      }
    }
  } else {
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < total;
         g += uint64_t(gridDim.x) * blockDim.x) {
      const uint64_t rank = g / P;
      const uint32_t k = uint32_t(g - rank * P);
      const uint32_t leaf = a.src ? __ldg(a.src + rank) : uint32_t(rank);
      if constexpr (kMode == 2) {
        uint64_t p64;
        const bool valid = image_code<Map, Grid>(a, pts, table, leaf, k, g, p64);
        a.valid_out[g] = valid ? 1 : 0;
        a.p64_out[g] = valid ? p64 : ~0ull;   // the invalid box (~0, 255) of PointToBox
      } else if constexpr (kMode >= 3) {
        uint64_t p64;
        const bool valid = image_code<Map, Grid>(a, pts, table, leaf, k, g, p64);
        const uint32_t b = inner_box_of(CmpIndex{a.cmp, a.tab, a.n, a.tab_bits}, a.code, a.dep, a.box_pos,
                                        a.inner_depth, valid, p64);
        if constexpr (kMode == 4) a.out[g] = b;
        else if (b != kInvalidIndex) a.box_hit[b] = 1;
      } else {
        const uint32_t t = image_of<Map, Grid>(a, pts, table, leaf, k, g);
        if constexpr (kMode == 1) a.out[g] = t;
        else if (t != kInvalidIndex) a.hit[t] = 1;
      }
    }
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

// the leaf of each of n point boxes given by the caller (the search of
// searchByIterators / setFlagsByIterators, ImplicitBoxTree.hpp:2394-2432): its index into
// `index`, or (index null) a hit mark on it
__global__ void point_box_kernel(const CmpIndex ix, const uint64_t* __restrict__ code,
                                 const uint8_t* __restrict__ dep, const uint64_t* __restrict__ p64,
                                 const uint8_t* __restrict__ valid, uint64_t n, uint32_t* index, uint8_t* hit)
{
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t t = locate_mixed(ix, code, dep, __ldg(valid + i) != 0, __ldg(p64 + i));
    if (index) index[i] = t;
    else if (t != kInvalidIndex) hit[t] = 1;
  }
}

// counts the leaves that break the tree's invariants: a depth above 64, bits above the
// depth, or a leaf that does not strictly precede the next one or contains it
__global__ void leaf_order_kernel(const uint64_t* code, const uint8_t* dep, uint32_t n, uint32_t* bad)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t d = dep[i];
    bool ok = d <= 64 && (d == 64 || (code[i] >> d) == 0);
    if (ok && i + 1 < n) {
      const uint32_t e = dep[i + 1];
      if (e > 64) {
        ok = false;
      } else {
        const uint32_t m = d < e ? d : e;
        const bool nested = m == 0 || (srs(code[i], d - m) == srs(code[i + 1], e - m));
        ok = comparable(code[i], d) < comparable(code[i + 1], e) && !nested;
      }
    }
    if (!ok) atomicAdd(bad, 1u);
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

// heads of the boxes at `depth` into t->row_count and their scan into t->rowptr (the box
// of a leaf j at least that deep is rowptr[j + 1] - 1); *n_boxes
b12g_status inner_boxes(b12g_tree* t, uint8_t depth, uint32_t* n_boxes)
{
  const uint32_t n = t->n;
  ST(t->row_count.ensure(uint64_t(n) + 1, "box heads"));
  ST(t->rowptr.ensure(uint64_t(n) + 1, "box positions"));
  box_head_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(t->codes(), dep_cur(t), n, depth, t->row_count.p);
  count_launches(1);
  return scan_marks(t, t->row_count.p, t->rowptr.p, n, n_boxes);
}

// every box's AND (into t->src) and OR (into t->out) of its leaves' flags
b12g_status box_flags(b12g_tree* t, uint8_t depth, uint32_t n_boxes)
{
  ST(t->src.ensure(std::max<uint32_t>(n_boxes, 1), "box flags"));
  ST(t->out.ensure(std::max<uint32_t>(n_boxes, 1), "box flags"));
  CK(cudaMemsetAsync(t->src.p, 0xFF, size_t(n_boxes) * 4, t->stream));
  CK(cudaMemsetAsync(t->out.p, 0, size_t(n_boxes) * 4, t->stream));
  box_combine_kernel<<<grid_for_n(t->n), kThreads, 0, t->stream>>>(t->flg(), dep_cur(t), t->n, depth, t->rowptr.p,
                                                                   t->src.p, t->out.p);
  count_launches(1);
  return B12G_OK;
}

b12g_status refresh_comparable(b12g_tree* t)
{
  ST(t->cmp.ensure(std::max<uint32_t>(t->n, 1), "comparable patterns"));
  comparable_kernel<<<grid_for_n(t->n), kThreads, 0, t->stream>>>(t->codes(), dep_cur(t), t->n, t->cmp.p);
  LAUNCHED("comparable patterns");
  // about two table entries per leaf, 4 .. 22 bits
  uint32_t bits = 4;
  while (bits < 22 && (1ull << bits) < 2ull * t->n) ++bits;
  t->cmp_bits = bits;
  ST(t->cmp_tab.ensure((size_t(1) << bits) + 1, "pattern prefix table"));
  cmp_table_kernel<<<grid_for_n((uint64_t(1) << bits) + 1), kThreads, 0, t->stream>>>(t->cmp.p, t->n, bits,
                                                                                       t->cmp_tab.p);
  LAUNCHED("pattern prefix table");
  count_launches(2);
  return B12G_OK;
}

// the scheme's source leaves: every leaf with all the scheme's flags
// the scheme's sources into a.src / a.n_src / a.src_depth: every leaf with all the
// scheme's flags, or at an inner source depth the boxes whose leaves all have them
b12g_status mixed_sources(b12g_tree* t, const b12g_scheme* sc, MixedArgs& a)
{
  const uint32_t n = t->n;
  a.src_depth = 0;
  if (sc->depth != B12G_LEAF_DEPTH) {
    const uint32_t d = sc->depth;
    if (d == 0 || d > 64)
      return fail(B12G_ERR_UNSUPPORTED_MIXED_DEPTH, "scheme source depth %u (inner depths 1..64 and 255)", d);
    a.src_depth = d;
    a.src = nullptr;
    a.n_src = 0;
    if (d > t->depth) return B12G_OK;      // no box that deep: no sources
    ST(t->isrc_head.ensure(uint64_t(n) + 1, "inner sources"));
    ST(t->isrc_pos.ensure(uint64_t(n) + 1, "inner sources"));
    ST(t->isrc_and.ensure(std::max<uint32_t>(n, 1), "inner sources"));
    ST(t->isrc.ensure(std::max<uint32_t>(n, 1), "inner sources"));
    box_head_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(t->codes(), dep_cur(t), n, d, t->isrc_head.p);
    uint32_t boxes = 0;
    ST(scan_marks(t, t->isrc_head.p, t->isrc_pos.p, n, &boxes));
    CK(cudaMemsetAsync(t->isrc_and.p, 0xFF, size_t(std::max<uint32_t>(boxes, 1)) * 4, t->stream));
    box_and_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(t->flg(), dep_cur(t), n, d, t->isrc_pos.p,
                                                               t->isrc_and.p);
    source_select_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(t->isrc_head.p, t->isrc_pos.p, t->isrc_and.p, n,
                                                                     sc->flags_to_check);
    uint32_t total = 0;
    ST(scan_marks(t, t->isrc_head.p, t->isrc_pos.p, n, &total));
    keep_scatter_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(nullptr, nullptr, nullptr, n, t->isrc_pos.p,
                                                                     nullptr, nullptr, nullptr, t->isrc.p);
    count_launches(4);
    a.src = t->isrc.p;
    a.n_src = total;
    return B12G_OK;
  }
  if (sc->flags_to_check == 0) {
    a.src = nullptr;
    a.n_src = n;
    return B12G_OK;
  }
  ST(t->row_count.ensure(uint64_t(n) + 1, "source marks"));
  ST(t->rowptr.ensure(uint64_t(n) + 1, "source positions"));
  ST(t->src.ensure(std::max<uint32_t>(n, 1), "source list"));
  keep_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(t->flg(), n, sc->flags_to_check, t->row_count.p);
  uint32_t total = 0;
  ST(scan_marks(t, t->row_count.p, t->rowptr.p, n, &total));
  keep_scatter_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(nullptr, nullptr, nullptr, n, t->rowptr.p,
                                                                   nullptr, nullptr, nullptr, t->src.p);
  count_launches(2);
  a.src = t->src.p;
  a.n_src = total;
  return B12G_OK;
}

b12g_status mixed_args(b12g_tree* t, const b12g_scheme* sc, MixedArgs& a)
{
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
  a.tab = t->cmp_tab.p;
  a.tab_bits = t->cmp_bits;
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
  LAUNCHED("depth range");
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
  ++t->leaf_gen;
  t->mixed = true;
  ST(set_ctr(t, t->ncur, n));
  ST(sync(t, "load leaves"));
  return mixed_settle(t);
}

// setFlags / unsetFlags / changeFlags (op 0 / 1 / 2) at a depth inside the tree: every
// leaf of a box at that depth changes (setFlagsByStencil, unsetFlagsByStencil,
// changeFlagsByStencil with a true stencil, ImplicitBoxTree.hpp:914-1058, 2805-2882,
// 3336-3411); *n_changed counts boxes as countIfFlags does (1104-1200).  A depth below
// no leaf changes nothing.
b12g_status mixed_flags_at_depth(b12g_tree* t, int op, uint8_t u, uint8_t f, uint8_t depth, uint32_t* n_changed)
{
  if (n_changed) *n_changed = 0;
  if (depth == 0 || depth > 64) return fail(B12G_ERR_INVALID, "inner depth %u", depth);
  if (depth > t->depth) return B12G_OK;
  ST(mixed_enter(t));
  const uint32_t n = t->n;
  uint32_t boxes = 0;
  ST(inner_boxes(t, depth, &boxes));
  if (boxes) {
    ST(box_flags(t, depth, boxes));
    ST(set_ctr(t, C_CHANGED, 0));
    box_apply_kernel<<<grid_for_n(std::max(n, boxes)), kThreads, 0, t->stream>>>(
        t->flg(), dep_cur(t), n, depth, t->rowptr.p, t->src.p, t->out.p, boxes, op, u, f, t->ctr.p + C_CHANGED);
    count_launches(1);
    ST(read_ctr(t, C_CHANGED, 1));
    if (n_changed) *n_changed = t->h_ctr[C_CHANGED];
  }
  return mixed_settle(t);
}

// flags f on every leaf of the boxes at `depth` marked in t->hit[0 .. n_boxes), which
// are cleared after; *n_changed (if not null) = marked boxes whose leaves did not all have f
b12g_status apply_box_hits(b12g_tree* t, uint8_t depth, uint32_t n_boxes, uint8_t f, uint32_t* n_changed)
{
  if (n_changed) *n_changed = 0;
  if (!n_boxes) return B12G_OK;
  ST(box_flags(t, depth, n_boxes));
  ST(set_ctr(t, C_CHANGED, 0));
  box_hit_apply_kernel<<<grid_for_n(std::max(t->n, n_boxes)), kThreads, 0, t->stream>>>(
      t->flg(), dep_cur(t), t->n, depth, t->rowptr.p, t->src.p, t->hit.p, n_boxes, f, t->ctr.p + C_CHANGED);
  CK(cudaMemsetAsync(t->hit.p, 0, n_boxes, t->stream));
  count_launches(1);
  ST(read_ctr(t, C_CHANGED, 1));
  if (n_changed) *n_changed = t->h_ctr[C_CHANGED];
  return B12G_OK;
}

// the images of the scheme's source leaves located at an inner depth: flags on the
// boxes hit (setFlagsByIterators, ImplicitBoxTree.hpp:2691-2694), or with search set
// each point's box index at that depth into t->out (searchByIterators, 2473-2566)
b12g_status mixed_image_at_depth(b12g_tree* t, const b12g_scheme* sc, uint8_t depth, uint8_t flags, bool search,
                                 uint64_t* n_points, uint32_t* n_changed)
{
  if (n_changed) *n_changed = 0;
  if (depth == 0 || depth > 64) return fail(B12G_ERR_UNSUPPORTED_MIXED_DEPTH, "image search at depth %u", depth);
  ST(mixed_enter(t));
  MixedArgs a;
  ST(mixed_args(t, sc, a));
  ST(mixed_sources(t, sc, a));
  const uint64_t np = uint64_t(a.n_src) * a.points;
  if (n_points) *n_points = np;
  uint32_t boxes = 0;
  ST(inner_boxes(t, depth, &boxes));   // no box below the deepest leaf: every search fails
  a.box_pos = t->rowptr.p;
  a.inner_depth = depth;
  a.box_hit = t->hit.p;
  if (search) {
    ST(t->out.ensure(std::max<uint64_t>(np, 1), "search output"));
    a.out = t->out.p;
  }
  if (np)
    CK(dispatch(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, [&](auto map, auto grid) -> cudaError_t {
      if (search) mixed_image_kernel<decltype(map), decltype(grid), 4><<<grid_for_n(np), kThreads, 0, t->stream>>>(a);
      else mixed_image_kernel<decltype(map), decltype(grid), 3><<<grid_for_n(np), kThreads, 0, t->stream>>>(a);
      return cudaGetLastError();
    }));
  count_launches(1);
  if (!search) ST(apply_box_hits(t, depth, boxes, flags, n_changed));
  if (search) return B12G_OK;       // t->out is read by the caller before the layout may change
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
  if (codes) CK(cudaMemcpyAsync(codes, t->codes(), size_t(t->n) * 8, cudaMemcpyDefault, t->stream));
  if (flags) CK(cudaMemcpyAsync(flags, t->flg(), t->n, cudaMemcpyDefault, t->stream));
  if (depths) CK(cudaMemcpyAsync(depths, dep_cur(t), t->n, cudaMemcpyDefault, t->stream));
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
  ++t->leaf_gen;
  t->ncur = no;
  t->n = total;
  ++t->leaf_gen;
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
  ++t->leaf_gen;
  t->ncur = no;
  t->n = kept;
  ++t->leaf_gen;
  ST(set_ctr(t, t->ncur, kept));
  ST(sync(t, "remove"));
  if (n_removed) *n_removed = n - kept;
  if (kept == 0) return set_root(t, B12G_NONE);  // insertSurroundingBoxIfEmpty; one depth again
  return mixed_settle(t);
}

b12g_status mixed_set_flags_by_image(b12g_tree* t, const b12g_scheme* sc, uint8_t flags, uint8_t depth,
                                     uint32_t* n_changed)
{
  if (depth != B12G_LEAF_DEPTH) return mixed_image_at_depth(t, sc, depth, flags, false, nullptr, n_changed);
  MixedArgs a;
  ST(mixed_args(t, sc, a));
  ST(mixed_sources(t, sc, a));
  if (t->hit.n < t->n) {
    // the hit marks are all clear between calls (apply_hits clears what it reads)
    ST(t->hit.ensure(t->n, "hit marks"));
    CK(cudaMemsetAsync(t->hit.p, 0, t->hit.n, t->stream));
  }
  a.hit = t->hit.p;
  CK(dispatch(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, [&](auto map, auto grid) -> cudaError_t {
    mixed_image_kernel<decltype(map), decltype(grid), 0>
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
  ST(mixed_sources(t, sc, a));
  const uint64_t np = uint64_t(a.n_src) * a.points;
  ST(t->out.ensure(std::max<uint64_t>(np, 1), "search output"));
  a.out = t->out.p;
  CK(dispatch(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, [&](auto map, auto grid) -> cudaError_t {
    mixed_image_kernel<decltype(map), decltype(grid), 1><<<grid_for_n(np), kThreads, 0, t->stream>>>(a);
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

// unsubdivide (ImplicitBoxTree.hpp:3414-3460); returns the number of parents made
b12g_status mixed_unsubdivide(b12g_tree* t, uint8_t flags, uint32_t* n_parents)
{
  ST(mixed_enter(t));
  const uint32_t n = t->n;
  ST(t->out.ensure(std::max<uint32_t>(n, 1), "unsubdivide marks"));
  ST(t->row_count.ensure(uint64_t(n) + 1, "keep marks"));
  ST(t->rowptr.ensure(uint64_t(n) + 1, "keep positions"));
  ST(set_ctr(t, C_CAND, 0));
  const int o = 1 - t->cur;
  unsub_mark_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(t->codes(), dep_cur(t), t->flg(), n, flags, t->out.p,
                                                                t->ctr.p + C_CAND);
  unsub_apply_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(t->codes(), dep_cur(t), t->flg(), n, t->out.p,
                                                                 t->code[o].p, t->dep[o].p, t->flags[o].p,
                                                                 t->row_count.p);
  count_launches(2);
  uint32_t kept = 0;
  ST(scan_marks(t, t->row_count.p, t->rowptr.p, n, &kept));
  keep_scatter_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(t->code[o].p, t->flags[o].p, t->dep[o].p, n,
                                                                   t->rowptr.p, t->codes(), t->flg(), dep_cur(t),
                                                                   nullptr);
  count_launches(1);
  ST(read_ctr(t, C_CAND, 1));
  const uint32_t marked = t->h_ctr[C_CAND];
  t->n = kept;
  ++t->leaf_gen;
  ST(set_ctr(t, t->ncur, kept));
  ST(sync(t, "unsubdivide"));
  if (n_parents) *n_parents = marked - (n - kept);
  return mixed_settle(t);
}

// insertByIterators (ImplicitBoxTree.hpp:1615-1910) for the np point boxes held in
// t->cand (depth-64 codes) and t->pvalid, at `depth` (255: the leaf depth), for trees of
// any depths; the caller handles depth 0.  *n_inserted gets the distinct new boxes.
b12g_status mixed_insert_boxes(b12g_tree* t, uint64_t np, uint8_t depth, uint8_t ins, uint8_t hit,
                               uint32_t* n_inserted)
{
  if (depth > 64 && depth != B12G_LEAF_DEPTH) return fail(B12G_ERR_INVALID, "insertion depth %u", depth);
  if (np > 0xFFFFFFF0ull) return fail(B12G_ERR_CAPACITY, "too many points in one insertion");
  const int mode = depth == B12G_LEAF_DEPTH ? 0 : (depth <= t->depth ? 2 : 3);
  if (n_inserted) *n_inserted = 0;
  ST(mixed_enter(t));
  ST(refresh_comparable(t));
  const uint32_t m_cap = uint32_t(std::max<uint64_t>(np, 1));
  ST(t->ins_code.ensure(m_cap, "new boxes"));
  ST(t->ins_dep.ensure(m_cap, "new box depths"));
  ST(set_ctr(t, C_CAND, 0));
  InsertArgs a{};
  a.p64 = t->cand.p;
  a.valid = t->pvalid.p;
  a.np = np;
  a.code = t->codes();
  a.dep = dep_cur(t);
  a.cmp = t->cmp.p;
  a.tab = t->cmp_tab.p;
  a.tab_bits = t->cmp_bits;
  a.n = t->n;
  a.depth = depth;
  a.mode = mode;
  a.hit = (mode == 0 && hit) ? t->hit.p : nullptr;
  a.out_code = t->ins_code.p;
  a.out_dep = t->ins_dep.p;
  a.count = t->ctr.p + C_CAND;
  a.cap = m_cap;
  a.error = t->ctr.p + C_ERROR;
  uint32_t inner = 0;   // boxes at an inner insertion depth, for the flags of the boxes hit
  if (mode == 2) {
    ST(inner_boxes(t, depth, &inner));
    a.box_pos = t->rowptr.p;
    a.box_hit = hit ? t->hit.p : nullptr;
  }
  if (np) insert_boxes_kernel<<<grid_for_n(np), kThreads, 0, t->stream>>>(a);
  count_launches(1);
  if (a.hit) {
    ST(set_ctr(t, C_CHANGED, 0));
    apply_hits_kernel<<<grid_for_n(t->n), kThreads, 0, t->stream>>>(t->flg(), t->hit.p, t->n, hit,
                                                                     t->ctr.p + C_CHANGED);
    count_launches(1);
  }
  if (a.box_hit) ST(apply_box_hits(t, depth, inner, hit, nullptr));
  ST(read_ctr(t, C_CAND, 1));
  ST(check_error(t, "insert"));
  const uint32_t m = t->h_ctr[C_CAND];
  if (m == 0) return mixed_settle(t);

  // the new boxes in tree order (deeper first among equal patterns), then distinct
  for (int q = 0; q < 2; ++q) {
    ST(t->ins_key[q].ensure(m, "new box keys"));
    ST(t->ins_idx[q].ensure(m, "new box order"));
  }
  ST(t->ins_pos.ensure(uint64_t(m) + 1, "new box heads"));
  ST(t->ins_head.ensure(uint64_t(m) + 1, "new box heads"));
  const uint64_t cells = sort_scratch_u32(m);
  ST(t->sort_idx.ensure(cells + 8, "new box sort"));
  uint32_t* scratch = t->sort_idx.p;
  depth_key_kernel<<<grid_for_n(m), kThreads, 0, t->stream>>>(t->ins_dep.p, m, t->ins_key[0].p, t->ins_idx[0].p);
  uint64_t* keys = nullptr;
  uint32_t* order = nullptr;
  CK(radix_sort_u64_values(t->ins_key[0].p, t->ins_key[1].p, t->ins_idx[0].p, t->ins_idx[1].p, t->ctr.p + C_CAND, m,
                           8, scratch, t->ctr.p + C_ERROR, &keys, &order, t->stream));
  uint32_t* order_alt = order == t->ins_idx[0].p ? t->ins_idx[1].p : t->ins_idx[0].p;
  pattern_key_kernel<<<grid_for_n(m), kThreads, 0, t->stream>>>(t->ins_code.p, t->ins_dep.p, order, m,
                                                                 t->ins_key[0].p);
  CK(radix_sort_u64_values(t->ins_key[0].p, t->ins_key[1].p, order, order_alt, t->ctr.p + C_CAND, m, 64, scratch,
                           t->ctr.p + C_ERROR, &keys, &order, t->stream));
  count_launches(2 + sort_launches(8) + sort_launches(64));   // key kernels and the two sorts
  ST(check_error(t, "new box sort"));
  new_heads_kernel<<<grid_for_n(m), kThreads, 0, t->stream>>>(t->ins_code.p, t->ins_dep.p, order, m, t->ins_head.p);
  count_launches(1);
  uint32_t u = 0;
  ST(scan_marks(t, t->ins_head.p, t->ins_pos.p, m, &u));
  uint64_t* ucode = keys == t->ins_key[0].p ? t->ins_key[1].p : t->ins_key[0].p;
  ST(t->ins_dep2.ensure(std::max<uint32_t>(u, 1), "distinct new boxes"));
  uint8_t* udep = t->ins_dep2.p;
  new_scatter_kernel<<<grid_for_n(m), kThreads, 0, t->stream>>>(t->ins_code.p, t->ins_dep.p, order, m,
                                                                 t->ins_pos.p, ucode, udep);
  count_launches(1);

  // sortBoxes of leaves + new boxes, the two HasSamePath scans and unique (1862-1897)
  const uint32_t n = t->n;
  const uint64_t total = uint64_t(n) + u;
  ST(reserve(t, total));
  ST(t->scan_code.ensure(total, "merge scan"));
  ST(t->scan_dep.ensure(total, "merge scan"));
  ST(t->scan_flags.ensure(total, "merge scan"));
  ST(t->row_count.ensure(total + 1, "keep marks"));
  ST(t->rowptr.ensure(total + 1, "keep positions"));
  const int o = 1 - t->cur;
  merge_boxes_kernel<<<grid_for_n(total), kThreads, 0, t->stream>>>(t->codes(), dep_cur(t), t->flg(), n, ucode, udep,
                                                                     ins, u, t->code[o].p, t->dep[o].p,
                                                                     t->flags[o].p);
  forward_scan_kernel<<<grid_for_n(total), kThreads, 0, t->stream>>>(t->code[o].p, t->dep[o].p, t->flags[o].p,
                                                                      uint32_t(total), t->scan_code.p,
                                                                      t->scan_dep.p, t->scan_flags.p);
  reverse_scan_kernel<<<grid_for_n(total), kThreads, 0, t->stream>>>(t->scan_code.p, t->scan_dep.p, t->scan_flags.p,
                                                                      uint32_t(total), t->code[o].p, t->dep[o].p,
                                                                      t->flags[o].p);
  path_heads_kernel<<<grid_for_n(total), kThreads, 0, t->stream>>>(t->code[o].p, t->dep[o].p, uint32_t(total),
                                                                    t->row_count.p);
  count_launches(4);
  uint32_t kept = 0;
  ST(scan_marks(t, t->row_count.p, t->rowptr.p, uint32_t(total), &kept));
  keep_scatter_kernel<<<grid_for_n(total), kThreads, 0, t->stream>>>(t->code[o].p, t->flags[o].p, t->dep[o].p,
                                                                       uint32_t(total), t->rowptr.p, t->codes(),
                                                                       t->flg(), dep_cur(t), nullptr);
  count_launches(1);
  t->n = kept;
  ++t->leaf_gen;
  ST(set_ctr(t, t->ncur, kept));
  ST(sync(t, "insert"));
  if (n_inserted) *n_inserted = u;
  return mixed_settle(t);
}

// the point boxes of n_points host points (row-major, dim doubles each) into t->cand / t->pvalid
b12g_status mixed_point_boxes(b12g_tree* t, const double* points, uint64_t n_points)
{
  const uint32_t D = t->domain.dim;
  if (D < 2) return fail(B12G_ERR_UNSUPPORTED_MIXED_DEPTH, "insertion at other depths needs dimension 2 to 4");
  ST(t->cand.ensure(std::max<uint64_t>(n_points, 256), "point boxes"));
  ST(t->pvalid.ensure(std::max<uint64_t>(n_points, 1), "point boxes"));
  if (n_points == 0) return B12G_OK;
  ST(t->points.ensure(n_points * D, "points"));
  CK(cudaMemcpyAsync(t->points.p, points, n_points * D * 8, cudaMemcpyHostToDevice, t->stream));
  const int g = grid_for_n(n_points);
  switch (D) {
    case 2: point_codes_kernel<2><<<g, kThreads, 0, t->stream>>>(t->points.p, n_points, t->dom, t->cand.p, t->pvalid.p); break;
    case 3: point_codes_kernel<3><<<g, kThreads, 0, t->stream>>>(t->points.p, n_points, t->dom, t->cand.p, t->pvalid.p); break;
    default: point_codes_kernel<4><<<g, kThreads, 0, t->stream>>>(t->points.p, n_points, t->dom, t->cand.p, t->pvalid.p); break;
  }
  CK(cudaGetLastError());
  count_launches(1);
  return B12G_OK;
}

// the point boxes of the images of the scheme's source leaves into t->cand / t->pvalid
b12g_status mixed_image_boxes(b12g_tree* t, const b12g_scheme* sc, uint64_t* n_points)
{
  ST(mixed_enter(t));
  MixedArgs a;
  ST(mixed_args(t, sc, a));
  ST(mixed_sources(t, sc, a));
  const uint64_t np = uint64_t(a.n_src) * a.points;
  ST(t->cand.ensure(std::max<uint64_t>(np, 256), "point boxes"));
  ST(t->pvalid.ensure(std::max<uint64_t>(np, 1), "point boxes"));
  a.p64_out = t->cand.p;
  a.valid_out = t->pvalid.p;
  if (np)
    CK(dispatch(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, [&](auto map, auto grid) -> cudaError_t {
      mixed_image_kernel<decltype(map), decltype(grid), 2><<<grid_for_n(np), kThreads, 0, t->stream>>>(a);
      return cudaGetLastError();
    }));
  count_launches(1);
  *n_points = np;
  return B12G_OK;
}

// the point boxes of the images of the scheme's sources into the caller's device buffers
// (codes, validity), source-major; CAPACITY with *n_points set when they do not fit
b12g_status mixed_image_point_boxes(b12g_tree* t, const b12g_scheme* sc, uint64_t* codes, uint8_t* valid,
                                    uint64_t capacity, uint64_t* n_points, bool distinct, uint8_t keep_depth)
{
  ST(mixed_enter(t));
  MixedArgs a;
  ST(mixed_args(t, sc, a));
  ST(mixed_sources(t, sc, a));
  const uint64_t np = uint64_t(a.n_src) * a.points;
  *n_points = np;
  if (np > capacity) {
    ST(mixed_settle(t));
    return fail(B12G_ERR_CAPACITY, "%llu image points, room for %llu", (unsigned long long)np,
                (unsigned long long)capacity);
  }
  if (np && (!codes || !valid)) {
    ST(mixed_settle(t));
    return fail(B12G_ERR_INVALID, "NULL output buffer");
  }
  a.p64_out = codes;
  a.valid_out = valid;
  a.p64_cap = capacity;
  a.p64_keep = keep_depth >= 64 ? ~0ull : keep_depth == 0 ? 0ull : ~((uint64_t(1) << (64 - keep_depth)) - 1ull);
  a.n_out = t->ctr.p + C_TMP;
  if (np) {
    if (distinct) ST(set_ctr(t, C_TMP, 0));
    CK(dispatch(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, [&](auto map, auto grid) -> cudaError_t {
      if (distinct)
        mixed_image_kernel<decltype(map), decltype(grid), 5><<<grid_for_n(np), kThreads, 0, t->stream>>>(a);
      else
        mixed_image_kernel<decltype(map), decltype(grid), 2><<<grid_for_n(np), kThreads, 0, t->stream>>>(a);
      return cudaGetLastError();
    }));
    count_launches(1);
  }
  if (distinct && np) {
    ST(read_ctr(t, C_TMP, 1));
    *n_points = t->h_ctr[C_TMP];
  } else {
    ST(sync(t, "image point boxes"));
  }
  return mixed_settle(t);
}

// the leaf of each given point box into index (device), or, with index null, `flags` set
// on every leaf that holds one; *n_changed counts the leaves whose flags changed
b12g_status mixed_point_box_search(b12g_tree* t, const uint64_t* codes, const uint8_t* valid, uint64_t n,
                                   uint32_t* index, uint8_t flags, uint32_t* n_changed)
{
  if (n_changed) *n_changed = 0;
  if (n && (!codes || !valid)) return fail(B12G_ERR_INVALID, "NULL point boxes");
  ST(mixed_enter(t));
  ST(refresh_comparable(t));
  const CmpIndex ix{t->cmp.p, t->cmp_tab.p, t->n, t->cmp_bits};
  if (!index && t->hit.n < t->n) {
    // the hit marks are all clear between calls (apply_hits clears what it reads)
    ST(t->hit.ensure(t->n, "hit marks"));
    CK(cudaMemsetAsync(t->hit.p, 0, t->hit.n, t->stream));
  }
  if (n) {
    point_box_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(ix, t->codes(), dep_cur(t), codes, valid, n, index,
                                                                 t->hit.p);
    CK(cudaGetLastError());
    count_launches(1);
  }
  if (!index) {
    ST(set_ctr(t, C_CHANGED, 0));
    apply_hits_kernel<<<grid_for_n(t->n), kThreads, 0, t->stream>>>(t->flg(), t->hit.p, t->n, flags,
                                                                     t->ctr.p + C_CHANGED);
    LAUNCHED("apply hits");
    count_launches(1);
    ST(read_ctr(t, C_CHANGED, 1));
    if (n_changed) *n_changed = t->h_ctr[C_CHANGED];
  } else {
    ST(sync(t, "search point boxes"));
  }
  return mixed_settle(t);
}

// leaves from device memory; the same checks as a load from the host, made on the device
b12g_status mixed_load_device(b12g_tree* t, const uint64_t* codes, const uint8_t* depths, const uint8_t* flags,
                              uint32_t n)
{
  if (n == 0) return set_root(t, B12G_NONE);
  ST(reserve(t, n));
  ST(ensure_dep(t, std::max<uint64_t>(t->code[0].n, n)));
  CK(cudaMemcpyAsync(t->codes(), codes, size_t(n) * 8, cudaMemcpyDeviceToDevice, t->stream));
  CK(cudaMemcpyAsync(t->flg(), flags, n, cudaMemcpyDeviceToDevice, t->stream));
  CK(cudaMemcpyAsync(dep_cur(t), depths, n, cudaMemcpyDeviceToDevice, t->stream));
  ST(set_ctr(t, C_TMP, 0));
  leaf_order_kernel<<<grid_for_n(n), kThreads, 0, t->stream>>>(t->codes(), dep_cur(t), n, t->ctr.p + C_TMP);
  CK(cudaGetLastError());
  count_launches(1);
  ST(read_ctr(t, C_TMP, 1));
  if (t->h_ctr[C_TMP] != 0) {
    const uint32_t bad = t->h_ctr[C_TMP];
    ST(set_root(t, B12G_NONE));
    return fail(B12G_ERR_INVALID, "%u leaves out of order, nested or deeper than 64", bad);
  }
  t->n = n;
  ++t->leaf_gen;
  t->mixed = true;
  ST(set_ctr(t, t->ncur, n));
  ST(sync(t, "load leaves"));
  return mixed_settle(t);
}

}  // namespace host
}  // namespace b12g
