// Kernel launch interface shared by the host library (api.cu) and the kernel files.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device.cuh"

namespace b12g {

// What an image kernel does with the leaf that a mapped point lands in.
enum class ImageMode : int {
  Hit = 0,     // hit[leaf] = 1                       (setFlagsByIterators)
  Search = 1,  // out[point] = leaf index or invalid  (searchByIterators)
  Insert = 2,  // not found -> candidate code         (insertByIterators)
  Mark = 3,    // the image's box marked in a bitmap of every box of the depth; the
               // boxes this launch marks first also in `fresh`, and counted
};

// One box-image launch over a uniform-depth leaf set.
constexpr int kSrcStride = 4;    // doubles per source in ImageArgs::src_c (two 16-byte loads)

struct ImageArgs {
  Domain dom;
  MapParams map;
  GridParams grid;
  const uint64_t* codes;     // sorted leaf codes (parents in children mode)
  const uint32_t* n_leaves;  // device count of `codes`
  int depth;                 // depth of the imaged boxes (children depth in children mode)
  DepthConst dc;             // constants of `depth` (launch_image / launch_rows fill them in)
  int children;              // 1: boxes are the 2n children of `codes`, never materialised
  const uint32_t* src;       // source leaf ranks -> leaf index (nullptr: all leaves)
  const uint32_t* n_src;     // device count of sources (nullptr: all leaves / children)
  uint32_t n_src_value;      // Mark mode: the count of sources itself (n_src unused)
  const double* src_c;       // optional: the centre of every source box by rank, kSrcStride
                             // doubles a source (the radius is dc's); nullptr: from the codes
  uint64_t points;           // points per box
  LeafHash hash;             // leaf lookup table (slots == nullptr: binary search)
  // outputs
  uint8_t* hit;
  uint32_t hit_cap;          // entries of `hit`; more boxes than this sets error bit 0
  uint32_t* targets;         // Hit mode, optional: every point's target box (kInvalidIndex:
                             // in no box; kOutsideIndex: it left the domain)
  uint64_t targets_cap;      // entries of `targets`; a point beyond sets *targets_over
  uint32_t* targets_over;
  uint32_t* out;
  uint64_t* cand;            // insert candidates: packed keys (pack_bits) of depth-d boxes
  uint32_t* cand_count;
  uint32_t cand_cap;
  uint32_t* bits;            // Mark mode: bit c = the box of depth-d code c is a leaf
  uint32_t* fresh;           // Mark mode: bit c = the box of code c was added by this launch
  int claim;                 // Insert mode: claim each new box in `hash` (a kept table,
                             // log2_use set), so every candidate is a distinct new box
  uint32_t* error;           // bit 0: capacity overflow
  unsigned long long* work;  // the image kernel's work-queue counter (launch_image zeroes it)
};

// Transition rows: warp per source box, up to kMaxRowPoints points.
constexpr uint32_t kMaxRowPoints = 128;
constexpr uint32_t kPadKey = 0xFFFFFFFFu;
constexpr uint32_t kLostKey = 0xFFFFFFFEu;

struct RowArgs {
  ImageArgs img;
  uint32_t* stage_col;       // n x points
  uint32_t* stage_cnt;       // n x points
  uint32_t* row_count;       // n
  int keep_lost;             // 1: lost points form a column `lost_col`
  uint32_t lost_col;
};

// Transition rows from the targets a subdivision step stored (child indices of that
// step's boxes) and its compaction ranks (rank[c] = survivors before child c, 2n + 1
// entries): a row per surviving child, a column per surviving target.
struct StoredRowArgs {
  const uint32_t* targets;   // children x points
  const uint32_t* rank;
  const uint64_t* codes;     // the survivors (the tree's leaves)
  uint32_t n_children;
  uint32_t n_leaves;
  uint32_t points;
  uint32_t* stage_col;
  uint32_t* stage_cnt;
  uint32_t* row_count;
  int keep_lost;
};
cudaError_t launch_stored_rows(const StoredRowArgs& a, cudaStream_t s);

// launch helpers (image.cu); return cudaSuccess or the launch error
cudaError_t launch_image(uint32_t map_kind, uint32_t arith, uint32_t grid_kind, uint32_t dim, ImageMode mode,
                         const ImageArgs& a, uint64_t max_points, cudaStream_t s);
cudaError_t launch_rows(uint32_t map_kind, uint32_t arith, uint32_t grid_kind, uint32_t dim,
                        const RowArgs& a, uint32_t max_rows, cudaStream_t s);
// true if the (map, arith, grid, dim) combination has compiled kernels
bool image_supported(uint32_t map_kind, uint32_t arith, uint32_t grid_kind, uint32_t dim);

// tree_ops.cu ---------------------------------------------------------------------
int device_sm_count();
// insert the n leaves of one depth (dim 2..4, depth <= kHashMaxDepth) into the lookup
// table with tag h.tag, keyed by their packed per-dimension indices (pack_bits), which
// also go to h.pk[i]; table slots = 2^h.log2_cap must be >= the slots hash_log2(n) asks
// for, or 2^h.log2_use when set (error bit 0 otherwise)
cudaError_t build_leaf_hash(const uint64_t* codes, const uint32_t* n, int depth, int dim, LeafHash h, uint32_t* error,
                            uint32_t max_n, cudaStream_t s);

// flags |= f on hit leaves (hit cleared); *changed += leaves that lacked f
cudaError_t apply_hits(uint8_t* flags, uint8_t* hit, const uint32_t* n, uint8_t f, uint32_t* changed,
                       uint32_t max_n, cudaStream_t s);
// op: 0 set, 1 unset, 2 change(u -> f); *changed counts as the reference returns it
cudaError_t flag_op(uint8_t* flags, const uint32_t* n, int op, uint8_t u, uint8_t f, uint32_t* changed,
                    uint32_t max_n, cudaStream_t s);
// count leaves with all `f` set (f == 0: all)
cudaError_t count_flags(const uint8_t* flags, const uint32_t* n, uint8_t f, uint32_t* count, uint32_t max_n,
                        cudaStream_t s);
// children: out_code[2i] = code<<1, out_code[2i+1] = code<<1|1; flags copied; *n_out = 2n
cudaError_t split_codes(const uint64_t* code, const uint8_t* flags, const uint32_t* n, uint64_t* out_code,
                        uint8_t* out_flags, uint32_t* n_out, uint32_t max_n, cudaStream_t s);

// stream compaction with a tile-count / tile-scan / scatter sequence.
struct CompactScratch {
  uint32_t* tile_counts;     // >= tiles(max_n)
  uint32_t* tile_offsets;    // >= tiles(max_n)
};
constexpr uint32_t kCompactTile = 4096;
inline uint32_t compact_tiles(uint64_t n) { return uint32_t((n + kCompactTile - 1) / kCompactTile); }

// keep leaf i iff flags[i] has all `f`; unset `clear` on kept leaves.  In children
// mode the input is the implicit children of `code` (n parents -> 2n children) and
// the keep predicate is hit[child]; hit is cleared.  *n_out gets the new count.
struct CompactArgs {
  const uint64_t* code;
  const uint8_t* flags;
  const uint32_t* n;         // input count (parents in children mode)
  uint8_t* hit;              // children mode keep mask
  int children;
  uint8_t keep_flags;
  uint8_t clear_flags;
  uint32_t hit_cap;          // entries of `hit` (children mode)
  uint64_t* out_code;
  uint8_t* out_flags;
  uint32_t* out_index;       // non-null: write the kept indices instead of code/flags
  uint32_t* n_out;
  uint32_t* n_out2;          // optional second copy of the new count
  uint32_t* out_rank;        // optional: out_rank[i] = kept elements before input i (n + 1 entries)
  int vec;                   // set by compact(): the mask and rank arrays take 16-byte accesses
  uint32_t out_cap;
  uint32_t* error;
};
cudaError_t compact(const CompactArgs& a, const CompactScratch& sc, uint32_t max_in, cudaStream_t s);
// kernels one compaction launches: count and scatter, and a scan between them when the
// elements make more than 4,096 tiles
int compact_launches(bool children, uint32_t max_in);

// exclusive scan of u32 -> u32 (out has n+1 entries; out[n] = total)
cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, const uint32_t* n, uint32_t* tile_sums,
                               uint32_t max_n, cudaStream_t s);

// csr.cu ---------------------------------------------------------------------------
cudaError_t gather_rows(const uint32_t* stage_col, const uint32_t* stage_cnt, uint32_t stride,
                        const uint32_t* row_count, const uint32_t* rowptr, const uint32_t* n_rows,
                        uint32_t* cols, double* vals, int absolute, double points, uint32_t max_rows,
                        cudaStream_t s);

// partition.cu -----------------------------------------------------------------------
// *found = 1 when some of the n values equals x (found is not cleared)
cudaError_t value_present(const uint32_t* v, uint64_t n, uint32_t x, uint32_t* found, cudaStream_t s);

}  // namespace b12g
