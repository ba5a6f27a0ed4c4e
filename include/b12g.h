/*
 * b12g - B200-native (sm_100a) box-image path of an implicit box tree.
 *
 * C ABI of libb12g.so.  It replaces, for the set-oriented box-image path, the
 * reference's C++ template class ImplicitBoxTree<A,DIM,REAL,N>
 * (B12c/src/include/ImplicitBoxTree.h:32-640) and the Matlab MEX dispatcher that binds
 * it (B12c/src/matlab/general_implicit_box_tree_interface_mex.hpp.in:21-1858).  Each
 * entry point below cites the reference member function it stands in for.
 *
 * Conventions
 *   - Every call returns a b12g_status; B12G_OK == 0.  b12g_last_error() gives a
 *     human-readable reason for the last failure on the calling thread.
 *   - A tree lives on one GPU (the device current at b12g_tree_create) and owns one
 *     CUDA stream.  Calls on one tree are not thread-safe (as in the reference);
 *     different trees may be used from different threads.
 *   - Depth is uint8_t as in the reference (TypeDefinitions.h:19-57): 255 means
 *     "leaves" (getLeafDepth), 254 "unsubdividable" (not supported here).
 *   - Leaf index results use 0xFFFFFFFF for "not found" (getInvalidNrBoxes).
 *   - Flags are the reference's 8-bit flags (Flags.h:10-23).
 *   - Leaves may have different depths, as in the reference (kept in the order of
 *     isStrictlyPreceding, Box.hpp:124-135).  A tree whose leaves share one depth runs
 *     the fused single-depth kernels; subdividing some of its leaves, or loading leaves
 *     of several depths, switches it to per-leaf depths until one depth is left.  At a
 *     depth inside the tree, flags (and image flags, insertion hit flags) change every
 *     leaf of each box at that depth, and searches return the box's index among the
 *     boxes at that depth.  A scheme's source depth may be 255 (the leaves) or a depth
 *     inside the tree (its boxes whose leaves all carry the scheme's flags).  Source
 *     depth 0 and the unsubdividable depth 254 are not offered; those calls return
 *     B12G_ERR_UNSUPPORTED_MIXED_DEPTH and leave the tree unchanged.
 *   - Host pointers are plain host memory (pinned or pageable); the library owns all
 *     device memory of a tree and of a CSR matrix.
 */
#ifndef B12G_H
#define B12G_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B12G_MAX_DIM 4
#define B12G_LEAF_DEPTH 255u
#define B12G_INVALID_INDEX 0xFFFFFFFFu

typedef enum {
  B12G_OK = 0,
  B12G_ERR_INVALID = 1,                 /* bad argument */
  B12G_ERR_OOM = 2,                     /* device allocation failed */
  B12G_ERR_CUDA = 3,                    /* CUDA runtime error (see b12g_last_error) */
  B12G_ERR_TIMEOUT = 4,                 /* a bounded device-side wait gave up */
  B12G_ERR_UNSUPPORTED_MIXED_DEPTH = 5, /* result would mix leaf depths */
  B12G_ERR_CAPACITY = 6,                /* a size limit of the call was exceeded */
  B12G_ERR_NO_DEVICE = 7                /* no CUDA device / kernels not loadable */
} b12g_status;

/* Flags.h:10-23 */
enum {
  B12G_NONE = 0x00, B12G_HIT = 0x01, B12G_INS = 0x02, B12G_EXPD = 0x04, B12G_SD = 0x08,
  B12G_EQU = 0x10, B12G_ENTR = 0x20, B12G_EXTR = 0x40, B12G_ALL = 0xFF
};

/* map functors (reference: Map_Henon.h, Map_Lorenz.h, MapTools.hpp; the coupled and
 * forced Duffing maps are user plug-ins in the reference's sense, B12_doc.tex:107-146) */
typedef enum {
  B12G_MAP_HENON = 1,           /* p = {a, b}; steps = iterates (IteratingMap) */
  B12G_MAP_LORENZ = 2,          /* p = {sigma, rho, beta}; h, steps (RK4Auto) */
  B12G_MAP_COUPLED_DUFFING = 3, /* h, steps (SymplecticIntegratorAuto, order 2) */
  B12G_MAP_FORCED_DUFFING = 4   /* p = {delta, alpha, beta, gamma}; h = period/steps */
} b12g_map_kind;

typedef enum {
  B12G_ARITH_STRICT = 0,        /* every FP64 op rounded separately (reference -fmad=false) */
  B12G_ARITH_FMA = 1            /* explicit fused multiply-adds (Lorenz only) */
} b12g_arith;

typedef enum {
  B12G_GRID_INNER = 1,          /* InnerGrid(n): n^DIM cell-centre points (Grids.hpp:103-134) */
  B12G_GRID_FULL = 2,           /* FullGrid(n, eps) (Grids.hpp:60-95) */
  B12G_GRID_PHILOX = 3          /* `points` uniform points from Philox4x32-10 keyed by (seed, point index) */
} b12g_grid_kind;

typedef struct {
  uint32_t dim;                 /* 1..B12G_MAX_DIM */
  uint32_t pad;
  double center[B12G_MAX_DIM];
  double radius[B12G_MAX_DIM];
} b12g_domain;

typedef struct {
  uint32_t kind;                /* b12g_map_kind */
  uint32_t arith;               /* b12g_arith */
  uint32_t steps;
  uint32_t pad;
  double h;
  double p[6];
} b12g_map;

typedef struct {
  uint32_t kind;                /* b12g_grid_kind */
  uint32_t n;                   /* points per dimension (inner, full) */
  uint64_t points;              /* points per box (philox) */
  uint64_t seed;                /* philox key */
  double eps;                   /* full grid stretch */
} b12g_grid;

/* A "scheme" is the Matlab driver's {grid, map, depth, flags} cell
 * (subdivision.m:5, continuation.m:24): the point iterator of
 * makePointIteratorPairOverLeaves / makePointIteratorPairByFlags
 * (ImplicitBoxTree.hpp:2167-2196, 2303-2341). */
typedef struct {
  b12g_map map;
  b12g_grid grid;
  uint8_t depth;                /* source depth; 255 = leaves */
  uint8_t flags_to_check;       /* only boxes with all these flags are mapped (0 = all) */
  uint8_t pad[6];
} b12g_scheme;

typedef struct b12g_tree b12g_tree;
typedef struct b12g_csr b12g_csr;

/* ---- library ---------------------------------------------------------------- */
const char* b12g_last_error(void);
const char* b12g_version(void);

/* ---- construction (ImplicitBoxTree.hpp:122-128, 28-45) ------------------------ */
/* ImplicitBoxTree(center, radius): one leaf, the surrounding box (0, depth 0, NONE) */
b12g_status b12g_tree_create(const b12g_domain* domain, b12g_tree** tree);
b12g_status b12g_tree_destroy(b12g_tree* tree);
/* reserve device capacity for `n_boxes` leaves (optional; trees grow on demand) */
b12g_status b12g_tree_reserve(b12g_tree* tree, uint64_t n_boxes);

/* ---- queries ------------------------------------------------------------------ */
/* count(depth) (ImplicitBoxTree.hpp:1061-1095) */
b12g_status b12g_count(b12g_tree* tree, uint8_t depth, uint32_t* count);
/* depth() (ImplicitBoxTree.hpp:1265-1271) */
b12g_status b12g_depth(b12g_tree* tree, uint8_t* depth);
/* the leaves in tree order: codes, depths, flags (host arrays of count(255) entries;
 * any pointer may be NULL).  Mirrors getBitPatternVector/getDepthVector/getFlagsVector. */
b12g_status b12g_leaves(b12g_tree* tree, uint64_t* codes, uint8_t* depths, uint8_t* flags);
/* replace the leaves (in tree order, none inside another; depths may differ) - the load
 * half of save/load */
b12g_status b12g_load_leaves(b12g_tree* tree, const uint64_t* codes, const uint8_t* depths,
                             const uint8_t* flags, uint32_t n);

/* ---- flags (ImplicitBoxTree.hpp:2684-2688, 3208-3411, 787-1058) ----------------- */
/* n_changed may be NULL: for the leaves' own depth (B12G_LEAF_DEPTH, or a one-depth
 * tree's depth) the update is then queued on the tree's stream without a read-back */
/* setFlags(flags, depth): returns the number of boxes that did not have them */
b12g_status b12g_set_flags(b12g_tree* tree, uint8_t flags, uint8_t depth, uint32_t* n_changed);
/* unsetFlags(flags, depth): returns the number of boxes that had any of them */
b12g_status b12g_unset_flags(b12g_tree* tree, uint8_t flags, uint8_t depth, uint32_t* n_changed);
/* changeFlags(to_unset, to_set, depth): boxes with all of to_unset get them replaced */
b12g_status b12g_change_flags(b12g_tree* tree, uint8_t to_unset, uint8_t to_set, uint8_t depth,
                              uint32_t* n_changed);

/* ---- structure ------------------------------------------------------------------ */
/* subdivide(flags) (ImplicitBoxTree.hpp:2884-2930): returns the leaves with all flags set;
 * those below depth 64 become their two halves */
b12g_status b12g_subdivide(b12g_tree* tree, uint8_t flags, uint32_t* n_subdivided);
/* remove(flags): drop leaves that do NOT have all `flags` (ImplicitBoxTree.hpp:2344-2371) */
b12g_status b12g_remove(b12g_tree* tree, uint8_t flags, uint32_t* n_removed);
/* unsubdivide(flags) (ImplicitBoxTree.hpp:3414-3460): a leaf with all flags becomes its
 * parent when its sibling is a leaf with them too (the two merge, flags ANDed) or when
 * its sibling's region holds no leaf; returns the number of parents made */
b12g_status b12g_unsubdivide(b12g_tree* tree, uint8_t flags, uint32_t* n_parents);
/* deleteDepth(depth) (ImplicitBoxTree.hpp:1217-1228); depth 0 and 255 supported */
b12g_status b12g_delete_depth(b12g_tree* tree, uint8_t depth, uint32_t* n_deleted);

/* ---- box images -------------------------------------------------------------------- */
/* setFlagsByIterators(makePointIteratorPair...(scheme), flags, depth)
 * (ImplicitBoxTree.hpp:2691-2694 via searchCompacted 2624-2681 and setFlagsBySearch 2717-2775) */
b12g_status b12g_set_flags_by_image(b12g_tree* tree, const b12g_scheme* scheme, uint8_t flags, uint8_t depth,
                                    uint32_t* n_changed);
/* searchByIterators(makePointIteratorPair...(scheme), depth) (ImplicitBoxTree.hpp:2375-2432):
 * one leaf index per mapped point, point index = source rank * points per box + grid index.
 * `out` is a host array of `capacity` entries; *n_points receives the number of points. */
b12g_status b12g_search_by_image(b12g_tree* tree, const b12g_scheme* scheme, uint8_t depth,
                                 uint32_t* out, uint64_t capacity, uint64_t* n_points);
/* insertByPoints(points, depth, ins, hit) (ImplicitBoxTree.hpp:1927-1946); points are
 * n_points x dim doubles, row-major.  depth 255 inserts at the leaf depth (each new box
 * the coarsest one that meets neither neighbour; a point in a leaf above depth 64 splits
 * it); a depth other than the leaves' merges new and old boxes on one path into the
 * deepest, flags ORed, as the reference does.  *n_inserted = distinct new boxes. */
b12g_status b12g_insert_points(b12g_tree* tree, const double* points, uint64_t n_points, uint8_t depth,
                               uint8_t flags_for_inserted, uint8_t flags_for_hit, uint32_t* n_inserted);
/* insertByIterators(makePointIteratorPairByFlags(scheme), depth, ins, hit)
 * (ImplicitBoxTree.hpp:1615-1910) */
b12g_status b12g_insert_by_image(b12g_tree* tree, const b12g_scheme* scheme, uint8_t depth,
                                 uint8_t flags_for_inserted, uint8_t flags_for_hit, uint32_t* n_inserted);

/* ---- range-partitioned trees ---------------------------------------------------------
 * One tree split over ranks, each holding a contiguous run of the leaves in the
 * reference's order.  A subdivision step sends every image point box to the rank whose
 * code range holds it; the reference is single-device, so these entries have no direct
 * counterpart: each is the named reference step restricted to the leaves of one rank.
 * Every pointer here is DEVICE memory (the buffers the collectives move); a point box is
 * a depth-64 code with a validity byte (0: the point left the domain, the reference's
 * invalid box (~0, 255)). */
/* the point boxes of the images of the scheme's sources (GridPointsFunctor +
 * PointToBox of makePointIteratorPairByFlags, ImplicitBoxTree.hpp:2624-2681),
 * source-major; CAPACITY with *n_points set when capacity is too small */
b12g_status b12g_image_point_boxes(b12g_tree* tree, const b12g_scheme* scheme, uint64_t* codes, uint8_t* valid,
                                   uint64_t capacity, uint64_t* n_points);
/* the same point boxes as a set for setFlagsByIterators (ImplicitBoxTree.hpp:2167-2196),
 * each code cut to its first `depth` bisections (the lower bits zero: the same leaves
 * hold it when no leaf is deeper than `depth`), each distinct (code, validity) pair of
 * 32 consecutive points once, in no fixed order; *n_boxes = how many were written;
 * capacity must hold one box per point (the number b12g_image_point_boxes reports),
 * else CAPACITY */
b12g_status b12g_image_distinct_point_boxes(b12g_tree* tree, const b12g_scheme* scheme, uint8_t depth,
                                            uint64_t* codes, uint8_t* valid, uint64_t capacity, uint64_t* n_boxes);
/* searchByIterators over n point boxes at the leaf depth (ImplicitBoxTree.hpp:2394-2432):
 * the leaf holding each, or B12G_INVALID_INDEX */
b12g_status b12g_search_point_boxes(b12g_tree* tree, const uint64_t* codes, const uint8_t* valid, uint64_t n,
                                    uint32_t* index);
/* setFlagsByIterators over n point boxes at the leaf depth (ImplicitBoxTree.hpp:2167-2196,
 * 2717-2775); *n_changed = leaves whose flags changed */
b12g_status b12g_set_flags_by_point_boxes(b12g_tree* tree, const uint64_t* codes, const uint8_t* valid, uint64_t n,
                                          uint8_t flags, uint32_t* n_changed);
/* the run-length step of transitionMatrixForLeaves (ImplicitBoxTree.hpp:2934-3090) for the
 * tree's leaves as rows: targets holds points_per_row column indices a row (< n_columns,
 * or B12G_INVALID_INDEX for a lost point), row-major; columns and the lost column follow
 * b12g_transition_matrix with n = n_columns */
b12g_status b12g_transition_rows(b12g_tree* tree, const uint32_t* targets, uint32_t points_per_row,
                                 uint32_t n_columns, int absolute, int invalid_column, b12g_csr** csr);
/* b12g_load_leaves from device buffers, with the same checks made on the device (a
 * failed check leaves the surrounding box); b12g_leaves copies into host or device
 * buffers alike */
b12g_status b12g_load_leaves_device(b12g_tree* tree, const uint64_t* codes, const uint8_t* depths,
                                    const uint8_t* flags, uint32_t n);
/* Routing of n point boxes (device buffers) to the ranks that own them (no counterpart
 * in the reference, which runs on one device): run r of the tree's leaves starts at the
 * depth-64 code run_starts[r] and lives on rank run_ranks[r] (host arrays of the n_runs
 * non-empty runs, both ascending); a valid box goes to the last run starting at or below
 * it, an invalid one to the last run.  out_codes / out_valid receive the boxes grouped by
 * rank, in their order within each rank; slot (device, may be NULL) the position of box
 * i in the output; counts (host, `world` entries) the boxes for each rank.  Uses the
 * tree's stream and scratch and returns after the work has finished. */
b12g_status b12g_route_point_boxes(b12g_tree* tree, const uint64_t* codes, const uint8_t* valid, uint64_t n,
                                   const uint64_t* run_starts, const uint32_t* run_ranks, uint32_t n_runs,
                                   uint32_t world, uint64_t* out_codes, uint8_t* out_valid, uint32_t* slot,
                                   uint64_t* counts);
/* one leaf (index in tree order) to the host: code, depth and flags (any may be NULL) */
b12g_status b12g_leaf_at(b12g_tree* tree, uint32_t index, uint64_t* code, uint8_t* depth, uint8_t* flags);

/* ---- transition matrix (ImplicitBoxTree.hpp:2934-3193, CooMatrix.hpp:14-56) ---------- */
/* transitionMatrixForLeaves<double>(grid, map, absolute, rowMajor=true, invalid):
 * row = source leaf, column = target leaf, value = count (absolute) or count / P.
 * With `invalid_column`, lost points go to column n + 1 and the matrix has n + 1 columns
 * if any point was lost, n otherwise (ImplicitBoxTree.hpp:3075-3090).
 * The result is a row-major CSR that stays on the device.  *csr must be NULL (a new
 * matrix is created) or a matrix from an earlier call, which is refilled in place. */
b12g_status b12g_transition_matrix(b12g_tree* tree, const b12g_scheme* scheme, int absolute,
                                   int invalid_column, b12g_csr** csr);
b12g_status b12g_csr_shape(const b12g_csr* csr, uint32_t* n_rows, uint32_t* n_cols, uint64_t* nnz);
/* copy to host: rowptr[n_rows+1], cols[nnz], vals[nnz] (any may be NULL) */
b12g_status b12g_csr_copy(const b12g_csr* csr, uint32_t* rowptr, uint32_t* cols, double* vals);
b12g_status b12g_csr_destroy(b12g_csr* csr);
/* invariant measure: v <- P^T v / |P^T v|_1, `iters` times from the uniform vector,
 * FP64 (the eigenvector step of subdivisionByNim.m:30-58).  v: host array of n_rows,
 * or NULL to keep the result on the device (b12g_csr_measure copies it later). */
b12g_status b12g_invariant_measure(b12g_csr* csr, uint32_t iters, double* v);
/* the same power iteration run until it settles, as subdivisionByNim.m:30-45 asks of
 * powerMethodMPE(P, 1e-14, 1e9) (not shipped with the reference): launches of
 * check_every iterations, each continuing from the last iterate, until the L1 change
 * made by one iteration, |v_k - v_(k-1)|_1, is at most `tol`, or max_iters iterations.
 * v: host array of n_rows (or NULL, the result stays on the device); *iters_done and
 * *last_change (either may be NULL) receive the iterations run and that change. */
b12g_status b12g_invariant_measure_tol(b12g_csr* csr, double tol, uint32_t max_iters, uint32_t check_every,
                                       double* v, uint32_t* iters_done, double* last_change);
/* copy the last invariant measure of `csr` to the host array v (n_rows entries) */
b12g_status b12g_csr_measure(const b12g_csr* csr, double* v);
/* Allocation-free invariant measure (no counterpart in the reference): for callers that
 * cannot let the library allocate device memory - a process whose own memory pool owns
 * the free HBM, or a latency-critical loop where cudaMalloc/cudaFree would synchronize
 * the device.  Same power iteration as b12g_invariant_measure, on the CSR of P^T given
 * as device arrays (tptr[n+1], trows[nnz], tvals[nnz]; sources ascending in each row),
 * result in the device array v[n].  Every row pointer must be non-decreasing from
 * tptr[0] = 0 and every source below n; a matrix that breaks this is refused with
 * B12G_ERR_INVALID (a check kernel reads tptr and trows once before the iteration).
 * Its scratch is one fixed __device__ array shared by all calls: at most 262,144 boxes
 * (B12G_ERR_CAPACITY above that), and calls that overlap on the GPU race.  The first
 * call on a device looks up the array's device address.  The call waits for `stream`
 * twice (after the check and after the iteration, to read their error words) and
 * returns after the work on `stream` has finished. */
b12g_status b12g_invariant_measure_noalloc(const uint32_t* tptr, const uint32_t* trows, const double* tvals,
                                           uint32_t n, uint32_t iters, double* v, void* stream);

/* ---- fused drivers ------------------------------------------------------------------- */
/* The subdivision loop of B12_doc.tex:269-290 / subdivision.m:18-45,
 *   setFlags(SD); repeat steps: subdivide(SD); setFlagsByIterators(scheme, HIT);
 *   remove(HIT); unsetFlags(HIT)
 * run on the device without host round trips.  counts[k] = leaves after step k+1
 * (host array of `steps` entries, may be NULL). */
b12g_status b12g_subdivision_run(b12g_tree* tree, const b12g_scheme* scheme, uint32_t steps, uint32_t* counts);
/* The continuation loop of continuation.m:13-44 at one depth: deleteDepth(0);
 * insertByPoints(x0, depth, INS); repeat { changeFlags(INS, EXPD); insert(scheme on
 * EXPD boxes, INS); unsetFlags(EXPD) } until the count stops growing (or max_sweeps).
 * counts: host array of max_sweeps entries (may be NULL); *n_sweeps receives the sweeps. */
b12g_status b12g_continuation_run(b12g_tree* tree, const b12g_scheme* scheme, const double* x0, uint64_t n_x0,
                                  uint8_t depth, uint32_t max_sweeps, uint32_t* counts, uint32_t* n_sweeps);

/* ---- selection steps that consume a transition matrix ------------------------------------
 * The Matlab drivers chainRecurrentSet.m:18-44 (keep the boxes of strongly connected
 * components of P's graph with at least two boxes; graphconncomp(P') there) and
 * subdivisionByNim.m:22-66 (keep the boxes whose invariant measure is at least 1e-9 / n;
 * an eigensolver there, the FP64 power iteration here). */
/* component label of every row's box: the largest box index of its strongly connected
 * component (self-loops join nothing; the lost column is ignored); comp: host, n_rows entries */
b12g_status b12g_csr_strong_components(b12g_csr* matrix, uint32_t* comp, uint32_t* n_components);
/* setFlags(stencil, flags) with the stencil "in a component of at least min_size boxes"
 * (chainRecurrentSet.m:29-37); the matrix's rows are the tree's leaves */
b12g_status b12g_set_flags_by_components(b12g_tree* tree, b12g_csr* matrix, uint32_t min_size, uint8_t flags,
                                         uint32_t* n_flagged);
/* setFlags(stencil, flags) with the stencil "measure >= threshold" on the matrix's last
 * invariant measure (subdivisionByNim.m:56-62 uses threshold 1e-9 / n) */
b12g_status b12g_set_flags_by_measure(b12g_tree* tree, b12g_csr* matrix, double threshold, uint8_t flags,
                                      uint32_t* n_flagged);
/* the two drivers: setFlags(SD); steps x {subdivide(SD); transition matrix; select with
 * HIT; remove(HIT); unsetFlags(HIT)}; counts: leaves after each step (may be NULL) */
b12g_status b12g_chain_recurrent_run(b12g_tree* tree, const b12g_scheme* scheme, uint32_t steps, uint32_t* counts);
/* fixedBoxes.m:15-17: flag every leaf one of whose own test points lands in it again
 * (search(scheme), then any(s == box index) per box) */
b12g_status b12g_set_flags_by_self_hit(b12g_tree* tree, const b12g_scheme* scheme, uint8_t flags,
                                       uint32_t* n_flagged);
/* fixedBoxes.m:10-22: deleteDepth(0); setFlags(SD); steps x {subdivide(SD); self-hit
 * selection with HIT; remove(HIT); unsetFlags(HIT)} */
b12g_status b12g_fixed_boxes_run(b12g_tree* tree, const b12g_scheme* scheme, uint32_t steps, uint32_t* counts);
b12g_status b12g_nim_run(b12g_tree* tree, const b12g_scheme* scheme, uint32_t steps, uint32_t power_iterations,
                         uint32_t* counts);
/* the NIM driver with the measure of every step run to the tolerance `tol`
 * (b12g_invariant_measure_tol, checked every 20 iterations, at most max_iters) */
b12g_status b12g_nim_run_tol(b12g_tree* tree, const b12g_scheme* scheme, uint32_t steps, double tol,
                             uint32_t max_iters, uint32_t* counts);

/* ---- JSON files in the reference's format ----------------------------------------------
 * Trees as written by ImplicitBoxTree::save (ImplicitBoxTree.hpp:435-528) and read by
 * ImplicitBoxTree(fileName) (ImplicitBoxTree.hpp:144-359, JSON files only): center,
 * radius, sdScheme, nLeaves, bitPatternVector, depthVector, flagsVector, nHostBufferBytes.
 * Matrices as written by CooMatrix::save (CooMatrix.hpp:473-525) and read by
 * CooMatrix(fileName) (CooMatrix.hpp:236-291): nRows, nColumns, nnz and the row-major
 * triples.  Files written here are byte for byte what the reference writes for the same
 * tree or matrix; ".json" is appended to a path without it, as the reference does.
 * Loading needs the default subdivision scheme. */
b12g_status b12g_tree_save_json(b12g_tree* tree, const char* path);
b12g_status b12g_tree_load_json(const char* path, b12g_tree** tree);
b12g_status b12g_csr_save_json(const b12g_csr* matrix, const char* path);
b12g_status b12g_csr_load_json(const char* path, b12g_csr** matrix);
/* the same files from and to host arrays (no device involved): *n is the capacity of the
 * arrays on entry (any array may be NULL to query the count) and the leaf count on return */
b12g_status b12g_json_write_leaves(const char* path, const b12g_domain* domain, const uint64_t* codes,
                                   const uint8_t* depths, const uint8_t* flags, uint64_t n);
b12g_status b12g_json_read_leaves(const char* path, b12g_domain* domain, uint64_t* codes, uint8_t* depths,
                                  uint8_t* flags, uint64_t* n);
/* CSR arrays (rowptr: n_rows + 1 entries); reading fills rowptr, cols, vals when not NULL */
b12g_status b12g_json_write_coo(const char* path, uint32_t n_rows, uint32_t n_cols, const uint32_t* rowptr,
                                const uint32_t* cols, const double* vals);
b12g_status b12g_json_read_coo(const char* path, uint32_t* n_rows, uint32_t* n_cols, uint32_t* rowptr,
                               uint32_t* cols, double* vals, uint64_t* nnz);

/* ---- batches of independent subdivision jobs --------------------------------------------
 * Many instances of the subdivision loop (subdivision.m:18-45) with one domain, map
 * kind, grid and arithmetic but per-instance map parameters and depths, advanced in
 * lockstep on one GPU: one persistent launch per subdivision step serves every
 * instance still subdividing, fed by a device work queue of point chunks; the steps
 * run as one CUDA graph; the launch shape is autotuned on the first run.  The reference
 * runs such scans one ImplicitBoxTree at a time.  Inner and full grids only. */
typedef struct b12g_batch b12g_batch;
/* params: n x 6 map parameters (b12g_map.p per instance); depths: n target depths 1..32 */
b12g_status b12g_batch_create(const b12g_domain* domain, const b12g_scheme* scheme, uint32_t n,
                              const double* params, const uint8_t* depths, b12g_batch** batch);
b12g_status b12g_batch_destroy(b12g_batch* batch);
/* run every instance's subdivision loop from the surrounding box */
b12g_status b12g_batch_run(b12g_batch* batch);
/* leaf counts of instance i after each of its steps (depth_i entries) */
b12g_status b12g_batch_counts(b12g_batch* batch, uint32_t i, uint32_t* counts);
/* final leaves of instance i (codes/flags may be NULL to query *n and *depth) */
b12g_status b12g_batch_leaves(b12g_batch* batch, uint32_t i, uint64_t* codes, uint8_t* flags, uint32_t* n,
                              uint8_t* depth);
/* every instance's transition matrix (transitionMatrixForLeaves), resident on the device */
b12g_status b12g_batch_transition_matrices(b12g_batch* batch, int absolute, int invalid_column);
/* instance i's CSR (host arrays, any may be NULL to query sizes) */
b12g_status b12g_batch_csr(b12g_batch* batch, uint32_t i, uint32_t* rowptr, uint32_t* cols, double* vals,
                           uint32_t* n_rows, uint64_t* nnz);
/* box-images of the last run, final boxes, nonzeros, and the autotuned launch shape */
b12g_status b12g_batch_info(b12g_batch* batch, uint64_t* box_images, uint64_t* final_boxes, uint64_t* nnz,
                            uint32_t* threads, uint32_t* points_per_thread, uint32_t* chunk);
b12g_status b12g_batch_stream(b12g_batch* batch, void** stream);

/* ---- job server: continuous batching of subdivision jobs ---------------------------------
 * No counterpart in the reference, which runs one ImplicitBoxTree per process.  A job is
 * `depth` steps of the subdivision loop (subdivision.m:18-45) from the surrounding box,
 * followed by transitionMatrixForLeaves (relative transition probabilities, points
 * leaving the leaves dropped).  Jobs of one family (domain, map kind, arithmetic,
 * integrator step and steps, grid) share an engine: a host thread and CUDA stream that
 * advances every job it holds by one subdivision step per tick in one batched launch
 * sequence; a job submitted while others run joins at the next tick, and leaves at the
 * end of its last step with its leaves and CSR resident on the device until released.
 * Families run concurrently.  Admission is by projected HBM footprint against the
 * server's cap (first come, first served within a family); a job's reservation lasts
 * until its result is released, so a client that holds results while waiting for later
 * jobs can stall admission once the cap is reached.  Inner and full grids with up
 * to 128 points per box. */
typedef struct b12g_server b12g_server;
typedef struct {
  b12g_domain domain;
  b12g_map map;          /* p[] is the job's own parameter set */
  b12g_grid grid;
  uint32_t depth;        /* subdivision steps, 1..32 */
  uint32_t pad;
} b12g_job;
enum { B12G_JOB_WAITING = 0, B12G_JOB_RUNNING = 1, B12G_JOB_DONE = 2, B12G_JOB_FAILED = 3 };
typedef struct {
  uint32_t state;
  uint32_t depth;
  uint32_t n_boxes;      /* final leaves (done jobs) */
  uint32_t pad;
  uint64_t nnz;
  double t_submit, t_start, t_done;   /* seconds on the server's steady clock */
} b12g_job_info;
/* hbm_cap_bytes: admission cap (0: 80% of the free device memory at creation) */
b12g_status b12g_server_create(uint64_t hbm_cap_bytes, b12g_server** server);
/* stops the engines after their current tick and frees every result */
b12g_status b12g_server_destroy(b12g_server* server);
b12g_status b12g_server_submit(b12g_server* server, const b12g_job* job, uint64_t* id);
/* ids of jobs finished (or failed) since the last poll, waiting up to wait_seconds for one */
b12g_status b12g_server_poll(b12g_server* server, uint64_t* ids, uint32_t max, uint32_t* n, double wait_seconds);
b12g_status b12g_server_job(b12g_server* server, uint64_t id, b12g_job_info* info);
/* a done job's leaf counts after each step (depth entries), final leaves (n_boxes codes at
 * the job's depth) and CSR; any pointer may be NULL */
b12g_status b12g_server_result(b12g_server* server, uint64_t id, uint64_t* codes, uint32_t* counts,
                               uint32_t* rowptr, uint32_t* cols, double* vals);
/* free a done or failed job's resident result and its admission reservation */
b12g_status b12g_server_release(b12g_server* server, uint64_t id);
b12g_status b12g_server_stats(b12g_server* server, uint64_t* ticks, uint64_t* box_images, uint64_t* in_use_bytes,
                              uint64_t* cap_bytes, uint32_t* waiting, uint32_t* running);
/* engine i (in order of creation): its map kind, ticks, finished jobs, and host seconds
 * spent in ticks (finishing included) and in finishing jobs; B12G_ERR_INVALID past the last */
b12g_status b12g_server_engine_stats(b12g_server* server, uint32_t i, uint32_t* map_kind, uint64_t* ticks,
                                     uint64_t* jobs_done, double* tick_seconds, double* finish_seconds);

/* ---- measurement hooks (no counterpart in the reference) ---------------------------------- */
/* the CUDA stream (cudaStream_t) every kernel of this tree runs on */
b12g_status b12g_tree_stream(b12g_tree* tree, void** stream);
/* time every box-image (kind 0) and transition-row (kind 1) kernel launch with CUDA
 * events on the tree's stream; read the accumulated device milliseconds and launches */
b12g_status b12g_profile_enable(b12g_tree* tree, int enable);
b12g_status b12g_profile_read(b12g_tree* tree, uint32_t kind, double* ms_total, uint64_t* launches, int reset);
/* kernels this process has launched through the library (graph replays included) */
b12g_status b12g_launch_count(uint64_t* launches);
/* FP64 fused multiply-add throughput of the current device (TFLOP/s, FMA = 2 FLOPs),
 * measured with a launch of about `seconds_hint` seconds */
b12g_status b12g_probe_fp64_fma(double seconds_hint, double* tflops, double* seconds);

#ifdef __cplusplus
}
#endif
#endif /* B12G_H */
