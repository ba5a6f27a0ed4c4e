/*
 * ORACLE - test infrastructure only.
 *
 * A plain-C restatement of the reference's set-oriented box-image path
 * (SON-GPU-Enabler/B12, B12c/src/include).  It is the checker for the CUDA library:
 * only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py may load
 * it.  The product never calls it and has no CPU fallback.
 *
 * Parity pin: the restatement is checked against outputs of the reference itself,
 * compiled from its own headers with the Thrust OMP backend (oracle/ref, built into
 * oracle/_ref) - per-step leaf sets and transition matrices are committed as golden
 * fixtures under tests/golden/.  The invariant measure has no reference implementation
 * (the Matlab driver's powerMethodMPE is not shipped): that part is unpinned.
 *
 * Arithmetic: compiled with -ffp-contract=off and without -march=native, so every
 * FP64 operation is rounded separately (the reference built with -fmad=false); the
 * explicit-FMA Lorenz variant calls the correctly rounded C99 fma().
 */
#ifndef B12_ORACLE_H
#define B12_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_DIM 4
#define ORC_LEAF_DEPTH 255u
#define ORC_INVALID 0xFFFFFFFFu

/* map ids (same numbering as the CUDA library's b12g_map_kind) */
enum { ORC_MAP_HENON = 1, ORC_MAP_LORENZ = 2, ORC_MAP_COUPLED_DUFFING = 3, ORC_MAP_FORCED_DUFFING = 4 };
/* grid ids */
enum { ORC_GRID_INNER = 1, ORC_GRID_FULL = 2, ORC_GRID_PHILOX = 3 };

typedef struct {
  uint32_t kind;        /* ORC_MAP_* */
  uint32_t fma;         /* 1: explicit-FMA arithmetic (Lorenz only) */
  uint32_t steps;       /* iterates / integrator steps */
  uint32_t pad;
  double h;             /* integrator step */
  double p[6];          /* parameters: Henon (a,b); Lorenz (sigma,rho,beta); forced Duffing (delta,alpha,beta,gamma) */
  const double* table;  /* forced Duffing: cos at t = j*h/2, j = 0..2*steps */
} orc_map;

typedef struct {
  uint32_t kind;        /* ORC_GRID_* */
  uint32_t n;           /* points per dimension (inner/full) */
  uint64_t points;      /* points per box (philox) */
  uint64_t seed;        /* philox key */
  double eps;           /* full grid stretch */
} orc_grid;

typedef struct {
  uint32_t dim;
  double center[ORC_MAX_DIM];
  double radius[ORC_MAX_DIM];
} orc_domain;

/* a tree of leaves kept sorted in the reference's tree order */
typedef struct {
  orc_domain dom;
  uint64_t n, cap;
  uint64_t* code;
  uint8_t* depth;
  uint8_t* flags;
} orc_tree;

/* ---- geometry and plug-ins ---- */
uint64_t orc_grid_points_per_box(const orc_grid* g, uint32_t dim);
void orc_grid_point(const orc_grid* g, uint32_t dim, uint64_t i, double* res);
void orc_map_apply(const orc_map* m, const double* x, double* res);
void orc_box_coordinates(const orc_domain* d, uint64_t code, uint32_t depth, double* center, double* radius);
/* depth-64 point code, as the reference computes it; returns 0 for points outside the domain */
int orc_point_code64(const orc_domain* d, const double* p, uint64_t* code64);
void orc_forced_duffing_table(uint32_t steps, double period, double* table);
void orc_philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1);

/* ---- tree ---- */
void orc_tree_init(orc_tree* t, const orc_domain* d);     /* surrounding box (0, 0, NONE) */
void orc_tree_free(orc_tree* t);
void orc_tree_load(orc_tree* t, const uint64_t* code, const uint8_t* depth, const uint8_t* flags, uint64_t n);
uint32_t orc_set_flags(orc_tree* t, uint8_t flags);
uint32_t orc_set_flags_mask(orc_tree* t, const uint8_t* mask, uint8_t flags);
uint32_t orc_unset_flags(orc_tree* t, uint8_t flags);
uint32_t orc_change_flags(orc_tree* t, uint8_t to_unset, uint8_t to_set);
uint32_t orc_subdivide(orc_tree* t, uint8_t flags);
uint32_t orc_remove(orc_tree* t, uint8_t flags);
/* search of a depth-64 point box among the leaves; ORC_INVALID if no leaf contains it */
uint32_t orc_search(const orc_tree* t, uint64_t code64, int valid);
/* point boxes of a range-partitioned tree */
void orc_image_point_boxes(const orc_tree* t, const orc_map* m, const orc_grid* g, uint64_t* codes, uint8_t* valid);
void orc_search_point_boxes(const orc_tree* t, const uint64_t* codes, const uint8_t* valid, uint64_t n,
                            uint32_t* out);
uint32_t orc_set_flags_by_point_boxes(orc_tree* t, const uint64_t* codes, const uint8_t* valid, uint64_t n,
                                      uint8_t flags);
uint64_t orc_transition_rows(uint32_t* tgt, uint64_t n, uint64_t P, uint32_t n_cols, int absolute, int invalid,
                             uint32_t* rowptr, uint32_t* cols, double* vals, uint32_t* out_n_cols);
/* per-point target leaf index of the image of grid point i of source leaf src[k] */
void orc_search_by_image(const orc_tree* t, const orc_map* m, const orc_grid* g,
                         const uint32_t* src, uint64_t n_src, uint32_t* out);
uint32_t orc_set_flags_by_image(orc_tree* t, const orc_map* m, const orc_grid* g, uint8_t flags);
/* continuation insert at uniform depth d: sources = leaves with flags_to_check */
uint32_t orc_insert_by_image(orc_tree* t, const orc_map* m, const orc_grid* g, uint8_t flags_to_check,
                             uint8_t ins, uint8_t hit);
uint32_t orc_insert_points(orc_tree* t, const double* pts, uint64_t n_points, uint32_t depth, uint8_t ins,
                           uint8_t hit);
void orc_delete_depth0(orc_tree* t);

/* trees of mixed depths: unsubdivide, and insertByIterators for any tree and depth
 * (255 = leaf depth) */
uint32_t orc_unsubdivide(orc_tree* t, uint8_t flags);
/* set / unset / change (op 0 / 1 / 2) flags of the boxes at an inner depth; for change, u
 * is unset and f set */
uint32_t orc_flags_at_depth(orc_tree* t, int op, uint8_t u, uint8_t f, uint32_t depth);
/* images of every leaf located at an inner depth d: flags on the boxes hit (returns the
 * hit boxes that lacked them), or with out != NULL each point's box index at d */
uint32_t orc_image_at_depth(orc_tree* t, const orc_map* m, const orc_grid* g, uint32_t d, uint8_t flags,
                            uint32_t* out);
/* the images of a scheme's sources (leaves with flags_to_check at src_depth 255, or the
 * boxes of an inner src_depth whose leaves all have them) located at `target` (255: the
 * leaves, else an inner depth): flags on what is hit, or each point's index into out */
uint32_t orc_image_search(orc_tree* t, const orc_map* m, const orc_grid* g, uint32_t src_depth, uint8_t flags_to_check,
                          uint32_t target, uint8_t flags, uint32_t* out, uint64_t* n_points);
uint32_t orc_insert_boxes(orc_tree* t, const uint64_t* code64, const uint8_t* valid, uint64_t n_points,
                          uint32_t depth, uint8_t ins, uint8_t hit, int* unsupported);
uint32_t orc_insert_points_general(orc_tree* t, const double* pts, uint64_t n_points, uint32_t depth, uint8_t ins,
                                   uint8_t hit, int* unsupported);
uint32_t orc_insert_by_image_general(orc_tree* t, const orc_map* m, const orc_grid* g, uint8_t flags_to_check,
                                     uint32_t depth, uint8_t ins, uint8_t hit, int* unsupported);
/* the same with the scheme's sources at src_depth (255: leaves; else the boxes of that
 * inner depth whose leaves all have flags_to_check) */
uint32_t orc_insert_by_image_src(orc_tree* t, const orc_map* m, const orc_grid* g, uint32_t src_depth,
                                 uint8_t flags_to_check, uint32_t depth, uint8_t ins, uint8_t hit, int* unsupported);

/* transition matrix on the leaves, row-major CSR; returns nnz.  Pass NULL arrays to
 * query nnz only.  absolute: values are counts; invalid: lost points go to column
 * n+1 as in the reference (nColumns becomes n+1). */
uint64_t orc_transition_matrix(const orc_tree* t, const orc_map* m, const orc_grid* g, int absolute, int invalid,
                               uint32_t* rowptr, uint32_t* cols, double* vals, uint32_t* n_cols);

/* v <- P^T v, L1-normalised, `iters` times from the uniform vector */
void orc_strong_components(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, uint32_t* comp);
void orc_invariant_measure(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const double* vals,
                           uint32_t iters, double* v);
void orc_invariant_measure_tol(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const double* vals,
                               double tol, uint32_t max_iters, uint32_t check_every, double* v, uint32_t* iters_done,
                               double* last_change);

/* whole subdivision loop; counts[k] = leaves after step k+1; returns box-images */
uint64_t orc_subdivision(orc_tree* t, const orc_map* m, const orc_grid* g, uint32_t steps, uint32_t* counts);

int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
