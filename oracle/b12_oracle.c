/*
 * ORACLE - test infrastructure only (see b12_oracle.h).
 *
 * Plain-C restatement of the reference's box-image path.  Every function cites the
 * reference file:line it restates (paths relative to B12c/src/include unless noted).
 * Build: gcc -O2 -fopenmp -ffp-contract=off -fPIC -shared (oracle/Makefile).
 */
#include "b12_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NONE_FLAGS 0u
#define INVALID_CODE (~(uint64_t)0)

int orc_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* safeLeftShift / safeRightShift for 64-bit patterns (BitPattern.hpp:3-28) */
static inline uint64_t sls(uint64_t b, int i) { return i <= 0 ? b : (i >= 64 ? 0 : b << i); }
static inline uint64_t srs(uint64_t b, int i) { return i <= 0 ? b : (i >= 64 ? 0 : b >> i); }

/* ------------------------------------------------------------------------------
 * grids (Grids.hpp:12-162)
 * ---------------------------------------------------------------------------- */
static uint64_t ipow_u64(uint64_t b, uint32_t e)
{
  uint64_t r = 1;
  while (e--) r *= b;
  return r;
}

/* getNumberOfPointsPerBox (Grids.hpp:79-83, 131-134, 158-162) */
uint64_t orc_grid_points_per_box(const orc_grid* g, uint32_t dim)
{
  return g->kind == ORC_GRID_PHILOX ? g->points : ipow_u64(g->n, dim);
}

/* Philox4x32-10 (Salmon et al., SC'11): published round multipliers and Weyl steps */
void orc_philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    c[0] = n0; c[1] = (uint32_t)p1; c[2] = n2; c[3] = (uint32_t)p0;
  }
}

static inline double philox_signed(uint32_t hi, uint32_t lo)
{
  const uint64_t m = (((uint64_t)hi << 32) | (uint64_t)lo) >> 11;
  return 2.0 * ((double)m * 0x1p-53) - 1.0;
}

void orc_grid_point(const orc_grid* g, uint32_t dim, uint64_t i, double* res)
{
  if (g->kind == ORC_GRID_INNER) {
    /* InnerGrid::operator() (Grids.hpp:105-120) */
    const uint64_t n = g->n;
    uint64_t tmp = 1;
    for (uint32_t j = 0; j < dim; ++j) {
      res[j] = (((double)((i / tmp) % n) * 2.0 + 1.0) - (double)n) / (double)n;
      tmp *= n;
    }
  } else if (g->kind == ORC_GRID_FULL) {
    /* FullGrid::operator() (Grids.hpp:67-83) */
    const uint64_t n = g->n;
    uint64_t tmp = 1;
    for (uint32_t j = 0; j < dim; ++j) {
      res[j] = ((double)((i / tmp) % n) * 2.0) / (double)(n - 1) - 1.0;
      res[j] *= 1.0 + g->eps;
      tmp *= n;
    }
  } else {
    /* Philox plug-in keyed by (seed, global point index), replacing UniformGrid
     * (Grids.hpp:143-162), whose host and device generators differ */
    for (uint32_t j = 0; j < dim; j += 2) {
      uint32_t c[4] = {(uint32_t)i, (uint32_t)(i >> 32), j / 2, 0u};
      orc_philox4x32_10(c, (uint32_t)g->seed, (uint32_t)(g->seed >> 32));
      res[j] = philox_signed(c[0], c[1]);
      if (j + 1 < dim) res[j + 1] = philox_signed(c[2], c[3]);
    }
  }
}

/* ------------------------------------------------------------------------------
 * maps
 * ---------------------------------------------------------------------------- */
/* HenonMap (Map_Henon.h:11-24) */
static inline void henon(const double* p, double a, double b, double* r)
{
  r[0] = (1.0 - (a * p[0]) * p[0]) + p[1];
  r[1] = b * p[0];
}

/* LorenzRHS (Map_Lorenz.h:10-24) */
static inline void lorenz_rhs(const double* s, const double* p, double* r)
{
  r[0] = s[0] * (p[1] - p[0]);
  r[1] = (s[1] * p[0] - p[1]) - p[0] * p[2];
  r[2] = (-s[2]) * p[2] + p[0] * p[1];
}

static inline void lorenz_rhs_fma(const double* s, const double* p, double* r)
{
  r[0] = s[0] * (p[1] - p[0]);
  r[1] = fma(-p[0], p[2], fma(s[1], p[0], -p[1]));
  r[2] = fma(p[0], p[1], (-s[2]) * p[2]);
}

/* RK4Auto::operator() (MapTools.hpp:118-182) with the Lorenz right-hand side */
static void lorenz_map(const orc_map* m, const double* x0, double* res)
{
  double x[3] = {x0[0], x0[1], x0[2]}, k[3], a[3];
  const double h = m->h;
  for (uint32_t s = 0; s < m->steps; ++s) {
    if (!m->fma) {
      lorenz_rhs(m->p, x, k);
      for (int j = 0; j < 3; ++j) res[j] = x[j] + (h / 6.0) * k[j];
      for (int j = 0; j < 3; ++j) a[j] = x[j] + (h / 2.0) * k[j];
      lorenz_rhs(m->p, a, k);
      for (int j = 0; j < 3; ++j) res[j] += (h / 3.0) * k[j];
      for (int j = 0; j < 3; ++j) a[j] = x[j] + (h / 2.0) * k[j];
      lorenz_rhs(m->p, a, k);
      for (int j = 0; j < 3; ++j) res[j] += (h / 3.0) * k[j];
      for (int j = 0; j < 3; ++j) a[j] = x[j] + h * k[j];
      lorenz_rhs(m->p, a, k);
      for (int j = 0; j < 3; ++j) res[j] += (h / 6.0) * k[j];
    } else {
      const double h6 = h / 6.0, h3 = h / 3.0, h2 = h / 2.0;
      lorenz_rhs_fma(m->p, x, k);
      for (int j = 0; j < 3; ++j) { res[j] = fma(h6, k[j], x[j]); a[j] = fma(h2, k[j], x[j]); }
      lorenz_rhs_fma(m->p, a, k);
      for (int j = 0; j < 3; ++j) { res[j] = fma(h3, k[j], res[j]); a[j] = fma(h2, k[j], x[j]); }
      lorenz_rhs_fma(m->p, a, k);
      for (int j = 0; j < 3; ++j) { res[j] = fma(h3, k[j], res[j]); a[j] = fma(h, k[j], x[j]); }
      lorenz_rhs_fma(m->p, a, k);
      for (int j = 0; j < 3; ++j) res[j] = fma(h6, k[j], res[j]);
    }
    for (int j = 0; j < 3; ++j) x[j] = res[j];
  }
}

/* SymplecticIntegratorAuto order 2 (MapTools.hpp:371-421) with the coupled-Duffing
 * right-hand sides: RHS1(p) = p, RHS2(q) = -grad V(q) */
static void coupled_duffing_map(const orc_map* m, const double* x0, double* res)
{
  double t[2];
  const double h = m->h;
  for (int j = 0; j < 4; ++j) res[j] = x0[j];
  for (uint32_t s = 0; s < m->steps; ++s) {
    t[0] = res[2]; t[1] = res[3];
    for (int j = 0; j < 2; ++j) res[j] += (0.5 * t[j]) * h;
    t[0] = (res[0] - (res[0] * res[0]) * res[0]) - ((0.2 * res[0]) * res[1]) * res[1];
    t[1] = (-1.69 * res[1]) - ((0.2 * res[0]) * res[0]) * res[1];
    for (int j = 0; j < 2; ++j) res[2 + j] += t[j] * h;
    t[0] = res[2]; t[1] = res[3];
    for (int j = 0; j < 2; ++j) res[j] += (0.5 * t[j]) * h;
  }
}

/* forced Duffing: exactly `steps` RK4 steps (the classical RK4 of MapTools.hpp:42-108
 * with the stage forcing read from a host cos table) */
static inline void forced_rhs(const double* q, double c, const double* p, double* r)
{
  r[0] = p[1];
  r[1] = (((-q[0] * p[1]) - q[1] * p[0]) - q[2] * ((p[0] * p[0]) * p[0])) + q[3] * c;
}

static void forced_duffing_map(const orc_map* m, const double* x0, double* res)
{
  const double h = m->h, h6 = h / 6.0, h3 = h / 3.0, h2 = h / 2.0;
  double x[2] = {x0[0], x0[1]}, k[2], a[2];
  for (uint32_t s = 0; s < m->steps; ++s) {
    const double c0 = m->table[2 * s], c1 = m->table[2 * s + 1], c2 = m->table[2 * s + 2];
    forced_rhs(m->p, c0, x, k);
    for (int j = 0; j < 2; ++j) { res[j] = x[j] + h6 * k[j]; a[j] = x[j] + h2 * k[j]; }
    forced_rhs(m->p, c1, a, k);
    for (int j = 0; j < 2; ++j) { res[j] += h3 * k[j]; a[j] = x[j] + h2 * k[j]; }
    forced_rhs(m->p, c1, a, k);
    for (int j = 0; j < 2; ++j) { res[j] += h3 * k[j]; a[j] = x[j] + h * k[j]; }
    forced_rhs(m->p, c2, a, k);
    for (int j = 0; j < 2; ++j) { res[j] += h6 * k[j]; x[j] = res[j]; }
  }
}

void orc_forced_duffing_table(uint32_t steps, double period, double* table)
{
  for (uint32_t j = 0; j <= 2 * steps; ++j) table[j] = cos((double)j * (period / (double)(2 * steps)));
}

void orc_map_apply(const orc_map* m, const double* x, double* res)
{
  switch (m->kind) {
    case ORC_MAP_HENON: {
      /* IteratingMap (MapTools.hpp:10-32) */
      uint32_t i = 0;
      double tmp[2];
      if (m->steps & 1u) { henon(x, m->p[0], m->p[1], res); i = 1; }
      else { res[0] = x[0]; res[1] = x[1]; }
      for (; i < m->steps; i += 2) { henon(res, m->p[0], m->p[1], tmp); henon(tmp, m->p[0], m->p[1], res); }
      break;
    }
    case ORC_MAP_LORENZ: lorenz_map(m, x, res); break;
    case ORC_MAP_COUPLED_DUFFING: coupled_duffing_map(m, x, res); break;
    case ORC_MAP_FORCED_DUFFING: forced_duffing_map(m, x, res); break;
    default: break;
  }
}

/* ------------------------------------------------------------------------------
 * geometry (coordinateFunctions.hpp)
 * ---------------------------------------------------------------------------- */
/* computeCoordinatesOfBoxFixedSdScheme (coordinateFunctions.hpp:130-159) */
void orc_box_coordinates(const orc_domain* d, uint64_t code, uint32_t depth, double* center, double* radius)
{
  const int D = (int)d->dim;
  for (int j = 0; j < D; ++j) {
    uint64_t bits = 0;
    const int initialShift = (D + (int)depth - 1 - j) % D;
    for (int i = 0; i * D < 64; ++i)
      bits |= srs(code, i * (D - 1) + initialShift) & sls(1, i);
    const int k = (int)depth / D + (j < (int)depth % D ? 1 : 0);
    radius[j] = ldexp(d->radius[j], -k);
    center[j] = ((ldexp((double)bits, -k) * 2.0 - 1.0) * d->radius[j] + d->center[j]) + radius[j];
  }
}

/* isPointInBox + computeBoxFromPointFixedSdScheme (coordinateFunctions.hpp:9-19, 63-93) */
int orc_point_code64(const orc_domain* d, const double* p, uint64_t* code64)
{
  const int D = (int)d->dim;
  for (int j = 0; j < D; ++j)
    if (!(d->center[j] - d->radius[j] <= p[j] && p[j] < d->center[j] + d->radius[j])) {
      *code64 = INVALID_CODE;
      return 0;
    }
  uint64_t res = 0;
  for (int j = 0; j < D; ++j) {
    const int m = 64 / D + (j < 64 % D ? 1 : 0);
    const uint64_t bits = (uint64_t)floor(ldexp(((p[j] - d->center[j]) / d->radius[j] + 1.0) / 2.0, m));
    const int initialShift = (63 - j) % D;
    for (int i = 0; i * D + initialShift < 64; ++i)
      res |= sls(bits, i * (D - 1) + initialShift) & sls(1, i * D + initialShift);
  }
  *code64 = res;
  return 1;
}

/* ------------------------------------------------------------------------------
 * tree order and search (Box.hpp:67-135, ImplicitBoxTree.hpp:2394-2432,
 * Functors.hpp:289-315)
 * ---------------------------------------------------------------------------- */
static inline uint64_t comparable(uint64_t code, uint32_t depth)
{
  const int d = 64 - (int)depth;
  return sls(code, d) | (sls(1, d - 1) - 1);
}

static inline int is_invalid_depth(uint32_t depth) { return depth > 64; }

/* isStrictlyPreceding (Box.hpp:124-135) */
static inline int strictly_preceding(uint64_t c1, uint32_t d1, uint64_t c2, uint32_t d2)
{
  if (is_invalid_depth(d1)) return 0;
  if (is_invalid_depth(d2)) return 1;
  const uint64_t b1 = comparable(c1, d1), b2 = comparable(c2, d2);
  return b1 < b2 || (b1 == b2 && d2 < d1);
}

/* hasSamePath (Box.hpp:76-83) */
static inline int same_path(uint64_t c1, uint32_t d1, uint64_t c2, uint32_t d2)
{
  const int diff = (int)d1 - (int)d2;
  return (is_invalid_depth(d1) && is_invalid_depth(d2)) || srs(c1, diff) == srs(c2, -diff);
}

uint32_t orc_search(const orc_tree* t, uint64_t code64, int valid)
{
  const uint32_t pd = valid ? 64u : ORC_LEAF_DEPTH;
  const uint64_t pc = valid ? code64 : INVALID_CODE;
  /* thrust::lower_bound with IsStrictlyPrecedingFunctor */
  uint64_t lo = 0, hi = t->n;
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo) / 2;
    if (strictly_preceding(t->code[mid], t->depth[mid], pc, pd)) lo = mid + 1;
    else hi = mid;
  }
  const uint32_t idx = (uint32_t)lo;
  /* ComputeSearchIndexFunctor: candidates Box[max(idx-1,0)] and Box[min(idx,n-1)] */
  const uint32_t a = idx > 0 ? idx - 1 : 0;
  const uint32_t b = idx < t->n - 1 ? idx : (uint32_t)(t->n - 1);
  if (pd >= t->depth[a] && same_path(pc, pd, t->code[a], t->depth[a])) return idx > 0 ? idx - 1 : 0;
  if (pd >= t->depth[b] && same_path(pc, pd, t->code[b], t->depth[b])) return idx;
  return ORC_INVALID;
}

/* ------------------------------------------------------------------------------
 * tree storage
 * ---------------------------------------------------------------------------- */
static void tree_reserve(orc_tree* t, uint64_t cap)
{
  if (cap <= t->cap) return;
  t->code = (uint64_t*)realloc(t->code, cap * 8);
  t->depth = (uint8_t*)realloc(t->depth, cap);
  t->flags = (uint8_t*)realloc(t->flags, cap);
  t->cap = cap;
}

void orc_tree_init(orc_tree* t, const orc_domain* d)
{
  memset(t, 0, sizeof *t);
  t->dom = *d;
  tree_reserve(t, 16);
  t->n = 1;
  t->code[0] = 0;
  t->depth[0] = 0;
  t->flags[0] = NONE_FLAGS;
}

void orc_tree_free(orc_tree* t)
{
  free(t->code); free(t->depth); free(t->flags);
  memset(t, 0, sizeof *t);
}

void orc_tree_load(orc_tree* t, const uint64_t* code, const uint8_t* depth, const uint8_t* flags, uint64_t n)
{
  tree_reserve(t, n ? n : 1);
  memcpy(t->code, code, n * 8);
  memcpy(t->depth, depth, n);
  memcpy(t->flags, flags, n);
  t->n = n;
}

/* insertSurroundingBoxIfEmpty (ImplicitBoxTree.hpp:1961-1970) */
static void insert_surrounding_if_empty(orc_tree* t)
{
  if (t->n == 0) { tree_reserve(t, 1); t->n = 1; t->code[0] = 0; t->depth[0] = 0; t->flags[0] = 0; }
}

static inline int flags_set(uint8_t f, uint8_t check) { return (uint8_t)(f & check) == check; }

/* setFlags / setFlagsByStencil on the leaves (ImplicitBoxTree.hpp:2684-2688) */
uint32_t orc_set_flags(orc_tree* t, uint8_t flags)
{
  uint32_t c = 0;
  for (uint64_t i = 0; i < t->n; ++i) { c += !flags_set(t->flags[i], flags); t->flags[i] |= flags; }
  return c;
}

/* setFlags(stencil, flags) with a logical vector over the leaves, as the Matlab drivers
 * call it (chainRecurrentSet.m:37, subdivisionByNim.m:62); returns the leaves flagged */
uint32_t orc_set_flags_mask(orc_tree* t, const uint8_t* mask, uint8_t flags)
{
  uint32_t c = 0;
  for (uint64_t i = 0; i < t->n; ++i)
    if (mask[i]) { t->flags[i] |= flags; ++c; }
  return c;
}

/* unsetFlags / unsetFlagsByStencil on the leaves (ImplicitBoxTree.hpp:3336-3360) */
uint32_t orc_unset_flags(orc_tree* t, uint8_t flags)
{
  uint32_t c = 0;
  for (uint64_t i = 0; i < t->n; ++i) { c += (t->flags[i] & flags) != 0; t->flags[i] &= (uint8_t)~flags; }
  return c;
}

/* changeFlags / changeFlagsByStencil on the leaves (ImplicitBoxTree.hpp:934-957, Flags.hpp:22-26) */
uint32_t orc_change_flags(orc_tree* t, uint8_t to_unset, uint8_t to_set)
{
  uint32_t c = 0;
  for (uint64_t i = 0; i < t->n; ++i)
    if (flags_set(t->flags[i], to_unset)) { ++c; t->flags[i] = (uint8_t)((t->flags[i] & ~to_unset) | to_set); }
  return c;
}

/* sortBoxes (helpFunctions.hpp:40-98): tree order = comparable pattern, then deeper first */
static const orc_tree* g_sort_tree;
static int cmp_box(const void* a, const void* b)
{
  const uint64_t i = *(const uint64_t*)a, j = *(const uint64_t*)b;
  const orc_tree* t = g_sort_tree;
  if (strictly_preceding(t->code[i], t->depth[i], t->code[j], t->depth[j])) return -1;
  if (strictly_preceding(t->code[j], t->depth[j], t->code[i], t->depth[i])) return 1;
  return i < j ? -1 : (i > j); /* stable */
}

static void sort_tree(orc_tree* t)
{
  uint64_t* idx = (uint64_t*)malloc(t->n * 8);
  for (uint64_t i = 0; i < t->n; ++i) idx[i] = i;
  g_sort_tree = t;
  qsort(idx, t->n, 8, cmp_box);
  uint64_t* c = (uint64_t*)malloc(t->n * 8);
  uint8_t* d = (uint8_t*)malloc(t->n);
  uint8_t* f = (uint8_t*)malloc(t->n);
  for (uint64_t i = 0; i < t->n; ++i) { c[i] = t->code[idx[i]]; d[i] = t->depth[idx[i]]; f[i] = t->flags[idx[i]]; }
  memcpy(t->code, c, t->n * 8); memcpy(t->depth, d, t->n); memcpy(t->flags, f, t->n);
  free(c); free(d); free(f); free(idx);
}

/* subdivide (ImplicitBoxTree.hpp:2884-2930): flagged leaves below the maximal depth
 * become their two halves (incrementDepthBy / computeOtherHalf, Box.hpp:140-147,
 * 234-239); flags are inherited; the result is re-sorted */
uint32_t orc_subdivide(orc_tree* t, uint8_t flags)
{
  /* returns countIfFlags(flags) over the leaves; leaves at depth 64 stay whole */
  uint64_t n = t->n, m = 0, flagged = 0;
  for (uint64_t i = 0; i < n; ++i) {
    flagged += flags_set(t->flags[i], flags);
    m += flags_set(t->flags[i], flags) && t->depth[i] < 64;
  }
  tree_reserve(t, n + m);
  uint64_t k = n;
  for (uint64_t i = 0; i < n; ++i) {
    if (flags_set(t->flags[i], flags) && t->depth[i] < 64) {
      t->code[i] <<= 1;
      t->depth[i] += 1;
      t->code[k] = t->code[i] | 1u;
      t->depth[k] = t->depth[i];
      t->flags[k] = t->flags[i];
      ++k;
    }
  }
  t->n = n + m;
  sort_tree(t);
  return (uint32_t)flagged;
}

/* remove (ImplicitBoxTree.hpp:2344-2371): keep leaves that have all `flags` set */
uint32_t orc_remove(orc_tree* t, uint8_t flags)
{
  uint64_t k = 0;
  const uint64_t n = t->n;
  for (uint64_t i = 0; i < n; ++i)
    if (flags_set(t->flags[i], flags)) { t->code[k] = t->code[i]; t->depth[k] = t->depth[i]; t->flags[k] = t->flags[i]; ++k; }
  t->n = k;
  insert_surrounding_if_empty(t);
  return (uint32_t)(n - k);
}

/* ------------------------------------------------------------------------------
 * box images: GridPointsFunctor::operator() (Functors.hpp:476-511) + search
 * ---------------------------------------------------------------------------- */
static uint32_t image_target(const orc_tree* t, const orc_map* m, const orc_grid* g,
                             uint64_t code, uint32_t depth, uint64_t i)
{
  const uint32_t D = t->dom.dim;
  double c[ORC_MAX_DIM], r[ORC_MAX_DIM], gp[ORC_MAX_DIM], y[ORC_MAX_DIM];
  orc_box_coordinates(&t->dom, code, depth, c, r);
  orc_grid_point(g, D, i, gp);
  for (uint32_t j = 0; j < D; ++j) c[j] += gp[j] * r[j];
  orc_map_apply(m, c, y);
  uint64_t code64;
  const int valid = orc_point_code64(&t->dom, y, &code64);
  return orc_search(t, code64, valid);
}

#define points_per_box orc_grid_points_per_box

void orc_search_by_image(const orc_tree* t, const orc_map* m, const orc_grid* g,
                         const uint32_t* src, uint64_t n_src, uint32_t* out)
{
  const uint64_t P = points_per_box(g, t->dom.dim);
  const int64_t total = (int64_t)(n_src * P);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < total; ++i) {
    const uint32_t b = src[(uint64_t)i / P];
    out[i] = image_target(t, m, g, t->code[b], t->depth[b], (uint64_t)i);
  }
}

/* setFlagsByIterators over makePointIteratorPairOverLeaves
 * (ImplicitBoxTree.hpp:2691-2694, 2624-2681, 2717-2775, 2167-2196) */
uint32_t orc_set_flags_by_image(orc_tree* t, const orc_map* m, const orc_grid* g, uint8_t flags)
{
  const uint64_t n = t->n, P = points_per_box(g, t->dom.dim);
  uint32_t* src = (uint32_t*)malloc(n * 4);
  for (uint64_t i = 0; i < n; ++i) src[i] = (uint32_t)i;
  uint32_t* tgt = (uint32_t*)malloc(n * P * 4);
  orc_search_by_image(t, m, g, src, n, tgt);
  uint8_t* hit = (uint8_t*)calloc(n, 1);
  for (uint64_t i = 0; i < n * P; ++i) if (tgt[i] != ORC_INVALID) hit[tgt[i]] = 1;
  uint32_t c = 0;
  for (uint64_t i = 0; i < n; ++i)
    if (hit[i]) { c += !flags_set(t->flags[i], flags); t->flags[i] |= flags; }
  free(hit); free(tgt); free(src);
  return c;
}

uint64_t orc_subdivision(orc_tree* t, const orc_map* m, const orc_grid* g, uint32_t steps, uint32_t* counts)
{
  /* subdivision loop (B12_doc.tex:269-290, subdivision.m:18-45) */
  uint64_t box_images = 0;
  orc_set_flags(t, 8u /* SD */);
  for (uint32_t s = 0; s < steps; ++s) {
    orc_subdivide(t, 8u);
    box_images += t->n;
    orc_set_flags_by_image(t, m, g, 1u /* HIT */);
    orc_remove(t, 1u);
    orc_unset_flags(t, 1u);
    if (counts) counts[s] = (uint32_t)t->n;
  }
  return box_images;
}

/* ------------------------------------------------------------------------------
 * transition matrix (ImplicitBoxTree.hpp:2934-3159): row = source leaf, column =
 * target leaf, value = count (absolute) or count / P; row-major, columns ascending;
 * lost points dropped, or sent to column n+1 with nColumns = n+1 (invalid, and only
 * when some point was lost: nColumns stays n otherwise)
 * ---------------------------------------------------------------------------- */
static int cmp_u32(const void* a, const void* b)
{
  const uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return x < y ? -1 : (x > y);
}

/* the run-length step of transitionMatrixForLeaves for n_rows rows of P targets each
 * (columns < n_cols, ORC_INVALID for a lost point); tgt is sorted row by row in place */
uint64_t orc_transition_rows(uint32_t* tgt, uint64_t n, uint64_t P, uint32_t n_cols, int absolute, int invalid,
                             uint32_t* rowptr, uint32_t* cols, double* vals, uint32_t* out_n_cols)
{
  /* the lost column exists only when some point was lost (ImplicitBoxTree.hpp:3075-3090) */
  int lost = 0;
  for (uint64_t i = 0; i < n * P && !lost; ++i) lost = tgt[i] == ORC_INVALID;
  const uint32_t nc = invalid && lost ? n_cols + 1 : n_cols;
  uint64_t nnz = 0;
  if (rowptr) rowptr[0] = 0;
  for (uint64_t r = 0; r < n; ++r) {
    uint32_t* row = tgt + r * P;
    qsort(row, P, 4, cmp_u32);
    for (uint64_t k = 0; k < P;) {
      uint64_t e = k;
      while (e < P && row[e] == row[k]) ++e;
      const uint32_t col = row[k];
      if (col != ORC_INVALID || invalid) {
        if (cols) {
          cols[nnz] = col == ORC_INVALID ? nc : col;
          vals[nnz] = absolute ? (double)(e - k) : (double)(e - k) / (double)P;
        }
        ++nnz;
      }
      k = e;
    }
    if (rowptr) rowptr[r + 1] = (uint32_t)nnz;
  }
  if (out_n_cols) *out_n_cols = nc;
  return nnz;
}

uint64_t orc_transition_matrix(const orc_tree* t, const orc_map* m, const orc_grid* g, int absolute, int invalid,
                               uint32_t* rowptr, uint32_t* cols, double* vals, uint32_t* n_cols)
{
  const uint64_t n = t->n, P = points_per_box(g, t->dom.dim);
  uint32_t* src = (uint32_t*)malloc(n * 4);
  for (uint64_t i = 0; i < n; ++i) src[i] = (uint32_t)i;
  uint32_t* tgt = (uint32_t*)malloc(n * P * 4);
  orc_search_by_image(t, m, g, src, n, tgt);
  const uint64_t nnz = orc_transition_rows(tgt, n, P, (uint32_t)n, absolute, invalid, rowptr, cols, vals, n_cols);
  free(tgt); free(src);
  return nnz;
}

/* ------------------------------------------------------------------------------
 * point boxes of a range-partitioned tree: the steps above restricted to given point
 * boxes (depth-64 codes with a validity byte)
 * ---------------------------------------------------------------------------- */
/* GridPointsFunctor + PointToBox of every leaf (ImplicitBoxTree.hpp:2624-2681), leaf-major */
void orc_image_point_boxes(const orc_tree* t, const orc_map* m, const orc_grid* g, uint64_t* codes, uint8_t* valid)
{
  const uint64_t n = t->n, P = points_per_box(g, t->dom.dim);
  const uint32_t D = t->dom.dim;
  const int64_t total = (int64_t)(n * P);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < total; ++i) {
    const uint64_t b = (uint64_t)i / P;
    double c[ORC_MAX_DIM], r[ORC_MAX_DIM], gp[ORC_MAX_DIM], y[ORC_MAX_DIM];
    orc_box_coordinates(&t->dom, t->code[b], t->depth[b], c, r);
    orc_grid_point(g, D, (uint64_t)i, gp);
    for (uint32_t j = 0; j < D; ++j) c[j] += gp[j] * r[j];
    orc_map_apply(m, c, y);
    valid[i] = (uint8_t)orc_point_code64(&t->dom, y, codes + i);
  }
}

/* searchByIterators over point boxes (ImplicitBoxTree.hpp:2394-2432) */
void orc_search_point_boxes(const orc_tree* t, const uint64_t* codes, const uint8_t* valid, uint64_t n,
                            uint32_t* out)
{
  for (uint64_t i = 0; i < n; ++i) out[i] = orc_search(t, codes[i], valid[i]);
}

/* setFlagsByIterators over point boxes (ImplicitBoxTree.hpp:2167-2196); returns the
 * leaves whose flags changed */
uint32_t orc_set_flags_by_point_boxes(orc_tree* t, const uint64_t* codes, const uint8_t* valid, uint64_t n,
                                      uint8_t flags)
{
  uint8_t* hit = (uint8_t*)calloc(t->n ? t->n : 1, 1);
  for (uint64_t i = 0; i < n; ++i) {
    const uint32_t b = orc_search(t, codes[i], valid[i]);
    if (b != ORC_INVALID) hit[b] = 1;
  }
  uint32_t c = 0;
  for (uint64_t i = 0; i < t->n; ++i)
    if (hit[i]) { c += !flags_set(t->flags[i], flags); t->flags[i] |= flags; }
  free(hit);
  return c;
}

/* ------------------------------------------------------------------------------
 * invariant measure: power iteration v <- P^T v / |P^T v|_1 from the uniform vector
 * (subdivisionByNim.m:30-58 computes it with eigs / powerMethodMPE, not shipped)
 * ---------------------------------------------------------------------------- */
void orc_invariant_measure(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const double* vals,
                           uint32_t iters, double* v)
{
  double* w = (double*)malloc((size_t)n * 8);
  for (uint32_t i = 0; i < n; ++i) v[i] = 1.0 / (double)n;
  for (uint32_t it = 0; it < iters; ++it) {
    memset(w, 0, (size_t)n * 8);
    for (uint32_t i = 0; i < n; ++i)
      for (uint32_t e = rowptr[i]; e < rowptr[i + 1]; ++e)
        if (cols[e] < n) w[cols[e]] += vals[e] * v[i];
    double s = 0.0;
    for (uint32_t j = 0; j < n; ++j) s += fabs(w[j]);
    for (uint32_t j = 0; j < n; ++j) v[j] = w[j] / s;
  }
  free(w);
}

/* The same iteration run until it settles (subdivisionByNim.m:30-45 asks
 * powerMethodMPE(P, 1e-14, 1e9), not shipped): after every check_every-th iteration, and
 * after max_iters, the L1 change made by that iteration, |v_k - v_(k-1)|_1, is compared
 * with tol; the run stops at the first check where it is at most tol. */
void orc_invariant_measure_tol(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const double* vals,
                               double tol, uint32_t max_iters, uint32_t check_every, double* v, uint32_t* iters_done,
                               double* last_change)
{
  double* w = (double*)malloc((size_t)n * 8);
  for (uint32_t i = 0; i < n; ++i) v[i] = 1.0 / (double)n;
  uint32_t k = 0;
  double change = 0.0;
  while (k < max_iters) {
    memset(w, 0, (size_t)n * 8);
    for (uint32_t i = 0; i < n; ++i)
      for (uint32_t e = rowptr[i]; e < rowptr[i + 1]; ++e)
        if (cols[e] < n) w[cols[e]] += vals[e] * v[i];
    double s = 0.0;
    for (uint32_t j = 0; j < n; ++j) s += fabs(w[j]);
    ++k;
    const int check = k % check_every == 0 || k == max_iters;
    change = 0.0;
    for (uint32_t j = 0; j < n; ++j) {
      const double x = w[j] / s;
      if (check) change += fabs(x - v[j]);
      v[j] = x;
    }
    if (check && change <= tol) break;
  }
  free(w);
  *iters_done = k;
  *last_change = change;
}

/* ------------------------------------------------------------------------------
 * continuation (insertByIterators at a uniform depth, ImplicitBoxTree.hpp:1615-1910,
 * makePointIteratorPairByFlags 2303-2341, insertByPoints 1927-1946, deleteDepth 1217-1228)
 * ---------------------------------------------------------------------------- */
void orc_delete_depth0(orc_tree* t)
{
  t->n = 0;
  insert_surrounding_if_empty(t);
}

static int cmp_u64(const void* a, const void* b)
{
  const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
  return x < y ? -1 : (x > y);
}

/* merge sorted unique new depth-d codes (flags `ins`) into a uniform-depth tree */
static void merge_new(orc_tree* t, const uint64_t* nc, uint64_t m, uint32_t depth, uint8_t ins)
{
  const uint64_t n = t->n;
  uint64_t* c = (uint64_t*)malloc((n + m) * 8);
  uint8_t* d = (uint8_t*)malloc(n + m);
  uint8_t* f = (uint8_t*)malloc(n + m);
  uint64_t i = 0, j = 0, k = 0;
  while (i < n || j < m) {
    if (j >= m || (i < n && t->code[i] < nc[j])) { c[k] = t->code[i]; d[k] = t->depth[i]; f[k] = t->flags[i]; ++i; }
    else { c[k] = nc[j]; d[k] = (uint8_t)depth; f[k] = ins; ++j; }
    ++k;
  }
  tree_reserve(t, n + m);
  memcpy(t->code, c, k * 8); memcpy(t->depth, d, k); memcpy(t->flags, f, k);
  t->n = k;
  free(c); free(d); free(f);
}

uint32_t orc_insert_points(orc_tree* t, const double* pts, uint64_t n_points, uint32_t depth, uint8_t ins,
                           uint8_t hit)
{
  /* insertByPoints (ImplicitBoxTree.hpp:1927-1946) at depth `depth` into a tree whose
   * leaves are all at that depth, or into the surrounding box alone, which merges
   * into the (single) new box (its path is shared by every box) */
  const uint32_t D = t->dom.dim;
  const int root_only = t->n == 1 && t->depth[0] == 0;
  uint64_t* nc = (uint64_t*)malloc((n_points ? n_points : 1) * 8);
  uint64_t m = 0;
  for (uint64_t p = 0; p < n_points; ++p) {
    uint64_t c64;
    if (!orc_point_code64(&t->dom, pts + p * D, &c64)) continue;
    if (!root_only) {
      const uint32_t f = orc_search(t, c64, 1);
      if (f != ORC_INVALID) { t->flags[f] |= hit; continue; }
    }
    nc[m++] = srs(c64, 64 - (int)depth);
  }
  qsort(nc, m, 8, cmp_u64);
  uint64_t u = 0;
  for (uint64_t k = 0; k < m; ++k) if (u == 0 || nc[k] != nc[u - 1]) nc[u++] = nc[k];
  uint8_t root_flags = root_only ? t->flags[0] : 0;
  if (root_only && u > 0) t->n = 0;
  merge_new(t, nc, u, depth, ins);
  if (root_only && u > 0) t->flags[0] |= root_flags;
  free(nc);
  return (uint32_t)u;
}

uint32_t orc_insert_by_image(orc_tree* t, const orc_map* m, const orc_grid* g, uint8_t flags_to_check,
                             uint8_t ins, uint8_t hit)
{
  const uint64_t n = t->n, P = points_per_box(g, t->dom.dim);
  const uint32_t depth = t->depth[0];
  uint64_t ns = 0;
  uint32_t* src = (uint32_t*)malloc((n ? n : 1) * 4);
  for (uint64_t i = 0; i < n; ++i) if (flags_set(t->flags[i], flags_to_check)) src[ns++] = (uint32_t)i;
  uint64_t* cand = (uint64_t*)malloc((ns * P > 0 ? ns * P : 1) * 8);
  uint32_t* tgt = (uint32_t*)malloc((ns * P > 0 ? ns * P : 1) * 4);
  const int64_t total = (int64_t)(ns * P);
  const uint32_t D = t->dom.dim;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < total; ++i) {
    const uint32_t b = src[(uint64_t)i / P];
    double c[ORC_MAX_DIM], r[ORC_MAX_DIM], gp[ORC_MAX_DIM], y[ORC_MAX_DIM];
    orc_box_coordinates(&t->dom, t->code[b], t->depth[b], c, r);
    orc_grid_point(g, D, (uint64_t)i, gp);
    for (uint32_t j = 0; j < D; ++j) c[j] += gp[j] * r[j];
    orc_map_apply(m, c, y);
    uint64_t code64;
    const int valid = orc_point_code64(&t->dom, y, &code64);
    tgt[i] = orc_search(t, code64, valid);
    cand[i] = valid && tgt[i] == ORC_INVALID ? srs(code64, 64 - (int)depth) : INVALID_CODE;
  }
  if (hit)
    for (int64_t i = 0; i < total; ++i) if (tgt[i] != ORC_INVALID) t->flags[tgt[i]] |= hit;
  qsort(cand, (size_t)total, 8, cmp_u64);
  uint64_t u = 0;
  for (int64_t k = 0; k < total && cand[k] != INVALID_CODE; ++k) if (u == 0 || cand[k] != cand[u - 1]) cand[u++] = cand[k];
  merge_new(t, cand, u, depth, ins);
  free(cand); free(tgt); free(src);
  return (uint32_t)u;
}

/* ------------------------------------------------------------------------------
 * trees of mixed depths: unsubdivide and the general insert
 * ---------------------------------------------------------------------------- */
typedef struct { uint64_t c; uint32_t d; uint8_t f; } obox;

static inline int box_same(obox a, obox b)
{
  return (is_invalid_depth(a.d) && is_invalid_depth(b.d)) || (a.c == b.c && a.d == b.d);
}
static inline int box_same_path(obox a, obox b) { return same_path(a.c, a.d, b.c, b.d); }

/* decrementDepthBy (Box.hpp:151-158) */
static inline obox decrement_by(obox b, uint32_t k)
{
  if (k > b.d) k = b.d;
  b.c = srs(b.c, (int)k);
  b.d -= k;
  return b;
}

/* IsUnsubdividableFunctor (Functors.hpp:343-364) on leaf i with its neighbours */
static int unsubdividable(const orc_tree* t, uint64_t i, uint8_t flags)
{
  const uint64_t n = t->n;
  const obox b = {t->code[i], t->depth[i], t->flags[i]};
  if (!(flags_set(b.f, flags) && b.d > 0)) return 0;
  const uint64_t j = (b.c & 1u) ? (i > 0 ? i - 1 : 0) : (i + 1 < n ? i + 1 : n - 1);
  const obox nb = {t->code[j], t->depth[j], t->flags[j]};
  const obox parent = decrement_by(b, 1);
  return box_same(parent, decrement_by(nb, 1)) ? flags_set(nb.f, flags) : !box_same_path(parent, nb);
}

/* unsubdivide (ImplicitBoxTree.hpp:3414-3460): leaves with `flags` whose sibling is a
 * leaf with them too, or whose sibling's region holds no leaf, become their parents;
 * two halves merge into one parent with the AND of their flags.  Returns the number of
 * parents made. */
uint32_t orc_unsubdivide(orc_tree* t, uint8_t flags)
{
  const uint64_t n = t->n;
  uint8_t* mask = (uint8_t*)malloc(n ? n : 1);
  uint64_t res = 0;
  for (uint64_t i = 0; i < n; ++i) res += (mask[i] = (uint8_t)unsubdividable(t, i, flags));
  for (uint64_t i = 0; i < n; ++i)
    if (mask[i]) { t->code[i] >>= 1; t->depth[i] -= 1; }
  /* reverse inclusive_scan_by_key of the flags over runs of equal boxes (AND) */
  for (uint64_t i = n; i-- > 1;) {
    const obox a = {t->code[i - 1], t->depth[i - 1], 0}, b = {t->code[i], t->depth[i], 0};
    if (box_same(b, a)) t->flags[i - 1] &= t->flags[i];
  }
  /* unique(IsSameBox): the first of each run stays */
  uint64_t k = 0;
  obox prev = {0, 0, 0};
  for (uint64_t i = 0; i < n; ++i) {
    const obox b = {t->code[i], t->depth[i], t->flags[i]};
    const int dup = i > 0 && box_same(prev, b);
    prev = b;
    if (dup) continue;
    t->code[k] = b.c; t->depth[k] = (uint8_t)b.d; t->flags[k] = b.f; ++k;
  }
  res -= n - k;
  t->n = k;
  free(mask);
  return (uint32_t)res;
}

/* setFlags / unsetFlags / changeFlags (op 0 / 1 / 2) at a depth that is neither the
 * leaves' own nor 0 (setFlagsByStencil, unsetFlagsByStencil, changeFlagsByStencil with a
 * true stencil, ImplicitBoxTree.hpp:914-1058, 2805-2882, 3336-3411; countIfFlags
 * 1104-1200): a box at that depth is a run of leaves at least that deep with one prefix;
 * its flags are its leaves' AND (set, change) or OR (unset).  Every leaf of the box
 * changes (change: only the boxes whose AND has all of u); the count is of the boxes
 * whose combined flags lacked f (set), had any of f (unset) or had all of u (change).
 * Depths above the deepest leaf change nothing. */
uint32_t orc_flags_at_depth(orc_tree* t, int op, uint8_t u, uint8_t f, uint32_t depth)
{
  const uint64_t n = t->n;
  uint32_t count = 0;
  uint64_t i = 0;
  while (i < n) {
    if (t->depth[i] < depth) { ++i; continue; }
    const uint64_t pre = t->code[i] >> (t->depth[i] - depth);
    uint64_t j = i;
    uint8_t all = 0xFF, any = 0;
    while (j < n && t->depth[j] >= depth && (t->code[j] >> (t->depth[j] - depth)) == pre) {
      all &= t->flags[j];
      any |= t->flags[j];
      ++j;
    }
    int hit;
    if (op == 0) hit = !flags_set(all, f);
    else if (op == 1) hit = (any & f) != 0;
    else hit = flags_set(all, u);
    count += hit;
    for (uint64_t k = i; k < j; ++k) {
      if (op == 0) t->flags[k] |= f;
      else if (op == 1) t->flags[k] &= (uint8_t)~f;
      else if (hit) t->flags[k] = (uint8_t)((t->flags[k] & ~u) | f);
    }
    i = j;
  }
  return count;
}

/* the index of every leaf's box at depth d (initializeIndicesInDepth,
 * ImplicitBoxTree.hpp:1399-1470): boxes counted in tree order; ORC_INVALID for leaves
 * shallower than d.  Caller frees. */
static uint32_t* boxes_at_depth(const orc_tree* t, uint32_t d, uint64_t* n_boxes)
{
  uint32_t* box = (uint32_t*)malloc((t->n ? t->n : 1) * 4);
  uint64_t b = 0;
  for (uint64_t i = 0; i < t->n; ++i) {
    if (t->depth[i] < d) { box[i] = ORC_INVALID; continue; }
    int fresh = i == 0 || t->depth[i - 1] < d;
    if (!fresh) fresh = (t->code[i - 1] >> (t->depth[i - 1] - d)) != (t->code[i] >> (t->depth[i] - d));
    if (fresh) ++b;
    box[i] = (uint32_t)(b - 1);
  }
  *n_boxes = b;
  return box;
}

/* searchByIterators at an inner depth d (ImplicitBoxTree.hpp:2473-2566): the lower
 * bound of the point box among the leaves, its two neighbours taken to depth d
 * (decrementDepthTo) when at least that deep, ComputeSearchIndexFunctor, then the
 * box index at depth d of the leaf found */
static uint32_t search_at_depth(const orc_tree* t, const uint32_t* box, uint64_t code64, int valid, uint32_t d)
{
  const uint64_t n = t->n;
  if (n == 0) return ORC_INVALID;
  const uint32_t pd = valid ? 64u : ORC_LEAF_DEPTH;
  const uint64_t pc = valid ? code64 : INVALID_CODE;
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo) / 2;
    if (strictly_preceding(t->code[mid], t->depth[mid], pc, pd)) lo = mid + 1;
    else hi = mid;
  }
  const uint64_t ia = lo > 0 ? lo - 1 : 0, ib = lo < n - 1 ? lo : n - 1;
  uint64_t found = ORC_INVALID;
  for (int c = 0; c < 2 && found == ORC_INVALID; ++c) {
    const uint64_t j = c == 0 ? ia : ib;
    if (t->depth[j] < d) continue;                        /* hasAtLeastDepth */
    const uint64_t cd = t->code[j] >> (t->depth[j] - d);  /* decrementDepthTo(d) */
    if (pd >= d && same_path(pc, pd, cd, d)) found = c == 0 ? (lo > 0 ? lo - 1 : 0) : lo;
  }
  return found == ORC_INVALID ? ORC_INVALID : box[found];
}

/* the sources of a scheme (initializeLeafIndicesFromDepth, ImplicitBoxTree.hpp:1476-1611):
 * at the leaf depth (255) the leaves with all of flags_to_check; at an inner depth d the
 * boxes at d whose leaves all have them, each as its first leaf taken to depth d
 * (DecrementDepthToFunctor in makePointIteratorPairByFlags, 2303-2341) */
static uint64_t scheme_sources(const orc_tree* t, uint32_t src_depth, uint8_t flags_to_check, uint64_t* code,
                               uint32_t* depth)
{
  uint64_t ns = 0;
  if (src_depth == ORC_LEAF_DEPTH) {
    for (uint64_t i = 0; i < t->n; ++i)
      if (flags_set(t->flags[i], flags_to_check)) { code[ns] = t->code[i]; depth[ns] = t->depth[i]; ++ns; }
    return ns;
  }
  uint64_t i = 0;
  while (i < t->n) {
    if (t->depth[i] < src_depth) { ++i; continue; }
    const uint64_t pre = t->code[i] >> (t->depth[i] - src_depth);
    uint64_t j = i;
    uint8_t all = 0xFF;
    while (j < t->n && t->depth[j] >= src_depth && (t->code[j] >> (t->depth[j] - src_depth)) == pre) all &= t->flags[j++];
    if (flags_set(all, flags_to_check)) { code[ns] = pre; depth[ns] = src_depth; ++ns; }
    i = j;
  }
  return ns;
}

/* the images of a scheme's sources located among the leaves (target 255: leaf index,
 * searchByIterators 2394-2432) or at an inner depth (the box index, 2473-2566).  With
 * out == NULL the hit leaves / every leaf of the hit boxes get `flags`
 * (setFlagsByIterators 2691-2694 via setFlagsBySearch 2717-2800), and the return value
 * counts the hit leaves / boxes that lacked them; with out != NULL each point's index is
 * written and nothing changes.  *n_points gets the number of points. */
uint32_t orc_image_search(orc_tree* t, const orc_map* m, const orc_grid* g, uint32_t src_depth, uint8_t flags_to_check,
                          uint32_t target, uint8_t flags, uint32_t* out, uint64_t* n_points)
{
  const uint64_t n = t->n, P = points_per_box(g, t->dom.dim);
  const uint32_t D = t->dom.dim;
  uint64_t* scode = (uint64_t*)malloc((n ? n : 1) * 8);
  uint32_t* sdep = (uint32_t*)malloc((n ? n : 1) * 4);
  const uint64_t ns = scheme_sources(t, src_depth, flags_to_check, scode, sdep);
  if (n_points) *n_points = ns * P;
  uint64_t nb = 0;
  uint32_t* box = target == ORC_LEAF_DEPTH ? NULL : boxes_at_depth(t, target, &nb);
  const uint64_t nt = target == ORC_LEAF_DEPTH ? n : nb;
  uint8_t* hit = (uint8_t*)calloc(nt ? nt : 1, 1);
  for (uint64_t i = 0; i < ns * P; ++i) {
    const uint64_t b = i / P;
    double c[ORC_MAX_DIM], r[ORC_MAX_DIM], gp[ORC_MAX_DIM], y[ORC_MAX_DIM];
    orc_box_coordinates(&t->dom, scode[b], sdep[b], c, r);
    orc_grid_point(g, D, i, gp);
    for (uint32_t j = 0; j < D; ++j) c[j] += gp[j] * r[j];
    orc_map_apply(m, c, y);
    uint64_t c64;
    const int valid = orc_point_code64(&t->dom, y, &c64);
    const uint32_t s = target == ORC_LEAF_DEPTH ? orc_search(t, c64, valid) : search_at_depth(t, box, c64, valid, target);
    if (out) out[i] = s;
    else if (s != ORC_INVALID) hit[s] = 1;
  }
  uint32_t count = 0;
  if (!out) {
    if (target == ORC_LEAF_DEPTH) {
      for (uint64_t i = 0; i < n; ++i)
        if (hit[i]) { count += !flags_set(t->flags[i], flags); t->flags[i] |= flags; }
    } else {
      uint8_t* all = (uint8_t*)malloc(nb ? nb : 1);
      memset(all, 0xFF, nb ? nb : 1);
      for (uint64_t i = 0; i < n; ++i) if (box[i] != ORC_INVALID) all[box[i]] &= t->flags[i];
      for (uint64_t b = 0; b < nb; ++b) count += hit[b] && !flags_set(all[b], flags);
      for (uint64_t i = 0; i < n; ++i) if (box[i] != ORC_INVALID && hit[box[i]]) t->flags[i] |= flags;
      free(all);
    }
  }
  free(hit);
  free(box);
  free(scode);
  free(sdep);
  return count;
}

/* images of every leaf located at an inner depth d (orc_image_search with the leaves as
 * sources) */
uint32_t orc_image_at_depth(orc_tree* t, const orc_map* m, const orc_grid* g, uint32_t d, uint8_t flags,
                            uint32_t* out)
{
  return orc_image_search(t, m, g, ORC_LEAF_DEPTH, 0, d, flags, out, NULL);
}

/* computeDepthOfMutualAncestor (Box.hpp:209-223) */
static inline uint32_t mutual_ancestor(obox a, obox b)
{
  const uint64_t x = sls(a.c, 64 - (int)a.d) ^ sls(b.c, 64 - (int)b.d);
  const uint32_t lz = x ? (uint32_t)__builtin_clzll(x) : 64u;
  const uint32_t m = a.d < b.d ? a.d : b.d;
  return lz < m ? lz : m;
}

/* changeDepthTo (Box.hpp:180-198) for depths 0..64 */
static inline obox change_depth_to(obox b, uint32_t depth)
{
  if (depth < b.d) {
    b.c = srs(b.c, (int)(b.d - depth));
    b.d = depth;
  } else if (depth > b.d && depth != ORC_LEAF_DEPTH) {
    if (depth > 64) depth = 64;
    b.c = sls(b.c, (int)(depth - b.d));
    b.d = depth;
  }
  return b;
}

static int cmp_obox(const void* x, const void* y)
{
  const obox* a = (const obox*)x;
  const obox* b = (const obox*)y;
  if (strictly_preceding(a->c, a->d, b->c, b->d)) return -1;
  if (strictly_preceding(b->c, b->d, a->c, a->d)) return 1;
  return 0;
}

/* a stable sort in tree order (qsort is not stable: sort (box, position) pairs) */
typedef struct { obox b; uint64_t pos; } opos;
static int cmp_opos(const void* x, const void* y)
{
  const opos* a = (const opos*)x;
  const opos* b = (const opos*)y;
  const int c = cmp_obox(&a->b, &b->b);
  return c ? c : (a->pos < b->pos ? -1 : (a->pos > b->pos));
}
static void stable_sort_boxes(obox* v, uint64_t n)
{
  opos* w = (opos*)malloc((n ? n : 1) * sizeof(opos));
  for (uint64_t i = 0; i < n; ++i) { w[i].b = v[i]; w[i].pos = i; }
  qsort(w, n, sizeof(opos), cmp_opos);
  for (uint64_t i = 0; i < n; ++i) v[i] = w[i].b;
  free(w);
}

/* insertByIterators (ImplicitBoxTree.hpp:1615-1910) for any tree, given the depth-64
 * point boxes (valid[k] = 0: the point left the domain).  depth 255 inserts at the
 * leaf depth (each new box the coarsest one that does not meet its neighbours,
 * AdaptDepthOfFirstBoxFunctor, Functors.hpp:381-389); new boxes are merged into the
 * leaves by the reference's two HasSamePath scans and unique (1875-1897).  At an inner
 * depth, flags for hit boxes go to every leaf of the box hit.  *unsupported stays 0.
 * Returns the number of distinct new boxes. */
uint32_t orc_insert_boxes(orc_tree* t, const uint64_t* c64, const uint8_t* valid, uint64_t np, uint32_t depth,
                          uint8_t ins, uint8_t hit, int* unsupported)
{
  *unsupported = 0;
  const uint64_t n = t->n;
  if (depth == 0) {
    int any = 0;
    for (uint64_t k = 0; k < np; ++k) any |= valid[k] != 0;
    if (hit && any) for (uint64_t i = 0; i < n; ++i) t->flags[i] |= hit;
    return 0;
  }
  if (!(depth == ORC_LEAF_DEPTH || depth <= 64)) return 0;
  uint32_t maxd = 0, uniform = 1;
  for (uint64_t i = 0; i < n; ++i) {
    if (t->depth[i] > maxd) maxd = t->depth[i];
    uniform &= t->depth[i] == t->depth[0];
  }
  const int leaf_search = depth == ORC_LEAF_DEPTH || (uniform && depth == t->depth[0]);
  const int inner_search = !leaf_search && depth <= maxd;
  uint64_t n_boxes = 0;
  uint32_t* box = inner_search ? boxes_at_depth(t, depth, &n_boxes) : NULL;
  uint8_t* box_hit = inner_search ? (uint8_t*)calloc(n_boxes ? n_boxes : 1, 1) : NULL;
  obox* nb = (obox*)malloc((np ? np : 1) * sizeof(obox));
  uint32_t* hits = (uint32_t*)malloc((np ? np : 1) * 4);
  uint64_t m = 0, nh = 0;
  for (uint64_t k = 0; k < np; ++k) {
    const obox p = valid[k] ? (obox){c64[k], 64u, ins} : (obox){INVALID_CODE, ORC_LEAF_DEPTH, 0};
    int to_insert;
    if (leaf_search) {
      const uint32_t s = orc_search(t, p.c, valid[k]);
      if (depth == ORC_LEAF_DEPTH)
        to_insert = s == ORC_INVALID ? valid[k] != 0 : t->depth[s] < 64;
      else
        to_insert = s == ORC_INVALID && valid[k];
      if (!to_insert && s != ORC_INVALID) hits[nh++] = s;
    } else if (inner_search) {
      /* the box at `depth` around the point (setFlagsBySearch marks it for hit flags) */
      const uint32_t s = search_at_depth(t, box, p.c, valid[k], depth);
      if (s != ORC_INVALID) box_hit[s] = 1;
      to_insert = valid[k] && s == ORC_INVALID;
    } else {
      to_insert = valid[k] != 0;
    }
    if (!to_insert) continue;
    obox b = p;
    if (depth == ORC_LEAF_DEPTH) {
      /* lower bound of the point box among the leaves; its two neighbours */
      uint64_t lo = 0, hi = n;
      while (lo < hi) {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (strictly_preceding(t->code[mid], t->depth[mid], p.c, p.d)) lo = mid + 1;
        else hi = mid;
      }
      const uint64_t ia = lo > 0 ? lo - 1 : 0, ib = lo < n - 1 ? lo : n - 1;
      const obox a = {t->code[ia], t->depth[ia], 0}, c = {t->code[ib], t->depth[ib], 0};
      const uint32_t x = mutual_ancestor(p, a), y = mutual_ancestor(p, c);
      b = change_depth_to(p, (x > y ? x : y) + 1);
    } else if (depth < b.d) {
      b.c = srs(b.c, (int)(b.d - depth));
      b.d = depth;
    }
    b.f = (uint8_t)(b.f | ins);
    nb[m++] = b;
  }
  for (uint64_t k = 0; k < nh; ++k) t->flags[hits[k]] |= hit;
  if (inner_search) {
    /* setFlagsByStencil at the inner depth: every leaf of a hit box */
    if (hit)
      for (uint64_t i = 0; i < n; ++i) if (box[i] != ORC_INVALID && box_hit[box[i]]) t->flags[i] |= hit;
    free(box);
    free(box_hit);
  }
  /* distinct new boxes in tree order */
  stable_sort_boxes(nb, m);
  uint64_t u = 0;
  for (uint64_t k = 0; k < m; ++k) if (u == 0 || !box_same(nb[u - 1], nb[k])) nb[u++] = nb[k];
  if (u > 0) {
    const uint64_t total = n + u;
    obox* all = (obox*)malloc(total * sizeof(obox));
    for (uint64_t i = 0; i < n; ++i) all[i] = (obox){t->code[i], t->depth[i], t->flags[i]};
    for (uint64_t k = 0; k < u; ++k) all[n + k] = nb[k];
    stable_sort_boxes(all, total);
    /* forward inclusive_scan_by_key: segments of adjacent boxes on one path (original keys) */
    obox* f = (obox*)malloc(total * sizeof(obox));
    for (uint64_t i = 0; i < total; ++i) {
      if (i > 0 && box_same_path(all[i - 1], all[i])) {
        f[i].c = f[i - 1].c > all[i].c ? f[i - 1].c : all[i].c;
        f[i].d = f[i - 1].d > all[i].d ? f[i - 1].d : all[i].d;
        f[i].f = (uint8_t)(f[i - 1].f | all[i].f);
      } else {
        f[i] = all[i];
      }
    }
    /* reverse scan, keyed by the forward scan's output */
    obox* r = all;
    for (uint64_t i = total; i-- > 0;) {
      if (i + 1 < total && box_same_path(f[i + 1], f[i])) {
        r[i].c = r[i + 1].c > f[i].c ? r[i + 1].c : f[i].c;
        r[i].d = r[i + 1].d > f[i].d ? r[i + 1].d : f[i].d;
        r[i].f = (uint8_t)(r[i + 1].f | f[i].f);
      } else {
        r[i] = f[i];
      }
    }
    /* unique(HasSamePath) with adjacent comparisons */
    tree_reserve(t, total);
    uint64_t k = 0;
    for (uint64_t i = 0; i < total; ++i) {
      if (i > 0 && box_same_path(r[i - 1], r[i])) continue;
      t->code[k] = r[i].c; t->depth[k] = (uint8_t)r[i].d; t->flags[k] = r[i].f; ++k;
    }
    t->n = k;
    free(f);
    free(all);
  }
  free(nb);
  free(hits);
  return (uint32_t)u;
}

/* insertByPoints (ImplicitBoxTree.hpp:1927-1946) through the general insert */
uint32_t orc_insert_points_general(orc_tree* t, const double* pts, uint64_t n_points, uint32_t depth, uint8_t ins,
                                   uint8_t hit, int* unsupported)
{
  const uint32_t D = t->dom.dim;
  uint64_t* c = (uint64_t*)malloc((n_points ? n_points : 1) * 8);
  uint8_t* v = (uint8_t*)malloc(n_points ? n_points : 1);
  for (uint64_t k = 0; k < n_points; ++k) v[k] = (uint8_t)orc_point_code64(&t->dom, pts + k * D, c + k);
  const uint32_t r = orc_insert_boxes(t, c, v, n_points, depth, ins, hit, unsupported);
  free(c); free(v);
  return r;
}

/* insertByIterators(makePointIteratorPairByFlags(255, flags_to_check, grid, map), ...)
 * through the general insert: the images of the leaves with flags_to_check */
uint32_t orc_insert_by_image_src(orc_tree* t, const orc_map* m, const orc_grid* g, uint32_t src_depth,
                                 uint8_t flags_to_check, uint32_t depth, uint8_t ins, uint8_t hit, int* unsupported)
{
  const uint64_t n = t->n, P = points_per_box(g, t->dom.dim);
  const uint32_t D = t->dom.dim;
  uint64_t* scode = (uint64_t*)malloc((n ? n : 1) * 8);
  uint32_t* sdep = (uint32_t*)malloc((n ? n : 1) * 4);
  const uint64_t ns = scheme_sources(t, src_depth, flags_to_check, scode, sdep);
  const uint64_t total = ns * P;
  uint64_t* c = (uint64_t*)malloc((total ? total : 1) * 8);
  uint8_t* v = (uint8_t*)malloc(total ? total : 1);
  for (uint64_t i = 0; i < total; ++i) {
    const uint64_t b = i / P;
    double ctr[ORC_MAX_DIM], r[ORC_MAX_DIM], gp[ORC_MAX_DIM], y[ORC_MAX_DIM];
    orc_box_coordinates(&t->dom, scode[b], sdep[b], ctr, r);
    orc_grid_point(g, D, i, gp);
    for (uint32_t j = 0; j < D; ++j) ctr[j] += gp[j] * r[j];
    orc_map_apply(m, ctr, y);
    v[i] = (uint8_t)orc_point_code64(&t->dom, y, c + i);
  }
  const uint32_t res = orc_insert_boxes(t, c, v, total, depth, ins, hit, unsupported);
  free(c); free(v); free(scode); free(sdep);
  return res;
}

uint32_t orc_insert_by_image_general(orc_tree* t, const orc_map* m, const orc_grid* g, uint8_t flags_to_check,
                                     uint32_t depth, uint8_t ins, uint8_t hit, int* unsupported)
{
  return orc_insert_by_image_src(t, m, g, ORC_LEAF_DEPTH, flags_to_check, depth, ins, hit, unsupported);
}

/* ------------------------------------------------------------------------------
 * strongly connected components of the graph of a transition matrix (row = source,
 * column = target; columns >= n, the lost column, ignored) - what graphconncomp(P')
 * gives chainRecurrentSet.m:29.  Tarjan's algorithm with an explicit stack; each
 * component is labelled by its largest vertex.
 * ---------------------------------------------------------------------------- */
void orc_strong_components(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, uint32_t* comp)
{
  const uint32_t NONE = 0xFFFFFFFFu;
  uint32_t* index = (uint32_t*)malloc((size_t)n * 4);
  uint32_t* low = (uint32_t*)malloc((size_t)n * 4);
  uint8_t* on = (uint8_t*)calloc(n, 1);
  uint32_t* stack = (uint32_t*)malloc((size_t)n * 4);
  uint32_t* call_v = (uint32_t*)malloc((size_t)n * 4);
  uint32_t* call_e = (uint32_t*)malloc((size_t)n * 4);
  uint32_t sp = 0, next = 0;
  for (uint32_t v = 0; v < n; ++v) index[v] = NONE;
  for (uint32_t r = 0; r < n; ++r) {
    if (index[r] != NONE) continue;
    uint32_t depth = 0;
    call_v[0] = r; call_e[0] = rowptr[r];
    index[r] = low[r] = next++; stack[sp++] = r; on[r] = 1;
    while (1) {
      const uint32_t v = call_v[depth];
      if (call_e[depth] < rowptr[v + 1]) {
        const uint32_t w = cols[call_e[depth]++];
        if (w >= n) continue;
        if (index[w] == NONE) {
          ++depth;
          call_v[depth] = w; call_e[depth] = rowptr[w];
          index[w] = low[w] = next++; stack[sp++] = w; on[w] = 1;
        } else if (on[w] && index[w] < low[v]) {
          low[v] = index[w];
        }
        continue;
      }
      if (low[v] == index[v]) {
        /* v is the root of a component: pop it, label by its largest vertex */
        uint32_t top = sp, label = 0;
        do { --top; if (stack[top] > label) label = stack[top]; } while (stack[top] != v);
        while (sp > top) { const uint32_t x = stack[--sp]; on[x] = 0; comp[x] = label; }
      }
      if (depth == 0) break;
      --depth;
      { const uint32_t u = call_v[depth]; if (low[v] < low[u]) low[u] = low[v]; }
    }
  }
  free(index); free(low); free(on); free(stack); free(call_v); free(call_e);
}
