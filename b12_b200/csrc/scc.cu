// Strongly connected components of a transition graph, the two selection steps that
// consume a transition matrix, and the fixed-box selection of fixedBoxes.m:
//   chain recurrent set: keep the boxes of strongly connected components with at least
//     two boxes (chainRecurrentSet.m:18-44, graphconncomp on P')
//   natural invariant measure: keep the boxes whose measure is at least 1e-9 / n
//     (subdivisionByNim.m:22-66, the stencil of lines 56-57)
//
// Components by forward-backward colouring on the device:
//   1. trim: a box without an edge to another remaining box, or without one from
//      another remaining box, is a component of its own (repeated until nothing changes);
//   2. colour every remaining box with the largest index that reaches it (pull over P^T
//      until nothing changes); a box whose colour is itself is a root;
//   3. the root's component is every box of its colour that reaches it (pull over P);
//   4. retire the assigned boxes and repeat from 2 until none remains.
// A component's label is its largest box index, so labels do not depend on the order of
// the parallel updates.  Self-loops never join a box to a component.
#include <algorithm>
#include <vector>

#include "tree.h"

using namespace b12g;
using namespace b12g::host;

namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr int kThreads = 256;
constexpr int kBatch = 8;   // sweeps launched between two reads of the change flag

int grid_for_n(uint32_t n) { return int(std::max<uint32_t>(1, std::min<uint32_t>((n + kThreads - 1) / kThreads,
                                                                                 uint32_t(device_sm_count()) * 8))); }

__global__ void init_kernel(uint32_t n, uint8_t* active, uint32_t* comp)
{
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    active[v] = 1;
    comp[v] = kNone;
  }
}

// a remaining box with no edge to, or no edge from, another remaining box is a component of its own
__global__ void trim_kernel(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const uint32_t* tptr,
                            const uint32_t* trows, uint8_t* active, uint32_t* comp, uint32_t* changed)
{
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    if (!active[v]) continue;
    bool out = false, in = false;
    for (uint32_t e = rowptr[v]; e < rowptr[v + 1] && !out; ++e) {
      const uint32_t w = cols[e];
      out = w < n && w != v && active[w];
    }
    for (uint32_t e = tptr[v]; e < tptr[v + 1] && !in; ++e) {
      const uint32_t u = trows[e];
      in = u != v && active[u];
    }
    if (!(out && in)) {
      active[v] = 0;
      comp[v] = v;
      *changed = 1;
    }
  }
}

__global__ void colour_init_kernel(uint32_t n, const uint8_t* active, uint32_t* colour)
{
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    colour[v] = active[v] ? v : kNone;
}

// colour(v) <- max over remaining u with u -> v of colour(u)  (colours only grow)
__global__ void colour_pull_kernel(uint32_t n, const uint32_t* tptr, const uint32_t* trows, const uint8_t* active,
                                   uint32_t* colour, uint32_t* changed)
{
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    if (!active[v]) continue;
    const uint32_t c0 = colour[v];
    uint32_t c = c0;
    for (uint32_t e = tptr[v]; e < tptr[v + 1]; ++e) {
      const uint32_t u = trows[e];
      if (u != v && active[u]) c = max(c, colour[u]);
    }
    if (c > c0) {
      colour[v] = c;
      *changed = 1;
    }
  }
}

__global__ void roots_kernel(uint32_t n, const uint8_t* active, const uint32_t* colour, uint32_t* comp)
{
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    if (active[v] && colour[v] == v) comp[v] = v;
}

// a remaining unassigned box joins the component of its colour when an edge leads it to a
// box already in that component
__global__ void back_pull_kernel(uint32_t n, const uint32_t* rowptr, const uint32_t* cols, const uint8_t* active,
                                 const uint32_t* colour, uint32_t* comp, uint32_t* changed)
{
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    if (!active[v] || comp[v] != kNone) continue;
    const uint32_t c = colour[v];
    for (uint32_t e = rowptr[v]; e < rowptr[v + 1]; ++e) {
      const uint32_t w = cols[e];
      if (w < n && w != v && active[w] && colour[w] == c && comp[w] == c) {
        comp[v] = c;
        *changed = 1;
        break;
      }
    }
  }
}

// assigned boxes leave the graph; counts the boxes that remain
__global__ void retire_kernel(uint32_t n, uint8_t* active, const uint32_t* comp, uint32_t* remaining)
{
  uint32_t left = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    if (!active[v]) continue;
    if (comp[v] != kNone) active[v] = 0;
    else ++left;
  }
  if (left) atomicAdd(remaining, left);
}

__global__ void size_kernel(uint32_t n, const uint32_t* comp, uint32_t* size)
{
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    atomicAdd(size + comp[v], 1u);
}

__global__ void flag_components_kernel(uint32_t n, const uint32_t* comp, const uint32_t* size, uint32_t min_size,
                                       uint8_t* flags, uint8_t f, uint32_t* count)
{
  uint32_t k = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    if (size[comp[v]] >= min_size) {
      flags[v] |= f;
      ++k;
    }
  if (k) atomicAdd(count, k);
}

// a leaf one of whose own test points lands in it again (fixedBoxes.m:15-17)
__global__ void flag_self_hit_kernel(uint32_t n, const uint32_t* target, uint32_t P, uint8_t* flags, uint8_t f,
                                     uint32_t* count)
{
  uint32_t k = 0;
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x) {
    bool self = false;
    for (uint32_t q = 0; q < P && !self; ++q) self = target[size_t(b) * P + q] == b;
    if (self) {
      flags[b] |= f;
      ++k;
    }
  }
  if (k) atomicAdd(count, k);
}

__global__ void flag_measure_kernel(uint32_t n, const double* v, double threshold, uint8_t* flags, uint8_t f,
                                    uint32_t* count)
{
  uint32_t k = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (v[i] >= threshold) {
      flags[i] |= f;
      ++k;
    }
  if (k) atomicAdd(count, k);
}

// runs `sweep` in batches until a batch changes nothing; false when `limit` sweeps did not settle
template<class Sweep>
b12g_status until_stable(cudaStream_t s, uint32_t* changed_dev, uint32_t limit, Sweep sweep, const char* what)
{
  for (uint32_t done = 0; done < limit; done += kBatch) {
    CK(cudaMemsetAsync(changed_dev, 0, 4, s));
    for (int k = 0; k < kBatch; ++k) sweep();
    count_launches(kBatch);
    uint32_t changed = 0;
    CK(cudaMemcpyAsync(&changed, changed_dev, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (!changed) return B12G_OK;
  }
  return fail(B12G_ERR_TIMEOUT, "strong components: %s did not settle", what);
}

// component labels of all n boxes into comp (device); the matrix's P^T must exist
b12g_status components(b12g_csr* m, uint32_t* comp, uint8_t* active, uint32_t* colour, uint32_t* word)
{
  const uint32_t n = m->n_rows;
  cudaStream_t s = m->stream;
  const int g = grid_for_n(n);
  const uint32_t* rowptr = m->rowptr.p;
  const uint32_t* cols = m->cols.p;
  const uint32_t* tptr = m->tptr.p;
  const uint32_t* trows = m->trows.p;
  init_kernel<<<g, kThreads, 0, s>>>(n, active, comp);
  count_launches(1);
  // a sweep settles within n + 1 sweeps: every change retires or recolours at least one box
  const uint32_t limit = n + 2 * kBatch;
  ST(until_stable(s, word, limit, [&] { trim_kernel<<<g, kThreads, 0, s>>>(n, rowptr, cols, tptr, trows, active,
                                                                         comp, word); }, "trimming"));
  for (uint32_t round = 0; round <= n; ++round) {
    CK(cudaMemsetAsync(word + 1, 0, 4, s));
    retire_kernel<<<g, kThreads, 0, s>>>(n, active, comp, word + 1);
    count_launches(1);
    uint32_t remaining = 0;
    CK(cudaMemcpyAsync(&remaining, word + 1, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (remaining == 0) return B12G_OK;
    colour_init_kernel<<<g, kThreads, 0, s>>>(n, active, colour);
    count_launches(1);
    ST(until_stable(s, word, limit, [&] { colour_pull_kernel<<<g, kThreads, 0, s>>>(n, tptr, trows, active, colour,
                                                                                   word); }, "colouring"));
    roots_kernel<<<g, kThreads, 0, s>>>(n, active, colour, comp);
    count_launches(1);
    ST(until_stable(s, word, limit, [&] { back_pull_kernel<<<g, kThreads, 0, s>>>(n, rowptr, cols, active, colour,
                                                                                 comp, word); }, "backward sweep"));
  }
  return fail(B12G_ERR_TIMEOUT, "strong components: rounds did not end");
}

struct SccScratch {
  Buf<uint32_t> comp, colour, size, word;
  Buf<uint8_t> active;
  b12g_status ensure(uint32_t n)
  {
    ST(comp.ensure(n, "components"));
    ST(colour.ensure(n, "components"));
    ST(size.ensure(n, "components"));
    ST(word.ensure(8, "components"));
    return active.ensure(n, "components");
  }
};

b12g_status label_components(b12g_csr* m, SccScratch& sc)
{
  ST(ensure_transpose(m));
  ST(sc.ensure(m->n_rows));
  return components(m, sc.comp.p, sc.active.p, sc.colour.p, sc.word.p);
}

}  // namespace

extern "C" {

b12g_status b12g_csr_strong_components(b12g_csr* m, uint32_t* comp, uint32_t* n_components)
{
  if (!m) return fail(B12G_ERR_INVALID, "NULL matrix");
  const uint32_t n = m->n_rows;
  if (n == 0) {
    if (n_components) *n_components = 0;
    return B12G_OK;
  }
  SccScratch sc;
  ST(label_components(m, sc));
  std::vector<uint32_t> h(n);
  CK(cudaMemcpyAsync(h.data(), sc.comp.p, size_t(n) * 4, cudaMemcpyDeviceToHost, m->stream));
  CK(cudaStreamSynchronize(m->stream));
  if (comp) std::copy(h.begin(), h.end(), comp);
  if (n_components) {
    uint32_t k = 0;
    for (uint32_t v = 0; v < n; ++v) k += h[v] == v ? 1u : 0u;
    *n_components = k;
  }
  return B12G_OK;
}

b12g_status b12g_set_flags_by_components(b12g_tree* t, b12g_csr* m, uint32_t min_size, uint8_t flags,
                                         uint32_t* n_flagged)
{
  if (!t || !m) return fail(B12G_ERR_INVALID, "NULL argument");
  if (m->n_rows != t->n) return fail(B12G_ERR_INVALID, "matrix of %u rows for %u leaves", m->n_rows, t->n);
  const uint32_t n = m->n_rows;
  SccScratch sc;
  ST(label_components(m, sc));
  cudaStream_t s = m->stream;
  CK(cudaMemsetAsync(sc.size.p, 0, size_t(n) * 4, s));
  CK(cudaMemsetAsync(sc.word.p + 2, 0, 4, s));
  const int g = grid_for_n(n);
  size_kernel<<<g, kThreads, 0, s>>>(n, sc.comp.p, sc.size.p);
  // the tree's own stream must not touch the flags meanwhile: wait for it first
  CK(cudaStreamSynchronize(t->stream));
  flag_components_kernel<<<g, kThreads, 0, s>>>(n, sc.comp.p, sc.size.p, std::max<uint32_t>(min_size, 1), t->flg(),
                                                flags, sc.word.p + 2);
  count_launches(2);
  uint32_t k = 0;
  CK(cudaMemcpyAsync(&k, sc.word.p + 2, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (n_flagged) *n_flagged = k;
  return B12G_OK;
}

b12g_status b12g_set_flags_by_measure(b12g_tree* t, b12g_csr* m, double threshold, uint8_t flags, uint32_t* n_flagged)
{
  if (!t || !m) return fail(B12G_ERR_INVALID, "NULL argument");
  if (m->n_rows != t->n) return fail(B12G_ERR_INVALID, "matrix of %u rows for %u leaves", m->n_rows, t->n);
  if (m->vout.n < m->n_rows) return fail(B12G_ERR_INVALID, "no invariant measure computed yet");
  const uint32_t n = m->n_rows;
  cudaStream_t s = m->stream;
  Buf<uint32_t> word;
  ST(word.ensure(1, "count"));
  CK(cudaMemsetAsync(word.p, 0, 4, s));
  CK(cudaStreamSynchronize(t->stream));
  flag_measure_kernel<<<grid_for_n(n), kThreads, 0, s>>>(n, m->vout.p, threshold, t->flg(), flags, word.p);
  count_launches(1);
  uint32_t k = 0;
  CK(cudaMemcpyAsync(&k, word.p, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  word.release();
  if (n_flagged) *n_flagged = k;
  return B12G_OK;
}

b12g_status b12g_set_flags_by_self_hit(b12g_tree* t, const b12g_scheme* sc, uint8_t flags, uint32_t* n_flagged)
{
  if (!t || !sc) return fail(B12G_ERR_INVALID, "NULL argument");
  if (sc->flags_to_check != 0 || (sc->depth != B12G_LEAF_DEPTH && sc->depth != t->depth))
    return fail(B12G_ERR_INVALID, "the self-hit selection images every leaf");
  if (t->mixed) {
    uint64_t np = 0;
    ST(mixed_search(t, sc, &np));
    const uint32_t P = t->n ? uint32_t(np / t->n) : 0u;
    ST(set_ctr(t, C_TMP, 0));
    flag_self_hit_kernel<<<grid_for_n(t->n), kThreads, 0, t->stream>>>(t->n, t->out.p, P, t->flg(), flags,
                                                                      t->ctr.p + C_TMP);
    count_launches(1);
    ST(read_ctr(t, C_TMP, 1));
    if (n_flagged) *n_flagged = t->h_ctr[C_TMP];
    return B12G_OK;
  }
  Prepared pr;
  ST(prepare(t, sc, pr));
  uint32_t n_src = 0;
  ST(select_sources(t, sc, pr, n_src));
  const uint64_t np = uint64_t(n_src) * pr.P;
  ST(t->out.ensure(std::max<uint64_t>(np, 1), "search output"));
  ST(build_current_hash(t, pr));
  pr.a.out = t->out.p;
  CK(launch_image(sc->map.kind, sc->map.arith, sc->grid.kind, t->domain.dim, ImageMode::Search, pr.a, np, t->stream));
  ST(set_ctr(t, C_TMP, 0));
  flag_self_hit_kernel<<<grid_for_n(n_src), kThreads, 0, t->stream>>>(n_src, t->out.p, uint32_t(pr.P), t->flg(), flags,
                                                                     t->ctr.p + C_TMP);
  count_launches(2);
  ST(read_ctr(t, C_TMP, 1));
  if (n_flagged) *n_flagged = t->h_ctr[C_TMP];
  return B12G_OK;
}

b12g_status b12g_fixed_boxes_run(b12g_tree* t, const b12g_scheme* sc, uint32_t steps, uint32_t* counts)
{
  if (!t || !sc) return fail(B12G_ERR_INVALID, "NULL argument");
  uint32_t k = 0;
  ST(b12g_delete_depth(t, 0, &k));
  ST(b12g_set_flags(t, B12G_SD, B12G_LEAF_DEPTH, &k));
  for (uint32_t i = 0; i < steps; ++i) {
    ST(b12g_subdivide(t, B12G_SD, &k));
    ST(b12g_set_flags_by_self_hit(t, sc, B12G_HIT, &k));
    ST(b12g_remove(t, B12G_HIT, &k));
    ST(b12g_unset_flags(t, B12G_HIT, B12G_LEAF_DEPTH, &k));
    if (counts) ST(b12g_count(t, B12G_LEAF_DEPTH, counts + i));
  }
  return B12G_OK;
}

// chainRecurrentSet.m:18-44 and subdivisionByNim.m:22-66 as device loops (the SCC and
// eigenvector steps of the Matlab drivers replaced by the functions above)
// by_measure: 0 components, 1 measure of `iters` iterations, 2 measure to tolerance `tol`
static b12g_status selection_run(b12g_tree* t, const b12g_scheme* sc, uint32_t steps, int by_measure, uint32_t iters,
                                 uint32_t* counts, double tol = 0.0)
{
  if (!t || !sc) return fail(B12G_ERR_INVALID, "NULL argument");
  uint32_t k = 0;
  ST(b12g_set_flags(t, B12G_SD, B12G_LEAF_DEPTH, &k));
  b12g_csr* m = nullptr;
  b12g_status st = B12G_OK;
  for (uint32_t i = 0; i < steps && st == B12G_OK; ++i) {
    st = b12g_subdivide(t, B12G_SD, &k);
    if (st == B12G_OK) st = b12g_transition_matrix(t, sc, 0, 0, &m);
    if (st == B12G_OK) {
      if (by_measure) {
        st = by_measure == 2 ? b12g_invariant_measure_tol(m, tol, iters, 20, nullptr, nullptr, nullptr)
                             : b12g_invariant_measure(m, iters, nullptr);
        if (st == B12G_OK) st = b12g_set_flags_by_measure(t, m, 1e-9 / double(m->n_rows), B12G_HIT, &k);
      } else {
        st = b12g_set_flags_by_components(t, m, 2, B12G_HIT, &k);
      }
    }
    if (st == B12G_OK) st = b12g_remove(t, B12G_HIT, &k);
    if (st == B12G_OK) st = b12g_unset_flags(t, B12G_HIT, B12G_LEAF_DEPTH, &k);
    if (st == B12G_OK && counts) st = b12g_count(t, B12G_LEAF_DEPTH, counts + i);
  }
  if (m) b12g_csr_destroy(m);
  return st;
}

b12g_status b12g_chain_recurrent_run(b12g_tree* t, const b12g_scheme* sc, uint32_t steps, uint32_t* counts)
{
  return selection_run(t, sc, steps, 0, 0, counts);
}

b12g_status b12g_nim_run(b12g_tree* t, const b12g_scheme* sc, uint32_t steps, uint32_t iters, uint32_t* counts)
{
  return selection_run(t, sc, steps, 1, iters, counts);
}

b12g_status b12g_nim_run_tol(b12g_tree* t, const b12g_scheme* sc, uint32_t steps, double tol, uint32_t max_iters,
                             uint32_t* counts)
{
  return selection_run(t, sc, steps, 2, max_iters, counts, tol);
}

}  // extern "C"
