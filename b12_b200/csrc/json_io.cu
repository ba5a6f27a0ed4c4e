// JSON files of trees and transition matrices, in the reference's own format so that
// files move both ways between B12 and this library:
//   tree:   ImplicitBoxTree::save (ImplicitBoxTree.hpp:435-528) and the file constructor
//           ImplicitBoxTree(fileName) (ImplicitBoxTree.hpp:144-359, JSON branch)
//   matrix: CooMatrix::save (CooMatrix.hpp:473-525) and CooMatrix(fileName)
//           (CooMatrix.hpp:236-291)
// Layout of a file: "{", then "\n  \"name\": value" entries separated by ",", arrays as
// "[" + "\n    value" items separated by "," + "\n  ]", then "\n}" (the matrix writer
// leaves a "," after its last entry, as the reference's does).  Doubles carry 17
// significant digits (max_digits10), integers are decimal.  Host code only.
#include <cerrno>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "tree.h"

using namespace b12g;
using namespace b12g::host;

namespace {

constexpr uint32_t kB12VersionMajor = 3;   // 'c' - 'a' + 1: the reference is B12c (TypeDefinitions.h:11-12)
constexpr uint32_t kB12VersionMinor = 1;
constexpr uint64_t kHostBufferBytes = 4ull << 30;  // the reference's default nHostBufferBytes
constexpr int kSdSchemeEntries = 64;       // sdScheme_ of a depth-64 tree: dimension i mod DIM at depth i

std::string with_extension(const char* path)
{
  std::string p(path);
  if (p.size() < 5 || p.compare(p.size() - 5, 5, ".json") != 0) p += ".json";
  return p;
}

// ---------------------------------------------------------------------------- writing
struct Writer {
  FILE* f = nullptr;
  bool ok = true;
  explicit Writer(const std::string& p) : f(std::fopen(p.c_str(), "wb")) { ok = f != nullptr; }
  ~Writer() { if (f) std::fclose(f); }
  void raw(const char* s) { if (ok && std::fputs(s, f) < 0) ok = false; }
  void name(const char* n)
  {
    if (ok && std::fprintf(f, "\n  \"%s\": ", n) < 0) ok = false;
  }
  void u64(uint64_t v) { if (ok && std::fprintf(f, "%" PRIu64, v) < 0) ok = false; }
  void f64(double v) { if (ok && std::fprintf(f, "%.17g", v) < 0) ok = false; }
  template<class Put>
  void array(const char* n, size_t count, Put put)
  {
    name(n);
    raw("[");
    for (size_t i = 0; i < count && ok; ++i) {
      raw(i ? ",\n    " : "\n    ");
      put(i);
    }
    raw("\n  ]");
  }
  bool close()
  {
    if (f && std::fclose(f) != 0) ok = false;
    f = nullptr;
    return ok;
  }
};

b12g_status write_tree(const std::string& p, const b12g_domain& d, const uint64_t* codes, const uint8_t* depths,
                       const uint8_t* flags, uint64_t n)
{
  Writer w(p);
  if (!w.ok) return fail(B12G_ERR_INVALID, "cannot open %s for writing: %s", p.c_str(), std::strerror(errno));
  w.raw("{");
  w.name("B12_VERSION_MAJOR"); w.u64(kB12VersionMajor); w.raw(",");
  w.name("B12_VERSION_MINOR"); w.u64(kB12VersionMinor); w.raw(",");
  w.array("center", d.dim, [&](size_t i) { w.f64(d.center[i]); }); w.raw(",");
  w.array("radius", d.dim, [&](size_t i) { w.f64(d.radius[i]); }); w.raw(",");
  w.array("sdScheme", kSdSchemeEntries, [&](size_t i) { w.u64(i % d.dim); }); w.raw(",");
  w.name("nLeaves"); w.u64(n); w.raw(",");
  w.array("bitPatternVector", n, [&](size_t i) { w.u64(codes[i]); }); w.raw(",");
  w.array("depthVector", n, [&](size_t i) { w.u64(depths[i]); }); w.raw(",");
  w.array("flagsVector", n, [&](size_t i) { w.u64(flags[i]); }); w.raw(",");
  w.name("nHostBufferBytes"); w.u64(kHostBufferBytes);
  w.raw("\n}");
  if (!w.close()) return fail(B12G_ERR_INVALID, "error while writing %s", p.c_str());
  return B12G_OK;
}

b12g_status write_coo(const std::string& p, uint32_t n_rows, uint32_t n_cols, const uint32_t* rowptr,
                      const uint32_t* cols, const double* vals)
{
  Writer w(p);
  if (!w.ok) return fail(B12G_ERR_INVALID, "cannot open %s for writing: %s", p.c_str(), std::strerror(errno));
  const uint64_t nnz = rowptr[n_rows];
  std::vector<uint32_t> rows(nnz);
  for (uint32_t r = 0; r < n_rows; ++r)
    for (uint32_t e = rowptr[r]; e < rowptr[r + 1]; ++e) rows[e] = r;
  w.raw("{");
  w.name("nRows"); w.u64(n_rows); w.raw(",");
  w.name("nColumns"); w.u64(n_cols); w.raw(",");
  w.name("nnz"); w.u64(nnz); w.raw(",");
  w.array("rowIndices", nnz, [&](size_t i) { w.u64(rows[i]); }); w.raw(",");
  w.array("columnIndices", nnz, [&](size_t i) { w.u64(cols[i]); }); w.raw(",");
  w.array("values", nnz, [&](size_t i) { w.f64(vals[i]); }); w.raw(",");
  w.raw("\n}");
  if (!w.close()) return fail(B12G_ERR_INVALID, "error while writing %s", p.c_str());
  return B12G_OK;
}

// ---------------------------------------------------------------------------- reading
bool read_file(const std::string& p, std::string& out)
{
  FILE* f = std::fopen(p.c_str(), "rb");
  if (!f) return false;
  char buf[1 << 16];
  size_t k;
  while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) out.append(buf, k);
  std::fclose(f);
  return true;
}

// position just after `"name"` and the following ':', or npos (getNumberFromJSONString's lookup)
size_t find_value(const std::string& s, const char* name)
{
  const std::string key = std::string("\"") + name + "\"";
  size_t at = 0;
  while ((at = s.find(key, at)) != std::string::npos) {
    size_t c = s.find_first_not_of(" \t\n\v\f\r", at + key.size());
    if (c != std::string::npos && s[c] == ':') return c + 1;
    at += key.size();
  }
  return std::string::npos;
}

bool read_number(const std::string& s, const char* name, double* d, uint64_t* u)
{
  size_t p = find_value(s, name);
  if (p == std::string::npos) return false;
  p = s.find_first_not_of(" \t\n\v\f\r\"", p);
  if (p == std::string::npos) return false;
  const char* b = s.c_str() + p;
  char* e = nullptr;
  errno = 0;
  if (u) *u = std::strtoull(b, &e, 10);
  else *d = std::strtod(b, &e);
  return e != b && errno == 0;
}

// the numbers of array `name`, as doubles or as unsigned integers
template<class T>
bool read_array(const std::string& s, const char* name, std::vector<T>& out)
{
  size_t p = find_value(s, name);
  if (p == std::string::npos) return false;
  p = s.find_first_not_of(" \t\n\v\f\r", p);
  if (p == std::string::npos || s[p] != '[') return false;
  const size_t end = s.find(']', p);
  if (end == std::string::npos) return false;
  const char* c = s.c_str() + p + 1;
  const char* stop = s.c_str() + end;
  out.clear();
  while (c < stop) {
    while (c < stop && (std::strchr(" \t\n\v\f\r\",", *c) != nullptr)) ++c;
    if (c >= stop) break;
    char* e = nullptr;
    errno = 0;
    if (std::is_floating_point<T>::value) out.push_back(T(std::strtod(c, &e)));
    else out.push_back(T(std::strtoull(c, &e, 10)));
    if (e == c || errno != 0) return false;
    c = e;
  }
  return true;
}

struct TreeFile {
  b12g_domain dom{};
  std::vector<uint64_t> codes;
  std::vector<uint64_t> depths, flags;
};

b12g_status read_tree(const std::string& p, TreeFile& t)
{
  std::string s;
  if (!read_file(p, s)) return fail(B12G_ERR_INVALID, "cannot open %s", p.c_str());
  std::vector<double> center, radius;
  std::vector<uint64_t> sd;
  uint64_t n = 0;
  if (!read_array(s, "center", center) || !read_array(s, "radius", radius) || !read_array(s, "sdScheme", sd) ||
      !read_number(s, "nLeaves", nullptr, &n) || !read_array(s, "bitPatternVector", t.codes) ||
      !read_array(s, "depthVector", t.depths) || !read_array(s, "flagsVector", t.flags))
    return fail(B12G_ERR_INVALID, "%s: not a tree file of the reference's JSON format", p.c_str());
  const size_t dim = center.size();
  if (dim < 1 || dim > B12G_MAX_DIM || radius.size() != dim)
    return fail(B12G_ERR_INVALID, "%s: %zu-dimensional domain (1..%d supported)", p.c_str(), dim, B12G_MAX_DIM);
  for (size_t i = 0; i < sd.size(); ++i)
    if (sd[i] != i % dim)
      return fail(B12G_ERR_INVALID, "%s: only the default subdivision scheme (dimension i mod %zu at depth i) "
                  "is supported", p.c_str(), dim);
  if (t.codes.size() != n || t.depths.size() != n || t.flags.size() != n)
    return fail(B12G_ERR_INVALID, "%s: nLeaves %llu does not match the leaf vectors", p.c_str(),
                (unsigned long long)n);
  t.dom.dim = uint32_t(dim);
  for (size_t i = 0; i < dim; ++i) {
    t.dom.center[i] = center[i];
    t.dom.radius[i] = radius[i];
  }
  for (uint64_t i = 0; i < n; ++i)
    if (t.depths[i] > 64 || t.flags[i] > 255 || (t.depths[i] < 64 && (t.codes[i] >> t.depths[i]) != 0))
      return fail(B12G_ERR_INVALID, "%s: leaf %llu has no valid (code, depth, flags)", p.c_str(),
                  (unsigned long long)i);
  return B12G_OK;
}

struct CooFile {
  uint64_t n_rows = 0, n_cols = 0;
  std::vector<uint32_t> rowptr, cols;
  std::vector<double> vals;
};

b12g_status read_coo(const std::string& p, CooFile& m)
{
  std::string s;
  if (!read_file(p, s)) return fail(B12G_ERR_INVALID, "cannot open %s", p.c_str());
  uint64_t nnz = 0;
  std::vector<uint64_t> rows, cols;
  if (!read_number(s, "nRows", nullptr, &m.n_rows) || !read_number(s, "nColumns", nullptr, &m.n_cols) ||
      !read_number(s, "nnz", nullptr, &nnz) || !read_array(s, "rowIndices", rows) ||
      !read_array(s, "columnIndices", cols) || !read_array(s, "values", m.vals))
    return fail(B12G_ERR_INVALID, "%s: not a matrix file of the reference's JSON format", p.c_str());
  if (rows.size() != nnz || cols.size() != nnz || m.vals.size() != nnz || m.n_rows > 0xFFFFFFFEull ||
      m.n_cols > 0xFFFFFFFEull)
    return fail(B12G_ERR_INVALID, "%s: inconsistent matrix sizes", p.c_str());
  // entries in row-major order (the reference writes them so); a matrix written otherwise
  // is reordered by a stable counting sort on the row
  m.rowptr.assign(m.n_rows + 1, 0);
  for (uint64_t e = 0; e < nnz; ++e) {
    // columns are kept as written: the reference's column of lost points is nColumns itself
    // (ImplicitBoxTree.hpp:3075-3090)
    if (rows[e] >= m.n_rows || cols[e] > 0xFFFFFFFFull)
      return fail(B12G_ERR_INVALID, "%s: index out of range", p.c_str());
    ++m.rowptr[rows[e] + 1];
  }
  for (uint64_t r = 0; r < m.n_rows; ++r) m.rowptr[r + 1] += m.rowptr[r];
  std::vector<uint32_t> at(m.rowptr.begin(), m.rowptr.end() - 1);
  std::vector<double> v(nnz);
  m.cols.resize(nnz);
  for (uint64_t e = 0; e < nnz; ++e) {
    const uint32_t d = at[rows[e]]++;
    m.cols[d] = uint32_t(cols[e]);
    v[d] = m.vals[e];
  }
  m.vals.swap(v);
  return B12G_OK;
}

}  // namespace

extern "C" {

b12g_status b12g_json_write_leaves(const char* path, const b12g_domain* domain, const uint64_t* codes,
                                   const uint8_t* depths, const uint8_t* flags, uint64_t n)
{
  if (!path || !domain || (n && (!codes || !depths || !flags))) return fail(B12G_ERR_INVALID, "NULL argument");
  if (domain->dim < 1 || domain->dim > B12G_MAX_DIM) return fail(B12G_ERR_INVALID, "bad domain dimension");
  return write_tree(with_extension(path), *domain, codes, depths, flags, n);
}

b12g_status b12g_json_read_leaves(const char* path, b12g_domain* domain, uint64_t* codes, uint8_t* depths,
                                  uint8_t* flags, uint64_t* n)
{
  if (!path || !n) return fail(B12G_ERR_INVALID, "NULL argument");
  TreeFile t;
  ST(read_tree(path, t));
  const uint64_t count = t.codes.size();
  if (domain) *domain = t.dom;
  if (codes || depths || flags) {
    if (*n < count) return fail(B12G_ERR_CAPACITY, "%llu leaves do not fit %llu entries", (unsigned long long)count,
                                (unsigned long long)*n);
    for (uint64_t i = 0; i < count; ++i) {
      if (codes) codes[i] = t.codes[i];
      if (depths) depths[i] = uint8_t(t.depths[i]);
      if (flags) flags[i] = uint8_t(t.flags[i]);
    }
  }
  *n = count;
  return B12G_OK;
}

b12g_status b12g_json_write_coo(const char* path, uint32_t n_rows, uint32_t n_cols, const uint32_t* rowptr,
                                const uint32_t* cols, const double* vals)
{
  if (!path || !rowptr || (rowptr[n_rows] && (!cols || !vals))) return fail(B12G_ERR_INVALID, "NULL argument");
  return write_coo(with_extension(path), n_rows, n_cols, rowptr, cols, vals);
}

b12g_status b12g_json_read_coo(const char* path, uint32_t* n_rows, uint32_t* n_cols, uint32_t* rowptr,
                               uint32_t* cols, double* vals, uint64_t* nnz)
{
  if (!path || !nnz) return fail(B12G_ERR_INVALID, "NULL argument");
  CooFile m;
  ST(read_coo(path, m));
  if (n_rows) *n_rows = uint32_t(m.n_rows);
  if (n_cols) *n_cols = uint32_t(m.n_cols);
  if (rowptr) std::memcpy(rowptr, m.rowptr.data(), m.rowptr.size() * 4);
  if (cols) std::memcpy(cols, m.cols.data(), m.cols.size() * 4);
  if (vals) std::memcpy(vals, m.vals.data(), m.vals.size() * 8);
  *nnz = m.vals.size();
  return B12G_OK;
}

b12g_status b12g_tree_save_json(b12g_tree* t, const char* path)
{
  if (!t || !path) return fail(B12G_ERR_INVALID, "NULL argument");
  uint32_t n = 0;
  ST(b12g_count(t, B12G_LEAF_DEPTH, &n));
  std::vector<uint64_t> codes(n);
  std::vector<uint8_t> depths(n), flags(n);
  ST(b12g_leaves(t, codes.data(), depths.data(), flags.data()));
  return write_tree(with_extension(path), t->domain, codes.data(), depths.data(), flags.data(), n);
}

b12g_status b12g_tree_load_json(const char* path, b12g_tree** out)
{
  if (!path || !out) return fail(B12G_ERR_INVALID, "NULL argument");
  TreeFile f;
  ST(read_tree(path, f));
  const uint64_t n = f.codes.size();
  if (n == 0 || n > 0xFFFFFFFEull) return fail(B12G_ERR_INVALID, "%s: %llu leaves", path, (unsigned long long)n);
  std::vector<uint64_t> codes(f.codes);
  std::vector<uint8_t> depths(n), flags(n);
  for (uint64_t i = 0; i < n; ++i) {
    depths[i] = uint8_t(f.depths[i]);
    flags[i] = uint8_t(f.flags[i]);
  }
  b12g_tree* t = nullptr;
  ST(b12g_tree_create(&f.dom, &t));
  const b12g_status st = b12g_load_leaves(t, codes.data(), depths.data(), flags.data(), uint32_t(n));
  if (st != B12G_OK) {
    b12g_tree_destroy(t);
    return st;
  }
  *out = t;
  return B12G_OK;
}

b12g_status b12g_csr_save_json(const b12g_csr* m, const char* path)
{
  if (!m || !path) return fail(B12G_ERR_INVALID, "NULL argument");
  std::vector<uint32_t> rowptr(m->n_rows + 1), cols(std::max<uint64_t>(m->nnz, 1));
  std::vector<double> vals(std::max<uint64_t>(m->nnz, 1));
  ST(b12g_csr_copy(m, rowptr.data(), cols.data(), vals.data()));
  return write_coo(with_extension(path), m->n_rows, m->n_cols, rowptr.data(), cols.data(), vals.data());
}

b12g_status b12g_csr_load_json(const char* path, b12g_csr** out)
{
  if (!path || !out) return fail(B12G_ERR_INVALID, "NULL argument");
  CooFile f;
  ST(read_coo(path, f));
  int dev = 0;
  cudaGetDevice(&dev);
  b12g_csr* m = new b12g_csr();
  m->device = dev;
  m->n_rows = uint32_t(f.n_rows);
  m->n_cols = uint32_t(f.n_cols);
  m->nnz = f.vals.size();
  b12g_status st = B12G_OK;
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess)
    st = cuda_fail(cudaGetLastError(), "stream");
  if (st == B12G_OK) st = m->rowptr.ensure(f.n_rows + 1, "rowptr");
  if (st == B12G_OK) st = m->cols.ensure(std::max<uint64_t>(m->nnz, 1), "cols");
  if (st == B12G_OK) st = m->vals.ensure(std::max<uint64_t>(m->nnz, 1), "vals");
  if (st == B12G_OK) st = m->ctr.ensure(256, "csr counters");
  if (st == B12G_OK) {
    cudaError_t e = cudaMemcpy(m->rowptr.p, f.rowptr.data(), f.rowptr.size() * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && m->nnz) e = cudaMemcpy(m->cols.p, f.cols.data(), m->nnz * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && m->nnz) e = cudaMemcpy(m->vals.p, f.vals.data(), m->nnz * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) st = cuda_fail(e, "csr upload");
  }
  if (st != B12G_OK) {
    b12g_csr_destroy(m);
    return st;
  }
  *out = m;
  return B12G_OK;
}

}  // extern "C"
