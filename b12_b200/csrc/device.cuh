// Device building blocks of the box-image path: arithmetic policies, box geometry,
// grids, maps and point location.  Everything here is FP64 and written with explicit
// rounding intrinsics, so the generated code does not depend on contraction flags:
//   strict  - __dmul_rn / __dadd_rn / __dsub_rn / __ddiv_rn, one rounding per op, the
//             same values as the reference built with -fmad=false on both sides;
//   fma     - __fma_rn where the map is written with explicit fused multiply-adds.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/b12g.h"

namespace b12g {

constexpr uint32_t kInvalidIndex = 0xFFFFFFFFu;
constexpr uint32_t kOutsideIndex = 0xFFFFFFFEu;   // stored image target: point left the domain
constexpr uint32_t kAbsentIndex = 0xFFFFFFFDu;   // leaf table: present, index not recorded
constexpr uint64_t kInvalidCode = ~uint64_t(0);

// ---------------------------------------------------------------------------------
// arithmetic policies
// ---------------------------------------------------------------------------------
struct Strict {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  // a*b + c with two roundings
  static __device__ __forceinline__ double madd(double a, double b, double c) { return __dadd_rn(__dmul_rn(a, b), c); }
};

struct Fused {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double madd(double a, double b, double c) { return __fma_rn(a, b, c); }
};

// exact multiplication by 2^e for |e| <= 1000 (the ldexp of the reference's
// coordinateFunctions.hpp for the normal range that box coordinates live in)
__device__ __forceinline__ double pow2(int e) { return __longlong_as_double((long long)(1023 + e) << 52); }

// ---------------------------------------------------------------------------------
// job constants shared by every kernel of one tree + scheme
// ---------------------------------------------------------------------------------
struct Domain {
  double c[B12G_MAX_DIM];
  double r[B12G_MAX_DIM];
  double lo[B12G_MAX_DIM];   // c - r, rounded as the reference does (isPointInBox)
  double hi[B12G_MAX_DIM];   // c + r
  double inv_r[B12G_MAX_DIM];  // RN(1 / r) for the point-code fast path, 0 where it is not used
};

// Depth-dependent constants of dimension j at one depth, k = bisections of j: powers of
// two and exact scalings, the same values whether the host computes them once for a
// launch (the single-tree image kernels read them from their launch parameters) or a
// kernel computes them for a depth of its own.
struct AxisConst {
  double rk;        // r_j 2^-k: the radius of a box
  double s1k;       // 2^(1-k)
  double yh;        // RN(1/r_j) 2^(k-1); 0 where the point-code fast path is off
  double half;      // 2^(k-1)
  double eps;       // 2^(k-49)
  double one_eps;   // 1 - 2^(k-49)
  double pk;        // 2^k
  uint32_t mask;    // 2^k - 1, for k <= 32
  int k;
};

// exact 2^e for |e| <= 1000
__host__ __device__ __forceinline__ double pow2_hd(int e)
{
  const unsigned long long b = (unsigned long long)(1023 + e) << 52;
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)b);
#else
  double d;
  __builtin_memcpy(&d, &b, sizeof d);
  return d;
#endif
}

__host__ __device__ __forceinline__ AxisConst axis_const(const Domain& dom, int j, int k)
{
  AxisConst x;
  x.rk = dom.r[j] * pow2_hd(-k);
  x.s1k = pow2_hd(1 - k);
  x.half = pow2_hd(k - 1);
  x.yh = dom.inv_r[j] * x.half;
  x.eps = pow2_hd(k - 49);
  x.one_eps = 1.0 - x.eps;
  x.pk = pow2_hd(k);
  x.mask = uint32_t((k >= 64 ? ~0ull : (1ull << k) - 1ull) & 0xFFFFFFFFull);
  x.k = k;
  return x;
}

// every dimension's constants at a launch's depth, and the bisections one depth up (the
// parents of children-mode launches)
struct DepthConst {
  AxisConst ax[B12G_MAX_DIM];
  int k[B12G_MAX_DIM];       // bisections of each dimension at the depth
  int kp[B12G_MAX_DIM];      // ... and at the depth above
  int jd;                    // the dimension the depth's last bisection splits
  int ks[B12G_MAX_DIM];      // code assembly: dimension j's bits move up by ks[j] = K - k[j]
  int cs;                    // ... and the spread code down by cs = D K - depth (K = ceil(depth / D))
  int c32;                   // 1: D K <= 32 and K is within the 32-bit spreading's range
};

// the constants of a launch at `depth` for a domain of `dim` dimensions
inline void fill_depth_const(const Domain& dom, int dim, int depth, DepthConst& dc)
{
  auto bis = [&](int d, int j) { return d <= 0 ? 0 : d / dim + (j < d % dim ? 1 : 0); };
  for (int j = 0; j < B12G_MAX_DIM; ++j) {
    const int k = j < dim ? bis(depth, j) : 0;
    dc.ax[j] = axis_const(dom, j < dim ? j : 0, k);
    dc.k[j] = k;
    dc.kp[j] = j < dim ? bis(depth - 1, j) : 0;
  }
  dc.jd = depth >= 1 ? (depth - 1) % dim : 0;
  const int K = (depth + dim - 1) / dim;
  for (int j = 0; j < B12G_MAX_DIM; ++j) dc.ks[j] = j < dim ? K - dc.k[j] : 0;
  dc.cs = dim * K - depth;
  const int kmax = dim == 2 ? 16 : dim == 3 ? 10 : dim == 4 ? 8 : 0;
  dc.c32 = (depth > 0 && K <= kmax && dim * K <= 32) ? 1 : 0;
}

struct MapParams {
  double h, h2, h3, h6;      // step and h/2, h/3, h/6 (the reference divides at every use; same values)
  double p[6];
  uint32_t steps;
  const double* table;       // forced Duffing cos table on the device
};

struct GridParams {
  uint32_t n;                // points per dimension
  uint64_t points;           // points per box
  uint64_t seed;
  double eps1;               // 1 + eps (full grid)
  double coord[64];          // 1-D grid coordinates for index 0..n-1 (inner / full, before eps)
};

// ---------------------------------------------------------------------------------
// box geometry (computeCoordinatesOfBoxFixedSdScheme, coordinateFunctions.hpp:130-159;
// computeBoxFromPointFixedSdScheme, coordinateFunctions.hpp:63-93)
// The depth-d code holds d bits; bit t counted from the top (t = 0 is the first
// bisection) lies at position d-1-t and bisects dimension t mod D.
// ---------------------------------------------------------------------------------
template<int D>
__device__ __forceinline__ int bisections(int depth, int j) { return depth / D + (j < depth % D ? 1 : 0); }

// bit spreading: bit i of x goes to bit D*i (magic-number shifts), and back
template<int D> struct Bits;
template<> struct Bits<1> {
  static constexpr int kMax = 64;
  static __device__ __forceinline__ uint64_t spread(uint64_t x) { return x; }
  static __device__ __forceinline__ uint64_t compact(uint64_t x) { return x; }
};
template<> struct Bits<2> {
  static constexpr int kMax = 32;
  static __device__ __forceinline__ uint64_t spread(uint64_t x)
  {
    x &= 0xFFFFFFFFull;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    return (x | (x << 1)) & 0x5555555555555555ull;
  }
  static __device__ __forceinline__ uint64_t compact(uint64_t x)
  {
    x &= 0x5555555555555555ull;
    x = (x ^ (x >> 1)) & 0x3333333333333333ull;
    x = (x ^ (x >> 2)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x ^ (x >> 4)) & 0x00FF00FF00FF00FFull;
    x = (x ^ (x >> 8)) & 0x0000FFFF0000FFFFull;
    return (x ^ (x >> 16)) & 0x00000000FFFFFFFFull;
  }
};
template<> struct Bits<3> {
  static constexpr int kMax = 21;
  static __device__ __forceinline__ uint64_t spread(uint64_t x)
  {
    x &= 0x1FFFFFull;
    x = (x | (x << 32)) & 0x1F00000000FFFFull;
    x = (x | (x << 16)) & 0x1F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    return (x | (x << 2)) & 0x1249249249249249ull;
  }
  static __device__ __forceinline__ uint64_t compact(uint64_t x)
  {
    x &= 0x1249249249249249ull;
    x = (x ^ (x >> 2)) & 0x10C30C30C30C30C3ull;
    x = (x ^ (x >> 4)) & 0x100F00F00F00F00Full;
    x = (x ^ (x >> 8)) & 0x1F0000FF0000FFull;
    x = (x ^ (x >> 16)) & 0x1F00000000FFFFull;
    return (x ^ (x >> 32)) & 0x1FFFFFull;
  }
};
template<> struct Bits<4> {
  static constexpr int kMax = 16;
  static __device__ __forceinline__ uint64_t spread(uint64_t x)
  {
    x &= 0xFFFFull;
    x = (x | (x << 24)) & 0x000000FF000000FFull;
    x = (x | (x << 12)) & 0x000F000F000F000Full;
    x = (x | (x << 6)) & 0x0303030303030303ull;
    return (x | (x << 3)) & 0x1111111111111111ull;
  }
  static __device__ __forceinline__ uint64_t compact(uint64_t x)
  {
    x &= 0x1111111111111111ull;
    x = (x ^ (x >> 3)) & 0x0303030303030303ull;
    x = (x ^ (x >> 6)) & 0x000F000F000F000Full;
    x = (x ^ (x >> 12)) & 0x000000FF000000FFull;
    return (x ^ (x >> 24)) & 0x000000000000FFFFull;
  }
};

// extract the k bits of dimension j from a depth-d code, first bisection = MSB.
// Padding the code to K = ceil(d/D) full rounds puts dimension j's bits at positions
// D*m + (D-1-j), so one compaction extracts them.
template<int D>
__device__ __forceinline__ uint32_t deinterleave(uint64_t code, int depth, int j)
{
  const int K = (depth + D - 1) / D;
  if (K <= Bits<D>::kMax && D * K <= 64) {
    const int k = depth / D + (j < depth % D ? 1 : 0);
    const uint64_t x = (code << (D * K - depth)) >> (D - 1 - j);
    return uint32_t(Bits<D>::compact(x) >> (K - k));
  }
  uint32_t bits = 0;
  for (int t = j; t < depth; t += D) bits = (bits << 1) | uint32_t((code >> (depth - 1 - t)) & 1u);
  return bits;
}

// the same spreading in 32 bits, for codes of at most 32 bits (D*K <= 32); the steps for
// three dimensions are the usual 10-bit Morton ones
template<int D> struct Spread32;
template<> struct Spread32<2> {
  static constexpr int kMax = 16;
  static __device__ __forceinline__ uint32_t f(uint32_t x)
  {
    x &= 0xFFFFu;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    return (x | (x << 1)) & 0x55555555u;
  }
};
template<> struct Spread32<3> {
  static constexpr int kMax = 10;
  static __device__ __forceinline__ uint32_t f(uint32_t x)
  {
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0xFF0000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    return (x | (x << 2)) & 0x09249249u;
  }
};
template<> struct Spread32<4> {
  static constexpr int kMax = 8;
  static __device__ __forceinline__ uint32_t f(uint32_t x)
  {
    x &= 0xFFu;
    x = (x | (x << 12)) & 0x000F000Fu;
    x = (x | (x << 6)) & 0x03030303u;
    return (x | (x << 3)) & 0x11111111u;
  }
};

template<int D>
__device__ __forceinline__ uint64_t interleave(const uint32_t (&bits)[D], const int (&k)[D], int depth)
{
  const int K = (depth + D - 1) / D;
  if (K <= Bits<D>::kMax && D * K <= 64) {
    uint64_t x = 0;
#pragma unroll
    for (int j = 0; j < D; ++j) x |= Bits<D>::spread(uint64_t(bits[j]) << (K - k[j])) << (D - 1 - j);
    return depth == 0 ? 0ull : x >> (D * K - depth);
  }
  uint64_t code = 0;
#pragma unroll 1
  for (int m = 0; m < K; ++m) {
#pragma unroll
    for (int j = 0; j < D; ++j)
      if (m * D + j < depth) code = (code << 1) | uint64_t((bits[j] >> (k[j] - 1 - m)) & 1u);
  }
  return code;
}

// the depth-d code of per-dimension indices with a launch's constants (32-bit spreading
// where the code fits 32 bits)
template<int D>
__device__ __forceinline__ uint64_t code_of_bits(const DepthConst& dc, const uint32_t (&bits)[D], int depth)
{
  if constexpr (D >= 2) {
    if (dc.c32) {
      uint32_t x = 0;
#pragma unroll
      for (int j = 0; j < D; ++j) x |= Spread32<D>::f(bits[j] << dc.ks[j]) << (D - 1 - j);
      return uint64_t(x >> dc.cs);
    }
  }
  int k[D];
#pragma unroll
  for (int j = 0; j < D; ++j) k[j] = dc.k[j];
  return interleave<D>(bits, k, depth);
}

// centre and radius of dimension j of a box whose index in that dimension is `bits`
// after k bisections
__device__ __forceinline__ void box_axis(const Domain& dom, const AxisConst& x, int j, uint32_t bits, double& c,
                                         double& r)
{
  r = x.rk;
  // t = 2 bits 2^-k - 1: the scalings are exact, so one fused rounding gives the value of
  // the reference's rounded subtraction
  const double t = __fma_rn(double(bits), x.s1k, -1.0);
  c = __dadd_rn(__dadd_rn(__dmul_rn(t, dom.r[j]), dom.c[j]), r);
}

__device__ __forceinline__ void box_axis(const Domain& dom, int j, uint32_t bits, int k, double& c, double& r)
{
  box_axis(dom, axis_const(dom, j, k), j, bits, c, r);
}

// centre and radius of a box
template<int D>
__device__ __forceinline__ void box_coordinates(const Domain& dom, uint64_t code, int depth, double* c, double* r)
{
#pragma unroll
  for (int j = 0; j < D; ++j) box_axis(dom, j, deinterleave<D>(code, depth, j), bisections<D>(depth, j), c[j], r[j]);
}

// The per-dimension indices of a depth-d box packed dimension 0 first: dimension j
// takes bisections(d, j) bits, so a packed key holds d bits.  The single-tree leaf
// lookup table is keyed by it (no bit interleaving on the lookup path); the order of
// packed keys is not the tree order.
template<int D>
__device__ __forceinline__ uint64_t pack_bits(const uint32_t* bits, int depth)
{
  uint64_t p = 0;
#pragma unroll
  for (int j = 0; j < D; ++j) p = (p << bisections<D>(depth, j)) | uint64_t(bits[j]);
  return p;
}

template<int D>
__device__ __forceinline__ uint64_t pack_bits_k(const uint32_t* bits, const int* k)
{
  uint64_t p = 0;
#pragma unroll
  for (int j = 0; j < D; ++j) p = (p << k[j]) | uint64_t(bits[j]);
  return p;
}

template<int D>
__device__ __forceinline__ void unpack_bits_k(uint64_t p, const int* k, uint32_t* bits)
{
#pragma unroll
  for (int j = D - 1; j >= 0; --j) {
    bits[j] = uint32_t(p & ((1ull << k[j]) - 1ull));
    p >>= k[j];
  }
}


// depth-d code of the box that contains p; false if p lies outside the domain.
// floor(u * 2^64bits) >> (64bits - k) == floor(u * 2^k) for u >= 0 and exact scaling,
// so the code equals the reference's depth-64 code shifted to depth d, including the
// u == 1.0 rounding case where the overflow bit is dropped.
//
// The index of p in dimension j after k bisections is floor(u 2^k) with
// u = RN(RN(RN(x / r) + 1) / 2), x = RN(p - c).  Since the halving is exact this is
// floor(RN(q + 1) 2^(k-1)) with q = RN(x / r), a non-decreasing function of q.  The fast
// path replaces the division by qa = RN(x RN(1/r)): two roundings of relative size
// 2^-53 each give |qa - x/r| <= 2^-52 |x/r| (1 + 2^-53), and |q - x/r| <= 2^-53 |x/r|,
// so |q - qa| < 2^-50.9 for |x/r| <= 1 + 2^-50 (p inside the domain).  The fast path
// takes sa = RN(x y 2^(k-1) + 2^(k-1)) (one fused operation; y 2^(k-1) is exact): it differs
// from (q + 1) 2^(k-1) by the division's and the reciprocal's errors and one rounding,
// and from the exact s = RN(q + 1) 2^(k-1) by less than 2^(k-50.5).  When sa is at least
// 2^(k-49) away from both neighbouring integers, floor(s) = floor(sa); otherwise
// (probability about 2^(k-48)) the IEEE division decides, exactly as before.
// (k <= 32: the index is returned in 32 bits)
__device__ __forceinline__ uint32_t axis_index(const Domain& dom, const AxisConst& a, int j, double pj)
{
  const double x = __dsub_rn(pj, dom.c[j]);
  if (a.yh != 0.0) {
    const double sa = __fma_rn(x, a.yh, a.half);
    const double fl = floor(sa);
    const double f = __dsub_rn(sa, fl);
    if (f >= a.eps && f <= a.one_eps) return uint32_t((unsigned long long)fl) & a.mask;
  }
  const double u = __dmul_rn(__dadd_rn(__ddiv_rn(x, dom.r[j]), 1.0), 0.5);
  return uint32_t((unsigned long long)floor(u * a.pk)) & a.mask;
}

__device__ __forceinline__ uint32_t axis_index(const Domain& dom, int j, double pj, int k)
{
  return axis_index(dom, axis_const(dom, j, k), j, pj);
}

// per-dimension indices of the depth-d box that contains p; false if p lies outside
// the domain
template<int D>
__device__ __forceinline__ bool point_bits(const Domain& dom, const double* p, int depth, uint32_t* bits)
{
  bool inside = true;
#pragma unroll
  for (int j = 0; j < D; ++j) inside = inside && (dom.lo[j] <= p[j]) && (p[j] < dom.hi[j]);
  if (!inside) return false;
#pragma unroll
  for (int j = 0; j < D; ++j) bits[j] = axis_index(dom, j, p[j], bisections<D>(depth, j));
  return true;
}

// the same with the launch's constants of that depth
template<int D>
__device__ __forceinline__ bool point_bits(const Domain& dom, const DepthConst& dc, const double* p, uint32_t* bits)
{
  bool inside = true;
#pragma unroll
  for (int j = 0; j < D; ++j) inside = inside && (dom.lo[j] <= p[j]) && (p[j] < dom.hi[j]);
  if (!inside) return false;
#pragma unroll
  for (int j = 0; j < D; ++j) bits[j] = axis_index(dom, dc.ax[j], j, p[j]);
  return true;
}

template<int D>
__device__ __forceinline__ bool point_code(const Domain& dom, const double* p, int depth, uint64_t& code)
{
  uint32_t bits[D];
  if (!point_bits<D>(dom, p, depth, bits)) return false;
  int k[D];
#pragma unroll
  for (int j = 0; j < D; ++j) k[j] = bisections<D>(depth, j);
  if constexpr (D == 3) {
    if (depth == 64) {
      // 22 + 21 + 21 bits: the first 63 bisections are 21 full rounds, the 64th is the
      // last bit of dimension 0
      const uint32_t top[3] = {bits[0] >> 1, bits[1], bits[2]};
      const int k21[3] = {21, 21, 21};
      code = (interleave<3>(top, k21, 63) << 1) | uint64_t(bits[0] & 1u);
      return true;
    }
  }
  code = interleave<D>(bits, k, depth);
  return true;
}

// ---------------------------------------------------------------------------------
// point location among sorted leaf codes of one depth (searchByIterators leaf branch,
// ImplicitBoxTree.hpp:2394-2432, with ComputeSearchIndexFunctor, Functors.hpp:289-315).
// For a uniform-depth tree the reference returns the index of the leaf whose code
// equals the point's depth-d code, else "invalid"; a point outside the domain is
// matched to the last leaf exactly when that leaf's code is 0 (hasSamePath of the
// invalid box with a zero code), which this reproduces.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t locate(const uint64_t* __restrict__ codes, uint32_t n, bool valid, uint64_t code)
{
  if (n == 0) return kInvalidIndex;
  if (!valid) return __ldg(codes + n - 1) == 0 ? n - 1 : kInvalidIndex;
  uint32_t lo = 0, len = n;
  while (len > 1) {
    const uint32_t half = len >> 1;
    const uint64_t v = __ldg(codes + lo + half);
    lo = (v <= code) ? lo + half : lo;
    len -= half;
  }
  return __ldg(codes + lo) == code ? lo : kInvalidIndex;
}

// ---------------------------------------------------------------------------------
// O(1) point location: an open-addressing hash of the leaf codes (linear probing,
// 16-byte slots {tag<<56 | code, leaf index}), built once per leaf set.  A slot whose
// tag differs from the current build's tag is empty, so a table is reused across
// builds without clearing; lookups return the same index the binary search would.
// ---------------------------------------------------------------------------------
struct LeafHash {
  ulonglong2* slots;         // nullptr: use the binary search
  uint32_t tag;              // 1..255
  uint32_t log2_cap;         // table capacity (slots allocated) = 2^log2_cap
  uint64_t* pk;              // single-tree tables: every leaf's packed key (pack_bits), which
                             // the image kernels read as their source box's indices
  uint32_t log2_use;         // nonzero: the table uses 2^log2_use slots whatever the leaf
                             // count (a table kept while boxes are added to it)
};

constexpr int kHashMaxDepth = 56;

// slots used for n keys: the smallest power of two >= 2n (load factor <= 1/2), >= 2^6
__device__ __forceinline__ int hash_log2(uint32_t n)
{
  return n <= 32 ? 6 : 64 - __clzll(2ull * n - 1ull);   // 2^l >= 2n > 2^(l-1)
}

__device__ __forceinline__ uint64_t hash_slot(uint64_t code, int log2)
{
  return (code * 0x9E3779B97F4A7C15ull) >> (64 - log2);
}

// log2 of the slots a table of n keys uses
__device__ __forceinline__ int table_log2(const LeafHash& h, uint32_t n)
{
  return h.log2_use ? int(h.log2_use) : hash_log2(n);
}

__device__ __forceinline__ uint32_t hash_locate(const LeafHash& h, uint32_t n, uint64_t code)
{
  const int l = table_log2(h, n);
  const uint64_t mask = (1ull << l) - 1ull;
  const uint64_t key = (uint64_t(h.tag) << 56) | code;
  uint64_t s = hash_slot(code, l);
  for (uint64_t probe = 0; probe <= mask; ++probe) {
    const ulonglong2 e = __ldg(h.slots + s);
    if (e.x == key) return uint32_t(e.y);
    if ((e.x >> 56) != h.tag) return kInvalidIndex;
    s = (s + 1) & mask;
  }
  return kInvalidIndex;
}

// Claims the box of packed key `code` in a table kept while boxes are added to it
// (h.log2_use set): true if this call added it (value kAbsentIndex: present, no leaf
// index), false if it was there already.  Linear probing with a CAS on the key word; a
// CAS lost to another claim re-reads the same slot.  Lookups running at the same time
// may read a slot before a claim lands; they then try the claim too and see the key.
// A table with no free slot sets bit 0 of `error`.
__device__ __forceinline__ bool hash_claim(const LeafHash& h, uint64_t code, uint32_t* error)
{
  const uint64_t mask = (1ull << h.log2_use) - 1ull;
  const unsigned long long key = (uint64_t(h.tag) << 56) | code;
  uint64_t s = hash_slot(code, int(h.log2_use));
  unsigned long long expect = 0;     // first guess for a slot: never used
  for (uint64_t step = 0; step <= 2 * mask + 64; ++step) {
    unsigned long long* kw = reinterpret_cast<unsigned long long*>(&h.slots[s].x);
    const unsigned long long cur = atomicCAS(kw, expect, key);
    if (cur == expect) {             // an empty slot (tag 0 or an old tag) now holds the key
      h.slots[s].y = kAbsentIndex;
      return true;
    }
    if (cur == key) return false;
    if ((cur >> 56) != h.tag) {
      expect = cur;                  // empty under an old tag: try it again with its value
      continue;
    }
    s = (s + 1) & mask;
    expect = 0;
  }
  atomicOr(error, 1u);
  return false;
}

// leaf index of the depth-d box with per-dimension indices `bits` (valid: inside the
// domain) among the leaves of a single tree: the table of packed keys when built, the
// binary search over the codes otherwise (with the out-of-domain rule of `locate`)
// the same with the bisection counts of `depth` given
template<int D>
__device__ __forceinline__ uint32_t find_leaf_bits(const LeafHash& h, const uint64_t* codes, uint32_t n, bool valid,
                                                   const uint32_t (&bits)[D], int depth, const int* k)
{
  if (h.slots && valid && n > 0) return hash_locate(h, n, pack_bits_k<D>(bits, k));
  if (!valid || n == 0) return locate(codes, n, valid, 0);
  int kk[D];
#pragma unroll
  for (int j = 0; j < D; ++j) kk[j] = k[j];
  return locate(codes, n, true, interleave<D>(bits, kk, depth));
}

template<int D>
__device__ __forceinline__ uint32_t find_leaf_bits(const LeafHash& h, const uint64_t* codes, uint32_t n, bool valid,
                                                   const uint32_t (&bits)[D], int depth)
{
  if (h.slots && valid && n > 0) return hash_locate(h, n, pack_bits<D>(bits, depth));
  if (!valid || n == 0) return locate(codes, n, valid, 0);
  int k[D];
#pragma unroll
  for (int j = 0; j < D; ++j) k[j] = bisections<D>(depth, j);
  return locate(codes, n, true, interleave<D>(bits, k, depth));
}

// ---------------------------------------------------------------------------------
// grids (Grids.hpp)
// ---------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11)
__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
    const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
  }
}

// 2 m 2^-53 - 1 for the top 53 bits m of (hi, lo), exactly: with m = b 2^52 + f, the
// double 1 + f 2^-52 has f as its fraction, and subtracting 2 - b from it is exact
// (Sterbenz), so no integer-to-double conversion is needed
__device__ __forceinline__ double philox_signed(uint32_t hi, uint32_t lo)
{
  const double x = __hiloint2double(int(0x3FF00000u | ((hi >> 11) & 0xFFFFFu)), int(__funnelshift_r(lo, hi, 11)));
  return __dsub_rn(x, (hi >> 31) ? 1.0 : 2.0);
}

// Inner and full grids read a per-block table of the P grid points (dimension-major,
// built from the 1-D coordinates at kernel start) instead of splitting the point index
// into digits for every point.
struct InnerGrid {
  static constexpr bool kTable = true;
  // InnerGrid::operator() (Grids.hpp:105-120): digit j of the point index picks coord[]
  static __device__ __forceinline__ double table_value(const GridParams& g, const double* coord, uint32_t k, int j)
  {
    for (int q = 0; q < j; ++q) k /= g.n;
    return coord[k % g.n];
  }
  template<int D>
  static __device__ __forceinline__ void point(const GridParams& g, const double* coord, uint64_t /*i*/,
                                               uint32_t k, double* res)
  {
#pragma unroll
    for (int j = 0; j < D; ++j) { res[j] = coord[k % g.n]; k /= g.n; }
  }
};

struct FullGrid {
  static constexpr bool kTable = true;
  // FullGrid::operator() (Grids.hpp:67-83), stretched by 1 + eps
  static __device__ __forceinline__ double table_value(const GridParams& g, const double* coord, uint32_t k, int j)
  {
    for (int q = 0; q < j; ++q) k /= g.n;
    return __dmul_rn(coord[k % g.n], g.eps1);
  }
  template<int D>
  static __device__ __forceinline__ void point(const GridParams& g, const double* coord, uint64_t /*i*/,
                                               uint32_t k, double* res)
  {
#pragma unroll
    for (int j = 0; j < D; ++j) { res[j] = __dmul_rn(coord[k % g.n], g.eps1); k /= g.n; }
  }
};

struct PhiloxGrid {
  static constexpr bool kTable = false;
  static __device__ __forceinline__ double table_value(const GridParams&, const double*, uint32_t, int) { return 0.0; }
  // uniform points in [-1,1)^D keyed by (seed, global point index i)
  template<int D>
  static __device__ __forceinline__ void point(const GridParams& g, const double* /*coord*/, uint64_t i,
                                               uint32_t /*k*/, double* res)
  {
#pragma unroll
    for (int j = 0; j < D; j += 2) {
      uint32_t c[4] = {uint32_t(i), uint32_t(i >> 32), uint32_t(j / 2), 0u};
      philox4x32_10(c, uint32_t(g.seed), uint32_t(g.seed >> 32));
      res[j] = philox_signed(c[0], c[1]);
      if (j + 1 < D) res[j + 1] = philox_signed(c[2], c[3]);
    }
  }
};

// ---------------------------------------------------------------------------------
// maps
// ---------------------------------------------------------------------------------
// Henon through IteratingMap (Map_Henon.h:11-40, MapTools.hpp:10-32)
struct HenonMap {
  static constexpr int D = 2;
  static __device__ __forceinline__ void step(const MapParams& m, const double* x, double* y)
  {
    y[0] = __dadd_rn(__dsub_rn(1.0, __dmul_rn(__dmul_rn(m.p[0], x[0]), x[0])), x[1]);
    y[1] = __dmul_rn(m.p[1], x[0]);
  }
  static __device__ __forceinline__ void apply(const MapParams& m, const double* x, double* res)
  {
    uint32_t i = 0;
    if (m.steps & 1u) { step(m, x, res); i = 1; }
    else { res[0] = x[0]; res[1] = x[1]; }
    for (; i < m.steps; i += 2) { double t[2]; step(m, res, t); step(m, t, res); }
  }
};

// Lorenz through RK4Auto (Map_Lorenz.h:10-44, MapTools.hpp:118-182)
template<class A>
struct LorenzMap {
  static constexpr int D = 3;
  static __device__ __forceinline__ void rhs(const MapParams& m, const double* x, double* r);
  static __device__ __forceinline__ void apply(const MapParams& m, const double* x0, double* res)
  {
    double x0_ = x0[0], x1 = x0[1], x2 = x0[2];
    double x[3] = {x0_, x1, x2}, k[3], a[3];
    auto step = [&]() {
      rhs(m, x, k);
#pragma unroll
      for (int j = 0; j < 3; ++j) { res[j] = A::madd(m.h6, k[j], x[j]); a[j] = A::madd(m.h2, k[j], x[j]); }
      rhs(m, a, k);
#pragma unroll
      for (int j = 0; j < 3; ++j) { res[j] = A::madd(m.h3, k[j], res[j]); a[j] = A::madd(m.h2, k[j], x[j]); }
      rhs(m, a, k);
#pragma unroll
      for (int j = 0; j < 3; ++j) { res[j] = A::madd(m.h3, k[j], res[j]); a[j] = A::madd(m.h, k[j], x[j]); }
      rhs(m, a, k);
#pragma unroll
      for (int j = 0; j < 3; ++j) { res[j] = A::madd(m.h6, k[j], res[j]); x[j] = res[j]; }
    };
    if (m.steps == 20) {
      // the configured step count with no loop instructions between the steps
#pragma unroll
      for (int s = 0; s < 20; ++s) step();
    } else {
      // four steps per trip: the loop's own counter and branch instructions would
      // otherwise take a twentieth of the issue slots at 20 steps
#pragma unroll 4
      for (uint32_t s = 0; s < m.steps; ++s) step();
    }
  }
};

// W independent Lorenz states integrated in one loop: the same operations per state as
// apply(), interleaved so that one thread keeps W dependency chains in flight
template<class A, int W>
__device__ __forceinline__ void lorenz_apply_multi(const MapParams& m, const double (&x0)[W][3], double (&res)[W][3])
{
  double x[W][3], k[W][3], a[W][3];
#pragma unroll
  for (int w = 0; w < W; ++w)
#pragma unroll
    for (int j = 0; j < 3; ++j) x[w][j] = x0[w][j];
#pragma unroll 1
  for (uint32_t s = 0; s < m.steps; ++s) {
#pragma unroll
    for (int w = 0; w < W; ++w) LorenzMap<A>::rhs(m, x[w], k[w]);
#pragma unroll
    for (int w = 0; w < W; ++w)
#pragma unroll
      for (int j = 0; j < 3; ++j) { res[w][j] = A::madd(m.h6, k[w][j], x[w][j]); a[w][j] = A::madd(m.h2, k[w][j], x[w][j]); }
#pragma unroll
    for (int w = 0; w < W; ++w) LorenzMap<A>::rhs(m, a[w], k[w]);
#pragma unroll
    for (int w = 0; w < W; ++w)
#pragma unroll
      for (int j = 0; j < 3; ++j) { res[w][j] = A::madd(m.h3, k[w][j], res[w][j]); a[w][j] = A::madd(m.h2, k[w][j], x[w][j]); }
#pragma unroll
    for (int w = 0; w < W; ++w) LorenzMap<A>::rhs(m, a[w], k[w]);
#pragma unroll
    for (int w = 0; w < W; ++w)
#pragma unroll
      for (int j = 0; j < 3; ++j) { res[w][j] = A::madd(m.h3, k[w][j], res[w][j]); a[w][j] = A::madd(m.h, k[w][j], x[w][j]); }
#pragma unroll
    for (int w = 0; w < W; ++w) LorenzMap<A>::rhs(m, a[w], k[w]);
#pragma unroll
    for (int w = 0; w < W; ++w)
#pragma unroll
      for (int j = 0; j < 3; ++j) { res[w][j] = A::madd(m.h6, k[w][j], res[w][j]); x[w][j] = res[w][j]; }
  }
}

// LorenzRHS (Map_Lorenz.h:10-24): (sigma (y-x), rho x - y - x z, -beta z + x y)
template<>
__device__ __forceinline__ void LorenzMap<Strict>::rhs(const MapParams& m, const double* x, double* r)
{
  r[0] = __dmul_rn(m.p[0], __dsub_rn(x[1], x[0]));
  r[1] = __dsub_rn(__dsub_rn(__dmul_rn(m.p[1], x[0]), x[1]), __dmul_rn(x[0], x[2]));
  r[2] = __dadd_rn(__dmul_rn(-m.p[2], x[2]), __dmul_rn(x[0], x[1]));
}

template<>
__device__ __forceinline__ void LorenzMap<Fused>::rhs(const MapParams& m, const double* x, double* r)
{
  r[0] = __dmul_rn(m.p[0], __dsub_rn(x[1], x[0]));
  r[1] = __fma_rn(-x[0], x[2], __fma_rn(m.p[1], x[0], -x[1]));
  r[2] = __fma_rn(x[0], x[1], __dmul_rn(-m.p[2], x[2]));
}

// coupled Duffing Hamiltonian through SymplecticIntegratorAuto order 2
// (MapTools.hpp:371-421): half q-step, full p-step, half q-step
struct CoupledDuffingMap {
  static constexpr int D = 4;
  static __device__ __forceinline__ void apply(const MapParams& m, const double* x, double* res)
  {
    double q0 = x[0], q1 = x[1], p0 = x[2], p1 = x[3];
    auto step = [&]() {
      q0 = __dadd_rn(q0, __dmul_rn(__dmul_rn(0.5, p0), m.h));
      q1 = __dadd_rn(q1, __dmul_rn(__dmul_rn(0.5, p1), m.h));
      const double f0 = __dsub_rn(__dsub_rn(q0, __dmul_rn(__dmul_rn(q0, q0), q0)),
                                  __dmul_rn(__dmul_rn(__dmul_rn(0.2, q0), q1), q1));
      const double f1 = __dsub_rn(__dmul_rn(-1.69, q1), __dmul_rn(__dmul_rn(__dmul_rn(0.2, q0), q0), q1));
      p0 = __dadd_rn(p0, __dmul_rn(f0, m.h));
      p1 = __dadd_rn(p1, __dmul_rn(f1, m.h));
      q0 = __dadd_rn(q0, __dmul_rn(__dmul_rn(0.5, p0), m.h));
      q1 = __dadd_rn(q1, __dmul_rn(__dmul_rn(0.5, p1), m.h));
    };
    if (m.steps == 10) {
      // the configured step count, without the loop's own instructions
#pragma unroll
      for (int s = 0; s < 10; ++s) step();
    } else {
#pragma unroll 2
      for (uint32_t s = 0; s < m.steps; ++s) step();
    }
    res[0] = q0; res[1] = q1; res[2] = p0; res[3] = p1;
  }
};

// forced Duffing x'' + delta x' + alpha x + beta x^3 = gamma cos t, exactly `steps`
// classical RK4 steps (MapTools.hpp:42-108 without the floating-point t loop), the
// forcing at the stage times read from a host-computed cos table
struct ForcedDuffingMap {
  static constexpr int D = 2;
  static __device__ __forceinline__ void rhs(const MapParams& m, double c, const double* x, double* r)
  {
    r[0] = x[1];
    r[1] = __dadd_rn(__dsub_rn(__dsub_rn(__dmul_rn(-m.p[0], x[1]), __dmul_rn(m.p[1], x[0])),
                               __dmul_rn(m.p[2], __dmul_rn(__dmul_rn(x[0], x[0]), x[0]))),
                     __dmul_rn(m.p[3], c));
  }
  static __device__ __forceinline__ void apply(const MapParams& m, const double* x0, double* res)
  {
    double x[2] = {x0[0], x0[1]}, k[2], a[2];
#pragma unroll 1
    for (uint32_t s = 0; s < m.steps; ++s) {
      const double c0 = __ldg(m.table + 2 * s), c1 = __ldg(m.table + 2 * s + 1), c2 = __ldg(m.table + 2 * s + 2);
      rhs(m, c0, x, k);
#pragma unroll
      for (int j = 0; j < 2; ++j) { res[j] = Strict::madd(m.h6, k[j], x[j]); a[j] = Strict::madd(m.h2, k[j], x[j]); }
      rhs(m, c1, a, k);
#pragma unroll
      for (int j = 0; j < 2; ++j) { res[j] = Strict::madd(m.h3, k[j], res[j]); a[j] = Strict::madd(m.h2, k[j], x[j]); }
      rhs(m, c1, a, k);
#pragma unroll
      for (int j = 0; j < 2; ++j) { res[j] = Strict::madd(m.h3, k[j], res[j]); a[j] = Strict::madd(m.h, k[j], x[j]); }
      rhs(m, c2, a, k);
#pragma unroll
      for (int j = 0; j < 2; ++j) { res[j] = Strict::madd(m.h6, k[j], res[j]); x[j] = res[j]; }
    }
  }
};

// ForcedDuffingMap::apply for W points sharing the map parameters, interleaved so that one
// thread keeps W dependency chains in flight; every point's operations and their order
// are those of apply()
template<int W>
__device__ __forceinline__ void duffing_apply_multi(const MapParams& m, const double (&x0)[W][2], double (&res)[W][2])
{
  double x[W][2], k[W][2], a[W][2];
#pragma unroll
  for (int w = 0; w < W; ++w) { x[w][0] = x0[w][0]; x[w][1] = x0[w][1]; }
#pragma unroll 1
  for (uint32_t s = 0; s < m.steps; ++s) {
    const double c0 = __ldg(m.table + 2 * s), c1 = __ldg(m.table + 2 * s + 1), c2 = __ldg(m.table + 2 * s + 2);
#pragma unroll
    for (int w = 0; w < W; ++w) ForcedDuffingMap::rhs(m, c0, x[w], k[w]);
#pragma unroll
    for (int w = 0; w < W; ++w)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        res[w][j] = Strict::madd(m.h6, k[w][j], x[w][j]);
        a[w][j] = Strict::madd(m.h2, k[w][j], x[w][j]);
      }
#pragma unroll
    for (int w = 0; w < W; ++w) ForcedDuffingMap::rhs(m, c1, a[w], k[w]);
#pragma unroll
    for (int w = 0; w < W; ++w)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        res[w][j] = Strict::madd(m.h3, k[w][j], res[w][j]);
        a[w][j] = Strict::madd(m.h2, k[w][j], x[w][j]);
      }
#pragma unroll
    for (int w = 0; w < W; ++w) ForcedDuffingMap::rhs(m, c1, a[w], k[w]);
#pragma unroll
    for (int w = 0; w < W; ++w)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        res[w][j] = Strict::madd(m.h3, k[w][j], res[w][j]);
        a[w][j] = Strict::madd(m.h, k[w][j], x[w][j]);
      }
#pragma unroll
    for (int w = 0; w < W; ++w) ForcedDuffingMap::rhs(m, c2, a[w], k[w]);
#pragma unroll
    for (int w = 0; w < W; ++w)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        res[w][j] = Strict::madd(m.h6, k[w][j], res[w][j]);
        x[w][j] = res[w][j];
      }
  }
}

}  // namespace b12g
