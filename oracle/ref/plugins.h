// Test infrastructure: user plug-ins and dump helpers for the reference harness.
//
// The reference's tree code (ImplicitBoxTree, compiled from its own headers with
// Architecture=OMP) is driven by user Grid and Map functors
// (B12c/doc/B12_doc.tex:107-146, B12c/src/include/Grids.h:11-98).  Four of the
// workloads need functors that the reference does not ship:
//
//   * LorenzFmaMap     - Lorenz RK4 (same steps as B12c/src/include/Map_Lorenz.h:10-44
//                        and MapTools.hpp:118-182) with every multiply-add written as
//                        an explicit fused multiply-add;
//   * CoupledDuffing   - the 2-DOF Hamiltonian
//                        H = (p1^2+p2^2)/2 - q1^2/2 + q1^4/4 + 1.69 q2^2/2 + 0.1 q1^2 q2^2
//                        as the two right-hand sides of the reference's
//                        SymplecticIntegratorAuto (MapTools.hpp:371-421, order 2);
//   * ForcedDuffingMap - x'' + 0.25 x' - x + x^3 = 0.3 cos t, period-2pi map as exactly
//                        200 classical RK4 steps (the reference's RK4 t-loop,
//                        MapTools.hpp:42-108, would run 201 steps), forcing taken from a
//                        host-computed cos table;
//   * PhiloxGrid       - uniform points in [-1,1)^DIM from Philox4x32-10 (Salmon et
//                        al., SC'11), keyed by (seed, global point index i), the index
//                        the reference passes to every grid (Functors.hpp:476-511).
//
// The same formulas, in the same operation order, are restated in oracle/b12_oracle.c
// and in the CUDA library; the tests check all three against each other.
// This file is only ever compiled into the oracle harness, never into the product.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "TypeDefinitions.h"
#include "mathFunctions.h"
#include "MapTools.h"
#include "Grids.h"

namespace b12 {

// ---------------------------------------------------------------------------------
// Lorenz with explicit FMA (RK4Auto operation order, MapTools.hpp:118-182)
// ---------------------------------------------------------------------------------
struct LorenzFmaMap : public thrust::binary_function<double*, double*, bool>
{
  double sigma_, rho_, beta_, h_;
  uint32_t steps_;

  __host__ __device__
  LorenzFmaMap(double sigma = 10.0, double rho = 28.0, double beta = 8.0 / 3.0,
               double h = 0.01, uint32_t steps = 20)
      : sigma_(sigma), rho_(rho), beta_(beta), h_(h), steps_(steps) {}

  __host__ __device__
  void rhs(const double* p, double* r) const
  {
    r[0] = sigma_ * (p[1] - p[0]);
    r[1] = fma(-p[0], p[2], fma(rho_, p[0], -p[1]));
    r[2] = fma(p[0], p[1], -beta_ * p[2]);
  }

  __host__ __device__
  bool operator()(const double* point, double* res) const
  {
    const double h6 = h_ / 6.0, h3 = h_ / 3.0, h2 = h_ / 2.0;
    double x[3] = {point[0], point[1], point[2]};
    double k[3], a[3];
    for (uint32_t s = 0; s < steps_; ++s) {
      rhs(x, k);
      for (int j = 0; j < 3; ++j) { res[j] = fma(h6, k[j], x[j]); a[j] = fma(h2, k[j], x[j]); }
      rhs(a, k);
      for (int j = 0; j < 3; ++j) { res[j] = fma(h3, k[j], res[j]); a[j] = fma(h2, k[j], x[j]); }
      rhs(a, k);
      for (int j = 0; j < 3; ++j) { res[j] = fma(h3, k[j], res[j]); a[j] = fma(h_, k[j], x[j]); }
      rhs(a, k);
      for (int j = 0; j < 3; ++j) { res[j] = fma(h6, k[j], res[j]); x[j] = res[j]; }
    }
    return false;
  }
};

// ---------------------------------------------------------------------------------
// Coupled Duffing Hamiltonian: right-hand sides for SymplecticIntegratorAuto.
// State (q1, q2, p1, p2); RHS1(p) = dq/dt = p, RHS2(q) = dp/dt = -grad V(q).
// ---------------------------------------------------------------------------------
struct CoupledDuffingRHS1
{
  __host__ __device__ void operator()(const double* p, double* r) const { r[0] = p[0]; r[1] = p[1]; }
};

struct CoupledDuffingRHS2
{
  __host__ __device__ void operator()(const double* q, double* r) const
  {
    // -dV/dq1 = q1 - q1^3 - 0.2 q1 q2^2 ;  -dV/dq2 = -1.69 q2 - 0.2 q1^2 q2
    r[0] = (q[0] - (q[0] * q[0]) * q[0]) - ((0.2 * q[0]) * q[1]) * q[1];
    r[1] = (-1.69 * q[1]) - ((0.2 * q[0]) * q[0]) * q[1];
  }
};

template<Dimension DIM, typename REAL>
struct CoupledDuffing : public thrust::binary_function<REAL*, REAL*, bool>
{
  SymplecticIntegratorAuto<4, double, CoupledDuffingRHS1, CoupledDuffingRHS2> integrator_;

  __host__ __device__
  CoupledDuffing(double h = 0.05, uint32_t steps = 10)
      : integrator_(2, CoupledDuffingRHS1(), CoupledDuffingRHS2(), h, steps) {}

  __host__ __device__
  bool operator()(const double* point, double* res) const { return integrator_(point, res); }
};

// ---------------------------------------------------------------------------------
// Forced Duffing: exactly `steps` RK4 steps over one forcing period.  The forcing
// cos(t) at the stage times t = j*h/2 (j = 0..2*steps) is read from a table that the
// caller fills with the host libm cos of (double)j * (period / (2*steps)).
// ---------------------------------------------------------------------------------
struct ForcedDuffingMap : public thrust::binary_function<double*, double*, bool>
{
  const double* cosTable_;  // 2*steps+1 entries
  double delta_, alpha_, beta_, gamma_, h_;
  uint32_t steps_;

  __host__ __device__
  ForcedDuffingMap(const double* cosTable, uint32_t steps, double h,
                   double delta = 0.25, double alpha = -1.0, double beta = 1.0, double gamma = 0.3)
      : cosTable_(cosTable), delta_(delta), alpha_(alpha), beta_(beta), gamma_(gamma), h_(h), steps_(steps) {}

  // x' = v ; v' = -delta v - alpha x - beta x^3 + gamma cos t
  __host__ __device__
  void rhs(double c, const double* p, double* r) const
  {
    r[0] = p[1];
    r[1] = (((-delta_ * p[1]) - alpha_ * p[0]) - beta_ * ((p[0] * p[0]) * p[0])) + gamma_ * c;
  }

  __host__ __device__
  bool operator()(const double* point, double* res) const
  {
    const double h6 = h_ / 6.0, h3 = h_ / 3.0, h2 = h_ / 2.0;
    double x[2] = {point[0], point[1]};
    double k[2], a[2];
    for (uint32_t s = 0; s < steps_; ++s) {
      const double c0 = cosTable_[2 * s], c1 = cosTable_[2 * s + 1], c2 = cosTable_[2 * s + 2];
      rhs(c0, x, k);
      for (int j = 0; j < 2; ++j) { res[j] = x[j] + h6 * k[j]; a[j] = x[j] + h2 * k[j]; }
      rhs(c1, a, k);
      for (int j = 0; j < 2; ++j) { res[j] += h3 * k[j]; a[j] = x[j] + h2 * k[j]; }
      rhs(c1, a, k);
      for (int j = 0; j < 2; ++j) { res[j] += h3 * k[j]; a[j] = x[j] + h_ * k[j]; }
      rhs(c2, a, k);
      for (int j = 0; j < 2; ++j) { res[j] += h6 * k[j]; x[j] = res[j]; }
    }
    return false;
  }
};

// ---------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy as
// 1, 2, 3", SC'11): 10 rounds of the 4x32 Philox S-box with the published round
// multipliers and Weyl key increments.
// ---------------------------------------------------------------------------------
__host__ __device__ inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    const uint64_t p0 = uint64_t(0xD2511F53u) * c[0];
    const uint64_t p1 = uint64_t(0xCD9E8D57u) * c[2];
    const uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0);
    const uint32_t hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
  }
}

// uniform double in [-1, 1): 53 random bits m, u = m * 2^-53, x = 2u - 1 (all exact)
__host__ __device__ inline double philoxToSigned(uint32_t hi, uint32_t lo)
{
  const uint64_t m = ((uint64_t(hi) << 32) | uint64_t(lo)) >> 11;
  return 2.0 * (double(m) * 0x1p-53) - 1.0;
}

template<Dimension DIM, typename REAL>
struct PhiloxGrid : public thrust::binary_function<NrPoints, REAL*, bool>
{
  NrPoints nPoints_;
  unsigned long long seed_;

  __host__ __device__ PhiloxGrid(NrPoints nPoints = 1, unsigned long long seed = 0)
      : nPoints_(nPoints), seed_(seed) {}

  __host__ __device__ bool operator()(NrPoints i, REAL* res) const
  {
    for (Dimension j = 0; j < DIM; j += 2) {
      uint32_t c[4] = {uint32_t(i), uint32_t(i >> 32), uint32_t(j / 2), 0u};
      philox4x32_10(c, uint32_t(seed_), uint32_t(seed_ >> 32));
      res[j] = philoxToSigned(c[0], c[1]);
      if (j + 1 < DIM) res[j + 1] = philoxToSigned(c[2], c[3]);
    }
    return false;
  }

  __host__ __device__ Dimension dim() const { return DIM; }
  __host__ __device__ NrPoints getNumberOfPointsPerBox() const { return nPoints_; }
};

} // namespace b12

// ---------------------------------------------------------------------------------
// dump helpers (little-endian binary files, read by tests/golden/make_golden.py)
// ---------------------------------------------------------------------------------
namespace harness {

inline FILE* openOut(const std::string& path)
{
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) { std::perror(path.c_str()); std::exit(2); }
  return f;
}

// leaves file: u64 n, then u64 codes[n], u8 depth[n], u8 flags[n]
template<class Tree>
inline void dumpLeaves(const Tree& t, const std::string& path)
{
  const uint64_t n = t.size();
  std::vector<uint64_t> codes(n);
  std::vector<uint8_t> depth(n), flags(n);
  uint64_t i = 0;
  for (auto it = t.begin(); it != t.end(); ++it, ++i) {
    auto b = *it;
    codes[i] = thrust::get<0>(b);
    depth[i] = thrust::get<1>(b);
    flags[i] = thrust::get<2>(b);
  }
  FILE* f = openOut(path);
  std::fwrite(&n, 8, 1, f);
  std::fwrite(codes.data(), 8, n, f);
  std::fwrite(depth.data(), 1, n, f);
  std::fwrite(flags.data(), 1, n, f);
  std::fclose(f);
}

// matrix file: u64 nnz, u32 nRows, u32 nCols, u32 rows[nnz], u32 cols[nnz], f64 vals[nnz]
template<class Coo>
inline void dumpCoo(const Coo& m, const std::string& path)
{
  const uint64_t nnz = m.values_.size();
  std::vector<uint32_t> r(m.rowIndices_.begin(), m.rowIndices_.end());
  std::vector<uint32_t> c(m.columnIndices_.begin(), m.columnIndices_.end());
  std::vector<double> v(m.values_.begin(), m.values_.end());
  FILE* f = openOut(path);
  const uint32_t nr = m.nRows_, nc = m.nColumns_;
  std::fwrite(&nnz, 8, 1, f);
  std::fwrite(&nr, 4, 1, f);
  std::fwrite(&nc, 4, 1, f);
  std::fwrite(r.data(), 4, nnz, f);
  std::fwrite(c.data(), 4, nnz, f);
  std::fwrite(v.data(), 8, nnz, f);
  std::fclose(f);
}

inline const char* arg(int argc, char** argv, const char* key, const char* dflt)
{
  for (int i = 1; i + 1 < argc; ++i)
    if (std::string(argv[i]) == key) return argv[i + 1];
  return dflt;
}

} // namespace harness
