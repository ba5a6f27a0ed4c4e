// Test infrastructure: drives the reference's own ImplicitBoxTree (Architecture=OMP)
// through the algorithm loops of its drivers and dumps every intermediate result.
//
//   subdivision loop : B12c/doc/B12_doc.tex:269-290, B12c/src/matlab/subdivision.m:18-45
//   transition matrix: ImplicitBoxTree.hpp:3180-3193 (transitionMatrixForLeaves)
//   continuation loop: B12c/src/matlab/continuation.m:13-44
//
// Output goes to --out DIR: leaves_XX.bin per step, tm.bin, and one JSON line on
// stdout with per-step counts and wall-clock times (the CPU baseline numbers).
#pragma once

#include <chrono>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "plugins.h"

#define INCLUDE_IMPLICIT_BOX_TREE_MEMBER_DEFINITIONS
#include "ImplicitBoxTree.h"
#undef INCLUDE_IMPLICIT_BOX_TREE_MEMBER_DEFINITIONS

namespace harness {

using clk = std::chrono::steady_clock;

inline double secs(clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); }

struct RunOpts
{
  int steps = 0;              // subdivision steps, or continuation depth
  uint64_t buf = 4ull << 30;  // nHostBufferBytes (reference default: 4 GiB)
  std::string out;            // dump directory ("" = no dumps)
  int dumpFrom = 0;           // dump leaves of steps >= dumpFrom
  int tm = 1;                 // 0: none, 1: relative, 2: absolute, 3: relative + invalid column
  std::string save;           // save the final tree and matrix as JSON (save(): ImplicitBoxTree.hpp:435-528,
                              // CooMatrix.hpp:473-525) to SAVE_tree.json / SAVE_tm.json
  int mixed = 0;              // steps of selective refinement after the uniform steps (mixed leaf depths)
};

inline RunOpts parseOpts(int argc, char** argv)
{
  RunOpts o;
  o.steps = std::atoi(arg(argc, argv, "--steps", "0"));
  o.buf = std::strtoull(arg(argc, argv, "--buf", "4294967296"), nullptr, 10);
  o.out = arg(argc, argv, "--out", "");
  o.dumpFrom = std::atoi(arg(argc, argv, "--dump-from", "0"));
  o.tm = std::atoi(arg(argc, argv, "--tm", "1"));
  o.save = arg(argc, argv, "--save", "");
  o.mixed = std::atoi(arg(argc, argv, "--mixed", "0"));
  return o;
}

// Selective refinement: SD stays only on the leaves in the lower half of the first
// coordinate (the first bisection bit is 0), set through setFlagsByStencil; then
// o.mixed steps of subdivide(SD) + image selection run on a tree whose leaves have
// different depths.  mixed_00.bin holds the flagged starting tree, mixed_KK.bin the
// tree after step KK.
template<class Tree, class Grid, class Map>
void runMixed(Tree& ibt, Grid grid, Map map, const RunOpts& o, std::ostringstream& js, uint64_t& boxImages)
{
  using namespace b12;
  ibt.unsetFlags(Flag::SD, getLeafDepth());
  const uint64_t n = ibt.size();
  ThrustSystem<OMP>::Vector<bool> lower(n);
  uint64_t i = 0;
  for (auto it = ibt.begin(); it != ibt.end(); ++it, ++i) {
    auto b = *it;
    const uint64_t code = thrust::get<0>(b);
    const int depth = thrust::get<1>(b);
    lower[i] = depth > 0 && (code >> (depth - 1)) == 0;
  }
  ibt.setFlagsByStencil(lower.begin(), Flag::SD, getLeafDepth());
  if (!o.out.empty()) dumpLeaves(ibt, o.out + "/mixed_00.bin");
  js << ", \"mixed\": [";
  for (int k = 1; k <= o.mixed; ++k) {
    auto a = clk::now();
    ibt.subdivide(Flag::SD);
    boxImages += ibt.count(getLeafDepth());
    auto itPair = ibt.makePointIteratorPairOverLeaves(grid, map);
    ibt.setFlagsByIterators(itPair, Flag::HIT, getLeafDepth());
    ibt.remove(Flag::HIT);
    ibt.unsetFlags(Flag::HIT, getLeafDepth());
    auto b = clk::now();
    js << (k > 1 ? ", " : "") << "[" << k << ", " << ibt.count(getLeafDepth()) << ", " << int(ibt.depth()) << ", "
       << secs(a, b) << "]";
    if (!o.out.empty()) {
      char fn[64];
      std::snprintf(fn, sizeof fn, "/mixed_%02d.bin", k);
      dumpLeaves(ibt, o.out + fn);
    }
  }
  js << "]";
}

template<b12::Dimension DIM, class Grid, class Map>
int runSubdivision(const std::vector<double>& c, const std::vector<double>& r,
                   Grid grid, Map map, const RunOpts& o, const std::string& name)
{
  using namespace b12;
  ThrustSystem<OMP>::Vector<double> center(c.begin(), c.end()), radius(r.begin(), r.end());
  ImplicitBoxTree<OMP, DIM, double, 64> ibt(center, radius);
  ibt.setNHostBufferBytes(o.buf);
  ibt.setFlags(Flag::SD, 0);

  std::ostringstream js;
  js << "{\"workload\": \"" << name << "\", \"buf\": " << o.buf << ", \"steps\": [";
  uint64_t boxImages = 0;
  auto t0 = clk::now();
  for (int i = 1; i <= o.steps; ++i) {
    auto a = clk::now();
    ibt.subdivide(Flag::SD);
    boxImages += ibt.count(getLeafDepth());
    auto itPair = ibt.makePointIteratorPairOverLeaves(grid, map);
    ibt.setFlagsByIterators(itPair, Flag::HIT, getLeafDepth());
    ibt.remove(Flag::HIT);
    ibt.unsetFlags(Flag::HIT, getLeafDepth());
    auto b = clk::now();
    js << (i > 1 ? ", " : "") << "[" << i << ", " << ibt.count(getLeafDepth()) << ", " << secs(a, b) << "]";
    if (!o.out.empty() && i >= o.dumpFrom) {
      char fn[64];
      std::snprintf(fn, sizeof fn, "/leaves_%02d.bin", i);
      dumpLeaves(ibt, o.out + fn);
    }
  }
  js << "]";
  if (o.mixed > 0) runMixed(ibt, grid, map, o, js, boxImages);
  auto t1 = clk::now();
  js << ", \"subdivision_s\": " << secs(t0, t1) << ", \"box_images\": " << boxImages;
  if (!o.save.empty()) ibt.save(o.save + "_tree.json");
  if (o.tm) {
    const bool absolute = (o.tm == 2), invalid = (o.tm == 3);
    auto P = ibt.template transitionMatrixForLeaves<double>(grid, map, absolute, true, invalid);
    auto t2 = clk::now();
    js << ", \"tm_s\": " << secs(t1, t2) << ", \"nnz\": " << P.values_.size()
       << ", \"tm_box_images\": " << ibt.count(getLeafDepth());
    if (!o.out.empty()) dumpCoo(P, o.out + "/tm.bin");
    if (!o.save.empty()) P.save(o.save + "_tm.json");
  }
  js << "}";
  std::cout << js.str() << std::endl;
  return 0;
}

// Continuation of an unstable manifold at one depth (continuation.m:13-44).
template<b12::Dimension DIM, class Grid, class Map>
int runContinuation(const std::vector<double>& c, const std::vector<double>& r, const std::vector<double>& x0,
                    Grid grid, Map map, const RunOpts& o, const std::string& name)
{
  using namespace b12;
  ThrustSystem<OMP>::Vector<double> center(c.begin(), c.end()), radius(r.begin(), r.end());
  ThrustSystem<OMP>::Vector<double> points(x0.begin(), x0.end());
  ImplicitBoxTree<OMP, DIM, double, 64> ibt(center, radius);
  ibt.setNHostBufferBytes(o.buf);
  const Depth d = Depth(o.steps);

  std::ostringstream js;
  js << "{\"workload\": \"" << name << "\", \"buf\": " << o.buf << ", \"depth\": " << int(d) << ", \"sweeps\": [";
  auto t0 = clk::now();
  ibt.deleteDepth(0);
  ibt.insertByPoints(points, d, Flag::INS, Flag::NONE);
  NrBoxes nb0 = 0, nb1 = ibt.count(d);
  uint64_t boxImages = 0;
  int k = 0;
  if (!o.out.empty()) dumpLeaves(ibt, o.out + "/cont_00.bin");
  while (nb1 > nb0) {
    auto a = clk::now();
    boxImages += ibt.changeFlags(Flag::INS, Flag::EXPD, d);
    ibt.insertByIterators(ibt.makePointIteratorPairByFlags(d, Flag::EXPD, grid, map), d, Flag::INS, Flag::NONE);
    ibt.unsetFlags(Flag::EXPD, getLeafDepth());
    nb0 = nb1;
    nb1 = ibt.count(d);
    ++k;
    auto b = clk::now();
    js << (k > 1 ? ", " : "") << "[" << k << ", " << nb1 << ", " << secs(a, b) << "]";
    if (!o.out.empty()) {
      char fn[64];
      std::snprintf(fn, sizeof fn, "/cont_%02d.bin", k);
      dumpLeaves(ibt, o.out + fn);
    }
  }
  auto t1 = clk::now();
  js << "], \"continuation_s\": " << secs(t0, t1) << ", \"box_images\": " << boxImages << "}";
  std::cout << js.str() << std::endl;
  return 0;
}

} // namespace harness
