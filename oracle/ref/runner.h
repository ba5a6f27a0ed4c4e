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
  int edits = 0;              // 1: unsubdivide / insert edits of the mixed tree afterwards (runEdits)
  std::string load;           // start from a tree the reference saved (ImplicitBoxTree(fileName),
                              // ImplicitBoxTree.hpp:144-359) instead of the surrounding box (runFromFile)
  int repeat = 1;             // runFromFile: load + steps + matrix this many times, each timed
  int maxSweeps = 0;          // continuation: stop after this many sweeps (0 = until the count stops growing)
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
  o.edits = std::atoi(arg(argc, argv, "--edits", "0"));
  o.load = arg(argc, argv, "--load", "");
  o.repeat = std::atoi(arg(argc, argv, "--repeat", "1"));
  o.maxSweeps = std::atoi(arg(argc, argv, "--max-sweeps", "0"));
  return o;
}

// n points uniform in the domain from SplitMix64 (seed), u = (x >> 11) * 2^-53 per
// coordinate in order; written to PATH as u64 n, u32 dim, f64 points[n][dim]
inline std::vector<double> domainPoints(const std::vector<double>& c, const std::vector<double>& r, uint64_t n,
                                        uint64_t seed, const std::string& path)
{
  const uint32_t dim = uint32_t(c.size());
  std::vector<double> p(n * dim);
  uint64_t s = seed;
  for (uint64_t k = 0; k < n * dim; ++k) {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = double(z >> 11) * (1.0 / 9007199254740992.0);
    const uint32_t j = uint32_t(k % dim);
    p[k] = (c[j] - r[j]) + 2.0 * r[j] * u;
  }
  if (!path.empty()) {
    FILE* f = openOut(path);
    std::fwrite(&n, 8, 1, f);
    std::fwrite(&dim, 4, 1, f);
    std::fwrite(p.data(), 8, p.size(), f);
    std::fclose(f);
  }
  return p;
}

// Edits of a tree of mixed depths, each dumped to edit_KK.bin and its return value
// recorded: unsubdivide (ImplicitBoxTree.hpp:3414-3460) twice, insertByPoints
// (1927-1946) at the leaf depth with flags for hit leaves, deeper than every leaf, and
// at an inner depth, then insertByIterators of the images of the INS leaves at the leaf
// depth, and one image selection step.  Before that, points inserted into a fresh tree
// (the surrounding box alone) at depth 6 go to root_insert.bin.
template<class Tree, class Grid, class Map>
void runEdits(Tree& ibt, const std::vector<double>& c, const std::vector<double>& r, Grid grid, Map map,
              const RunOpts& o, std::ostringstream& js)
{
  using namespace b12;
  using Vec = ThrustSystem<OMP>::Vector<double>;
  const std::string dir = o.out;
  auto pts = [&](uint64_t n, uint64_t seed, const char* name) {
    std::vector<double> p = domainPoints(c, r, n, seed, dir.empty() ? "" : dir + "/" + name);
    return Vec(p.begin(), p.end());
  };
  auto dump = [&](int k) {
    if (dir.empty()) return;
    char fn[64];
    std::snprintf(fn, sizeof fn, "/edit_%02d.bin", k);
    dumpLeaves(ibt, dir + fn);
  };
  {
    ThrustSystem<OMP>::Vector<double> center(c.begin(), c.end()), radius(r.begin(), r.end());
    Tree fresh(center, radius);
    fresh.setFlags(Flag::SD, 0);
    fresh.insertByPoints(pts(40, 7, "points_root.bin"), 6, Flag::INS, Flag::HIT);
    if (!dir.empty()) dumpLeaves(fresh, dir + "/root_insert.bin");
  }
  js << ", \"edits\": [";
  NrBoxes v = ibt.unsubdivide(Flag::SD);
  js << v;
  dump(1);
  v = ibt.unsubdivide(Flag::SD);
  js << ", " << v;
  dump(2);
  const int maxd = int(ibt.depth());
  ibt.insertByPoints(pts(300, 1, "points_3.bin"), getLeafDepth(), Flag::INS, Flag::HIT);
  js << ", " << ibt.count(getLeafDepth());
  dump(3);
  ibt.insertByPoints(pts(300, 2, "points_4.bin"), Depth(maxd + 2), Flag::INS, Flag::NONE);
  js << ", " << ibt.count(getLeafDepth());
  dump(4);
  ibt.insertByPoints(pts(300, 3, "points_5.bin"), Depth(maxd - 1), Flag::EXPD, Flag::NONE);
  js << ", " << ibt.count(getLeafDepth());
  dump(5);
  ibt.insertByIterators(ibt.makePointIteratorPairByFlags(getLeafDepth(), Flag::INS, grid, map), getLeafDepth(),
                        Flag::EXPD, Flag::NONE);
  js << ", " << ibt.count(getLeafDepth());
  dump(6);
  ibt.setFlagsByIterators(ibt.makePointIteratorPairOverLeaves(grid, map), Flag::HIT, getLeafDepth());
  ibt.remove(Flag::HIT);
  ibt.unsetFlags(Flag::HIT, getLeafDepth());
  js << ", " << ibt.count(getLeafDepth());
  dump(7);
  // flags of the boxes at inner depths (setFlags / changeFlags / unsetFlags with a depth
  // below the deepest leaf: every leaf of such a box changes, ImplicitBoxTree.hpp:914-1058,
  // 2805-2882, 3336-3411); the return values count the boxes
  const int md = int(ibt.depth());
  js << ", " << ibt.setFlags(Flag::EXPD, Depth(md - 2));
  dump(8);
  js << ", " << ibt.changeFlags(Flag::EXPD, Flag::INS, Depth(md - 3));
  dump(9);
  js << ", " << ibt.unsetFlags(Flag::INS, Depth(md - 1));
  dump(10);
  // images located at inner depths: flags on the boxes hit (setFlagsByIterators,
  // 2691-2694), the boxes' indices at that depth (searchByIterators, 2375-2572), and
  // flags for hit boxes of an insertion at an inner depth (1700-1712)
  js << ", " << ibt.setFlagsByIterators(ibt.makePointIteratorPairOverLeaves(grid, map), Flag::HIT, Depth(md - 2));
  dump(11);
  {
    auto s = ibt.searchByIterators(ibt.makePointIteratorPairOverLeaves(grid, map), Depth(md - 3));
    std::vector<uint32_t> h(s.begin(), s.end());
    if (!dir.empty()) {
      FILE* f = openOut(dir + "/search_12.bin");
      const uint64_t n = h.size();
      std::fwrite(&n, 8, 1, f);
      std::fwrite(h.data(), 4, n, f);
      std::fclose(f);
    }
    js << ", " << h.size();
  }
  ibt.insertByPoints(pts(300, 4, "points_13.bin"), Depth(md - 1), Flag::INS, Flag::EXPD);
  js << ", " << ibt.count(getLeafDepth());
  dump(13);
  // images of the boxes of an inner depth (makePointIteratorPairByFlags / OverDepth below
  // the leaves, 2267-2341, sources from initializeLeafIndicesFromDepth 1476-1611)
  js << ", " << ibt.setFlagsByIterators(ibt.makePointIteratorPairByFlags(Depth(md - 3), Flag::EXPD, grid, map),
                                        Flag::ENTR, getLeafDepth());
  dump(14);
  {
    auto s = ibt.searchByIterators(ibt.makePointIteratorPairOverDepth(Depth(md - 2), grid, map), getLeafDepth());
    std::vector<uint32_t> h(s.begin(), s.end());
    if (!dir.empty()) {
      FILE* f = openOut(dir + "/search_15.bin");
      const uint64_t n = h.size();
      std::fwrite(&n, 8, 1, f);
      std::fwrite(h.data(), 4, n, f);
      std::fclose(f);
    }
    js << ", " << h.size();
  }
  js << "], \"edit_max_depth\": " << maxd << ", \"edit_flag_depth\": " << md;
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
  if (o.edits > 0) runEdits(ibt, c, r, grid, map, o, js);
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

// The subdivision loop and the transition matrix from a tree the reference saved: each
// of o.repeat rounds constructs the tree from the file (untimed), then times o.steps
// steps (subdivide(SD), image flags, remove, unset) and transitionMatrixForLeaves.
// One JSON line: per round [subdivision s, matrix s, box-images, leaves, nonzeros].
template<b12::Dimension DIM, class Grid, class Map>
int runFromFile(Grid grid, Map map, const RunOpts& o, const std::string& name)
{
  using namespace b12;
  std::ostringstream js;
  js << "{\"workload\": \"" << name << "\", \"buf\": " << o.buf << ", \"load\": \"" << o.load << "\", \"rounds\": [";
  for (int rep = 0; rep < o.repeat; ++rep) {
    ImplicitBoxTree<OMP, DIM, double, 64> ibt(o.load);
    ibt.setNHostBufferBytes(o.buf);
    uint64_t boxImages = 0;
    auto t0 = clk::now();
    for (int i = 1; i <= o.steps; ++i) {
      ibt.subdivide(Flag::SD);
      boxImages += ibt.count(getLeafDepth());
      auto itPair = ibt.makePointIteratorPairOverLeaves(grid, map);
      ibt.setFlagsByIterators(itPair, Flag::HIT, getLeafDepth());
      ibt.remove(Flag::HIT);
      ibt.unsetFlags(Flag::HIT, getLeafDepth());
    }
    auto t1 = clk::now();
    uint64_t nnz = 0;
    if (o.tm) {
      auto P = ibt.template transitionMatrixForLeaves<double>(grid, map, o.tm == 2, true, o.tm == 3);
      nnz = P.values_.size();
    }
    auto t2 = clk::now();
    js << (rep ? ", " : "") << "[" << secs(t0, t1) << ", " << secs(t1, t2) << ", " << boxImages << ", "
       << ibt.count(getLeafDepth()) << ", " << nnz << "]";
  }
  js << "]}";
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
  while (nb1 > nb0 && (o.maxSweeps <= 0 || k < o.maxSweeps)) {
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
