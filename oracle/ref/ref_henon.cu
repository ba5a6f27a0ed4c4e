// Test infrastructure: reference Henon subdivision + transition matrix (see runner.h).
// Map: B12c/src/include/Map_Henon.h:9-40; grid: Grids.hpp:103-134 (InnerGrid).
#include "runner.h"
#include "Map_Henon.h"

int main(int argc, char** argv)
{
  using namespace b12;
  harness::RunOpts o = harness::parseOpts(argc, argv);
  const double a = std::atof(harness::arg(argc, argv, "--a", "1.4"));
  const double b = std::atof(harness::arg(argc, argv, "--b", "0.3"));
  const int n = std::atoi(harness::arg(argc, argv, "--grid", "4"));
  return harness::runSubdivision<2>({0.0, 0.0}, {1.5, 0.45}, InnerGrid<2, double>(n),
                                    Henon<2, double>(a, b, 1), o, "henon");
}
