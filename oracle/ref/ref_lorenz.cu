// Test infrastructure: reference Lorenz subdivision + transition matrix (see runner.h).
// Map: B12c/src/include/Map_Lorenz.h:10-44 (RK4Auto, MapTools.hpp:118-182), or the
// explicit-FMA plug-in LorenzFmaMap (plugins.h) with --fma 1.  With --load FILE the
// steps start from a tree the reference saved (runner.h, runFromFile).
#include "runner.h"
#include "Map_Lorenz.h"

int main(int argc, char** argv)
{
  using namespace b12;
  harness::RunOpts o = harness::parseOpts(argc, argv);
  const double rho = std::atof(harness::arg(argc, argv, "--rho", "28"));
  const int fmaMode = std::atoi(harness::arg(argc, argv, "--fma", "0"));
  const int n = std::atoi(harness::arg(argc, argv, "--grid", "5"));
  const std::vector<double> c = {0.0, 0.0, 27.0}, r = {30.0, 30.0, 40.0};
  if (!o.load.empty()) {
    if (fmaMode)
      return harness::runFromFile<3>(InnerGrid<3, double>(n), LorenzFmaMap(10.0, rho, 8.0 / 3.0, 0.01, 20), o,
                                     "lorenz-fma");
    return harness::runFromFile<3>(InnerGrid<3, double>(n), Lorenz<3, double>(10.0, rho, 8.0 / 3.0, 0.01, 20), o,
                                   "lorenz");
  }
  if (fmaMode)
    return harness::runSubdivision<3>(c, r, InnerGrid<3, double>(n),
                                      LorenzFmaMap(10.0, rho, 8.0 / 3.0, 0.01, 20), o, "lorenz-fma");
  return harness::runSubdivision<3>(c, r, InnerGrid<3, double>(n),
                                    Lorenz<3, double>(10.0, rho, 8.0 / 3.0, 0.01, 20), o, "lorenz");
}
