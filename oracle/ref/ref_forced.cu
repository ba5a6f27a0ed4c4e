// Test infrastructure: reference subdivision for the forced Duffing period map
// (plugins.h: ForcedDuffingMap, 200 RK4 steps, forcing from a host cos table).
#include "runner.h"

int main(int argc, char** argv)
{
  using namespace b12;
  harness::RunOpts o = harness::parseOpts(argc, argv);
  const int steps = 200;
  const double period = 2.0 * 3.14159265358979323846;
  std::vector<double> table(2 * steps + 1);
  for (int j = 0; j <= 2 * steps; ++j) table[j] = std::cos(double(j) * (period / double(2 * steps)));
  const int n = std::atoi(harness::arg(argc, argv, "--grid", "4"));
  return harness::runSubdivision<2>({0.0, 0.0}, {2.0, 2.0}, InnerGrid<2, double>(n),
                                    ForcedDuffingMap(table.data(), steps, period / double(steps)), o,
                                    "forced-duffing");
}
