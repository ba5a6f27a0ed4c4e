// Test infrastructure: reference continuation (continuation.m:13-44) of the unstable
// manifold of the origin for the coupled Duffing Hamiltonian (plugins.h), 64 Philox
// points per box, Stormer-Verlet h=0.05 x 10 (SymplecticIntegratorAuto order 2).
#include "runner.h"

int main(int argc, char** argv)
{
  using namespace b12;
  harness::RunOpts o = harness::parseOpts(argc, argv);
  const unsigned long long seed = std::strtoull(harness::arg(argc, argv, "--seed", "0"), nullptr, 10);
  const int np = std::atoi(harness::arg(argc, argv, "--points", "64"));
  return harness::runContinuation<4>({0, 0, 0, 0}, {2, 2, 2, 2}, {0, 0, 0, 0},
                                     PhiloxGrid<4, double>(np, seed), CoupledDuffing<4, double>(0.05, 10),
                                     o, "coupled-duffing");
}
