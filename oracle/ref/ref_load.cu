// Test infrastructure: reads JSON files with the reference's own loaders
// (ImplicitBoxTree(fileName): ImplicitBoxTree.hpp:144-359; CooMatrix(fileName):
// CooMatrix.hpp:236-291) and dumps what they read in the harness's binary layout.
//   ref_load --dim D --tree FILE.json --leaves OUT.bin   (leaf codes, depths, flags)
//   ref_load --coo FILE.json --out OUT.bin               (row, column, value triples)
#include "runner.h"

template<b12::Dimension DIM>
int loadTree(const std::string& in, const std::string& out)
{
  b12::ImplicitBoxTree<b12::OMP, DIM, double, 64> ibt(in);
  harness::dumpLeaves(ibt, out);
  std::cout << "{\"leaves\": " << ibt.size() << "}" << std::endl;
  return 0;
}

int main(int argc, char** argv)
{
  using namespace b12;
  const std::string tree = harness::arg(argc, argv, "--tree", "");
  const std::string coo = harness::arg(argc, argv, "--coo", "");
  if (!tree.empty()) {
    const std::string out = harness::arg(argc, argv, "--leaves", "leaves.bin");
    switch (std::atoi(harness::arg(argc, argv, "--dim", "2"))) {
      case 2: return loadTree<2>(tree, out);
      case 3: return loadTree<3>(tree, out);
      case 4: return loadTree<4>(tree, out);
      default: return 2;
    }
  }
  if (!coo.empty()) {
    CooMatrix<OMP, double> m(coo);
    harness::dumpCoo(m, harness::arg(argc, argv, "--out", "coo.bin"));
    std::cout << "{\"nnz\": " << m.values_.size() << "}" << std::endl;
    return 0;
  }
  return 1;
}
