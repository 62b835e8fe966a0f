// Driver that links the reference's own partition generator
// (modules/partitions/integer_partitions.cu, compiled from the reference
// sources by oracle/Makefile into oracle/_ref/) and prints the basis it
// builds, one line per row: "ROW <dL> <sector_size> <part>x<mult> ...".
// Used only to generate the golden fixture tests/golden/partitions_ref.json.
// Without a GPU the reference's device copy and print kernel fail with a
// printed CUDA error; the host-side partitions are unaffected.
#include <cstdio>
#include <cstdlib>

#include "integer_partitions.h"

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s N dL [dL ...]\n", argv[0]);
    return 2;
  }
  const int N = std::atoi(argv[1]);
  vector<int> sectors(argc - 2);
  for (int i = 2; i < argc; ++i) sectors[i - 2] = std::atoi(argv[i]);
  // leaked on purpose: the reference destructor frees device pointers that a
  // GPU-less run never allocated
  auto* P = new iparts::integer_partitions(N, sectors);
  iparts::integer_partitions::partition* rows = P->getHostPartitions();
  std::printf("META %d %d %d\n", P->subspaceDimension, P->maximalDegree, P->longestPartitionLenght);
  for (int r = 0; r < P->subspaceDimension; ++r) {
    std::printf("ROW %d %d", rows[r].dM, rows[r].subspaceSize);
    for (int k = 0; k < rows[r].size; ++k)
      std::printf(" %dx%d", rows[r].partitionArray[k].number, rows[r].partitionArray[k].repetitions);
    std::printf("\n");
  }
  return 0;
}
