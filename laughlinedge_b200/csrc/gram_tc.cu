// placeholder replaced by the tcgen05 implementation
#include "lemc_internal.h"
namespace lemc {
int launch_gram_tc(const float*, int, const float*, int, int, const TcTile*, int, int, double*,
                   int, int, int*, cudaStream_t) {
  return LEMC_ERR_ARG;
}
int launch_gram_tc_reduce(const double*, const TcTile*, int, int, const int32_t*, const int32_t*,
                          const int32_t*, int, double*, cudaStream_t) {
  return LEMC_ERR_ARG;
}
}  // namespace lemc
