// Instantiations of the general pencil pass (zpass.cuh) for 1 and 2 angle stacks.
#include "zpass.cuh"

namespace crava {

cudaError_t launch_zpass_n12(const ZParams& zp, int threads, cudaStream_t st) {
  return zp.nth == 1 ? launch_zpass_t<1>(zp, threads, st) : launch_zpass_t<2>(zp, threads, st);
}

}  // namespace crava
