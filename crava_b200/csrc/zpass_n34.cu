// Instantiations of the general pencil pass (zpass.cuh) for 3 and 4 angle stacks.
#include "zpass.cuh"

namespace crava {

cudaError_t launch_zpass_n34(const ZParams& zp, int threads, cudaStream_t st) {
  return zp.nth == 3 ? launch_zpass_t<3>(zp, threads, st) : launch_zpass_t<4>(zp, threads, st);
}

}  // namespace crava
