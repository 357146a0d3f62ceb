// Instantiations of the general pencil pass (zpass.cuh) for 7 and 8 angle stacks.
#include "zpass.cuh"

namespace crava {

cudaError_t launch_zpass_n78(const ZParams& zp, int threads, cudaStream_t st) {
  return zp.nth == 7 ? launch_zpass_t<7>(zp, threads, st) : launch_zpass_t<8>(zp, threads, st);
}

}  // namespace crava
