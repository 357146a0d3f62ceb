// Instantiations of the general pencil pass (zpass.cuh) for 5 and 6 angle stacks.
#include "zpass.cuh"

namespace crava {

cudaError_t launch_zpass_n56(const ZParams& zp, int threads, cudaStream_t st) {
  return zp.nth == 5 ? launch_zpass_t<5>(zp, threads, st) : launch_zpass_t<6>(zp, threads, st);
}

}  // namespace crava
