// Launcher of the eigen-form pencil pass (kernel in pencil.cuh, instantiated per z split in
// pencil_s1.cu, pencil_s2.cu and pencil_s3.cu).
#include "pencil.cuh"

namespace crava {

size_t pencil_smem_bytes(int W, int nzp, int nth, int SB) {
  const int G = nth + 3 > 9 ? nth + 3 : 9;
  return sizeof(float2) * ((size_t)nzp + (size_t)(G + 3 * SB) * W * nzp);
}

cudaError_t launch_pencil(const ZParams& zp, int threads, cudaStream_t st, int* nlaunch) {
  if ((zp.W & (zp.W - 1)) || (1 << zp.logW) != zp.W || !zp.eig || threads < 32 || threads > 512 || zp.SB < 0 ||
      zp.SB > kMaxSim || zp.nth < 1 || zp.nth > kMaxTheta)
    return cudaErrorInvalidValue;
  if (nlaunch) (*nlaunch)++;
  switch (zp.zsplit) {
    case 1: return launch_pencil_split1(zp, threads, st);
    case 2: return launch_pencil_split2(zp, threads, st);
    case 3: return launch_pencil_split3(zp, threads, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace crava
