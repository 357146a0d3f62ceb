// Launcher of the general pencil pass (kernel in zpass.cuh, instantiated by angle count in
// zpass_n12.cu, zpass_n34.cu, zpass_n56.cu and zpass_n78.cu).
#include "zpass.cuh"

namespace crava {

size_t zpass_smem_bytes(int W, int nzp, int nth, int GT, int SB) {
  int G = nth + 3 > 9 ? nth + 3 : 9;
  return sizeof(float2) * ((size_t)nzp + (size_t)(G + GT + 3 * SB) * W * nzp);
}

size_t zpass_smem_bytes(int W, int nzp, int nth) { return zpass_smem_bytes(W, nzp, nth, 3, 1); }

cudaError_t launch_zpass(const ZParams& zp_in, int threads, cudaStream_t st, int* nlaunch) {
  ZParams zp = zp_in;
  if (zp.GT <= 0) zp.GT = 3;  // unset: the three-slot layout
  if (zp.SB <= 0) zp.SB = 1;
  if ((zp.W & (zp.W - 1)) || (1 << zp.logW) != zp.W) return cudaErrorInvalidValue;
  if (3 * zp.SB > zp.GT) return cudaErrorInvalidValue;
  if (nlaunch) (*nlaunch)++;
  switch (zp.nth) {
    case 1: case 2: return launch_zpass_n12(zp, threads, st);
    case 3: case 4: return launch_zpass_n34(zp, threads, st);
    case 5: case 6: return launch_zpass_n56(zp, threads, st);
    case 7: case 8: return launch_zpass_n78(zp, threads, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace crava
