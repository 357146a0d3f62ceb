// Instantiations of the eigen-form pencil pass (pencil.cuh) for the 16x8 z split (nzp 128),
// one translation unit per split so that they compile side by side.
#include "pencil.cuh"

namespace crava {

cudaError_t launch_pencil_split3(const ZParams& zp, int threads, cudaStream_t st) {
  if (zp.nzp != 128) return cudaErrorInvalidValue;
  switch (zp.nth) {
    case 1: return launch_pencil_t<1, 16, 8>(zp, threads, st);
    case 2: return launch_pencil_t<2, 16, 8>(zp, threads, st);
    case 3: return launch_pencil_t<3, 16, 8>(zp, threads, st);
    case 4: return launch_pencil_t<4, 16, 8>(zp, threads, st);
    case 5: return launch_pencil_t<5, 16, 8>(zp, threads, st);
    case 6: return launch_pencil_t<6, 16, 8>(zp, threads, st);
    case 7: return launch_pencil_t<7, 16, 8>(zp, threads, st);
    case 8: return launch_pencil_t<8, 16, 8>(zp, threads, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace crava
