// Four-step launchers (fft4.cuh, fft4_facies.cuh) for part 2 of the size table in fft4.cu; the parts are
// separate translation units so that they compile side by side.
#include "fft4_facies.cuh"

namespace crava {

#define CRAVA_FOUR_STEP_PART(X) \
  X(18, 6, 3) \
  X(28, 7, 4) \
  X(42, 7, 6) \
  X(56, 8, 7) \
  X(75, 15, 5) \
  X(98, 14, 7) \
  X(125, 25, 5) \
  X(147, 21, 7) \
  X(180, 15, 12) \
  X(216, 18, 12) \
  X(252, 18, 14) \
  X(300, 20, 15) \
  X(360, 20, 18) \
  X(405, 27, 15) \
  X(480, 24, 20) \
  X(540, 27, 20) \
  X(625, 25, 25) \
  X(700, 28, 25) \
  X(784, 28, 28) \
  X(900, 30, 30)

cudaError_t four_step_line4_p2(const GridSet& gs, int ni, int n, size_t pstride, int no, size_t ostride,
                                const float2* tw, float sign, cudaStream_t st) {
  switch (n) {
#define CRAVA_CASE(NN, A, B) \
  case NN:                   \
    return line4<A, B>(gs, ni, pstride, no, ostride, tw, sign, st);
    CRAVA_FOUR_STEP_PART(CRAVA_CASE)
#undef CRAVA_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t four_step_x4_p2(bool fwd, const GridSet& gs, int h, int rows, const float2* tw, const float2* twn,
                             cudaStream_t st) {
  switch (h) {
#define CRAVA_CASE(NN, A, B) \
  case NN:                   \
    return x4<A, B>(fwd, gs, rows, tw, twn, st);
    CRAVA_FOUR_STEP_PART(CRAVA_CASE)
#undef CRAVA_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t four_step_x4_facies_p2(const FaciesFuse& F, const FaciesCorners& C, int h, int rows, const float2* tw,
                                    const float2* twn, cudaStream_t st) {
  switch (h) {
#define CRAVA_CASE(NN, A, B) \
  case NN:                   \
    return x4_facies<A, B>(F, C, rows, tw, twn, st);
    CRAVA_FOUR_STEP_PART(CRAVA_CASE)
#undef CRAVA_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace crava
