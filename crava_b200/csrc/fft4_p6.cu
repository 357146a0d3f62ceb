// Four-step launchers (fft4.cuh, fft4_facies.cuh) for part 6 of the size table in fft4.cu; the parts are
// separate translation units so that they compile side by side.
#include "fft4_facies.cuh"

namespace crava {

#define CRAVA_FOUR_STEP_PART(X) \
  X(25, 5, 5) \
  X(36, 6, 6) \
  X(50, 10, 5) \
  X(70, 10, 7) \
  X(90, 10, 9) \
  X(112, 14, 8) \
  X(140, 14, 10) \
  X(168, 14, 12) \
  X(200, 20, 10) \
  X(243, 27, 9) \
  X(288, 18, 16) \
  X(336, 21, 16) \
  X(392, 28, 14) \
  X(448, 28, 16) \
  X(512, 32, 16) \
  X(588, 28, 21) \
  X(672, 28, 24) \
  X(756, 28, 27) \
  X(864, 32, 27)

cudaError_t four_step_line4_p6(const GridSet& gs, int ni, int n, size_t pstride, int no, size_t ostride,
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

cudaError_t four_step_x4_p6(bool fwd, const GridSet& gs, int h, int rows, const float2* tw, const float2* twn,
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

cudaError_t four_step_x4_facies_p6(const FaciesFuse& F, const FaciesCorners& C, int h, int rows, const float2* tw,
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
