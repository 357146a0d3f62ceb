// Four-step launchers (fft4.cuh, fft4_facies.cuh) for part 1 of the size table in fft4.cu; the parts are
// separate translation units so that they compile side by side.
#include "fft4_facies.cuh"

namespace crava {

#define CRAVA_FOUR_STEP_PART(X) \
  X(16, 4, 4) \
  X(27, 9, 3) \
  X(40, 8, 5) \
  X(54, 9, 6) \
  X(72, 9, 8) \
  X(96, 12, 8) \
  X(120, 12, 10) \
  X(144, 12, 12) \
  X(175, 25, 7) \
  X(210, 15, 14) \
  X(250, 25, 10) \
  X(294, 21, 14) \
  X(350, 25, 14) \
  X(400, 20, 20) \
  X(450, 25, 18) \
  X(525, 25, 21) \
  X(600, 25, 24) \
  X(675, 27, 25) \
  X(768, 32, 24) \
  X(896, 32, 28)

cudaError_t four_step_line4_p1(const GridSet& gs, int ni, int n, size_t pstride, int no, size_t ostride,
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

cudaError_t four_step_x4_p1(bool fwd, const GridSet& gs, int h, int rows, const float2* tw, const float2* twn,
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

cudaError_t four_step_x4_facies_p1(const FaciesFuse& F, const FaciesCorners& C, int h, int rows, const float2* tw,
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
