// Four-step launchers (fft4.cuh, fft4_facies.cuh) for part 3 of the size table in fft4.cu; the parts are
// separate translation units so that they compile side by side.
#include "fft4_facies.cuh"

namespace crava {

#define CRAVA_FOUR_STEP_PART(X) \
  X(20, 5, 4) \
  X(30, 6, 5) \
  X(45, 9, 5) \
  X(60, 10, 6) \
  X(80, 10, 8) \
  X(100, 10, 10) \
  X(126, 14, 9) \
  X(150, 15, 10) \
  X(189, 21, 9) \
  X(224, 16, 14) \
  X(256, 16, 16) \
  X(315, 21, 15) \
  X(375, 25, 15) \
  X(420, 21, 20) \
  X(486, 27, 18) \
  X(560, 28, 20) \
  X(630, 30, 21) \
  X(720, 30, 24) \
  X(800, 32, 25) \
  X(960, 32, 30)

cudaError_t four_step_line4_p3(const GridSet& gs, int ni, int n, size_t pstride, int no, size_t ostride,
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

cudaError_t four_step_x4_p3(bool fwd, const GridSet& gs, int h, int rows, const float2* tw, const float2* twn,
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

cudaError_t four_step_x4_facies_p3(const FaciesFuse& F, const FaciesCorners& C, int h, int rows, const float2* tw,
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
