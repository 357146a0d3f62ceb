// Four-step launchers (fft4.cuh, fft4_facies.cuh) for part 4 of the size table in fft4.cu; the parts are
// separate translation units so that they compile side by side.
#include "fft4_facies.cuh"

namespace crava {

#define CRAVA_FOUR_STEP_PART(X) \
  X(21, 7, 3) \
  X(32, 8, 4) \
  X(48, 8, 6) \
  X(63, 9, 7) \
  X(81, 9, 9) \
  X(105, 15, 7) \
  X(128, 16, 8) \
  X(160, 16, 10) \
  X(192, 16, 12) \
  X(225, 15, 15) \
  X(270, 18, 15) \
  X(320, 20, 16) \
  X(378, 21, 18) \
  X(432, 24, 18) \
  X(500, 25, 20) \
  X(567, 27, 21) \
  X(640, 32, 20) \
  X(729, 27, 27) \
  X(810, 30, 27) \
  X(1024, 32, 32)

cudaError_t four_step_line4_p4(const GridSet& gs, int ni, int n, size_t pstride, int no, size_t ostride,
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

cudaError_t four_step_x4_p4(bool fwd, const GridSet& gs, int h, int rows, const float2* tw, const float2* twn,
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

cudaError_t four_step_x4_facies_p4(const FaciesFuse& F, const FaciesCorners& C, int h, int rows, const float2* tw,
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
