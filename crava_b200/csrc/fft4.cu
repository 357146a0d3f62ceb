// Dispatch of the four-step transforms (kernels and launch templates in fft4.cuh) over the
// size table below, and the fused xy pass (opt-in) for a few (nxp, nyp) pairs.
#include "fft4_facies.cuh"

namespace crava {

// Lengths with a four-step split N = N1 N2 (N1 >= N2, both at most 32): every 2,3,5,7-smooth
// length from 16 to 1024 that has one, the most balanced split (the launchers sit in the
// translation units fft4_p1.cu .. fft4_p6.cu; the second column names the unit).
#define CRAVA_FOUR_STEP_SIZES(X) \
  X(16, 1, 4, 4) \
  X(18, 2, 6, 3) \
  X(20, 3, 5, 4) \
  X(21, 4, 7, 3) \
  X(24, 5, 6, 4) \
  X(25, 6, 5, 5) \
  X(27, 1, 9, 3) \
  X(28, 2, 7, 4) \
  X(30, 3, 6, 5) \
  X(32, 4, 8, 4) \
  X(35, 5, 7, 5) \
  X(36, 6, 6, 6) \
  X(40, 1, 8, 5) \
  X(42, 2, 7, 6) \
  X(45, 3, 9, 5) \
  X(48, 4, 8, 6) \
  X(49, 5, 7, 7) \
  X(50, 6, 10, 5) \
  X(54, 1, 9, 6) \
  X(56, 2, 8, 7) \
  X(60, 3, 10, 6) \
  X(63, 4, 9, 7) \
  X(64, 5, 8, 8) \
  X(70, 6, 10, 7) \
  X(72, 1, 9, 8) \
  X(75, 2, 15, 5) \
  X(80, 3, 10, 8) \
  X(81, 4, 9, 9) \
  X(84, 5, 12, 7) \
  X(90, 6, 10, 9) \
  X(96, 1, 12, 8) \
  X(98, 2, 14, 7) \
  X(100, 3, 10, 10) \
  X(105, 4, 15, 7) \
  X(108, 5, 12, 9) \
  X(112, 6, 14, 8) \
  X(120, 1, 12, 10) \
  X(125, 2, 25, 5) \
  X(126, 3, 14, 9) \
  X(128, 4, 16, 8) \
  X(135, 5, 15, 9) \
  X(140, 6, 14, 10) \
  X(144, 1, 12, 12) \
  X(147, 2, 21, 7) \
  X(150, 3, 15, 10) \
  X(160, 4, 16, 10) \
  X(162, 5, 18, 9) \
  X(168, 6, 14, 12) \
  X(175, 1, 25, 7) \
  X(180, 2, 15, 12) \
  X(189, 3, 21, 9) \
  X(192, 4, 16, 12) \
  X(196, 5, 14, 14) \
  X(200, 6, 20, 10) \
  X(210, 1, 15, 14) \
  X(216, 2, 18, 12) \
  X(224, 3, 16, 14) \
  X(225, 4, 15, 15) \
  X(240, 5, 16, 15) \
  X(243, 6, 27, 9) \
  X(250, 1, 25, 10) \
  X(252, 2, 18, 14) \
  X(256, 3, 16, 16) \
  X(270, 4, 18, 15) \
  X(280, 5, 20, 14) \
  X(288, 6, 18, 16) \
  X(294, 1, 21, 14) \
  X(300, 2, 20, 15) \
  X(315, 3, 21, 15) \
  X(320, 4, 20, 16) \
  X(324, 5, 18, 18) \
  X(336, 6, 21, 16) \
  X(350, 1, 25, 14) \
  X(360, 2, 20, 18) \
  X(375, 3, 25, 15) \
  X(378, 4, 21, 18) \
  X(384, 5, 24, 16) \
  X(392, 6, 28, 14) \
  X(400, 1, 20, 20) \
  X(405, 2, 27, 15) \
  X(420, 3, 21, 20) \
  X(432, 4, 24, 18) \
  X(441, 5, 21, 21) \
  X(448, 6, 28, 16) \
  X(450, 1, 25, 18) \
  X(480, 2, 24, 20) \
  X(486, 3, 27, 18) \
  X(500, 4, 25, 20) \
  X(504, 5, 24, 21) \
  X(512, 6, 32, 16) \
  X(525, 1, 25, 21) \
  X(540, 2, 27, 20) \
  X(560, 3, 28, 20) \
  X(567, 4, 27, 21) \
  X(576, 5, 24, 24) \
  X(588, 6, 28, 21) \
  X(600, 1, 25, 24) \
  X(625, 2, 25, 25) \
  X(630, 3, 30, 21) \
  X(640, 4, 32, 20) \
  X(648, 5, 27, 24) \
  X(672, 6, 28, 24) \
  X(675, 1, 27, 25) \
  X(700, 2, 28, 25) \
  X(720, 3, 30, 24) \
  X(729, 4, 27, 27) \
  X(750, 5, 30, 25) \
  X(756, 6, 28, 27) \
  X(768, 1, 32, 24) \
  X(784, 2, 28, 28) \
  X(800, 3, 32, 25) \
  X(810, 4, 30, 27) \
  X(840, 5, 30, 28) \
  X(864, 6, 32, 27) \
  X(896, 1, 32, 28) \
  X(900, 2, 30, 30) \
  X(960, 3, 32, 30) \
  X(1024, 4, 32, 32)

// the launchers of each translation unit (fft4_p1.cu .. fft4_p6.cu)
#define CRAVA_PART_DECL(K)                                                                               \
  cudaError_t four_step_line4_p##K(const GridSet& gs, int ni, int n, size_t pstride, int no, size_t ostride, \
                                   const float2* tw, float sign, cudaStream_t st);                         \
  cudaError_t four_step_x4_p##K(bool fwd, const GridSet& gs, int h, int rows, const float2* tw,              \
                                const float2* twn, cudaStream_t st);                                          \
  cudaError_t four_step_x4_facies_p##K(const FaciesFuse& F, const FaciesCorners& C, int h, int rows,           \
                                       const float2* tw, const float2* twn, cudaStream_t st);
CRAVA_PART_DECL(1)
CRAVA_PART_DECL(2)
CRAVA_PART_DECL(3)
CRAVA_PART_DECL(4)
CRAVA_PART_DECL(5)
CRAVA_PART_DECL(6)
#undef CRAVA_PART_DECL

static int four_step_part(int n) {
  switch (n) {
#define CRAVA_CASE(NN, K, A, B) \
  case NN:                      \
    return K;
    CRAVA_FOUR_STEP_SIZES(CRAVA_CASE)
#undef CRAVA_CASE
    default:
      return 0;
  }
}

bool four_step_supported(int n) { return four_step_part(n) > 0 && four_step_enabled(n); }

cudaError_t launch_line4(const GridSet& gs, int ni, int n, size_t pstride, int no, size_t ostride, const float2* tw,
                         float sign, cudaStream_t st, int* nlaunch) {
  if (nlaunch) (*nlaunch)++;
  switch (four_step_part(n)) {
    case 1: return four_step_line4_p1(gs, ni, n, pstride, no, ostride, tw, sign, st);
    case 2: return four_step_line4_p2(gs, ni, n, pstride, no, ostride, tw, sign, st);
    case 3: return four_step_line4_p3(gs, ni, n, pstride, no, ostride, tw, sign, st);
    case 4: return four_step_line4_p4(gs, ni, n, pstride, no, ostride, tw, sign, st);
    case 5: return four_step_line4_p5(gs, ni, n, pstride, no, ostride, tw, sign, st);
    case 6: return four_step_line4_p6(gs, ni, n, pstride, no, ostride, tw, sign, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_x4(bool fwd, const GridSet& gs, int nxp, int rows, const float2* tw, const float2* twn,
                      cudaStream_t st, int* nlaunch) {
  if (nxp & 1) return cudaErrorInvalidValue;
  const int h = nxp / 2;
  if (nlaunch) (*nlaunch)++;
  switch (four_step_part(h)) {
    case 1: return four_step_x4_p1(fwd, gs, h, rows, tw, twn, st);
    case 2: return four_step_x4_p2(fwd, gs, h, rows, tw, twn, st);
    case 3: return four_step_x4_p3(fwd, gs, h, rows, tw, twn, st);
    case 4: return four_step_x4_p4(fwd, gs, h, rows, tw, twn, st);
    case 5: return four_step_x4_p5(fwd, gs, h, rows, tw, twn, st);
    case 6: return four_step_x4_p6(fwd, gs, h, rows, tw, twn, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_x4_facies(const FaciesFuse& F, const FaciesCornersHost& hc, int nxp, int rows, const float2* tw,
                             const float2* twn, cudaStream_t st, int* nlaunch) {
  if (nxp & 1) return cudaErrorInvalidValue;
  const int h = nxp / 2;
  const FaciesCorners C = facies_corners(hc);
  if (nlaunch) (*nlaunch)++;
  switch (four_step_part(h)) {
    case 1: return four_step_x4_facies_p1(F, C, h, rows, tw, twn, st);
    case 2: return four_step_x4_facies_p2(F, C, h, rows, tw, twn, st);
    case 3: return four_step_x4_facies_p3(F, C, h, rows, tw, twn, st);
    case 4: return four_step_x4_facies_p4(F, C, h, rows, tw, twn, st);
    case 5: return four_step_x4_facies_p5(F, C, h, rows, tw, twn, st);
    case 6: return four_step_x4_facies_p6(F, C, h, rows, tw, twn, st);
    default: return cudaErrorInvalidValue;
  }
}

template <int HX1, int HX2, int NY1, int NY2>
static cudaError_t xy4(bool fwd, const GridSet& gs, int nzp, const float2* twx, const float2* twn, const float2* twy,
                       cudaStream_t st) {
  constexpr int H = HX1 * HX2, NY = NY1 * NY2;
  const int T = 256;
  const int rpc = std::max(1, T / HX1);
  int W = 8, lw = 3;
  const int SK = (((W - NY2 * W) % 16) + 16) % 16;
  const int C = std::max(1, std::min(16, tuned("xy_cluster", H, 8)));
  const size_t work = std::max(x4_smem<HX1, HX2>(false, rpc), line4_smem<NY1, NY2>(W, SK));
  const size_t smem = sizeof(float2) * (2 * (size_t)H + NY) + work;
  const void* fn = fwd ? (const void*)k_xy4<HX1, HX2, NY1, NY2, true> : (const void*)k_xy4<HX1, HX2, NY1, NY2, false>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (C > 8 && (e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess)
    return e;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(C);
  int nclusters = 0;
  if ((e = cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg)) != cudaSuccess) return e;
  if (nclusters < 1) return cudaErrorInvalidConfiguration;
  const int planes = gs.n * nzp;
  cfg.gridDim = dim3((unsigned)(std::min(nclusters, planes) * C));
  if (fwd) return cudaLaunchKernelEx(&cfg, k_xy4<HX1, HX2, NY1, NY2, true>, gs, nzp, rpc, W, lw, SK, twx, twn, twy);
  return cudaLaunchKernelEx(&cfg, k_xy4<HX1, HX2, NY1, NY2, false>, gs, nzp, rpc, W, lw, SK, twx, twn, twy);
}

// (nxp, nyp) pairs with a fused xy pass
#define CRAVA_XY_PAIRS(X)   \
  X(64, 64, 8, 4, 8, 8)     \
  X(540, 540, 18, 15, 27, 20) \
  X(768, 768, 24, 16, 32, 24)

// Opt-in (schedule key xy_fused, n = nxp): at 540^2 and 768^2 the two separate passes are
// still faster, both being bound by latency rather than by HBM traffic.
static bool xy_enabled(int nxp) { return tuned("xy_fused", nxp, 0) != 0; }

bool xy_fused_supported(int nxp, int nyp) {
  if (!xy_enabled(nxp) || !four_step_enabled(nxp)) return false;
#define CRAVA_CASE(NX, NY, A, B, C2, D) \
  if (nxp == NX && nyp == NY) return true;
  CRAVA_XY_PAIRS(CRAVA_CASE)
#undef CRAVA_CASE
  return false;
}

cudaError_t launch_xy4(bool fwd, const GridSet& gs, int nxp, int nyp, int nzp, const float2* twx, const float2* twn,
                       const float2* twy, cudaStream_t st, int* nlaunch) {
  if (nlaunch) (*nlaunch)++;
#define CRAVA_CASE(NX, NY, A, B, C2, D) \
  if (nxp == NX && nyp == NY) return xy4<A, B, C2, D>(fwd, gs, nzp, twx, twn, twy, st);
  CRAVA_XY_PAIRS(CRAVA_CASE)
#undef CRAVA_CASE
  return cudaErrorInvalidValue;
}

}  // namespace crava
