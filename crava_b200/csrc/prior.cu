// Prior covariance grids generated on the device (sm_100a), for GRIDS-mode jobs:
//
//   SeismicParametersHolder::InitializeCorrelations (src/seismicparametersholder.cpp:235-353):
//   without estimated covariance six grids fillInParamCorr(corrXY, circCorrT, gradI, gradJ)
//   x float(priorVar0(a, b)) (FFTGrid::fillInParamCorr, src/fftgrid.cpp:878-928,
//   multiplyByScalar); with it FillInLateralCorr(corrXY, circAutoCov_ab, gradI, gradJ)
//   (src/fftgrid.cpp:830-876), the same interpolation of each grid's own temporal function;
//   FFTGrid::fillInErrCorr(corrXY, gradI, gradJ) (src/fftgrid.cpp:777-828).
//
// One thread per voxel writes all seven grids: 28 bytes per voxel of HBM writes instead of
// seven host uploads.  The arithmetic is the reference's float arithmetic, every operation
// explicitly rounded (no contraction into FMA), so the grids equal the reference's float
// grids bit for bit.
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"

namespace crava {

namespace {

__global__ void k_fill_prior(const __grid_constant__ PriorFill P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= P.nxp) return;
  const int nzp = P.nzp;
  const int ci = (i < P.nxp - i) ? i : i - P.nxp;   // cycleI: the nearer of i and i - nxp
  const int cj = (j < P.nyp - j) ? j : j - P.nyp;
  // subK = k + cycleI*gradI + cycleJ*gradJ, float, left to right
  const float sub = __fadd_rn(__fadd_rn((float)k, __fmul_rn((float)ci, P.gi)), __fmul_rn((float)cj, P.gj));
  const float cxy = __ldg(P.cxy + (size_t)j * P.nxp + i);
  const size_t o = ((size_t)k * P.nyp + j) * P.rnxp + i;
  // fillInParamCorr: linear interpolation of circCorrT at subK (cyclic), times corrXY; with
  // estimated covariance FillInLateralCorr, the same with each grid's own auto-covariance
  {
    int base = (int)floorf(sub);
    const float s = __fsub_rn(sub, (float)base);
    base %= nzp;
    if (base < 0) base += nzp;
    const int nxt = base != nzp - 1 ? base + 1 : 0;
    if (P.act) {
#pragma unroll
      for (int q = 0; q < 6; q++) {
        const float* t = P.act + (size_t)q * nzp;
        float v = __fmul_rn(__fsub_rn(1.f, s), __ldg(t + base));
        v = __fadd_rn(v, __fmul_rn(s, __ldg(t + nxt)));
        P.cov[q][o] = __fmul_rn(v, cxy);
      }
    } else {
      float v = __fmul_rn(__fsub_rn(1.f, s), __ldg(P.ct + base));
      v = __fadd_rn(v, __fmul_rn(s, __ldg(P.ct + nxt)));
      v = __fmul_rn(v, cxy);
#pragma unroll
      for (int q = 0; q < 6; q++) P.cov[q][o] = __fmul_rn(v, P.pv[q]);
    }
  }
  // fillInErrCorr: corrXY weighted by the distance of subK to the nearest multiple of nzp,
  // zero beyond one sample
  {
    float v = 0.f;
    if (fabsf(sub) < 1.0f || fabsf(__fsub_rn(sub, (float)nzp)) < 1.0f) {
      int base = (int)sub;
      float s = __fsub_rn(sub, (float)base);
      while (base < -1) base += nzp;   // |sub| < 1 or |sub - nzp| < 1: at most one step
      while (base >= 1) base -= nzp;
      if (base < 0) s = __fsub_rn(1.f, s);
      v = __fmul_rn(__fsub_rn(1.f, s), cxy);
    }
    P.err[o] = v;
  }
}

}  // namespace

cudaError_t launch_fill_prior(const PriorFill& P, cudaStream_t st, int* nlaunch) {
  dim3 grid((unsigned)((P.nxp + 127) / 128), (unsigned)P.nyp, (unsigned)P.nzp);
  k_fill_prior<<<grid, 128, 0, st>>>(P);
  if (nlaunch) (*nlaunch)++;
  return cudaGetLastError();
}

}  // namespace crava
