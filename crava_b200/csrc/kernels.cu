// Transform kernels of the FFT-domain AVO inversion hot path (sm_100a).
//
//   k_x_r2c      forward transform along x of every row: real -> half spectrum, in place
//                (first pass of FFTGrid::fftInPlace, src/fftgrid.cpp:1587-1612)
//   k_x_c2r      inverse along x: half spectrum -> real, scaled (last pass of
//                FFTGrid::invFFTInPlace, src/fftgrid.cpp:1615-1643)
//   k_line_fft   complex transform along a strided axis (y, or z for prior grids)
//   (the fused pencil pass is in zpass.cu)
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "fft_core.cuh"
#include "kernels.cuh"

namespace crava {

constexpr int kThreads = 256;

// ------------------------------------------------------------------ x transforms

__global__ void __launch_bounds__(512) k_x_r2c(const __grid_constant__ GridSet gs, int nxp, int rows, int rpc, LinePlan pl,
                                                const float2* __restrict__ twg) {
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* buf = sm + nxp;
  float2* scr = buf + rpc * nxp;
  const int T = blockDim.x, tid = threadIdx.x;
  float* g = gs.p[blockIdx.y];
  const float scale = gs.scale[blockIdx.y];
  const int row0 = blockIdx.x * rpc;
  const int nr = min(rpc, rows - row0);
  const int rnxp = 2 * (nxp / 2 + 1), cnxp = nxp / 2 + 1;
  for (int t = tid; t < nxp; t += T) tw[t] = twg[t];
  const float* src = gs.src[blockIdx.y] + (size_t)row0 * rnxp;
  for (int e = tid; e < nr * nxp; e += T) {
    int r = e / nxp, p = e - r * nxp;
    buf[e] = make_float2(src[(size_t)r * rnxp + p] * scale, 0.f);
  }
  __syncthreads();
  fft_lines<true>(buf, scr, nr, nxp, 1, pl, tw, -1.f);
  float2* dst = reinterpret_cast<float2*>(g) + (size_t)row0 * cnxp;
  for (int e = tid; e < nr * cnxp; e += T) {
    int r = e / cnxp, p = e - r * cnxp;
    dst[e] = buf[r * nxp + p];
  }
}

__global__ void __launch_bounds__(512) k_x_c2r(const __grid_constant__ GridSet gs, int nxp, int rows, int rpc, LinePlan pl,
                                                const float2* __restrict__ twg) {
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* buf = sm + nxp;
  float2* scr = buf + rpc * nxp;
  const int T = blockDim.x, tid = threadIdx.x;
  float* g = gs.p[blockIdx.y];
  const float scale = gs.scale[blockIdx.y];
  const int row0 = blockIdx.x * rpc;
  const int nr = min(rpc, rows - row0);
  const int rnxp = 2 * (nxp / 2 + 1), cnxp = nxp / 2 + 1;
  for (int t = tid; t < nxp; t += T) tw[t] = twg[t];
  const float2* src = reinterpret_cast<const float2*>(g) + (size_t)row0 * cnxp;
  // Hermitian extension of each row; the imaginary parts of the DC and Nyquist terms do
  // not enter a real-output inverse (halfcomplex input has no slot for them)
  for (int e = tid; e < nr * nxp; e += T) {
    int r = e / nxp, p = e - r * nxp;
    float2 v;
    if (p < cnxp) {
      v = src[(size_t)r * cnxp + p];
      if (p == 0 || 2 * p == nxp) v.y = 0.f;
    } else {
      v = src[(size_t)r * cnxp + (nxp - p)];
      v.y = -v.y;
    }
    buf[e] = v;
  }
  __syncthreads();
  fft_lines<true>(buf, scr, nr, nxp, 1, pl, tw, 1.f);
  float* dst = g + (size_t)row0 * rnxp;
  for (int e = tid; e < nr * rnxp; e += T) {
    int r = e / rnxp, p = e - r * rnxp;
    dst[e] = (p < nxp) ? buf[r * nxp + p].x * scale : 0.f;
  }
}

// ------------------------------------------------------------------ strided line transform

__global__ void __launch_bounds__(512) k_line_fft(const __grid_constant__ GridSet gs, int ni, int n, size_t pstride, int no,
                                                   size_t ostride, int W, int nIT, LinePlan pl,
                                                   const float2* __restrict__ twg, float sign) {
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* buf = sm + n;
  float2* scr = buf + W * n;
  const int T = blockDim.x, tid = threadIdx.x;
  const int it = blockIdx.x % nIT;
  const int o = blockIdx.x / nIT;
  const int i0 = it * W;
  const int nw = min(W, ni - i0);
  float2* g = reinterpret_cast<float2*>(gs.p[blockIdx.y]) + (size_t)o * ostride + i0;
  for (int t = tid; t < n; t += T) tw[t] = twg[t];
  for (int e = tid; e < n * W; e += T) {
    int p = e / W, w = e - p * W;
    buf[e] = (w < nw) ? g[(size_t)p * pstride + w] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_lines<false>(buf, scr, W, 1, W, pl, tw, sign);
  for (int e = tid; e < n * W; e += T) {
    int p = e / W, w = e - p * W;
    if (w < nw) g[(size_t)p * pstride + w] = buf[e];
  }
}

// ------------------------------------------------------------------ launchers

static int round_threads(int t) {
  t = (t + 31) / 32 * 32;
  return t < 64 ? 64 : t;
}

cudaError_t launch_x_r2c(const GridSet& gs, int nxp, int rows, const LinePlan& pl, const float2* tw,
                         cudaStream_t st, int* nlaunch) {
  int rpc = std::max(1, std::min(64, 4096 / nxp));
  int T = std::min(512, round_threads(rpc * nxp / 8));
  size_t smem = sizeof(float2) * (size_t)(nxp + 2 * rpc * nxp);
  dim3 grid((rows + rpc - 1) / rpc, gs.n);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_x_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_x_r2c<<<grid, T, smem, st>>>(gs, nxp, rows, rpc, pl, tw);
  if (nlaunch) (*nlaunch)++;
  return cudaGetLastError();
}

cudaError_t launch_x_c2r(const GridSet& gs, int nxp, int rows, const LinePlan& pl, const float2* tw,
                         cudaStream_t st, int* nlaunch) {
  int rpc = std::max(1, std::min(64, 4096 / nxp));
  int T = std::min(512, round_threads(rpc * nxp / 8));
  size_t smem = sizeof(float2) * (size_t)(nxp + 2 * rpc * nxp);
  dim3 grid((rows + rpc - 1) / rpc, gs.n);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_x_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_x_c2r<<<grid, T, smem, st>>>(gs, nxp, rows, rpc, pl, tw);
  if (nlaunch) (*nlaunch)++;
  return cudaGetLastError();
}

cudaError_t launch_line_fft(const GridSet& gs, int ni, int n, size_t pstride, int no, size_t ostride,
                            const LinePlan& pl, const float2* tw, float sign, cudaStream_t st, int* nlaunch) {
  int W = 16;
  while (W > 1 && W * n > 8192) W /= 2;
  if (W > ni) W = ni < 1 ? 1 : ni;
  int T = std::min(512, round_threads(W * n / 8));
  int nIT = (ni + W - 1) / W;
  size_t smem = sizeof(float2) * (size_t)(n + 2 * W * n);
  dim3 grid((unsigned)(nIT * no), gs.n);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_line_fft, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_line_fft<<<grid, T, smem, st>>>(gs, ni, n, pstride, no, ostride, W, nIT, pl, tw, sign);
  if (nlaunch) (*nlaunch)++;
  return cudaGetLastError();
}

}  // namespace crava
