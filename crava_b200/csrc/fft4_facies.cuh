// The inverse x transform of the three posterior-mean grids with the facies probabilities
// evaluated in the same pass (sm_100a): the rows of the three grids go through the c2r
// transform of k_xc2r4 (written back as the real posterior mean, the FFTGrid::invFFTInPlace
// output), stay in shared memory, and every voxel of those rows is evaluated there by
// facies_voxel (FaciesProb::calculateFaciesProb, src/faciesprob.cpp:1909-2075), so the
// posterior mean is not read back from memory for the facies pass.
#pragma once
#include "facies.cuh"
#include "fft4.cuh"

namespace crava {

// rows r = j + nyp k of rpc-row chunks; shared: twiddle tables, the work rows Z, the staged
// half spectra Xs and the real rows V of the three grids (3 x rpc x h sample pairs).
template <int N1, int N2>
__global__ void __launch_bounds__(256) k_xc2r4_facies(const __grid_constant__ FaciesFuse F,
                                                      const __grid_constant__ FaciesCorners C, int rows, int rpc,
                                                      const float2* __restrict__ twg, const float2* __restrict__ twn) {
  using L = RowLayout<N1, N2>;
  constexpr int H = N1 * N2, CN = H + 1;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* twh = tw + H;
  float2* Z = twh + H;
  float2* Xs = Z + rpc * L::PITCH;
  float2* V = Xs + rpc * CN;
  const int row0 = blockIdx.x * rpc, nr = min(rpc, rows - row0);
  for (int t = threadIdx.x; t < H; t += blockDim.x) {
    tw[t] = twg[t];
    twh[t] = twn[t];
  }
  for (int a = 0; a < 3; a++) {
    float2* g = reinterpret_cast<float2*>(F.mean[a]) + (size_t)row0 * CN;
    const uint32_t xb = smem_addr(Xs);
    for (int e = threadIdx.x; e < nr * CN; e += blockDim.x) cp_async8(xb + 8u * (uint32_t)e, g + e);
    cp_async_commit();
    cp_async_wait_0();
    __syncthreads();
    xc2r4_staged<N1, N2, true>(Xs, g, nr, F.scale, tw, twh, Z, V + a * rpc * H);
  }
  const float* Vf = reinterpret_cast<const float*>(V);
  for (int e = threadIdx.x; e < nr * F.rnxp_out; e += blockDim.x) {
    const int r = e / F.rnxp_out, i = e - r * F.rnxp_out;
    const int row = row0 + r, k = row / F.nyp, j = row - k * F.nyp;
    if (j >= F.ny || k >= F.nz) continue;
    const size_t o = (size_t)i + (size_t)F.rnxp_out * ((size_t)j + (size_t)F.ny * k);
    if (i >= F.nx) {
      for (int f = 0; f <= F.nf; f++) F.out.p[f][o] = kRMissing;
      if (F.seis_lh) F.seis_lh[o] = kRMissing;
      continue;
    }
    const int s = 2 * r * H + i;   // sample i of row r in a grid's block of 2 rpc H floats
    const float v[3] = {Vf[s], Vf[2 * rpc * H + s], Vf[4 * rpc * H + s]};
    float val[kMaxFacies];
    const float sum = facies_voxel(v, i, j, F.nx, F.ny, C, F.nf, F.pr, F.undef_sum, val);
    for (int f = 0; f < F.nf; f++) F.out.p[f][o] = val[f] / sum;
    F.out.p[F.nf][o] = F.undef_sum / sum;
    if (F.seis_lh) F.seis_lh[o] = sum;
  }
}

// threads per CTA: schedule key x4_facies_threads (n = h), default 128; rows per CTA T / N1
template <int N1, int N2>
static cudaError_t x4_facies(const FaciesFuse& F, const FaciesCorners& C, int rows, const float2* tw,
                             const float2* twn, cudaStream_t st) {
  using L = RowLayout<N1, N2>;
  constexpr int H = N1 * N2;
  const int T = std::max(32, std::min(256, tuned("x4_facies_threads", H, 128) / 32 * 32));
  const int rpc = std::max(1, T / N1);
  const size_t smem = sizeof(float2) * (2 * (size_t)H + (size_t)rpc * (L::PITCH + H + 1) + 3 * (size_t)rpc * H);
  cudaError_t e = cudaFuncSetAttribute(k_xc2r4_facies<N1, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_xc2r4_facies<N1, N2><<<(unsigned)((rows + rpc - 1) / rpc), T, smem, st>>>(F, C, rows, rpc, tw, twn);
  return cudaGetLastError();
}

}  // namespace crava
