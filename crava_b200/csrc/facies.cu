// Facies probabilities from the posterior elastic parameters (sm_100a).
//
//   k_facies_prob_corners  per voxel: trilinear lookup of every facies density volume at the
//                   posterior (ln Vp, ln Vs, ln rho), prior-weighted, normalised with the
//                   undefined-facies floor (FaciesProb::calculateFaciesProb and findDensity,
//                   src/faciesprob.cpp:1909-2075, 1307-1423), with local noise over 2^nang
//                   corner volumes weighted by the trace's relative noise scales
//   k_facies_pack   the density volumes repacked facies-interleaved for those lookups
//   k_spec_mul      spectrum product for the Gaussian smoothing of the facies histograms
//                   (FaciesProb::makeFaciesDens, src/faciesprob.cpp:440-522)
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "facies.cuh"

namespace crava {

__global__ void k_facies_prob_corners(const float* __restrict__ vp, const float* __restrict__ vs,
                                      const float* __restrict__ rho, int nx, int ny, int nz, int rnxp_in, int nyp_in,
                                      int rnxp_out, const __grid_constant__ FaciesCorners C, int nf, FaciesPrior pr,
                                      float undef_sum, FaciesOut out, float* __restrict__ seis_lh) {
  const size_t n_out = (size_t)rnxp_out * ny * nz;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n_out; e += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(e % rnxp_out);
    size_t r = e / rnxp_out;
    int j = (int)(r % ny);
    int k = (int)(r / ny);
    if (i >= nx) {
      for (int f = 0; f <= nf; f++) out.p[f][e] = kRMissing;
      if (seis_lh) seis_lh[e] = kRMissing;
      continue;
    }
    size_t gi = (size_t)i + (size_t)rnxp_in * ((size_t)j + (size_t)nyp_in * k);
    const float v[3] = {vp[gi], vs[gi], rho[gi]};
    float val[kMaxFacies];
    const float sum = facies_voxel(v, i, j, nx, ny, C, nf, pr, undef_sum, val);
    for (int f = 0; f < nf; f++) out.p[f][e] = val[f] / sum;
    out.p[nf][e] = undef_sum / sum;
    if (seis_lh) seis_lh[e] = sum;
  }
}

// Packs one density volume: cell (j, k, l) <- the nf facies values max(0, dens_f(j, k, l)),
// four per float4 (zero beyond nf); dens_f at src + f * fstride + j + rs (k + nb1 l).
__global__ void k_facies_pack(const float* __restrict__ src, int nb0, int nb1, int nb2, int rs, size_t fstride,
                              int nf, float4* __restrict__ dst) {
  const int nf4 = (nf + 3) / 4;
  const size_t ncell = (size_t)nb0 * nb1 * nb2;
  for (size_t cidx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; cidx < ncell * nf4;
       cidx += (size_t)gridDim.x * blockDim.x) {
    const size_t cell = cidx / nf4;
    const int g = (int)(cidx % nf4);
    const int j = (int)(cell % nb0);
    const size_t kl = cell / nb0;
    const int kk = (int)(kl % nb1), l = (int)(kl / nb1);
    const size_t o = (size_t)j + (size_t)rs * ((size_t)kk + (size_t)nb1 * l);
    float x[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int f = 4 * g + u;
      x[u] = f < nf ? fmaxf(0.f, __ldg(src + fstride * f + o)) : 0.f;
    }
    dst[cidx] = make_float4(x[0], x[1], x[2], x[3]);
  }
}

// a <- a * b (complex) over n bins
__global__ void k_spec_mul(float2* __restrict__ a, const float2* __restrict__ b, size_t n) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    float2 x = a[e], y = b[e];
    a[e] = make_float2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
  }
}

cudaError_t launch_facies_prob_corners(const float* vp, const float* vs, const float* rho, int nx, int ny, int nz,
                                       int rnxp_in, int nyp_in, int rnxp_out, const FaciesCornersHost& hc, int nf,
                                       const float* prior, float undef_sum, float* const* out, float* seis_lh,
                                       cudaStream_t st) {
  if (nf < 1 || nf > kMaxFacies || hc.nang < 0 || hc.nang > kMaxFaciesAngles) return cudaErrorInvalidValue;
  cudaError_t e = launch_facies_pack(hc, nf, st);
  if (e != cudaSuccess) return e;
  return launch_facies_eval(vp, vs, rho, nx, ny, nz, rnxp_in, nyp_in, rnxp_out, hc, nf, prior, undef_sum, out, seis_lh,
                            st);
}

cudaError_t launch_facies_eval(const float* vp, const float* vs, const float* rho, int nx, int ny, int nz, int rnxp_in,
                               int nyp_in, int rnxp_out, const FaciesCornersHost& hc, int nf, const float* prior,
                               float undef_sum, float* const* out, float* seis_lh, cudaStream_t st) {
  if (nf < 1 || nf > kMaxFacies || hc.nang < 0 || hc.nang > kMaxFaciesAngles) return cudaErrorInvalidValue;
  FaciesPrior pr;
  FaciesOut po;
  for (int f = 0; f < nf; f++) pr.p[f] = prior[f];
  for (int f = 0; f <= nf; f++) po.p[f] = out[f];
  const FaciesCorners C = facies_corners(hc);
  size_t n = (size_t)rnxp_out * ny * nz;
  int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_facies_prob_corners<<<blocks, 256, 0, st>>>(vp, vs, rho, nx, ny, nz, rnxp_in, nyp_in, rnxp_out, C, nf, pr,
                                                undef_sum, po, seis_lh);
  return cudaGetLastError();
}

cudaError_t launch_facies_pack(const FaciesCornersHost& hc, int nf, cudaStream_t st) {
  if (nf < 1 || nf > kMaxFacies || hc.nang < 0 || hc.nang > kMaxFaciesAngles) return cudaErrorInvalidValue;
  const int nf4 = (nf + 3) / 4;
  for (int c = 0; c < (1 << hc.nang); c++) {
    const size_t units = (size_t)hc.box[c].nb[0] * hc.box[c].nb[1] * hc.box[c].nb[2] * nf4;
    const int pb = (int)std::min<size_t>((units + 255) / 256, 148 * 8);
    k_facies_pack<<<pb, 256, 0, st>>>(hc.dens[c], hc.box[c].nb[0], hc.box[c].nb[1], hc.box[c].nb[2], hc.box[c].rs,
                                      hc.box[c].fstride, nf, hc.packed[c]);
  }
  return cudaGetLastError();
}

FaciesCorners facies_corners(const FaciesCornersHost& hc) {
  FaciesCorners C;
  C.nang = hc.nang;
  C.t = hc.t;
  for (int c = 0; c < (1 << hc.nang); c++) {
    for (int d = 0; d < 3; d++) {
      C.box[c].nb[d] = hc.box[c].nb[d];
      C.box[c].vmin[d] = hc.box[c].vmin[d];
      C.box[c].dv[d] = hc.box[c].dv[d];
    }
    C.box[c].rs = hc.box[c].rs;
    C.box[c].fstride = hc.box[c].fstride;
    C.dens[c] = hc.packed[c];
  }
  return C;
}

size_t facies_packed_bytes(const FaciesBoxHost& b, int nf) {
  return sizeof(float4) * (size_t)b.nb[0] * b.nb[1] * b.nb[2] * ((nf + 3) / 4);
}

cudaError_t launch_spec_mul(float2* a, const float2* b, size_t n, cudaStream_t st) {
  int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_spec_mul<<<blocks, 256, 0, st>>>(a, b, n);
  return cudaGetLastError();
}

}  // namespace crava
