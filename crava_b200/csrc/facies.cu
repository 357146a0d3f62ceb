// Facies probabilities from the posterior elastic parameters (sm_100a).
//
//   k_facies_prob   per voxel: trilinear lookup of every facies density cube at the
//                   posterior (ln Vp, ln Vs, ln rho), prior-weighted, normalised with the
//                   undefined-facies floor (FaciesProb::calculateFaciesProb and findDensity,
//                   src/faciesprob.cpp:1909-2075, 1307-1423; the single-volume case)
//   k_facies_prob_corners  the same with local noise: 2^nang corner volumes weighted by the
//                   trace's relative noise scales
//   k_spec_mul      spectrum product for the Gaussian smoothing of the facies histograms
//                   (FaciesProb::makeFaciesDens, src/faciesprob.cpp:440-522)
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "kernels.cuh"

namespace crava {

constexpr float kRMissing = -99999.0f;

// Box of one density volume: bins (nb), lower edges (vmin) and inverse widths (idv) along
// vp, vs, rho; density cube f at dens + f*fstride, element (j, k, l) at
// j + rs*k + rs*nb[1]*l (rs = row stride, FFTGrid-padded or dense).
struct FaciesBox {
  int nb[3];
  double vmin[3];
  double dv[3];
  int rs;
  size_t fstride;
};

struct FaciesCorners {
  int nang;                          // angles with a noise scale: 2^nang corner volumes
  const float* t;                    // nang x ny x nx relative noise scales in [0, 1]
  FaciesBox box[1 << kMaxFaciesAngles];
  const float* dens[1 << kMaxFaciesAngles];
};

// Index along one axis as Simbox::getInterpolationIndexes (value at bin centres, in
// double as the reference) and the clamping of findDensity: below the first centre or
// beyond the last the value of the edge bin is used.
__device__ __forceinline__ void axis_weights(float v, double vmin, double dv, int nb, int& i1, int& i2, float& w) {
  double f = ((double)v - vmin) / dv - 0.5;
  int i = (int)floor(f);
  if (i < 0) { i1 = i2 = 0; w = 0.f; }
  else if (i >= nb - 1) { i1 = i2 = nb - 1; w = 0.f; }
  else { i1 = i; i2 = i + 1; w = (float)(f - (double)i); }
}

__global__ void k_facies_prob(const float* __restrict__ vp, const float* __restrict__ vs, const float* __restrict__ rho,
                              int nx, int ny, int nz, int rnxp_in, int nyp_in, int rnxp_out,
                              const float* __restrict__ dens, FaciesBox box, int nf,
                              FaciesPrior pr, float undef_sum, FaciesOut out, float* __restrict__ seis_lh) {
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
    float v[3] = {vp[gi], vs[gi], rho[gi]};
    int a1[3], a2[3];
    float w[3];
#pragma unroll
    for (int d = 0; d < 3; d++) axis_weights(v[d], box.vmin[d], box.dv[d], box.nb[d], a1[d], a2[d], w[d]);
    const size_t sk = (size_t)box.rs, sl = (size_t)box.rs * box.nb[1];
    const size_t o111 = a1[0] + sk * a1[1] + sl * a1[2], o112 = a1[0] + sk * a1[1] + sl * a2[2];
    const size_t o121 = a1[0] + sk * a2[1] + sl * a1[2], o122 = a1[0] + sk * a2[1] + sl * a2[2];
    const size_t o211 = a2[0] + sk * a1[1] + sl * a1[2], o212 = a2[0] + sk * a1[1] + sl * a2[2];
    const size_t o221 = a2[0] + sk * a2[1] + sl * a1[2], o222 = a2[0] + sk * a2[1] + sl * a2[2];
    const float wj = w[0], wk = w[1], wl = w[2];
    float sum = undef_sum;
    float val[16];
    for (int f = 0; f < nf; f++) {
      const float* D = dens + box.fstride * f;
      float d = 0.f;
      d += (1.0f - wj) * (1.0f - wk) * (1.0f - wl) * fmaxf(0.f, __ldg(D + o111));
      d += (1.0f - wj) * (1.0f - wk) * wl * fmaxf(0.f, __ldg(D + o112));
      d += (1.0f - wj) * wk * (1.0f - wl) * fmaxf(0.f, __ldg(D + o121));
      d += (1.0f - wj) * wk * wl * fmaxf(0.f, __ldg(D + o122));
      d += wj * (1.0f - wk) * (1.0f - wl) * fmaxf(0.f, __ldg(D + o211));
      d += wj * (1.0f - wk) * wl * fmaxf(0.f, __ldg(D + o212));
      d += wj * wk * (1.0f - wl) * fmaxf(0.f, __ldg(D + o221));
      d += wj * wk * wl * fmaxf(0.f, __ldg(D + o222));
      if (!(d > 0.f)) d = 0.f;
      float x = pr.p[f] * d;
      if (f < 16) val[f] = x;
      sum += x;
    }
    for (int f = 0; f < nf && f < 16; f++) out.p[f][e] = val[f] / sum;
    out.p[nf][e] = undef_sum / sum;
    if (seis_lh) seis_lh[e] = sum;
  }
}

// findDensity with local noise (src/faciesprob.cpp:1307-1423): 2^nang density volumes, one per
// corner of the angles' noise-scale box, each with its own Simbox; a voxel's density is
// sum_c prod_a (t_a or 1 - t_a by bit a of c) * trilinear_c, t_a the trace's relative noise
// scale of angle a (calculateFaciesProb, :1961-1977).  Corner c's cubes at dens[c] + f*fstride.
__global__ void k_facies_prob_corners(const float* __restrict__ vp, const float* __restrict__ vs,
                                      const float* __restrict__ rho, int nx, int ny, int nz, int rnxp_in, int nyp_in,
                                      int rnxp_out, const __grid_constant__ FaciesCorners C, int nf, FaciesPrior pr,
                                      float undef_sum, FaciesOut out, float* __restrict__ seis_lh) {
  const size_t n_out = (size_t)rnxp_out * ny * nz;
  const int nc = 1 << C.nang;
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
    float t[kMaxFaciesAngles];
    for (int a = 0; a < C.nang; a++) t[a] = __ldg(C.t + ((size_t)a * ny + j) * nx + i);
    float sum = undef_sum;
    float val[16];
    for (int f = 0; f < nf; f++) {
      float dsum = 0.f;
      for (int c = 0; c < nc; c++) {
        const FaciesBox& box = C.box[c];
        int a1[3], a2[3];
        float w[3];
#pragma unroll
        for (int d = 0; d < 3; d++) axis_weights(v[d], box.vmin[d], box.dv[d], box.nb[d], a1[d], a2[d], w[d]);
        const size_t sk = (size_t)box.rs, sl = (size_t)box.rs * box.nb[1];
        const float* D = C.dens[c] + box.fstride * f;
        const float wj = w[0], wk = w[1], wl = w[2];
        float d = 0.f;
        d += (1.0f - wj) * (1.0f - wk) * (1.0f - wl) * fmaxf(0.f, __ldg(D + a1[0] + sk * a1[1] + sl * a1[2]));
        d += (1.0f - wj) * (1.0f - wk) * wl * fmaxf(0.f, __ldg(D + a1[0] + sk * a1[1] + sl * a2[2]));
        d += (1.0f - wj) * wk * (1.0f - wl) * fmaxf(0.f, __ldg(D + a1[0] + sk * a2[1] + sl * a1[2]));
        d += (1.0f - wj) * wk * wl * fmaxf(0.f, __ldg(D + a1[0] + sk * a2[1] + sl * a2[2]));
        d += wj * (1.0f - wk) * (1.0f - wl) * fmaxf(0.f, __ldg(D + a2[0] + sk * a1[1] + sl * a1[2]));
        d += wj * (1.0f - wk) * wl * fmaxf(0.f, __ldg(D + a2[0] + sk * a1[1] + sl * a2[2]));
        d += wj * wk * (1.0f - wl) * fmaxf(0.f, __ldg(D + a2[0] + sk * a2[1] + sl * a1[2]));
        d += wj * wk * wl * fmaxf(0.f, __ldg(D + a2[0] + sk * a2[1] + sl * a2[2]));
        for (int a = 0; a < C.nang; a++) d *= (c >> a) & 1 ? t[a] : (1.0f - t[a]);
        dsum += d;
      }
      if (!(dsum > 0.f)) dsum = 0.f;
      const float x = pr.p[f] * dsum;
      if (f < 16) val[f] = x;
      sum += x;
    }
    for (int f = 0; f < nf && f < 16; f++) out.p[f][e] = val[f] / sum;
    out.p[nf][e] = undef_sum / sum;
    if (seis_lh) seis_lh[e] = sum;
  }
}

// a <- a * b (complex) over n bins
__global__ void k_spec_mul(float2* __restrict__ a, const float2* __restrict__ b, size_t n) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    float2 x = a[e], y = b[e];
    a[e] = make_float2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
  }
}

cudaError_t launch_facies_prob(const float* vp, const float* vs, const float* rho, int nx, int ny, int nz,
                               int rnxp_in, int nyp_in, int rnxp_out, const float* dens, const FaciesBoxHost& hb,
                               int nf, const float* prior, float undef_sum, float* const* out, float* seis_lh,
                               cudaStream_t st) {
  if (nf < 1 || nf > kMaxFacies) return cudaErrorInvalidValue;
  FaciesPrior pr;
  FaciesOut po;
  for (int f = 0; f < nf; f++) pr.p[f] = prior[f];
  for (int f = 0; f <= nf; f++) po.p[f] = out[f];
  FaciesBox box;
  for (int d = 0; d < 3; d++) {
    box.nb[d] = hb.nb[d];
    box.vmin[d] = hb.vmin[d];
    box.dv[d] = hb.dv[d];
  }
  box.rs = hb.rs;
  box.fstride = hb.fstride;
  size_t n = (size_t)rnxp_out * ny * nz;
  int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_facies_prob<<<blocks, 256, 0, st>>>(vp, vs, rho, nx, ny, nz, rnxp_in, nyp_in, rnxp_out, dens, box, nf, pr,
                                        undef_sum, po, seis_lh);
  return cudaGetLastError();
}

cudaError_t launch_facies_prob_corners(const float* vp, const float* vs, const float* rho, int nx, int ny, int nz,
                                       int rnxp_in, int nyp_in, int rnxp_out, const FaciesCornersHost& hc, int nf,
                                       const float* prior, float undef_sum, float* const* out, float* seis_lh,
                                       cudaStream_t st) {
  if (nf < 1 || nf > kMaxFacies || hc.nang < 0 || hc.nang > kMaxFaciesAngles) return cudaErrorInvalidValue;
  FaciesPrior pr;
  FaciesOut po;
  for (int f = 0; f < nf; f++) pr.p[f] = prior[f];
  for (int f = 0; f <= nf; f++) po.p[f] = out[f];
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
    C.dens[c] = hc.dens[c];
  }
  size_t n = (size_t)rnxp_out * ny * nz;
  int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_facies_prob_corners<<<blocks, 256, 0, st>>>(vp, vs, rho, nx, ny, nz, rnxp_in, nyp_in, rnxp_out, C, nf, pr,
                                                undef_sum, po, seis_lh);
  return cudaGetLastError();
}

cudaError_t launch_spec_mul(float2* a, const float2* b, size_t n, cudaStream_t st) {
  int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_spec_mul<<<blocks, 256, 0, st>>>(a, b, n);
  return cudaGetLastError();
}

}  // namespace crava
