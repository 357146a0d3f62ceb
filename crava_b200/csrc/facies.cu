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
  const float4* dens[1 << kMaxFaciesAngles];   // packed volumes (k_facies_pack)
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

// findDensity with local noise (src/faciesprob.cpp:1307-1423): 2^nang density volumes, one per
// corner of the angles' noise-scale box, each with its own Simbox; a voxel's density is
// sum_c prod_a (t_a or 1 - t_a by bit a of c) * trilinear_c, t_a the trace's relative noise
// scale of angle a (calculateFaciesProb, :1961-1977).  nang = 0 is the single volume.
//
// The volumes are read packed (k_facies_pack): cell (j, k, l) of corner c holds its nf4 =
// ceil(nf / 4) float4 of the facies densities, already clamped at zero, so a voxel makes one
// vector load per cell corner and facies group and computes the cell indexes once per
// volume.  The float operations per facies are the reference's, in its order.
__global__ void k_facies_prob_corners(const float* __restrict__ vp, const float* __restrict__ vs,
                                      const float* __restrict__ rho, int nx, int ny, int nz, int rnxp_in, int nyp_in,
                                      int rnxp_out, const __grid_constant__ FaciesCorners C, int nf, FaciesPrior pr,
                                      float undef_sum, FaciesOut out, float* __restrict__ seis_lh) {
  const size_t n_out = (size_t)rnxp_out * ny * nz;
  const int nc = 1 << C.nang;
  const int nf4 = (nf + 3) / 4;
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
    float dsum[16];
    for (int f = 0; f < nf; f++) dsum[f] = 0.f;
    for (int c = 0; c < nc; c++) {
      const FaciesBox& box = C.box[c];
      int a1[3], a2[3];
      float w[3];
#pragma unroll
      for (int d = 0; d < 3; d++) axis_weights(v[d], box.vmin[d], box.dv[d], box.nb[d], a1[d], a2[d], w[d]);
      const size_t sk = (size_t)box.nb[0], sl = (size_t)box.nb[0] * box.nb[1];
      const float wj = w[0], wk = w[1], wl = w[2];
      // the eight cell corners in findDensity's order with their weights
      const size_t cell[8] = {a1[0] + sk * a1[1] + sl * a1[2], a1[0] + sk * a1[1] + sl * a2[2],
                              a1[0] + sk * a2[1] + sl * a1[2], a1[0] + sk * a2[1] + sl * a2[2],
                              a2[0] + sk * a1[1] + sl * a1[2], a2[0] + sk * a1[1] + sl * a2[2],
                              a2[0] + sk * a2[1] + sl * a1[2], a2[0] + sk * a2[1] + sl * a2[2]};
      const float w8[8] = {(1.0f - wj) * (1.0f - wk) * (1.0f - wl), (1.0f - wj) * (1.0f - wk) * wl,
                           (1.0f - wj) * wk * (1.0f - wl),          (1.0f - wj) * wk * wl,
                           wj * (1.0f - wk) * (1.0f - wl),          wj * (1.0f - wk) * wl,
                           wj * wk * (1.0f - wl),                   wj * wk * wl};
      const float4* P4 = C.dens[c];
      for (int g = 0; g < nf4; g++) {
        float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const float4 x = __ldg(P4 + cell[q] * nf4 + g);
          d[0] += w8[q] * x.x;
          d[1] += w8[q] * x.y;
          d[2] += w8[q] * x.z;
          d[3] += w8[q] * x.w;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int f = 4 * g + u;
          if (f >= nf) break;
          float val = d[u];
          for (int a = 0; a < C.nang; a++) val *= (c >> a) & 1 ? t[a] : (1.0f - t[a]);
          dsum[f] += val;
        }
      }
    }
    float sum = undef_sum;
    float val[16];
    for (int f = 0; f < nf; f++) {
      const float dn = dsum[f] > 0.f ? dsum[f] : 0.f;
      val[f] = pr.p[f] * dn;
      sum += val[f];
    }
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
  FaciesPrior pr;
  FaciesOut po;
  for (int f = 0; f < nf; f++) pr.p[f] = prior[f];
  for (int f = 0; f <= nf; f++) po.p[f] = out[f];
  FaciesCorners C;
  C.nang = hc.nang;
  C.t = hc.t;
  const int nf4 = (nf + 3) / 4;
  for (int c = 0; c < (1 << hc.nang); c++) {
    for (int d = 0; d < 3; d++) {
      C.box[c].nb[d] = hc.box[c].nb[d];
      C.box[c].vmin[d] = hc.box[c].vmin[d];
      C.box[c].dv[d] = hc.box[c].dv[d];
    }
    C.box[c].rs = hc.box[c].rs;
    C.box[c].fstride = hc.box[c].fstride;
    C.dens[c] = hc.packed[c];
    const size_t units = (size_t)hc.box[c].nb[0] * hc.box[c].nb[1] * hc.box[c].nb[2] * nf4;
    const int pb = (int)std::min<size_t>((units + 255) / 256, 148 * 8);
    k_facies_pack<<<pb, 256, 0, st>>>(hc.dens[c], hc.box[c].nb[0], hc.box[c].nb[1], hc.box[c].nb[2], hc.box[c].rs,
                                      hc.box[c].fstride, nf, hc.packed[c]);
  }
  size_t n = (size_t)rnxp_out * ny * nz;
  int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_facies_prob_corners<<<blocks, 256, 0, st>>>(vp, vs, rho, nx, ny, nz, rnxp_in, nyp_in, rnxp_out, C, nf, pr,
                                                undef_sum, po, seis_lh);
  return cudaGetLastError();
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
