// Facies density evaluation per voxel (FaciesProb::calculateFaciesProb / findDensity,
// src/faciesprob.cpp:1909-2075, 1307-1423), shared by the standalone facies pass (facies.cu)
// and the inverse x transform of the posterior mean that evaluates it on the fly (fft4.cuh).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

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
//
// facies_voxel: the densities of voxel (i, j) of trace row j at the parameters v, prior-
// weighted: val[f] = prior_f max(0, dens_f) and the returned sum = undef_sum + sum_f val[f]
// (the voxel's probabilities are val[f] / sum and undef_sum / sum).
__device__ __forceinline__ float facies_voxel(const float (&v)[3], int i, int j, int nx, int ny,
                                              const FaciesCorners& C, int nf, const FaciesPrior& pr,
                                              float undef_sum, float (&val)[kMaxFacies]) {
  const int nc = 1 << C.nang;
  const int nf4 = (nf + 3) / 4;
  float t[kMaxFaciesAngles];
  for (int a = 0; a < C.nang; a++) t[a] = __ldg(C.t + ((size_t)a * ny + j) * nx + i);
  float dsum[kMaxFacies];
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
        float vf = d[u];
        for (int a = 0; a < C.nang; a++) vf *= (c >> a) & 1 ? t[a] : (1.0f - t[a]);
        dsum[f] += vf;
      }
    }
  }
  float sum = undef_sum;
  for (int f = 0; f < nf; f++) {
    const float dn = dsum[f] > 0.f ? dsum[f] : 0.f;
    val[f] = pr.p[f] * dn;
    sum += val[f];
  }
  return sum;
}

// The host-side description of a facies evaluation as kernel parameters.
FaciesCorners facies_corners(const FaciesCornersHost& hc);

}  // namespace crava
