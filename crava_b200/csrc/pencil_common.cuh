// Device helpers shared by the two pencil-pass kernels (zpass.cu, pencil.cu): the
// counter-based noise of product-mode realisations, the reference-semantics Cholesky
// factorisation of small Hermitian matrices and the eigen-form per-bin posterior of a
// separable prior (its derivation is in pencil.cuh).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_core.cuh"

namespace crava {

// ------------------------------------------------------------------ noise (product mode)

// Philox-4x32 (Salmon, Moraes, Dror, Shaw, SC'11) with 7 rounds, which the authors
// report passes TestU01 BigCrush.
__device__ __forceinline__ uint4 philox4x32_7(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 7; r++) {
    uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// Box-Muller with the hardware approximations of log, sine and cosine: their absolute
// errors (about 2^-21 on these ranges) are far below what the normals' statistics can show.
// u1 from a 26-bit integer a (radius: the largest |normal| is sqrt(2 ln 2^27) = 6.1), the angle
// from a 16-bit integer b (resolution 2 pi / 65536).
__device__ __forceinline__ void box_muller(uint32_t a, uint32_t b, float& n0, float& n1) {
  float u1 = ((float)a + 0.5f) * 1.4901161193847656e-08f;        // (a + 1/2) / 2^26, in (0, 1)
  float u2 = ((float)b + 0.5f) * 1.52587890625e-05f - 0.5f;      // (b + 1/2) / 2^16 - 1/2
  float rad = sqrtf(-2.0f * __logf(u1));
  float sn, cs;
  __sincosf(6.283185307179586f * u2, &sn, &cs);   // angle in (-pi, pi)
  n0 = rad * cs;
  n1 = rad * sn;
}

// Three standard complex normals (one per parameter) for bin (i,j,k) of realisation s,
// Hermitian-consistent on the planes whose x-bin is its own mirror (i = 0, and
// i = nxp/2 for even nxp): the pair (j,k) / (-j,-k) share one draw (conjugated),
// self-mirrored bins are real with unit variance, all others have variance 1/2 per
// component (the properties FFTGrid::fillInComplexNoise gives its noise,
// src/fftgrid.cpp:997-1055, with the mirror-plane test done on the x index).  One
// Philox block (128 bits) per bin and realisation feeds the three Box-Muller pairs: three
// 26-bit radius words (the top bits of words 0-2) and three 16-bit angle words (word 3's two
// halves, and the low 6 + 6 + 4 bits of words 0-2).
__device__ __forceinline__ void device_noise3(uint64_t seed, int s, int i, int j, int k, int nyp, int nzp,
                                              int cnxp, bool nxp_even, float2 (&z)[3]) {
  bool mirror_plane = (i == 0) || (nxp_even && i == cnxp - 1);
  int jj = j, kk = k;
  bool conj = false, self = false;
  if (mirror_plane) {
    int jc = j == 0 ? 0 : nyp - j;
    int kc = k == 0 ? 0 : nzp - k;
    long long a = (long long)j + (long long)nyp * k, b = (long long)jc + (long long)nyp * kc;
    if (a == b) self = true;
    else if (b < a) { jj = jc; kk = kc; conj = true; }
  }
  uint64_t bin = ((uint64_t)kk * nyp + jj) * cnxp + i;
  uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
  const uint4 r = philox4x32_7(make_uint4((uint32_t)bin, (uint32_t)(bin >> 32), (uint32_t)s, 0u), key);
  const uint32_t b2 = (r.x & 63u) | ((r.y & 63u) << 6) | ((r.z & 15u) << 12);
  float n[6];
  box_muller(r.x >> 6, r.w & 0xFFFFu, n[0], n[1]);
  box_muller(r.y >> 6, r.w >> 16, n[2], n[3]);
  box_muller(r.z >> 6, b2, n[4], n[5]);
  const float h = self ? 1.0f : 0.70710678118654752f;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    z[c] = make_float2(h * n[2 * c], self ? 0.f : h * n[2 * c + 1]);
    if (conj) z[c].y = -z[c].y;
  }
}

// ------------------------------------------------------------------ per-bin algebra

// lib_matrCholCpx (libs/lib/lib_matr.c:78-168) on the lower triangle of a Hermitian
// n x n matrix a[][]: the reference scales by a00, rejects a00 <= 0, a scaled diagonal
// <= 1e-20 before its update or an updated pivot <= 1e-20, factors and rescales by
// sqrt(a00).  Here the factor is computed unscaled with the two pivot tests applied as
// a_ii > 1e-20 a00 (the same comparisons up to rounding), and each pivot's reciprocal
// comes from one reciprocal square root.  No division.  The diagonal entry holds
// (L_ii, 1 / L_ii): its imaginary part, zero for a Hermitian factor, carries the reciprocal.
template <int N>
__device__ __forceinline__ bool chol_ref(float2 (&a)[N][N]) {
  const float f = a[0][0].x;
  if (!(f > 0.f)) return false;
  const float tol = 1e-20f * f;
#pragma unroll
  for (int i = 0; i < N; i++) {
    if (!(a[i][i].x > tol)) return false;
#pragma unroll
    for (int j = 0; j < i; j++) {
      float2 s = a[i][j];
#pragma unroll
      for (int k = 0; k < j; k++) {  // - L_ik conj(L_jk)
        s.x -= a[i][k].x * a[j][k].x + a[i][k].y * a[j][k].y;
        s.y -= -(a[i][k].x * a[j][k].y) + a[i][k].y * a[j][k].x;
      }
      a[i][j] = make_float2(s.x * a[j][j].y, s.y * a[j][j].y);
    }
    float r = a[i][i].x;
#pragma unroll
    for (int k = 0; k < i; k++) r -= a[i][k].x * a[i][k].x + a[i][k].y * a[i][k].y;
    if (!(r > tol)) return false;
    const float rs = rsqrtf(r);
    a[i][i] = make_float2(r * rs, rs);
  }
  return true;
}

// ------------------------------------------------------------------ eigen-form per-bin step

// Section of N floats (N % 4 == 0) of the row of position p: group g at e[g * stride].
template <int N>
__device__ __forceinline__ void ldrow(float (&out)[N], const float4* __restrict__ e, int stride) {
#pragma unroll
  for (int g = 0; g < N / 4; g++) {
    const float4 v = __ldg(e + g * stride);
    out[4 * g] = v.x;
    out[4 * g + 1] = v.y;
    out[4 * g + 2] = v.z;
    out[4 * g + 3] = v.w;
  }
}

constexpr int pad4(int x) { return (x + 3) / 4 * 4; }

// mu_post, S_post (order 00 11 22 01 02 12) and the residual (in d) of NB bins of one z
// position from that position's row e (float4 groups at stride nzp), laid out as EigLayout:
// the angles' rows are streamed one at a time and every row load serves all NB bins.
template <int NTH, int NB>
__device__ __forceinline__ void bin_posterior_eig(const ZParams& P, const float4* __restrict__ e,
                                                  const float (&lam)[NB], const float (&rho)[NB],
                                                  const float2 (&mu)[NB][3], float2 (&d)[NB][NTH],
                                                  float2 (&mu_post)[NB][3], float2 (&sp)[NB][6]) {
  constexpr int VP = pad4(2 * NTH), OKW = 0, OL = VP, OR = OL + pad4(NTH), RS = VP + 16;
  const int st = P.nzp;
  float kw[VP];
  ldrow(kw, e + (OKW / 4) * st, st);
  float Lm[pad4(NTH)];
  ldrow(Lm, e + (OL / 4) * st, st);
  // y = d - K mu, K = diag(kw) A
  float2 y[NB][NTH];
#pragma unroll
  for (int b = 0; b < NB; b++)
#pragma unroll
    for (int l = 0; l < NTH; l++) {
      float2 am = make_float2(0.f, 0.f);
#pragma unroll
      for (int a = 0; a < 3; a++)
        am = make_float2(am.x + P.A[l][a] * mu[b][a].x, am.y + P.A[l][a] * mu[b][a].y);
      y[b][l] = csub(d[b][l], cmul(make_float2(kw[2 * l], kw[2 * l + 1]), am));
    }
  float2 mp[NB][3];
  float s00[NB], s11[NB], s22[NB];
  float2 s01[NB], s02[NB], s12[NB];
#pragma unroll
  for (int b = 0; b < NB; b++) {
#pragma unroll
    for (int a = 0; a < 3; a++) mp[b][a] = mu[b][a];
    s00[b] = rho[b] * P.pv[0];
    s11[b] = rho[b] * P.pv[1];
    s22[b] = rho[b] * P.pv[2];
    s01[b] = make_float2(rho[b] * P.pv[3], 0.f);
    s02[b] = make_float2(rho[b] * P.pv[4], 0.f);
    s12[b] = make_float2(rho[b] * P.pv[5], 0.f);
  }
#pragma unroll
  for (int l = 0; l < NTH; l++) {
    // r_l = (V y)_l, s_l = r_l lam / (lam Lam_l + 1), w_l = lam^2 / (lam Lam_l + 1)
    float V[VP];
    ldrow(V, e + ((OR + l * RS) / 4) * st, st);
    float QH[16];
    ldrow(QH, e + ((OR + l * RS + VP) / 4) * st, st);
    const float* h = QH + 6;
#pragma unroll
    for (int b = 0; b < NB; b++) {
      float2 r = make_float2(0.f, 0.f);
#pragma unroll
      for (int m = 0; m < NTH; m++) r = cadd(r, cmul(make_float2(V[2 * m], V[2 * m + 1]), y[b][m]));
      const float inv = __frcp_rn(fmaf(lam[b], Lm[l], 1.0f));
      const float f = lam[b] * inv;
      const float2 sl = make_float2(r.x * f, r.y * f);
      const float wl = lam[b] * f;
      // mu_post += conj(Q_l.) s_l;  S_post -= w_l H_l, H_l = (|Q_l0|^2, |Q_l1|^2, |Q_l2|^2,
      // conj(Q_l0) Q_l1, conj(Q_l0) Q_l2, conj(Q_l1) Q_l2)
#pragma unroll
      for (int a = 0; a < 3; a++) {
        const float qr = QH[2 * a], qi = QH[2 * a + 1];
        mp[b][a].x += qr * sl.x + qi * sl.y;
        mp[b][a].y += qr * sl.y - qi * sl.x;
      }
      s00[b] -= wl * h[0];
      s11[b] -= wl * h[1];
      s22[b] -= wl * h[2];
      s01[b] = make_float2(s01[b].x - wl * h[3], s01[b].y - wl * h[4]);
      s02[b] = make_float2(s02[b].x - wl * h[5], s02[b].y - wl * h[6]);
      s12[b] = make_float2(s12[b].x - wl * h[7], s12[b].y - wl * h[8]);
    }
  }
#pragma unroll
  for (int b = 0; b < NB; b++) {
#pragma unroll
    for (int a = 0; a < 3; a++) mu_post[b][a] = mp[b][a];
    sp[b][0] = make_float2(s00[b], 0.f);
    sp[b][1] = make_float2(s11[b], 0.f);
    sp[b][2] = make_float2(s22[b], 0.f);
    sp[b][3] = s01[b];
    sp[b][4] = s02[b];
    sp[b][5] = s12[b];
    // residual d - K mu_post = y - K (mu_post - mu) (the data spectrum itself where the row
    // is zero: kz not inverted)
#pragma unroll
    for (int l = 0; l < NTH; l++) {
      float2 am = make_float2(0.f, 0.f);
#pragma unroll
      for (int a = 0; a < 3; a++)
        am = make_float2(am.x + P.A[l][a] * (mp[b][a].x - mu[b][a].x), am.y + P.A[l][a] * (mp[b][a].y - mu[b][a].y));
      d[b][l] = csub(y[b][l], cmul(make_float2(kw[2 * l], kw[2 * l + 1]), am));
    }
  }
}

}  // namespace crava
