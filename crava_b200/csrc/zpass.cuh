// The fused pencil pass of the AVO inversion (sm_100a): per (x-tile, y) pencil, forward z
// transform of every input spectrum, the per-bin posterior of
// AVOInversion::computePostMeanResidAndFFTCov (src/avoinversion.cpp:944-1091), the per-bin
// simulation of AVOInversion::simulate (src/avoinversion.cpp:1421-1460) and the inverse z
// transform of every output spectrum.  Spectra never leave the CTA between the forward and
// the inverse z transform.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "fft2.cuh"
#include "fft_core.cuh"
#include "kernels.cuh"
#include "pencil_common.cuh"

namespace crava {


struct BinOut {
  float2 mu[3];
  float2 sp[6];
  float cond;   // (max / min Cholesky pivot)^2 of Sd, an estimate of its condition number
};

// Posterior of one bin.  Follows src/avoinversion.cpp:1036-1061 with
//   Sd = K S K^H + Se, K = diag(kw) A, S real symmetric (so K S K^H = (kw kw^H) o (A S A^T)),
//   L L^H = Sd (reference Cholesky), Y = L^{-1} K S,
//   S_post = S - Y^H Y, mu_post = mu + Y^H L^{-1} (d - K mu), res = d - K mu_post,
// which is the reference's  KS <- Sd^{-1} KS; S - KS_old^H KS;  mu + KS^H (d - K mu)
// regrouped through the Cholesky factor.
// SEP: separable prior.  Then S = rho P0, so K S K^H = rho (kw kw^H) o G0 and K S = rho
// diag(kw) AP with G0 = A P0 A^T and AP = A P0 job constants, and the error part of Sd is
// lam M2 with M2 = ec o (e1 e1^H + e2 e2^H) read per kz from the job's table (lower
// triangle, row by row), in place of the per-bin products.
template <int NTH, bool SEP>
__device__ __forceinline__ bool bin_posterior(const ZParams& P, int k, const float (&S)[6], float lam, float rho,
                                              const float2 (&mu)[3], float2 (&d)[NTH], BinOut& o) {
  constexpr int TRI = NTH * (NTH + 1) / 2;
  float2 kw[NTH];
#pragma unroll
  for (int l = 0; l < NTH; l++) kw[l] = __ldg(P.kz.kw + k * NTH + l);
  float2 Sd[NTH][NTH];
  float2 Y[NTH][3];  // K S, then L^{-1} K S
  if constexpr (SEP) {
    const float2* m2 = P.septab + (size_t)k * TRI;
#pragma unroll
    for (int l = 0; l < NTH; l++) {
#pragma unroll
      for (int m = 0; m <= l; m++) {
        const float2 b = __ldg(m2 + l * (l + 1) / 2 + m);
        const float g = rho * P.G0[l][m];
        // rho G0_lm kw_l conj(kw_m) + lam M2_lm
        Sd[l][m] = make_float2(g * (kw[l].x * kw[m].x + kw[l].y * kw[m].y) + lam * b.x,
                               g * (kw[l].y * kw[m].x - kw[l].x * kw[m].y) + lam * b.y);
      }
      Sd[l][l] = make_float2(Sd[l][l].x + __ldg(P.kz.ed + k * NTH + l), 0.f);
#pragma unroll
      for (int j = 0; j < 3; j++) {
        const float a = rho * P.AP[l][j];
        Y[l][j] = make_float2(kw[l].x * a, kw[l].y * a);
      }
    }
  } else {
    float2 e1[NTH], e2[NTH];
#pragma unroll
    for (int l = 0; l < NTH; l++) {
      e1[l] = __ldg(P.kz.e1 + k * NTH + l);
      e2[l] = __ldg(P.kz.e2 + k * NTH + l);
    }
    // AS = A S (NTH x 3), G = A S A^T
    float AS[NTH][3];
#pragma unroll
    for (int l = 0; l < NTH; l++) {
      AS[l][0] = P.A[l][0] * S[0] + P.A[l][1] * S[3] + P.A[l][2] * S[4];
      AS[l][1] = P.A[l][0] * S[3] + P.A[l][1] * S[1] + P.A[l][2] * S[5];
      AS[l][2] = P.A[l][0] * S[4] + P.A[l][1] * S[5] + P.A[l][2] * S[2];
    }
#pragma unroll
    for (int l = 0; l < NTH; l++) {
#pragma unroll
      for (int m = 0; m <= l; m++) {
        float g = AS[l][0] * P.A[m][0] + AS[l][1] * P.A[m][1] + AS[l][2] * P.A[m][2];
        // kw_l conj(kw_m)
        float2 kk = make_float2(kw[l].x * kw[m].x + kw[l].y * kw[m].y, kw[l].y * kw[m].x - kw[l].x * kw[m].y);
        float c = P.ec[l][m] * lam;
        float2 ee = make_float2(e1[l].x * e1[m].x + e1[l].y * e1[m].y + e2[l].x * e2[m].x + e2[l].y * e2[m].y,
                                e1[l].y * e1[m].x - e1[l].x * e1[m].y + e2[l].y * e2[m].x - e2[l].x * e2[m].y);
        Sd[l][m] = make_float2(kk.x * g + c * ee.x, kk.y * g + c * ee.y);
        if (l == m)
          Sd[l][m] = make_float2(Sd[l][m].x + __ldg(P.kz.ed + k * NTH + l), 0.f);
      }
#pragma unroll
      for (int j = 0; j < 3; j++) Y[l][j] = make_float2(kw[l].x * AS[l][j], kw[l].y * AS[l][j]);
    }
  }
  if (!chol_ref<NTH>(Sd)) return false;
  {
    float dmax = Sd[0][0].x, rmax = Sd[0][0].y;
#pragma unroll
    for (int l = 1; l < NTH; l++) {
      dmax = fmaxf(dmax, Sd[l][l].x);
      rmax = fmaxf(rmax, Sd[l][l].y);
    }
    o.cond = (dmax * rmax) * (dmax * rmax);
  }
  // Y = L^{-1} KS (forward substitution in place)
#pragma unroll
  for (int l = 0; l < NTH; l++) {
#pragma unroll
    for (int j = 0; j < 3; j++) {
      float2 acc = Y[l][j];
#pragma unroll
      for (int m = 0; m < l; m++) acc = csub(acc, cmul(Sd[l][m], Y[m][j]));
      Y[l][j] = make_float2(acc.x * Sd[l][l].y, acc.y * Sd[l][l].y);
    }
  }
  // S_post = S - Y^H Y
  const int qa[6] = {0, 1, 2, 0, 0, 1}, qb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int q = 0; q < 6; q++) {
    float2 r = make_float2(0.f, 0.f);
#pragma unroll
    for (int l = 0; l < NTH; l++) {  // conj(Y[l][a]) Y[l][b]
      r.x += Y[l][qa[q]].x * Y[l][qb[q]].x + Y[l][qa[q]].y * Y[l][qb[q]].y;
      r.y += Y[l][qa[q]].x * Y[l][qb[q]].y - Y[l][qa[q]].y * Y[l][qb[q]].x;
    }
    o.sp[q] = make_float2(S[q] - r.x, -r.y);
  }
  // yd = L^{-1} (d - K mu)
  float2 yd[NTH];
#pragma unroll
  for (int l = 0; l < NTH; l++) {
    float2 am = make_float2(0.f, 0.f);
#pragma unroll
    for (int j = 0; j < 3; j++) am = make_float2(am.x + P.A[l][j] * mu[j].x, am.y + P.A[l][j] * mu[j].y);
    float2 acc = csub(d[l], cmul(kw[l], am));
#pragma unroll
    for (int m = 0; m < l; m++) acc = csub(acc, cmul(Sd[l][m], yd[m]));
    yd[l] = make_float2(acc.x * Sd[l][l].y, acc.y * Sd[l][l].y);
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    float2 r = mu[a];
#pragma unroll
    for (int l = 0; l < NTH; l++) {  // conj(Y[l][a]) yd[l]
      r.x += Y[l][a].x * yd[l].x + Y[l][a].y * yd[l].y;
      r.y += Y[l][a].x * yd[l].y - Y[l][a].y * yd[l].x;
    }
    o.mu[a] = r;
  }
  // residual d - K mu_post, returned in d
#pragma unroll
  for (int l = 0; l < NTH; l++) {
    float2 am = make_float2(0.f, 0.f);
#pragma unroll
    for (int j = 0; j < 3; j++) am = make_float2(am.x + P.A[l][j] * o.mu[j].x, am.y + P.A[l][j] * o.mu[j].y);
    d[l] = csub(d[l], cmul(kw[l], am));
  }
  return true;
}

// ------------------------------------------------------------------ FP64 re-factorisation

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// lib_matrCholCpx semantics (libs/lib/lib_matr.c:78-168) in double.
template <int N>
__device__ __forceinline__ bool chol_ref_d(double2 (&a)[N][N]) {
  const double TOLD = 1e-20;
  double f = a[0][0].x;
  if (!(f > 0.0)) return false;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j <= i; j++) a[i][j] = make_double2(a[i][j].x / f, a[i][j].y / f);
#pragma unroll
  for (int i = 0; i < N; i++) {
    if (!(a[i][i].x > TOLD)) return false;
#pragma unroll
    for (int j = 0; j < i; j++) {
      double2 s = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < j; k++) {
        s.x += a[i][k].x * a[j][k].x + a[i][k].y * a[j][k].y;
        s.y += -(a[i][k].x * a[j][k].y) + a[i][k].y * a[j][k].x;
      }
      double dd = a[j][j].x;
      a[i][j] = make_double2((a[i][j].x - s.x) / dd, (a[i][j].y - s.y) / dd);
    }
    double r = 0.0;
#pragma unroll
    for (int k = 0; k < i; k++) r += a[i][k].x * a[i][k].x + a[i][k].y * a[i][k].y;
    r = a[i][i].x - r;
    if (!(r > TOLD)) return false;
    a[i][i] = make_double2(sqrt(r), 0.0);
  }
  double sf = sqrt(f);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j <= i; j++) a[i][j] = make_double2(a[i][j].x * sf, a[i][j].y * sf);
  return true;
}

// The per-bin posterior of bin_posterior re-done in double for a bin the FP32 pass flagged
// as ill-conditioned, with one step of iterative refinement of the data solve
// x = Sd^{-1} (d - K mu): x0 from the factor, r = (d - K mu) - Sd x0, x = x0 + Sd^{-1} r.
// Out of line: only flagged bins call it, and only the REFINE instantiation of the pencil
// kernel carries the call.
template <int NTH>
__device__ __noinline__ bool bin_posterior_fp64(const ZParams& P, int k, const float (&Sf)[6], float lamf,
                                                const float2 (&mu)[3], float2 (&d)[NTH], BinOut& o) {
  double2 kw[NTH], e1[NTH], e2[NTH];
#pragma unroll
  for (int l = 0; l < NTH; l++) {
    kw[l] = P.kz.kwd[k * NTH + l];
    e1[l] = P.kz.e1d[k * NTH + l];
    e2[l] = P.kz.e2d[k * NTH + l];
  }
  double S[6];
#pragma unroll
  for (int q = 0; q < 6; q++) S[q] = Sf[q];
  const double lam = lamf;
  double AS[NTH][3];
#pragma unroll
  for (int l = 0; l < NTH; l++) {
    AS[l][0] = P.Ad[l][0] * S[0] + P.Ad[l][1] * S[3] + P.Ad[l][2] * S[4];
    AS[l][1] = P.Ad[l][0] * S[3] + P.Ad[l][1] * S[1] + P.Ad[l][2] * S[5];
    AS[l][2] = P.Ad[l][0] * S[4] + P.Ad[l][1] * S[5] + P.Ad[l][2] * S[2];
  }
  double2 Sd[NTH][NTH], Sfull[NTH][NTH];
#pragma unroll
  for (int l = 0; l < NTH; l++) {
#pragma unroll
    for (int m = 0; m <= l; m++) {
      double g = AS[l][0] * P.Ad[m][0] + AS[l][1] * P.Ad[m][1] + AS[l][2] * P.Ad[m][2];
      double2 kk = make_double2(kw[l].x * kw[m].x + kw[l].y * kw[m].y, kw[l].y * kw[m].x - kw[l].x * kw[m].y);
      double c = P.ecd[l][m] * lam;
      double2 ee = make_double2(e1[l].x * e1[m].x + e1[l].y * e1[m].y + e2[l].x * e2[m].x + e2[l].y * e2[m].y,
                                e1[l].y * e1[m].x - e1[l].x * e1[m].y + e2[l].y * e2[m].x - e2[l].x * e2[m].y);
      Sd[l][m] = make_double2(kk.x * g + c * ee.x, kk.y * g + c * ee.y);
      if (l == m) Sd[l][m] = make_double2(Sd[l][m].x + (P.kz.edd ? P.kz.edd[k * NTH + l] : P.edd[l]), 0.0);
      Sfull[l][m] = Sd[l][m];
      Sfull[m][l] = make_double2(Sd[l][m].x, -Sd[l][m].y);
    }
  }
  if (!chol_ref_d<NTH>(Sd)) return false;
  // Y = L^{-1} K S, S_post = S - Y^H Y
  double2 Y[NTH][3];
#pragma unroll
  for (int l = 0; l < NTH; l++) {
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double2 acc = make_double2(kw[l].x * AS[l][j], kw[l].y * AS[l][j]);
#pragma unroll
      for (int m = 0; m < l; m++) acc = zsub(acc, zmul(Sd[l][m], Y[m][j]));
      Y[l][j] = make_double2(acc.x / Sd[l][l].x, acc.y / Sd[l][l].x);
    }
  }
  const int qa[6] = {0, 1, 2, 0, 0, 1}, qb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int q = 0; q < 6; q++) {
    double2 r = make_double2(0.0, 0.0);
#pragma unroll
    for (int l = 0; l < NTH; l++) {
      r.x += Y[l][qa[q]].x * Y[l][qb[q]].x + Y[l][qa[q]].y * Y[l][qb[q]].y;
      r.y += Y[l][qa[q]].x * Y[l][qb[q]].y - Y[l][qa[q]].y * Y[l][qb[q]].x;
    }
    o.sp[q] = make_float2((float)(S[q] - r.x), (float)(-r.y));
  }
  // b = d - K mu; x = Sd^{-1} b with one refinement step
  double2 b[NTH], x[NTH], t[NTH];
#pragma unroll
  for (int l = 0; l < NTH; l++) {
    double2 am = make_double2(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < 3; j++) am = make_double2(am.x + P.Ad[l][j] * mu[j].x, am.y + P.Ad[l][j] * mu[j].y);
    b[l] = zsub(make_double2(d[l].x, d[l].y), zmul(kw[l], am));
  }
  auto solve = [&](const double2 (&rhs)[NTH], double2 (&out)[NTH]) {
#pragma unroll
    for (int l = 0; l < NTH; l++) {
      double2 acc = rhs[l];
#pragma unroll
      for (int m = 0; m < l; m++) acc = zsub(acc, zmul(Sd[l][m], t[m]));
      t[l] = make_double2(acc.x / Sd[l][l].x, acc.y / Sd[l][l].x);
    }
#pragma unroll
    for (int l = NTH - 1; l >= 0; l--) {
      double2 acc = t[l];
#pragma unroll
      for (int m = l + 1; m < NTH; m++) acc = zsub(acc, zmul(make_double2(Sd[m][l].x, -Sd[m][l].y), out[m]));
      out[l] = make_double2(acc.x / Sd[l][l].x, acc.y / Sd[l][l].x);
    }
  };
  solve(b, x);
  double2 r[NTH], dx[NTH];
#pragma unroll
  for (int l = 0; l < NTH; l++) {
    double2 acc = b[l];
#pragma unroll
    for (int m = 0; m < NTH; m++) acc = zsub(acc, zmul(Sfull[l][m], x[m]));
    r[l] = acc;
  }
  solve(r, dx);
#pragma unroll
  for (int l = 0; l < NTH; l++) x[l] = make_double2(x[l].x + dx[l].x, x[l].y + dx[l].y);
  // mu_post = mu + (K S)^H x, residual d - K mu_post
  double2 mp[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    double2 acc = make_double2(mu[a].x, mu[a].y);
#pragma unroll
    for (int l = 0; l < NTH; l++) {  // conj(kw_l AS[l][a]) x_l
      double2 ks = make_double2(kw[l].x * AS[l][a], -kw[l].y * AS[l][a]);
      acc = make_double2(acc.x + ks.x * x[l].x - ks.y * x[l].y, acc.y + ks.x * x[l].y + ks.y * x[l].x);
    }
    mp[a] = acc;
    o.mu[a] = make_float2((float)acc.x, (float)acc.y);
  }
#pragma unroll
  for (int l = 0; l < NTH; l++) {
    double2 am = make_double2(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < 3; j++) am = make_double2(am.x + P.Ad[l][j] * mp[j].x, am.y + P.Ad[l][j] * mp[j].y);
    double2 rr = zsub(make_double2(d[l].x, d[l].y), zmul(kw[l], am));
    d[l] = make_float2((float)rr.x, (float)rr.y);
  }
  return true;
}

// ------------------------------------------------------------------ the fused z pass

// Shared-memory layout of one pencil tile (W consecutive x-bins at one y, all nzp kz):
//   tw  [nzp]             z twiddles
//   R   [nzp][G][W]       G = max(nth + 3, 9) slots per bin: inputs data 0..nth-1 and
//                         mean nth..nth+2; after the per-bin step outputs S_post 0..5 and
//                         mu_post 6..8 (each bin's slots are owned by the thread of that bin)
//   SC  [GT * W * nzp]    transform scratch: the z transforms run GT slots per call
//   S3  [nzp][3 SB][W]    the output spectra of SB realisations, transformed together
// Element (slot g, kz k, x-offset w) of R is R[(k * G + g) * W + w].  3 SB <= GT.


// z transform of nl lines of a pencil tile by the four-step passes (fft2.cuh): line l at
// in + l, point p at in + l + p * ps; pass 1 in place, pass 2 into out at the same
// offsets, so the result (natural order) is in out and in is overwritten.
template <int N1, int N2, int DIR>
__device__ __forceinline__ void zfft4(float2* in, float2* out, int nl, int ps, const float2* tw) {
  const int T = blockDim.x;
  const float rl = __frcp_rn((float)nl);
  const int mstep = N2 * ps;
  for (int q = threadIdx.x; q < nl * N2; q += T) {
    int l;
    const int t = fdivmod(q, nl, rl, l);
    float2* x = in + l + t * ps;
    four_step_pass1<N1, N2, DIR>(
        t, tw, [&](int, int m) { return x[m * mstep]; }, [&](int, int k2, float2 v) { x[k2 * mstep] = v; });
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nl * N1; q += T) {
    int l;
    const int k2 = fdivmod(q, nl, rl, l);
    const float2* y = in + l + k2 * mstep;
    float2 v[N2];
    four_step_pass2<N1, N2, DIR>(k2, [&](int, int t) { return y[t * ps]; }, v);
    float2* o = out + l + k2 * ps;
#pragma unroll
    for (int k1 = 0; k1 < N2; k1++) o[k1 * N1 * ps] = v[k1];
  }
  __syncthreads();
}

// Four-step z transform for the lengths with a split (P.zsplit 1: 16x16, 2: 20x16,
// 3: 16x8); returns false for the others.
template <int DIR>
__device__ __forceinline__ bool z_four_step(const ZParams& P, float2* in, float2* out, int nl, int ps,
                                            const float2* tw) {
  switch (P.zsplit) {
    case 1: zfft4<16, 16, DIR>(in, out, nl, ps, tw); return true;
    case 2: zfft4<20, 16, DIR>(in, out, nl, ps, tw); return true;
    case 3: zfft4<16, 8, DIR>(in, out, nl, ps, tw); return true;
    default: return false;
  }
}

// REFINE instantiates the FP64 re-factorisation of flagged bins; the FP32-only kernel is
// a separate instantiation so that its register allocation does not carry the call.
template <int NTH, bool REFINE>
__global__ void __launch_bounds__(512) k_zpass(const __grid_constant__ ZParams P) {
  extern __shared__ float2 sm[];
  const int nzp = P.nzp, W = P.W, lw = P.logW;
  const int TS = W * nzp;
  constexpr int G = NTH + 3 > 9 ? NTH + 3 : 9;
  constexpr int GIN = NTH + 3;
  const int GT = P.GT, SB = P.SB;
  float2* tw = sm;
  float2* R = tw + nzp;
  float2* SC = R + G * TS;
  float2* S3 = SC + GT * TS;
  // four-step z transforms write into the other G-slot buffer, which then takes over
  const bool four = P.zsplit != 0 && GT >= G;
  __shared__ unsigned long long cnt[4];
  const int T = blockDim.x, tid = threadIdx.x;
  const int it = blockIdx.x % P.nIT;
  const int j = blockIdx.x / P.nIT;
  const int i0 = it * W;
  const int nw = min(W, P.cnxp - i0);
  const size_t kstride = (size_t)P.nyp * P.cnxp;
  const size_t base = (size_t)j * P.cnxp + i0;

  if (tid < 4) cnt[tid] = 0;
  for (int t = tid; t < nzp; t += T) tw[t] = P.twz[t];
  // ---- load inputs: slot g <- data[g] (g < NTH) or mean[g - NTH]; every copy is issued
  //      before the first is waited for (cp.async), x-bins beyond the grid are zero-filled
  {
    const uint32_t rb = smem_addr(R);
    for (int e = tid; e < TS; e += T) {
      const int w = e & (W - 1), k = e >> lw;
      const bool ok = w < nw;
      const size_t go = base + (ok ? (size_t)k * kstride + w : 0);   // nothing is read when !ok
      const uint32_t sa = rb + 8u * (uint32_t)(k * G * W + w);
#pragma unroll
      for (int g = 0; g < GIN; g++)
        cp_async8_zfill(sa + 8u * (uint32_t)(g * W), (g < NTH ? P.data[g] : P.mean[g - NTH]) + go, ok);
    }
    cp_async_commit();
    cp_async_wait_0();
  }
  __syncthreads();
  // forward z transforms, GT slots per call
  if (four) {
    z_four_step<-1>(P, R, SC, GIN * W, G * W, tw);
    float2* t = R;
    R = SC;
    SC = t;
  } else {
#pragma unroll 1
    for (int g0 = 0; g0 < GIN; g0 += GT) {
      int ng = min(GT, GIN - g0);
      fft_lines<true, -1>(R + g0 * W, SC, ng * W, 1, G * W, P.zp, tw);
    }
  }

  // A NaN or Inf anywhere in a data or prior-mean grid reaches every bin through the three
  // transforms, so one bin per tile tells whether the inputs were finite.
  if (tid == 0 && P.counters) {
    float s = 0.f;
#pragma unroll
    for (int g = 0; g < GIN; g++) s += fabsf(R[g * W].x) + fabsf(R[g * W].y);
    if (!isfinite(s)) atomicAdd(P.counters + 4, 1ull);
  }
  // ---- per-bin posterior (src/avoinversion.cpp:1016-1082)
  unsigned long long n_inv = 0, n_fail = 0, n_zero_bins = 0, n_fp64 = 0;
  for (int b = tid; b < TS; b += T) {
    int k = b >> lw, w = b & (W - 1);
    if (w >= nw) continue;
    int i = i0 + w;
    size_t gidx = base + (size_t)k * kstride + w;
    float2* slot = R + k * G * W + w;   // slot g at slot[g * W]
    float S[6], lam, rho = 0.f;
    if (P.separable) {
      float2 cx = __ldg(P.cxy + (size_t)j * P.cnxp + i);
      float2 c_t = __ldg(P.ct + k);
      rho = fabsf(cx.x * c_t.x - cx.y * c_t.y);
#pragma unroll
      for (int q = 0; q < 6; q++) S[q] = P.pv[q] * rho;
      lam = fabsf(cx.x);
    } else {
      // getNextParameterCovariance: |Re/pv| pv (no division when pv == 0); a base prior's
      // pairs share |Re/pv| of the one spectrum transformed (pv[0] != 0)
      if (P.base_prior) {
        const float r0 = fabsf(P.cov[0][gidx].x / P.pv[0]);
#pragma unroll
        for (int q = 0; q < 6; q++) S[q] = r0 * P.pv[q];
      } else {
#pragma unroll
        for (int q = 0; q < 6; q++) {
          float re = P.cov[q][gidx].x;
          float pv = P.pv[q];
          if (pv != 0.f) re = re / pv;
          S[q] = fabsf(re) * pv;
        }
      }
      lam = fabsf(P.errspec[gidx].x);
    }
    float2 mu[3], d[NTH];
#pragma unroll
    for (int a = 0; a < 3; a++) mu[a] = slot[(NTH + a) * W];
#pragma unroll
    for (int l = 0; l < NTH; l++) d[l] = slot[l * W];
    BinOut o;
    bool inv = P.kz.inv[k] != 0;
    bool ok = false;
    if (!REFINE && P.eig) {
      // separable prior with a real temporal spectrum: the eigen form of the per-bin step
      // (bin_posterior_eig, tables in natural kz order), which never needs a fallback (the
      // host bounds the lateral factor against the reference's pivot test before choosing it)
      const float lam1[1] = {lam}, rho1[1] = {rho};
      float2 mu1[1][3], d1[1][NTH], mp1[1][3], sp1[1][6];
#pragma unroll
      for (int a = 0; a < 3; a++) mu1[0][a] = mu[a];
#pragma unroll
      for (int l = 0; l < NTH; l++) d1[0][l] = d[l];
      bin_posterior_eig<NTH, 1>(P, P.eig + k, lam1, rho1, mu1, d1, mp1, sp1);
#pragma unroll
      for (int a = 0; a < 3; a++) o.mu[a] = mp1[0][a];
#pragma unroll
      for (int q = 0; q < 6; q++) o.sp[q] = sp1[0][q];
#pragma unroll
      for (int l = 0; l < NTH; l++) d[l] = d1[0][l];
      if (inv) n_inv++;
      ok = true;
    } else if (inv) {
      n_inv++;
      ok = P.septab ? bin_posterior<NTH, true>(P, k, S, lam, rho, mu, d, o)
                    : bin_posterior<NTH, false>(P, k, S, lam, rho, mu, d, o);
      if constexpr (REFINE) {
        if (ok) {
          float ratio = 1.f;
#pragma unroll
          for (int a = 0; a < 3; a++)
            if (S[a] > 0.f) ratio = fminf(ratio, o.sp[a].x / S[a]);
          if (o.cond > P.fp64_threshold || ratio * P.fp64_threshold < 1.f) {
            // the data are still in their slots: restart from them
            float2 d64[NTH];
#pragma unroll
            for (int l = 0; l < NTH; l++) d64[l] = slot[l * W];
            if (bin_posterior_fp64<NTH>(P, k, S, lam, mu, d64, o)) {
              n_fp64++;
#pragma unroll
              for (int l = 0; l < NTH; l++) d[l] = d64[l];
            }
          }
        }
      }
      if (!ok) n_fail++;
    }
    if (!ok) {
#pragma unroll
      for (int a = 0; a < 3; a++) o.mu[a] = mu[a];
#pragma unroll
      for (int q = 0; q < 6; q++) o.sp[q] = make_float2(S[q], 0.f);
    }
    if (P.keep_resid) {
#pragma unroll
      for (int l = 0; l < NTH; l++) P.data[l][gidx] = d[l];
    }
    // Factor S_post once for all realisations (lib_matrCholCpx(3), simulate :1425-1443).
    // Slots 0..5 then hold L (diagonal real, slot 0 imaginary part set to -1 as the mark)
    // or, where the factorisation fails, S_post itself; the covariance output is rebuilt
    // as L L^H before its inverse transform.
    float2 C[3][3];
    C[0][0] = o.sp[0]; C[1][1] = o.sp[1]; C[2][2] = o.sp[2];
    C[0][1] = o.sp[3]; C[0][2] = o.sp[4]; C[1][2] = o.sp[5];
    C[1][0] = make_float2(o.sp[3].x, -o.sp[3].y);
    C[2][0] = make_float2(o.sp[4].x, -o.sp[4].y);
    C[2][1] = make_float2(o.sp[5].x, -o.sp[5].y);
    if (P.nsim > 0 && chol_ref<3>(C)) {
      slot[0] = make_float2(C[0][0].x, -1.f);
      slot[W] = make_float2(C[1][1].x, 0.f);
      slot[2 * W] = make_float2(C[2][2].x, 0.f);
      slot[3 * W] = C[1][0];
      slot[4 * W] = C[2][0];
      slot[5 * W] = C[2][1];
    } else {
      if (P.nsim > 0) n_zero_bins++;
#pragma unroll
      for (int q = 0; q < 6; q++) slot[q * W] = o.sp[q];
    }
#pragma unroll
    for (int a = 0; a < 3; a++) slot[(6 + a) * W] = o.mu[a];
  }
  __syncthreads();

  // ---- realisations (src/avoinversion.cpp:1401-1511), mean added in the spectral domain;
  //      SB realisations per batch share one transform call
#pragma unroll 1
  for (int s0 = 0; s0 < P.nsim; s0 += SB) {
    const int nb = min(SB, P.nsim - s0);
    const int SG = 3 * nb;  // slots of this batch
    for (int b = tid; b < TS; b += T) {
      int k = b >> lw, w = b & (W - 1);
      float2* o3 = S3 + k * SG * W + w;
      if (w >= nw) {
        for (int q = 0; q < SG; q++) o3[q * W] = make_float2(0.f, 0.f);
        continue;
      }
      int i = i0 + w;
      size_t gidx = base + (size_t)k * kstride + w;
      const float2* slot = R + k * G * W + w;
      const float2 l0 = slot[0];
      const float2 m0 = slot[6 * W], m1 = slot[7 * W], m2 = slot[8 * W];
#pragma unroll 1
      for (int sb = 0; sb < nb; sb++) {
        const int s = s0 + sb;
        float2 sd[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
        if (l0.y == -1.f) {
          float2 z[3];
          if (P.host_noise) {
#pragma unroll
            for (int c = 0; c < 3; c++) z[c] = P.noise[3 * s + c][gidx];
          } else {
            device_noise3(P.seed, s, i, j, k, P.nyp, nzp, P.cnxp, P.nxp_even, z);
          }
          const float2 l1 = slot[W], l2 = slot[2 * W], l10 = slot[3 * W], l20 = slot[4 * W], l21 = slot[5 * W];
          sd[0] = make_float2(l0.x * z[0].x, l0.x * z[0].y);
          sd[1] = cadd(cmul(l10, z[0]), make_float2(l1.x * z[1].x, l1.x * z[1].y));
          sd[2] = cadd(cadd(cmul(l20, z[0]), cmul(l21, z[1])), make_float2(l2.x * z[2].x, l2.x * z[2].y));
        }
        o3[(3 * sb + 0) * W] = cadd(m0, sd[0]);
        o3[(3 * sb + 1) * W] = cadd(m1, sd[1]);
        o3[(3 * sb + 2) * W] = cadd(m2, sd[2]);
      }
    }
    __syncthreads();
    const float2* res = S3;
    if (four) {
      z_four_step<1>(P, S3, SC, SG * W, SG * W, tw);
      res = SC;
    } else {
      fft_lines<true, 1>(S3, SC, SG * W, 1, SG * W, P.zp, tw);
    }
    for (int e = tid; e < TS; e += T) {
      const int w = e & (W - 1), k = e >> lw;
      if (w >= nw) continue;
      const size_t go = base + (size_t)k * kstride + w;
      const float2* r = res + k * SG * W + w;
#pragma unroll
      for (int q = 0; q < 6; q++)
        if (q < SG) P.sim[3 * s0 + q][go] = r[q * W];
    }
    __syncthreads();
  }
  // ---- rebuild S_post = L L^H where slots 0..5 hold the factor
  if (P.nsim > 0) {
    for (int b = tid; b < TS; b += T) {
      int k = b >> lw, w = b & (W - 1);
      float2* slot = R + k * G * W + w;
      const float2 l0 = slot[0];
      if (l0.y != -1.f) continue;
      const float2 l1 = slot[W], l2 = slot[2 * W], l10 = slot[3 * W], l20 = slot[4 * W], l21 = slot[5 * W];
      // S_ab = sum_c L_ac conj(L_bc)
      slot[0] = make_float2(l0.x * l0.x, 0.f);
      slot[W] = make_float2(l10.x * l10.x + l10.y * l10.y + l1.x * l1.x, 0.f);
      slot[2 * W] = make_float2(l20.x * l20.x + l20.y * l20.y + l21.x * l21.x + l21.y * l21.y + l2.x * l2.x, 0.f);
      slot[3 * W] = make_float2(l0.x * l10.x, -l0.x * l10.y);
      slot[4 * W] = make_float2(l0.x * l20.x, -l0.x * l20.y);
      slot[5 * W] = make_float2(l10.x * l20.x + l10.y * l20.y + l1.x * l21.x,
                                l10.y * l20.x - l10.x * l20.y - l1.x * l21.y);
    }
    __syncthreads();
  }

  // ---- inverse z transform of posterior covariance (slots 0..5, unless it stays spectral)
  //      and mean (6..8)
  const int gs0 = P.cov_spectral ? 6 : 0;
  if (four) {
    z_four_step<1>(P, R + gs0 * W, SC + gs0 * W, (9 - gs0) * W, G * W, tw);
  } else {
#pragma unroll 1
    for (int g0 = gs0; g0 < 9; g0 += GT)
      fft_lines<true, 1>(R + g0 * W, SC, min(GT, 9 - g0) * W, 1, G * W, P.zp, tw);
  }
  for (int e = tid; e < TS; e += T) {
    const int w = e & (W - 1), k = e >> lw;
    if (w >= nw) continue;
    const size_t go = base + (size_t)k * kstride + w;
    const int so = k * G * W + w;
#pragma unroll
    for (int g = 0; g < 9; g++) {
      const float2* src = (four && g >= gs0) ? SC : R;
      (g < 6 ? P.cov[g] : P.mean[g - 6])[go] = src[so + g * W];
    }
  }

  // counters
  unsigned long long n_zero = n_zero_bins * (unsigned long long)P.nsim;
  for (int off = 16; off > 0; off >>= 1) {
    n_inv += __shfl_down_sync(0xffffffffu, n_inv, off);
    n_fail += __shfl_down_sync(0xffffffffu, n_fail, off);
    n_zero += __shfl_down_sync(0xffffffffu, n_zero, off);
    n_fp64 += __shfl_down_sync(0xffffffffu, n_fp64, off);
  }
  if ((tid & 31) == 0) {
    atomicAdd(&cnt[0], n_inv);
    atomicAdd(&cnt[1], n_fail);
    atomicAdd(&cnt[2], n_zero);
    atomicAdd(&cnt[3], n_fp64);
  }
  __syncthreads();
  if (tid == 0 && P.counters) {
    atomicAdd(P.counters + 0, cnt[0]);
    atomicAdd(P.counters + 1, cnt[1]);
    atomicAdd(P.counters + 2, cnt[2]);
    atomicAdd(P.counters + 3, cnt[3]);
  }
}

// ------------------------------------------------------------------ launch templates

template <int NTH, bool REFINE>
inline cudaError_t launch_zpass_r(const ZParams& zp, int threads, cudaStream_t st) {
  size_t smem = zpass_smem_bytes(zp.W, zp.nzp, zp.nth, zp.GT, zp.SB);
  cudaError_t e = cudaFuncSetAttribute(k_zpass<NTH, REFINE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)(zp.nIT * zp.nyp));
  k_zpass<NTH, REFINE><<<grid, threads, smem, st>>>(zp);
  return cudaGetLastError();
}

template <int NTH>
inline cudaError_t launch_zpass_t(const ZParams& zp, int threads, cudaStream_t st) {
  return zp.fp64_threshold > 0.f ? launch_zpass_r<NTH, true>(zp, threads, st)
                                 : launch_zpass_r<NTH, false>(zp, threads, st);
}

// the general kernel's launchers by angle count (zpass_n12.cu, zpass_n34.cu, zpass_n56.cu,
// zpass_n78.cu): one translation unit per pair so that they compile side by side
cudaError_t launch_zpass_nth(const ZParams& zp, int threads, cudaStream_t st);
cudaError_t launch_zpass_n12(const ZParams& zp, int threads, cudaStream_t st);
cudaError_t launch_zpass_n34(const ZParams& zp, int threads, cudaStream_t st);
cudaError_t launch_zpass_n56(const ZParams& zp, int threads, cudaStream_t st);
cudaError_t launch_zpass_n78(const ZParams& zp, int threads, cudaStream_t st);

}  // namespace crava
