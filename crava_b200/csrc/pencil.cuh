// The separable-prior pencil pass in its eigen form (sm_100a).
//
// Per (x-tile, y) pencil, like k_zpass (zpass.cu): forward z transform of the data and
// prior-mean spectra, the per-bin posterior of AVOInversion::computePostMeanResidAndFFTCov
// (src/avoinversion.cpp:944-1091), the realisations of AVOInversion::simulate
// (src/avoinversion.cpp:1401-1511) and the inverse z transform of every output spectrum,
// with the spectra kept on chip between the two transforms.
//
// The per-bin algebra.  With a separable prior whose temporal factor has a real spectrum
// (a symmetric circular correlation, as SeismicParametersHolder::computeCircCorrT builds it,
// src/seismicparametersholder.cpp:624-660), every bin of one kz has the data covariance
//     Sd = lam M_k + E_k,   M_k = |ct_k| (kw kw^H) o G0 + M2_k,   E_k = diag(ed_k) > 0,
// with lam = |Re corrXY-spectrum(i, j)| the only lateral variable, and K S = lam |ct_k|
// diag(kw) A P0.  From the Hermitian eigen-decomposition E^-1/2 M_k E^-1/2 = U diag(Lam) U^H
// (per kz, on the host, in double) and V = U^H E^-1/2, Q = |ct_k| V diag(kw) A P0:
//     mu_post = mu + lam Q^H diag(1 / (lam Lam + 1)) V (d - K mu)
//     S_post  = rho P0 - lam^2 sum_l conj(Q_la) Q_lb / (lam Lam_l + 1)
//     resid   = d - K mu_post
// which equals the reference's Sd^-1 regrouping exactly in exact arithmetic: a few small
// matrix-vector products per bin instead of a per-bin Cholesky factorisation and solves.
// Sd is positive definite for every lam >= 0 (Sd >= E_k), so the reference's Cholesky
// never falls back here; the host checks that before it chooses this kernel.
//
// The z transforms run in place: the forward four-step transform leaves kz = k2 + N1 k1 at
// position k1 + N2 k2 (no scratch buffer), the per-bin step reads its tables in that
// position order, and the inverse transform takes that order back to natural order.  With
// no transform scratch the tile needs (G + 3) slots of W x nzp complex values, so two CTAs
// share an SM at nzp = 256 with one realisation per batch.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft2.cuh"
#include "fft_core.cuh"
#include "kernels.cuh"
#include "pencil_common.cuh"

namespace crava {

// ------------------------------------------------------------------ in-place z transforms

// Forward transform of nl lines (line l at x + l, point p at x + l + p ps) of length
// N1 N2, natural order in, position k1 + N2 k2 <- X[k2 + N1 k1] out.
template <int N1, int N2>
__device__ __forceinline__ void zfwd_inplace(float2* x, int nl, int ps, const float2* tw) {
  const int T = blockDim.x;
  const float rl = __frcp_rn((float)nl);
  const int mstep = N2 * ps;
  // pass 1, item t < N2: N1-point DFT over positions t + N2 m, twiddle w^(t k2), back to
  // positions t + N2 k2
  for (int q = threadIdx.x; q < nl * N2; q += T) {
    int l;
    const int t = fdivmod(q, nl, rl, l);
    float2* y = x + l + t * ps;
    four_step_pass1<N1, N2, -1>(
        t, tw, [&](int, int m) { return y[m * mstep]; }, [&](int, int k2, float2 v) { y[k2 * mstep] = v; });
  }
  __syncthreads();
  // pass 2, item k2 < N1: N2-point DFT over the run t + N2 k2 (t < N2), X[k2 + N1 k1] back to
  // position k1 + N2 k2
  for (int q = threadIdx.x; q < nl * N1; q += T) {
    int l;
    const int k2 = fdivmod(q, nl, rl, l);
    float2* y = x + l + k2 * mstep;
    float2 v[N2];
#pragma unroll
    for (int t = 0; t < N2; t++) v[t] = y[t * ps];
    Dft<N2>::run(v, -1.f);
#pragma unroll
    for (int k1 = 0; k1 < N2; k1++) y[k1 * ps] = v[k1];
  }
  __syncthreads();
}

// Inverse transform (unnormalised, e^{+2 pi i}) of nl lines holding X[k2 + N1 k1] at position
// k1 + N2 k2; natural order out:
//   x[t + N2 m] = sum_k2 w1^(-m k2) w^(-t k2) sum_k1 w2^(-t k1) X[k2 + N1 k1].
template <int N1, int N2>
__device__ __forceinline__ void zinv_inplace(float2* x, int nl, int ps, const float2* tw) {
  const int T = blockDim.x;
  const float rl = __frcp_rn((float)nl);
  const int mstep = N2 * ps;
  // pass A, item k2 < N1: N2-point inverse DFT over the run k1 + N2 k2, twiddle w^(-t k2),
  // back to positions t + N2 k2
  for (int q = threadIdx.x; q < nl * N1; q += T) {
    int l;
    const int k2 = fdivmod(q, nl, rl, l);
    float2* y = x + l + k2 * mstep;
    float2 v[N2];
#pragma unroll
    for (int k1 = 0; k1 < N2; k1++) v[k1] = y[k1 * ps];
    Dft<N2>::run(v, 1.f);
#pragma unroll
    for (int t = 1; t < N2; t++) {
      float2 w = tw[t * k2];   // t k2 < N1 N2
      v[t] = cmul(v[t], make_float2(w.x, -w.y));
    }
#pragma unroll
    for (int t = 0; t < N2; t++) y[t * ps] = v[t];
  }
  __syncthreads();
  // pass B, item t < N2: N1-point inverse DFT over positions t + N2 k2, natural order back
  for (int q = threadIdx.x; q < nl * N2; q += T) {
    int l;
    const int t = fdivmod(q, nl, rl, l);
    float2* y = x + l + t * ps;
    float2 v[N1];
#pragma unroll
    for (int k2 = 0; k2 < N1; k2++) v[k2] = y[k2 * mstep];
    Dft<N1>::run(v, 1.f);
#pragma unroll
    for (int m = 0; m < N1; m++) y[m * mstep] = v[m];
  }
  __syncthreads();
}

// The same inverse transform with its last pass writing each line's natural-order outputs
// straight out through store(l, k, value) (line l, z index k) instead of back to x; x is
// free for reuse after the closing barrier.
template <int N1, int N2, class Store>
__device__ __forceinline__ void zinv_store(float2* x, int nl, int ps, const float2* tw, Store store) {
  const int T = blockDim.x;
  const float rl = __frcp_rn((float)nl);
  const int mstep = N2 * ps;
  for (int q = threadIdx.x; q < nl * N1; q += T) {
    int l;
    const int k2 = fdivmod(q, nl, rl, l);
    float2* y = x + l + k2 * mstep;
    float2 v[N2];
#pragma unroll
    for (int k1 = 0; k1 < N2; k1++) v[k1] = y[k1 * ps];
    Dft<N2>::run(v, 1.f);
#pragma unroll
    for (int t = 1; t < N2; t++) {
      float2 w = tw[t * k2];
      v[t] = cmul(v[t], make_float2(w.x, -w.y));
    }
#pragma unroll
    for (int t = 0; t < N2; t++) y[t * ps] = v[t];
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nl * N2; q += T) {
    int l;
    const int t = fdivmod(q, nl, rl, l);
    const float2* y = x + l + t * ps;
    float2 v[N1];
#pragma unroll
    for (int k2 = 0; k2 < N1; k2++) v[k2] = y[k2 * mstep];
    Dft<N1>::run(v, 1.f);
#pragma unroll
    for (int m = 0; m < N1; m++) store(l, t + N2 * m, v[m]);
  }
  __syncthreads();
}

// ------------------------------------------------------------------ per-bin algebra

// Writes one bin's results into its slots: the residual (KEEP_RESIDUAL, at global index
// gidx), S_post's realisation factor (lib_matrCholCpx(3), simulate :1425-1443) in slots 0..5
// with slot 0's imaginary part -1 as the mark, or S_post itself where that factorisation
// fails, and mu_post in slots 6..8.  Returns 1 for a bin whose realisations stay zero.
template <int NTH>
__device__ __forceinline__ int store_bin(const ZParams& P, float2* slot, int W, const float2 (&d)[NTH],
                                         const float2 (&mp)[3], const float2 (&sp)[6], size_t gidx) {
  if (P.keep_resid) {
#pragma unroll
    for (int l = 0; l < NTH; l++) P.data[l][gidx] = d[l];
  }
  float2 C[3][3];
  C[0][0] = sp[0]; C[1][1] = sp[1]; C[2][2] = sp[2];
  C[0][1] = sp[3]; C[0][2] = sp[4]; C[1][2] = sp[5];
  C[1][0] = make_float2(sp[3].x, -sp[3].y);
  C[2][0] = make_float2(sp[4].x, -sp[4].y);
  C[2][1] = make_float2(sp[5].x, -sp[5].y);
  int zero = 0;
  if (P.nsim > 0 && chol_ref<3>(C)) {
    slot[0] = make_float2(C[0][0].x, -1.f);
    slot[W] = make_float2(C[1][1].x, 0.f);
    slot[2 * W] = make_float2(C[2][2].x, 0.f);
    slot[3 * W] = C[1][0];
    slot[4 * W] = C[2][0];
    slot[5 * W] = C[2][1];
  } else {
    if (P.nsim > 0) zero = 1;
#pragma unroll
    for (int q = 0; q < 6; q++) slot[q * W] = sp[q];
  }
#pragma unroll
  for (int a = 0; a < 3; a++) slot[(6 + a) * W] = mp[a];
  return zero;
}

// S_post = L L^H of a bin whose slots 0..5 hold its realisation factor (written back there).
// The products and sums are spelled out as explicit fused multiply-adds so that every call site
// rounds them alike (the two realisation forms call it from different code).
__device__ __forceinline__ void store_llh(float2* slot, int W, float2 l0, float2 l1, float2 l2, float2 l10,
                                          float2 l20, float2 l21) {
  slot[0] = make_float2(__fmul_rn(l0.x, l0.x), 0.f);
  slot[W] = make_float2(__fmaf_rn(l10.x, l10.x, __fmaf_rn(l10.y, l10.y, __fmul_rn(l1.x, l1.x))), 0.f);
  slot[2 * W] = make_float2(
      __fmaf_rn(l20.x, l20.x,
                __fmaf_rn(l20.y, l20.y, __fmaf_rn(l21.x, l21.x, __fmaf_rn(l21.y, l21.y, __fmul_rn(l2.x, l2.x))))),
      0.f);
  slot[3 * W] = make_float2(__fmul_rn(l0.x, l10.x), -__fmul_rn(l0.x, l10.y));
  slot[4 * W] = make_float2(__fmul_rn(l0.x, l20.x), -__fmul_rn(l0.x, l20.y));
  slot[5 * W] = make_float2(__fmaf_rn(l10.x, l20.x, __fmaf_rn(l10.y, l20.y, __fmul_rn(l1.x, l21.x))),
                            __fmaf_rn(l10.y, l20.x, __fmaf_rn(-l10.x, l20.y, -__fmul_rn(l1.x, l21.y))));
}

// ------------------------------------------------------------------ the kernel

// Shared-memory layout of one tile (W consecutive x-bins at one y, all NZ = N1 N2 positions):
//   tw  [NZ]             z twiddles e^{-2 pi i t / NZ}
//   R   [NZ][G][W]       G = max(nth + 3, 9) slots per bin: data 0..nth-1, mean nth..nth+2;
//                        after the per-bin step S_post (or its realisation factor) 0..5 and
//                        mu_post 6..8
//   S3  [NZ][3 SB][W]    the output spectra of SB realisations, transformed together
// Element (slot g, position p, x-offset w) of R is R[(p G + g) W + w].
// DENSE: bounded for two 384-thread CTAs per SM (at most 80 registers), the other form for
// one CTA of up to 512 threads (up to 128 registers).
template <int NTH, int N1, int N2, bool DENSE>
__global__ void __launch_bounds__(DENSE ? 384 : 512, DENSE ? 2 : 1) k_pencil(const __grid_constant__ ZParams P) {
  extern __shared__ float2 sm[];
  constexpr int NZ = N1 * N2;
  constexpr int G = NTH + 3 > 9 ? NTH + 3 : 9;
  constexpr int GIN = NTH + 3;
  const int W = P.W, lw = P.logW, SB = P.SB;
  const int TS = W * NZ;
  float2* tw = sm;
  float2* R = tw + NZ;
  float2* S3 = R + G * TS;
  __shared__ unsigned long long cnt[2];
  const int T = blockDim.x, tid = threadIdx.x;
  const int it = blockIdx.x % P.nIT;
  const int j = blockIdx.x / P.nIT;
  const int i0 = it * W;
  const int nw = min(W, P.cnxp - i0);
  const size_t kstride = (size_t)P.nyp * P.cnxp;
  const size_t base = (size_t)j * P.cnxp + i0;

  if (tid < 2) cnt[tid] = 0;
  for (int t = tid; t < NZ; t += T) tw[t] = P.twz[t];
  // ---- inputs: slot g <- data[g] (g < NTH) or mean[g - NTH], natural kz order; x-bins
  //      beyond the grid are zero-filled
  {
    const uint32_t rb = smem_addr(R);
    for (int e = tid; e < TS; e += T) {
      const int w = e & (W - 1), k = e >> lw;
      const bool ok = w < nw;
      const size_t go = base + (ok ? (size_t)k * kstride + w : 0);
      const uint32_t sa = rb + 8u * (uint32_t)(k * G * W + w);
#pragma unroll
      for (int g = 0; g < GIN; g++)
        cp_async8_zfill(sa + 8u * (uint32_t)(g * W), (g < NTH ? P.data[g] : P.mean[g - NTH]) + go, ok);
    }
    cp_async_commit();
    cp_async_wait_0();
  }
  __syncthreads();
  zfwd_inplace<N1, N2>(R, GIN * W, G * W, tw);
  // a NaN or Inf in any input grid reaches every bin through the transforms
  if (tid == 0 && P.counters) {
    float s = 0.f;
#pragma unroll
    for (int g = 0; g < GIN; g++) s += fabsf(R[g * W].x) + fabsf(R[g * W].y);
    if (!isfinite(s)) atomicAdd(P.counters + 4, 1ull);
  }

  // ---- per-bin posterior; bin at position p holds kz = p / N2 + N1 (p % N2).  A thread takes
  //      NB bins of one position (x-offsets w, w + W/NB, ...), so each table row it loads
  //      serves all of them
  unsigned long long n_zero_bins = 0;
  const int NB = (W >= 2 && P.nb2) ? 2 : 1;
  const int WB = W / NB, lwb = NB == 2 ? lw - 1 : lw;
  for (int b = tid; b < TS / NB; b += T) {
    const int p = b >> lwb, w0 = b & (WB - 1);
    const int kz = p / N2 + N1 * (p % N2);
    const float ctk = __ldg(P.ct + kz).x;
    if (NB == 2) {
      float lam[2], rho[2];
      float2 mu[2][3], d[2][NTH], mp[2][3], sp[2][6];
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int w = w0 + u * WB;
        const bool ok = w < nw;
        const float2 cx = ok ? __ldg(P.cxy + (size_t)j * P.cnxp + i0 + w) : make_float2(0.f, 0.f);
        lam[u] = fabsf(cx.x);
        rho[u] = fabsf(cx.x * ctk);
        const float2* slot = R + p * G * W + w;
#pragma unroll
        for (int a = 0; a < 3; a++) mu[u][a] = slot[(NTH + a) * W];
#pragma unroll
        for (int l = 0; l < NTH; l++) d[u][l] = slot[l * W];
      }
      bin_posterior_eig<NTH, 2>(P, P.eig + p, lam, rho, mu, d, mp, sp);
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int w = w0 + u * WB;
        if (w < nw) n_zero_bins += store_bin<NTH>(P, R + p * G * W + w, W, d[u], mp[u], sp[u],
                                                  base + (size_t)kz * kstride + w);
      }
    } else {
      const int w = w0;
      if (w >= nw) continue;
      const float2 cx = __ldg(P.cxy + (size_t)j * P.cnxp + i0 + w);
      float lam[1] = {fabsf(cx.x)}, rho[1] = {fabsf(cx.x * ctk)};
      float2 mu[1][3], d[1][NTH], mp[1][3], sp[1][6];
      const float2* slot = R + p * G * W + w;
#pragma unroll
      for (int a = 0; a < 3; a++) mu[0][a] = slot[(NTH + a) * W];
#pragma unroll
      for (int l = 0; l < NTH; l++) d[0][l] = slot[l * W];
      bin_posterior_eig<NTH, 1>(P, P.eig + p, lam, rho, mu, d, mp, sp);
      n_zero_bins += store_bin<NTH>(P, R + p * G * W + w, W, d[0], mp[0], sp[0], base + (size_t)kz * kstride + w);
    }
  }
  __syncthreads();

  // ---- SB = 0: no realisation slots.  The posterior mean (slots 6..8) is transformed and
  //      stored first; each realisation's L z then goes through those slots and the stored mean
  //      is added in the last pass (IFFT(mu + L z) = IFFT(mu) + IFFT(L z)); the covariance last.
  //      The tile needs G slots instead of G + 3, so wider tiles fit at the longer z lengths.
  if (SB == 0) {
    zinv_store<N1, N2>(R + 6 * W, 3 * W, G * W, tw, [&](int l, int k, float2 v) {
      const int w = l & (W - 1);
      if (w < nw) P.mean[l >> lw][base + (size_t)k * kstride + w] = v;
    });
#pragma unroll 1
    for (int s = 0; s < P.nsim; s++) {
      for (int b = tid; b < TS; b += T) {
        const int p = b >> lw, w = b & (W - 1);
        const float2* slot = R + p * G * W + w;
        float2* o3 = R + (p * G + 6) * W + w;
        float2 sd[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
        const float2 l0 = slot[0];
        if (w < nw && l0.y == -1.f) {
          const int kz = p / N2 + N1 * (p % N2);
          float2 z[3];
          if (P.host_noise) {
            const size_t gidx = base + (size_t)kz * kstride + w;
#pragma unroll
            for (int c = 0; c < 3; c++) z[c] = P.noise[3 * s + c][gidx];
          } else {
            device_noise3(P.seed, s, i0 + w, j, kz, P.nyp, NZ, P.cnxp, P.nxp_even, z);
          }
          const float2 l1 = slot[W], l2 = slot[2 * W], l10 = slot[3 * W], l20 = slot[4 * W], l21 = slot[5 * W];
          sd[0] = make_float2(l0.x * z[0].x, l0.x * z[0].y);
          sd[1] = cadd(cmul(l10, z[0]), make_float2(l1.x * z[1].x, l1.x * z[1].y));
          sd[2] = cadd(cadd(cmul(l20, z[0]), cmul(l21, z[1])), make_float2(l2.x * z[2].x, l2.x * z[2].y));
          // the last realisation leaves S_post in slots 0..5 for the covariance output
          if (s == P.nsim - 1) store_llh(R + p * G * W + w, W, l0, l1, l2, l10, l20, l21);
        }
        o3[0] = sd[0];
        o3[W] = sd[1];
        o3[2 * W] = sd[2];
      }
      __syncthreads();
      // the mean this CTA stored above (visible after the barriers), read at L2
      zinv_store<N1, N2>(R + 6 * W, 3 * W, G * W, tw, [&](int l, int k, float2 v) {
        const int w = l & (W - 1);
        if (w < nw) {
          const size_t idx = base + (size_t)k * kstride + w;
          P.sim[3 * s + (l >> lw)][idx] = cadd(__ldcg(P.mean[l >> lw] + idx), v);
        }
      });
    }
  }
  // ---- realisations (src/avoinversion.cpp:1401-1511), the mean added in the spectral
  //      domain; SB realisations per batch share one transform call
#pragma unroll 1
  for (int s0 = 0; SB > 0 && s0 < P.nsim; s0 += SB) {
    const int nb = min(SB, P.nsim - s0);
    const int SG = 3 * SB;   // slot stride of S3
    for (int b = tid; b < TS; b += T) {
      const int p = b >> lw, w = b & (W - 1);
      float2* o3 = S3 + p * SG * W + w;
      if (w >= nw) {
        for (int q = 0; q < 3 * nb; q++) o3[q * W] = make_float2(0.f, 0.f);
        continue;
      }
      const int kz = p / N2 + N1 * (p % N2);
      const int i = i0 + w;
      const float2* slot = R + p * G * W + w;
      const float2 l0 = slot[0];
      const float2 m0 = slot[6 * W], m1 = slot[7 * W], m2 = slot[8 * W];
      const bool fac = l0.y == -1.f;
      float2 l1 = make_float2(0.f, 0.f), l2 = l1, l10 = l1, l20 = l1, l21 = l1;
      if (fac) {
        l1 = slot[W]; l2 = slot[2 * W]; l10 = slot[3 * W]; l20 = slot[4 * W]; l21 = slot[5 * W];
      }
#pragma unroll 1
      for (int sb = 0; sb < nb; sb++) {
        const int s = s0 + sb;
        float2 sd[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
        if (fac) {
          float2 z[3];
          if (P.host_noise) {
            const size_t gidx = base + (size_t)kz * kstride + w;
#pragma unroll
            for (int c = 0; c < 3; c++) z[c] = P.noise[3 * s + c][gidx];
          } else {
            device_noise3(P.seed, s, i, j, kz, P.nyp, NZ, P.cnxp, P.nxp_even, z);
          }
          sd[0] = make_float2(l0.x * z[0].x, l0.x * z[0].y);
          sd[1] = cadd(cmul(l10, z[0]), make_float2(l1.x * z[1].x, l1.x * z[1].y));
          sd[2] = cadd(cadd(cmul(l20, z[0]), cmul(l21, z[1])), make_float2(l2.x * z[2].x, l2.x * z[2].y));
        }
        o3[(3 * sb) * W] = cadd(m0, sd[0]);
        o3[(3 * sb + 1) * W] = cadd(m1, sd[1]);
        o3[(3 * sb + 2) * W] = cadd(m2, sd[2]);
      }
      // the last batch leaves S_post in slots 0..5 for the covariance output
      if (fac && s0 + nb == P.nsim) store_llh(R + p * G * W + w, W, l0, l1, l2, l10, l20, l21);
    }
    __syncthreads();
    // inverse z transform, the last pass storing the realisations' spectra (line l: grid
    // 3 s0 + l / W, x-offset l % W)
    zinv_store<N1, N2>(S3, 3 * nb * W, SG * W, tw, [&](int l, int k, float2 v) {
      const int w = l & (W - 1);
      if (w < nw) P.sim[3 * s0 + (l >> lw)][base + (size_t)k * kstride + w] = v;
    });
  }
  // (S_post = L L^H is back in slots 0..5: the last realisation wrote it)
  // ---- inverse z transform of posterior covariance (slots 0..5, unless it stays spectral)
  //      and mean (6..8); spectral covariance slots stay in position order
  if (!P.cov_spectral) {
    // slots 0..5 to cov[0..5], 6..8 to mean[0..2] (already stored when SB = 0), stored by the
    // last pass
    zinv_store<N1, N2>(R, (SB == 0 ? 6 : 9) * W, G * W, tw, [&](int l, int k, float2 v) {
      const int g = l >> lw, w = l & (W - 1);
      if (w < nw) (g < 6 ? P.cov[g] : P.mean[g - 6])[base + (size_t)k * kstride + w] = v;
    });
  } else {
    // spectral covariance: slots 0..5 stay in position order, stored at their kz (the mean,
    // slots 6..8, is already stored when SB = 0)
    if (SB > 0) zinv_inplace<N1, N2>(R + 6 * W, 3 * W, G * W, tw);
    for (int e = tid; e < TS; e += T) {
      const int w = e & (W - 1), k = e >> lw;
      if (w >= nw) continue;
      const size_t go = base + (size_t)k * kstride + w;
      const int so = k * G * W + w;
      const int kz = k / N2 + N1 * (k % N2);
#pragma unroll
      for (int g = 0; g < 6; g++) P.cov[g][base + (size_t)kz * kstride + w] = R[so + g * W];
      if (SB > 0) {
#pragma unroll
        for (int a = 0; a < 3; a++) P.mean[a][go] = R[so + (6 + a) * W];
      }
    }
  }

  // counters: inverted bins per tile column from the host's count of inverted kz
  unsigned long long n_zero = n_zero_bins * (unsigned long long)P.nsim;
  for (int off = 16; off > 0; off >>= 1) n_zero += __shfl_down_sync(0xffffffffu, n_zero, off);
  if ((tid & 31) == 0 && n_zero) atomicAdd(&cnt[0], n_zero);
  __syncthreads();
  if (tid == 0 && P.counters) {
    atomicAdd(P.counters + 0, (unsigned long long)P.n_inv_rows * (unsigned long long)nw);
    if (cnt[0]) atomicAdd(P.counters + 2, cnt[0]);
  }
}

// ------------------------------------------------------------------ launch templates

template <int NTH, int N1, int N2, bool DENSE>
inline cudaError_t launch_pencil_d(const ZParams& zp, int threads, cudaStream_t st) {
  const size_t smem = pencil_smem_bytes(zp.W, zp.nzp, zp.nth, zp.SB);
  auto fn = k_pencil<NTH, N1, N2, DENSE>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  fn<<<dim3((unsigned)(zp.nIT * zp.nyp)), threads, smem, st>>>(zp);
  return cudaGetLastError();
}

// The dense form is instantiated for up to 6 angle stacks and 256 / 320 points (the
// production and precision-study lengths).
template <int NTH, int N1, int N2>
inline cudaError_t launch_pencil_t(const ZParams& zp, int threads, cudaStream_t st) {
  if constexpr (NTH <= 6 && N2 == 16) {
    if (zp.dense && threads <= 384) return launch_pencil_d<NTH, N1, N2, true>(zp, threads, st);
  }
  return launch_pencil_d<NTH, N1, N2, false>(zp, threads, st);
}


// launchers of one z split each (pencil_s1.cu 16x16, pencil_s2.cu 20x16, pencil_s3.cu 16x8)
cudaError_t launch_pencil_split1(const ZParams& zp, int threads, cudaStream_t st);
cudaError_t launch_pencil_split2(const ZParams& zp, int threads, cudaStream_t st);
cudaError_t launch_pencil_split3(const ZParams& zp, int threads, cudaStream_t st);

}  // namespace crava
