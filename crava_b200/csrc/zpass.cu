// The fused pencil pass of the AVO inversion (sm_100a): per (x-tile, y) pencil, forward z
// transform of every input spectrum, the per-bin posterior of
// AVOInversion::computePostMeanResidAndFFTCov (src/avoinversion.cpp:944-1091), the per-bin
// simulation of AVOInversion::simulate (src/avoinversion.cpp:1421-1460) and the inverse z
// transform of every output spectrum.  Spectra never leave the CTA between the forward and
// the inverse z transform.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "fft_core.cuh"
#include "kernels.cuh"

namespace crava {

constexpr int kThreads = 256;

// ------------------------------------------------------------------ noise (product mode)

// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// Standard complex normal for bin (i,j,k) of noise grid g, Hermitian-consistent on the
// planes whose x-bin is its own mirror (i = 0, and i = nxp/2 for even nxp): the pair
// (j,k) / (-j,-k) share one draw (conjugated), self-mirrored bins are real with unit
// variance, all others have variance 1/2 per component (FFTGrid::fillInComplexNoise,
// src/fftgrid.cpp:997-1055, with the mirror plane test done on the x index).
__device__ __forceinline__ float2 device_noise(uint64_t seed, int g, int i, int j, int k, int nyp, int nzp,
                                               int cnxp, bool nxp_even) {
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
  uint4 r = philox4x32_10(make_uint4((uint32_t)bin, (uint32_t)(bin >> 32), (uint32_t)g, 0x43524156u),
                          make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
  float u1 = ((float)r.x + 0.5f) * 2.3283064365386963e-10f;
  float u2 = (float)r.y * 2.3283064365386963e-10f;
  float rad = sqrtf(-2.0f * logf(u1));
  float sn, cs;
  sincospif(2.0f * u2, &sn, &cs);
  if (self) return make_float2(rad * cs, 0.f);
  const float h = 0.70710678118654752f;
  float2 z = make_float2(h * rad * cs, h * rad * sn);
  if (conj) z.y = -z.y;
  return z;
}

// ------------------------------------------------------------------ per-bin algebra

// lib_matrCholCpx (libs/lib/lib_matr.c:78-168) on the lower triangle of a Hermitian
// n x n matrix stored row-major in a[]: scale by a00, reject a00 <= 0, a scaled diagonal
// <= 1e-20 or an updated pivot <= 1e-20, factor, rescale by sqrt(a00).
template <int N>
__device__ __forceinline__ bool chol_ref(float2 (&a)[N][N]) {
  const float TOLF = 1e-20f;
  float f = a[0][0].x;
  if (!(f > 0.f)) return false;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j <= i; j++) a[i][j] = make_float2(a[i][j].x / f, a[i][j].y / f);
#pragma unroll
  for (int i = 0; i < N; i++) {
    if (!(a[i][i].x > TOLF)) return false;
#pragma unroll
    for (int j = 0; j < i; j++) {
      float2 s = make_float2(0.f, 0.f);
#pragma unroll
      for (int k = 0; k < j; k++) {  // L_ik conj(L_jk)
        s.x += a[i][k].x * a[j][k].x + a[i][k].y * a[j][k].y;
        s.y += -(a[i][k].x * a[j][k].y) + a[i][k].y * a[j][k].x;
      }
      float d = a[j][j].x;  // real pivot
      a[i][j] = make_float2((a[i][j].x - s.x) / d, (a[i][j].y - s.y) / d);
    }
    float r = 0.f;
#pragma unroll
    for (int k = 0; k < i; k++) r += a[i][k].x * a[i][k].x + a[i][k].y * a[i][k].y;
    r = a[i][i].x - r;
    if (!(r > TOLF)) return false;
    a[i][i] = make_float2(sqrtf(r), 0.f);
  }
  float sf = sqrtf(f);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j <= i; j++) a[i][j] = make_float2(a[i][j].x * sf, a[i][j].y * sf);
  return true;
}

struct BinOut {
  float2 mu[3];
  float2 sp[6];
};

// Posterior of one bin.  Follows src/avoinversion.cpp:1036-1061 with
//   Sd = K S K^H + Se, K = diag(kw) A, S real symmetric (so K S K^H = (kw kw^H) o (A S A^T)),
//   L L^H = Sd (reference Cholesky), Y = L^{-1} K S,
//   S_post = S - Y^H Y, mu_post = mu + Y^H L^{-1} (d - K mu), res = d - K mu_post,
// which is the reference's  KS <- Sd^{-1} KS; S - KS_old^H KS;  mu + KS^H (d - K mu)
// regrouped through the Cholesky factor.
template <int NTH>
__device__ __forceinline__ bool bin_posterior(const ZParams& P, int k, const float (&S)[6], float lam,
                                              const float2 (&mu)[3], float2 (&d)[NTH], BinOut& o) {
  float2 kw[NTH], e1[NTH], e2[NTH];
#pragma unroll
  for (int l = 0; l < NTH; l++) {
    kw[l] = __ldg(P.kz.kw + k * NTH + l);
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
  float2 Sd[NTH][NTH];
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
      if (l == m) Sd[l][m] = make_float2(Sd[l][m].x + P.ed[l], 0.f);
    }
  }
  if (!chol_ref<NTH>(Sd)) return false;
  // Y = L^{-1} KS, KS[l][j] = kw_l AS[l][j]
  float2 Y[NTH][3];
#pragma unroll
  for (int l = 0; l < NTH; l++) {
#pragma unroll
    for (int j = 0; j < 3; j++) {
      float2 acc = make_float2(kw[l].x * AS[l][j], kw[l].y * AS[l][j]);
#pragma unroll
      for (int m = 0; m < l; m++) acc = csub(acc, cmul(Sd[l][m], Y[m][j]));
      float inv = 1.f / Sd[l][l].x;
      Y[l][j] = make_float2(acc.x * inv, acc.y * inv);
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
    float inv = 1.f / Sd[l][l].x;
    yd[l] = make_float2(acc.x * inv, acc.y * inv);
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

// ------------------------------------------------------------------ the fused z pass

template <int NTH>
__global__ void __launch_bounds__(kThreads) k_zpass(const __grid_constant__ ZParams P) {
  extern __shared__ float2 sm[];
  const int nzp = P.nzp, W = P.W;
  const int TS = W * nzp;                      // points per tile
  constexpr int NR1 = NTH > 6 ? NTH : 6;
  float2* tw = sm;                             // nzp
  float2* R1 = tw + nzp;                       // NR1 tiles: data, then S_post
  float2* R2 = R1 + NR1 * TS;                  // 3 tiles: mean, then mu_post
  float2* R3 = R2 + 3 * TS;                    // 1 tile: realisation output
  float2* SC = R3 + TS;                        // 1 tile: transform scratch
  __shared__ unsigned long long cnt[3];
  const int T = blockDim.x, tid = threadIdx.x;
  const int it = blockIdx.x % P.nIT;
  const int j = blockIdx.x / P.nIT;
  const int i0 = it * W;
  const int nw = min(W, P.cnxp - i0);
  const size_t kstride = (size_t)P.nyp * P.cnxp;
  const size_t base = (size_t)j * P.cnxp + i0;

  if (tid < 3) cnt[tid] = 0;
  for (int t = tid; t < nzp; t += T) tw[t] = P.twz[t];
  auto load_tile = [&](float2* dst, const float2* g) {
    for (int e = tid; e < TS; e += T) {
      int k = e / W, w = e - k * W;
      dst[e] = (w < nw) ? g[base + (size_t)k * kstride + w] : make_float2(0.f, 0.f);
    }
  };
  auto store_tile = [&](float2* g, const float2* src) {
    for (int e = tid; e < TS; e += T) {
      int k = e / W, w = e - k * W;
      if (w < nw) g[base + (size_t)k * kstride + w] = src[e];
    }
  };
#pragma unroll 1
  for (int l = 0; l < NTH; l++) load_tile(R1 + l * TS, P.data[l]);
#pragma unroll 1
  for (int a = 0; a < 3; a++) load_tile(R2 + a * TS, P.mean[a]);
  __syncthreads();
  // forward z transform of the inputs (completes FFTGrid::fftInPlace)
#pragma unroll 1
  for (int l = 0; l < NTH; l++) fft_lines<false>(R1 + l * TS, SC, W, 1, W, P.zp, tw, -1.f);
#pragma unroll 1
  for (int a = 0; a < 3; a++) fft_lines<false>(R2 + a * TS, SC, W, 1, W, P.zp, tw, -1.f);

  // ---- per-bin posterior (src/avoinversion.cpp:1016-1082)
  unsigned long long n_inv = 0, n_fail = 0;
  for (int b = tid; b < TS; b += T) {
    int k = b / W, w = b - k * W;
    if (w >= nw) continue;
    int i = i0 + w;
    size_t gidx = base + (size_t)k * kstride + w;
    float S[6], lam;
    if (P.separable) {
      float2 cx = __ldg(P.cxy + (size_t)j * P.cnxp + i);
      float2 c_t = __ldg(P.ct + k);
      float rho = fabsf(cx.x * c_t.x - cx.y * c_t.y);
#pragma unroll
      for (int q = 0; q < 6; q++) S[q] = P.pv[q] * rho;
      lam = fabsf(cx.x);
    } else {
      // getNextParameterCovariance: |Re/pv| pv (no division when pv == 0)
#pragma unroll
      for (int q = 0; q < 6; q++) {
        float re = P.cov[q][gidx].x;
        float pv = P.pv[q];
        if (pv != 0.f) re = re / pv;
        S[q] = fabsf(re) * pv;
      }
      lam = fabsf(P.errspec[gidx].x);
    }
    float2 mu[3], d[NTH];
#pragma unroll
    for (int a = 0; a < 3; a++) mu[a] = R2[a * TS + b];
#pragma unroll
    for (int l = 0; l < NTH; l++) d[l] = R1[l * TS + b];
    BinOut o;
    bool inv = P.kz.inv[k] != 0;
    bool ok = false;
    if (inv) {
      n_inv++;
      ok = bin_posterior<NTH>(P, k, S, lam, mu, d, o);
      if (!ok) n_fail++;
    }
    if (!ok) {
#pragma unroll
      for (int a = 0; a < 3; a++) o.mu[a] = mu[a];
#pragma unroll
      for (int q = 0; q < 6; q++) o.sp[q] = make_float2(S[q], 0.f);
#pragma unroll
      for (int l = 0; l < NTH; l++) d[l] = R1[l * TS + b];
    }
    if (P.keep_resid) {
#pragma unroll
      for (int l = 0; l < NTH; l++) P.data[l][gidx] = d[l];
    }
#pragma unroll
    for (int a = 0; a < 3; a++) R2[a * TS + b] = o.mu[a];
#pragma unroll
    for (int q = 0; q < 6; q++) R1[q * TS + b] = o.sp[q];
  }
  __syncthreads();

  // ---- realisations (src/avoinversion.cpp:1401-1511), spectral sum with the mean
  unsigned long long n_zero = 0;
#pragma unroll 1
  for (int s = 0; s < P.nsim; s++) {
#pragma unroll 1
    for (int a = 0; a < 3; a++) {
      for (int b = tid; b < TS; b += T) {
        int k = b / W, w = b - k * W;
        float2 out = make_float2(0.f, 0.f);
        if (w < nw) {
          int i = i0 + w;
          size_t gidx = base + (size_t)k * kstride + w;
          float2 C[3][3];
          C[0][0] = R1[0 * TS + b];
          C[1][1] = R1[1 * TS + b];
          C[2][2] = R1[2 * TS + b];
          float2 c01 = R1[3 * TS + b], c02 = R1[4 * TS + b], c12 = R1[5 * TS + b];
          C[1][0] = make_float2(c01.x, -c01.y);
          C[2][0] = make_float2(c02.x, -c02.y);
          C[2][1] = make_float2(c12.x, -c12.y);
          C[0][1] = c01; C[0][2] = c02; C[1][2] = c12;
          float2 z[3];
#pragma unroll
          for (int c = 0; c < 3; c++) {
            if (c > a) { z[c] = make_float2(0.f, 0.f); continue; }
            z[c] = P.host_noise ? P.noise[3 * s + c][gidx]
                                : device_noise(P.seed, 3 * s + c, i, j, k, P.nyp, nzp, P.cnxp, P.nxp_even);
          }
          float2 seed = make_float2(0.f, 0.f);
          if (chol_ref<3>(C)) {
#pragma unroll
            for (int c = 0; c < 3; c++)
              if (c <= a) seed = cadd(seed, cmul(C[a][c], z[c]));
          } else if (a == 0) {
            n_zero++;
          }
          out = cadd(R2[a * TS + b], seed);
        }
        R3[b] = out;
      }
      __syncthreads();
      fft_lines<false>(R3, SC, W, 1, W, P.zp, tw, 1.f);
      store_tile(P.sim[3 * s + a], R3);
      __syncthreads();
    }
  }

  // ---- inverse z transform of posterior covariance and mean
#pragma unroll 1
  for (int q = 0; q < 6; q++) {
    fft_lines<false>(R1 + q * TS, SC, W, 1, W, P.zp, tw, 1.f);
    store_tile(P.cov[q], R1 + q * TS);
  }
#pragma unroll 1
  for (int a = 0; a < 3; a++) {
    fft_lines<false>(R2 + a * TS, SC, W, 1, W, P.zp, tw, 1.f);
    store_tile(P.mean[a], R2 + a * TS);
  }

  // counters
  for (int off = 16; off > 0; off >>= 1) {
    n_inv += __shfl_down_sync(0xffffffffu, n_inv, off);
    n_fail += __shfl_down_sync(0xffffffffu, n_fail, off);
    n_zero += __shfl_down_sync(0xffffffffu, n_zero, off);
  }
  if ((tid & 31) == 0) {
    atomicAdd(&cnt[0], n_inv);
    atomicAdd(&cnt[1], n_fail);
    atomicAdd(&cnt[2], n_zero);
  }
  __syncthreads();
  if (tid == 0 && P.counters) {
    atomicAdd(P.counters + 0, cnt[0]);
    atomicAdd(P.counters + 1, cnt[1]);
    atomicAdd(P.counters + 2, cnt[2]);
  }
}

// ------------------------------------------------------------------ launchers

size_t zpass_smem_bytes(int W, int nzp, int nth) {
  int nr1 = nth > 6 ? nth : 6;
  return sizeof(float2) * ((size_t)nzp + (size_t)(nr1 + 3 + 2) * W * nzp);
}

template <int NTH>
static cudaError_t launch_zpass_t(const ZParams& zp, cudaStream_t st) {
  size_t smem = zpass_smem_bytes(zp.W, zp.nzp, zp.nth);
  cudaError_t e = cudaFuncSetAttribute(k_zpass<NTH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)(zp.nIT * zp.nyp));
  k_zpass<NTH><<<grid, kThreads, smem, st>>>(zp);
  return cudaGetLastError();
}

cudaError_t launch_zpass(const ZParams& zp, cudaStream_t st, int* nlaunch) {
  if (nlaunch) (*nlaunch)++;
  switch (zp.nth) {
    case 1: return launch_zpass_t<1>(zp, st);
    case 2: return launch_zpass_t<2>(zp, st);
    case 3: return launch_zpass_t<3>(zp, st);
    case 4: return launch_zpass_t<4>(zp, st);
    case 5: return launch_zpass_t<5>(zp, st);
    case 6: return launch_zpass_t<6>(zp, st);
    case 7: return launch_zpass_t<7>(zp, st);
    case 8: return launch_zpass_t<8>(zp, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace crava
