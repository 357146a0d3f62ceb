// Local-noise shrinkage of the posterior (sm_100a): AVOInversion::correctVpVsRho with
// newPosteriorCovPointwise (src/avoinversion.cpp:2028-2302) and the local-noise mixing of the
// realisations in AVOInversion::simulate (src/avoinversion.cpp:1485-1504).
//
// Per trace (i, j) the angle stacks' noise is scaled by s_l = scale_l(i, j) / min scale_l; with
// D = diag(sqrt(s)), the local data covariance is  M = G Sm G^T + D SigmaTheta D  and
//   delta = Sm G^T M^-1 G Sm           (variance explained by the data, 3 x 3)
//   smd   = Sm - delta                 (the local posterior covariance)
//   S     = delta^1/2 (Sm - Smd)^-1/2   (map of the posterior deviation from the prior mean)
//   Msim  = smd^1/2 Smd^-1/2           (map of a realisation's deviation from the posterior)
// with G, Sm = priorVar0, Smd = postVar0 and the job-constant matrices from the host.  Every
// voxel of the trace then becomes
//   post' = mean + S (post - mean),   sim' = post' + Msim (sim - post)
// (the reference adds the corrected posterior to the mixed noise field; here each realisation
// already holds post + noise).  Square roots are spectral (eigenvalues <= 0 dropped), so the
// eigenvectors' order and signs do not enter.  The reference inverts M through its
// eigen-decomposition, dropping eigenvalues below 1e-8; M is symmetric positive definite for
// positive scales, and the Cholesky solve used here equals that inverse wherever all its
// eigenvalues exceed the threshold.
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"

namespace crava {

namespace {

// Cyclic Jacobi eigen-decomposition of a symmetric 3 x 3 matrix in double: a = V diag(w) V^T.
__device__ void sym3_eig(double (&a)[3][3], double (&w)[3], double (&v)[3][3]) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int k = 0; k < 3; k++) v[i][k] = i == k ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 12; sweep++) {
    const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    const double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off <= 1e-30 * diag || off == 0.0) break;
#pragma unroll
    for (int pq = 0; pq < 3; pq++) {
      const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
      const double apq = a[p][q];
      if (apq == 0.0) continue;
      const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
      const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      const double c = rsqrt(t * t + 1.0), s = t * c;
#pragma unroll
      for (int k = 0; k < 3; k++) {   // A <- A R
        const double akp = a[k][p], akq = a[k][q];
        a[k][p] = c * akp - s * akq;
        a[k][q] = s * akp + c * akq;
        const double vkp = v[k][p], vkq = v[k][q];
        v[k][p] = c * vkp - s * vkq;
        v[k][q] = s * vkp + c * vkq;
      }
#pragma unroll
      for (int k = 0; k < 3; k++) {   // A <- R^T A
        const double apk = a[p][k], aqk = a[q][k];
        a[p][k] = c * apk - s * aqk;
        a[q][k] = s * apk + c * aqk;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 3; i++) w[i] = a[i][i];
}

// Spectral square root of a symmetric 3 x 3 matrix, eigenvalues <= 0 dropped.
__device__ void sym3_sqrt(const double (&m)[3][3], double (&r)[3][3]) {
  double a[3][3], w[3], v[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int k = 0; k < 3; k++) a[i][k] = 0.5 * (m[i][k] + m[k][i]);
  sym3_eig(a, w, v);
  double sw[3];
#pragma unroll
  for (int i = 0; i < 3; i++) sw[i] = w[i] > 0.0 ? sqrt(w[i]) : 0.0;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int k = 0; k < 3; k++) r[i][k] = v[i][0] * sw[0] * v[k][0] + v[i][1] * sw[1] * v[k][1] + v[i][2] * sw[2] * v[k][2];
}

}  // namespace

// Two kernels: k_local_noise_maps computes every trace's two maps (one thread per trace, the
// double-precision solves) into a table of 18 floats per trace; k_local_noise_apply streams
// the voxels through them, a block of 32 consecutive traces (threadIdx.x) x 8 slices of their
// z range (threadIdx.y), so a warp reads 32 consecutive x of one plane and each trace has
// eight independent streams in flight.
constexpr int kLnTraces = 32, kLnSlices = 8;

template <int NTH>
__device__ __forceinline__ void trace_maps(const LocalNoiseParams& P, int i, int j, float (&Sf)[3][3],
                                           float (&Mf)[3][3]);

template <int NTH>
__global__ void __launch_bounds__(128) k_local_noise_maps(const __grid_constant__ LocalNoiseParams P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= P.nx || j >= P.ny) return;
  float Sf[3][3], Mf[3][3];
  trace_maps<NTH>(P, i, j, Sf, Mf);
  float* m = P.maps + 18 * ((size_t)j * P.nx + i);
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      m[3 * a + b] = Sf[a][b];
      m[9 + 3 * a + b] = Mf[a][b];
    }
}

__global__ void __launch_bounds__(kLnTraces * kLnSlices) k_local_noise_apply(const __grid_constant__ LocalNoiseParams P) {
  const int i = blockIdx.x * kLnTraces + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= P.nx || j >= P.ny) return;
  float S[3][3], Ms[3][3];
  const float* m = P.maps + 18 * ((size_t)j * P.nx + i);
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      S[a][b] = __ldg(m + 3 * a + b);
      Ms[a][b] = __ldg(m + 9 + 3 * a + b);
    }
  const size_t plane = (size_t)P.rnxp * P.nyp;
  const size_t t0 = (size_t)j * P.rnxp + i;
  for (int k = threadIdx.y; k < P.nz; k += kLnSlices) {
    const size_t o = t0 + (size_t)k * plane;
    float pm[3], pr[3], pn[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      pm[a] = P.prior_mean[a][o];
      pr[a] = P.post[a][o];
    }
    const float dv = pr[0] - pm[0], ds = pr[1] - pm[1], dr = pr[2] - pm[2];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      pn[a] = pm[a] + S[a][0] * dv + S[a][1] * ds + S[a][2] * dr;
      P.post[a][o] = pn[a];
    }
    for (int s = 0; s < P.nsim; s++) {
      float n3[3];
#pragma unroll
      for (int a = 0; a < 3; a++) n3[a] = P.sim[3 * s + a][o] - pr[a];
#pragma unroll
      for (int a = 0; a < 3; a++) P.sim[3 * s + a][o] = pn[a] + (Ms[a][0] * n3[0] + Ms[a][1] * n3[1] + Ms[a][2] * n3[2]);
    }
  }
}

// The trace's maps S and Msim (double arithmetic, rounded to float for the voxel loop).
template <int NTH>
__device__ __forceinline__ void trace_maps(const LocalNoiseParams& P, int i, int j, float (&Sf)[3][3],
                                           float (&Mf)[3][3]) {
  // M = G Sm G^T + D SigmaTheta D, then delta = B^T M^-1 B with B = G Sm
  double d[NTH];
#pragma unroll
  for (int l = 0; l < NTH; l++) d[l] = sqrt((double)P.scale[(size_t)l * P.nx * P.ny + (size_t)j * P.nx + i] * P.inv_min[l]);
  double L[NTH][NTH];
#pragma unroll
  for (int l = 0; l < NTH; l++)
#pragma unroll
    for (int m = 0; m <= l; m++) L[l][m] = P.gsg[l][m] + d[l] * P.sth[l][m] * d[m];
  bool ok = true;
#pragma unroll
  for (int c = 0; c < NTH; c++) {   // Cholesky, lower triangle in place
    double s = L[c][c];
#pragma unroll
    for (int k = 0; k < c; k++) s -= L[c][k] * L[c][k];
    if (!(s > 0.0)) ok = false;
    const double lc = sqrt(fmax(s, 1e-300));
    L[c][c] = lc;
#pragma unroll
    for (int r = c + 1; r < NTH; r++) {
      double t = L[r][c];
#pragma unroll
      for (int k = 0; k < c; k++) t -= L[r][k] * L[c][k];
      L[r][c] = t / lc;
    }
  }
  double delta[3][3];
  {
    double X[NTH][3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
#pragma unroll
      for (int r = 0; r < NTH; r++) {   // forward: L y = B
        double t = P.b[r][a];
#pragma unroll
        for (int k = 0; k < r; k++) t -= L[r][k] * X[k][a];
        X[r][a] = t / L[r][r];
      }
    }
    // delta = (L^-1 B)^T (L^-1 B)
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) {
        double t = 0;
#pragma unroll
        for (int r = 0; r < NTH; r++) t += X[r][a] * X[r][b];
        delta[a][b] = t;
      }
  }
  if (!ok) {   // a scale that leaves M singular: no correction of this trace
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) delta[a][b] = 0.0;
  }
  double smd[3][3], rs[3][3], rd[3][3], S[3][3], Ms[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) smd[a][b] = P.sm[a][b] - delta[a][b];
  sym3_sqrt(smd, rs);
  sym3_sqrt(delta, rd);
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      S[a][b] = rd[a][0] * P.sdel[0][b] + rd[a][1] * P.sdel[1][b] + rd[a][2] * P.sdel[2][b];
      Ms[a][b] = rs[a][0] * P.smdi[0][b] + rs[a][1] * P.smdi[1][b] + rs[a][2] * P.smdi[2][b];
    }
  if (!ok) {   // keep the trace as it is
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) S[a][b] = Ms[a][b] = a == b ? 1.0 : 0.0;
  }
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      Sf[a][b] = (float)S[a][b];
      Mf[a][b] = (float)Ms[a][b];
    }
}

cudaError_t launch_local_noise(const LocalNoiseParams& P, cudaStream_t st, int* nlaunch) {
  if (!P.maps) return cudaErrorInvalidValue;
  const dim3 mgrid((unsigned)((P.nx + 127) / 128), (unsigned)P.ny);
  switch (P.nth) {
#define LN_CASE(n) \
  case n: k_local_noise_maps<n><<<mgrid, 128, 0, st>>>(P); break;
    LN_CASE(1) LN_CASE(2) LN_CASE(3) LN_CASE(4) LN_CASE(5) LN_CASE(6) LN_CASE(7) LN_CASE(8)
#undef LN_CASE
    default: return cudaErrorInvalidValue;
  }
  const dim3 grid((unsigned)((P.nx + kLnTraces - 1) / kLnTraces), (unsigned)P.ny);
  k_local_noise_apply<<<grid, dim3(kLnTraces, kLnSlices), 0, st>>>(P);
  if (nlaunch) (*nlaunch) += 2;
  return cudaGetLastError();
}

}  // namespace crava
