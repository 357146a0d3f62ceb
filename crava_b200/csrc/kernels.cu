// Transform kernels of the FFT-domain AVO inversion hot path (sm_100a).
//
//   k_x_r2c      forward transform along x of every row: real -> half spectrum, in place
//                (first pass of FFTGrid::fftInPlace, src/fftgrid.cpp:1587-1612)
//   k_x_c2r      inverse along x: half spectrum -> real, scaled (last pass of
//                FFTGrid::invFFTInPlace, src/fftgrid.cpp:1615-1643)
//   k_line_fft   complex transform along a strided axis (y, or z for prior grids)
//   (the fused pencil pass is in zpass.cu)
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdlib>

#include "fft_core.cuh"
#include "kernels.cuh"

namespace crava {

constexpr int kThreads = 256;

// ------------------------------------------------------------------ x transforms
//
// Even nxp (h = nxp/2): a row x is read as h complex values z[m] = x[2m] + i x[2m+1]
// (the same bytes), transformed with a length-h complex FFT, and split into the half
// spectrum with w = e^{-2 pi i/nxp}:
//   E = (Z[k] + conj Z[h-k]) / 2,  O = (Z[k] - conj Z[h-k]) / 2i,
//   X[k] = E + w^k O,  X[h-k] = conj(E - w^k O),  X[0] = Re+Im Z[0], X[h] = Re-Im Z[0].
// The inverse runs the same steps backwards:
//   P = X[k] + conj X[h-k], Q = (X[k] - conj X[h-k]) conj(w^k),
//   Z'[k] = P + iQ, Z'[h-k] = conj P + i conj Q, Z'[0] from Re X[0], Re X[h] only
// (a real-output inverse has no slot for Im X[0], Im X[h]), then a length-h inverse
// FFT gives nxp * (x[2m] + i x[2m+1]).  Odd nxp uses a full-length complex transform.

__global__ void __launch_bounds__(512, 2) k_x_r2c(const __grid_constant__ GridSet gs, int nxp, int rows, int rpc,
                                                const __grid_constant__ LinePlan pl, const float2* __restrict__ twg,
                                                const float2* __restrict__ twn) {
  extern __shared__ float2 sm[];
  const int T = blockDim.x, tid = threadIdx.x;
  const bool even = (nxp & 1) == 0;
  const int n = even ? nxp / 2 : nxp;       // transform length
  const int cnxp = nxp / 2 + 1;
  const float rn = __frcp_rn((float)n);
  float2* tw = sm;                          // n
  float2* twh = tw + n;                     // nxp/2 (even only): e^{-2 pi i k / nxp}
  float2* buf = twh + (even ? nxp / 2 : 0);
  float2* scr = buf + rpc * n;
  float* g = gs.p[blockIdx.y];
  const float scale = gs.scale[blockIdx.y];
  const int row0 = blockIdx.x * rpc;
  const int nr = min(rpc, rows - row0);
  for (int t = tid; t < n; t += T) tw[t] = twg[t];
  if (even)
    for (int t = tid; t < nxp / 2; t += T) twh[t] = twn[t];
  if (even) {
    const float2* src = reinterpret_cast<const float2*>(gs.src[blockIdx.y]) + (size_t)row0 * cnxp;
    for (int e = tid; e < nr * n; e += T) {
      int m;
      int r = fdivmod(e, n, rn, m);
      float2 v = src[(size_t)r * cnxp + m];
      buf[e] = make_float2(v.x * scale, v.y * scale);
    }
  } else {
    const float* src = gs.src[blockIdx.y] + (size_t)row0 * 2 * cnxp;
    for (int e = tid; e < nr * n; e += T) {
      int p;
      int r = fdivmod(e, n, rn, p);
      buf[e] = make_float2(src[(size_t)r * 2 * cnxp + p] * scale, 0.f);
    }
  }
  __syncthreads();
  fft_lines<false, -1, false>(buf, scr, nr, n, 1, pl, tw);
  float2* dst = reinterpret_cast<float2*>(g) + (size_t)row0 * cnxp;
  if (even) {
    const int h = n, np = h / 2 + 1;  // pairs (k, h-k), k = 0..h/2
    const float rnp = __frcp_rn((float)np);
    for (int e = tid; e < nr * np; e += T) {
      int k;
      int r = fdivmod(e, np, rnp, k);
      const float2* Z = buf + r * h;
      float2* X = dst + (size_t)r * cnxp;
      if (k == 0) {
        float2 z0 = Z[0];
        X[0] = make_float2(z0.x + z0.y, 0.f);
        X[h] = make_float2(z0.x - z0.y, 0.f);
        continue;
      }
      float2 A = Z[k], Bc = Z[h - k];  // B = conj(Bc)
      float2 E = make_float2(0.5f * (A.x + Bc.x), 0.5f * (A.y - Bc.y));
      // O = (A - B) / 2i = -i (A - B) / 2
      float2 D = make_float2(A.x - Bc.x, A.y + Bc.y);
      float2 O = make_float2(0.5f * D.y, -0.5f * D.x);
      float2 t = cmul(twh[k], O);
      X[k] = cadd(E, t);
      if (2 * k != h) {
        float2 m = csub(E, t);
        X[h - k] = make_float2(m.x, -m.y);
      }
    }
  } else {
    const float rc = __frcp_rn((float)cnxp);
    for (int e = tid; e < nr * cnxp; e += T) {
      int p;
      int r = fdivmod(e, cnxp, rc, p);
      dst[e] = buf[r * n + p];
    }
  }
}

__global__ void __launch_bounds__(512, 2) k_x_c2r(const __grid_constant__ GridSet gs, int nxp, int rows, int rpc,
                                                const __grid_constant__ LinePlan pl, const float2* __restrict__ twg,
                                                const float2* __restrict__ twn) {
  extern __shared__ float2 sm[];
  const int T = blockDim.x, tid = threadIdx.x;
  const bool even = (nxp & 1) == 0;
  const int n = even ? nxp / 2 : nxp;
  const int cnxp = nxp / 2 + 1;
  const float rn = __frcp_rn((float)n);
  float2* tw = sm;
  float2* twh = tw + n;
  float2* buf = twh + (even ? nxp / 2 : 0);
  float2* scr = buf + rpc * n;
  float* g = gs.p[blockIdx.y];
  const float scale = gs.scale[blockIdx.y];
  const int row0 = blockIdx.x * rpc;
  const int nr = min(rpc, rows - row0);
  for (int t = tid; t < n; t += T) tw[t] = twg[t];
  if (even)
    for (int t = tid; t < nxp / 2; t += T) twh[t] = twn[t];
  __syncthreads();
  const float2* src = reinterpret_cast<const float2*>(g) + (size_t)row0 * cnxp;
  if (even) {
    const int h = n, np = h / 2 + 1;
    const float rnp = __frcp_rn((float)np);
    for (int e = tid; e < nr * np; e += T) {
      int k;
      int r = fdivmod(e, np, rnp, k);
      const float2* X = src + (size_t)r * cnxp;
      float2* Z = buf + r * h;
      if (k == 0) {
        float a = X[0].x, b = X[h].x;
        Z[0] = make_float2(a + b, a - b);
        continue;
      }
      float2 xk = X[k], xm = X[h - k];
      float2 P = make_float2(xk.x + xm.x, xk.y - xm.y);       // X[k] + conj X[h-k]
      float2 M = make_float2(xk.x - xm.x, xk.y + xm.y);       // X[k] - conj X[h-k]
      float2 w = twh[k];
      float2 Q = make_float2(M.x * w.x + M.y * w.y, M.y * w.x - M.x * w.y);  // M conj(w)
      Z[k] = make_float2(P.x - Q.y, P.y + Q.x);               // P + iQ
      if (2 * k != h) Z[h - k] = make_float2(P.x + Q.y, -P.y + Q.x);  // conj P + i conj Q
    }
  } else {
    // Hermitian extension; Im X[0] (and Im X[nxp/2]) do not enter a real-output inverse
    for (int e = tid; e < nr * n; e += T) {
      int p;
      int r = fdivmod(e, n, rn, p);
      float2 v;
      if (p < cnxp) {
        v = src[(size_t)r * cnxp + p];
        if (p == 0) v.y = 0.f;
      } else {
        v = src[(size_t)r * cnxp + (n - p)];
        v.y = -v.y;
      }
      buf[e] = v;
    }
  }
  __syncthreads();
  fft_lines<false, 1, false>(buf, scr, nr, n, 1, pl, tw);
  if (even) {
    float2* dst = reinterpret_cast<float2*>(g) + (size_t)row0 * cnxp;
    const float rc = __frcp_rn((float)cnxp);
    for (int e = tid; e < nr * cnxp; e += T) {
      int m;
      int r = fdivmod(e, cnxp, rc, m);
      float2 v = (m < n) ? buf[r * n + m] : make_float2(0.f, 0.f);
      dst[e] = make_float2(v.x * scale, v.y * scale);
    }
  } else {
    float* dst = g + (size_t)row0 * 2 * cnxp;
    const float r2c = __frcp_rn((float)(2 * cnxp));
    for (int e = tid; e < nr * 2 * cnxp; e += T) {
      int p;
      int r = fdivmod(e, 2 * cnxp, r2c, p);
      dst[e] = (p < n) ? buf[r * n + p].x * scale : 0.f;
    }
  }
}

// ------------------------------------------------------------------ strided line transform

__global__ void __launch_bounds__(512, 2) k_line_fft(const __grid_constant__ GridSet gs, int ni, int n, size_t pstride, int no,
                                                   size_t ostride, int W, int nIT, const __grid_constant__ LinePlan pl,
                                                   const float2* __restrict__ twg, float sign) {
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* buf = sm + n;
  float2* scr = buf + W * n;
  const int T = blockDim.x, tid = threadIdx.x;
  const int it = blockIdx.x % nIT;
  const int o = blockIdx.x / nIT;
  const int i0 = it * W;
  const int nw = min(W, ni - i0);
  float2* g = reinterpret_cast<float2*>(gs.p[blockIdx.y]) + (size_t)o * ostride + i0;
  for (int t = tid; t < n; t += T) tw[t] = twg[t];
  const int lw = 31 - __clz(W);  // W is a power of two
  for (int e = tid; e < n * W; e += T) {
    int p = e >> lw, w = e & (W - 1);
    buf[e] = (w < nw) ? g[(size_t)p * pstride + w] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  if (sign < 0.f) fft_lines<true, -1, false>(buf, scr, W, 1, W, pl, tw);
  else fft_lines<true, 1, false>(buf, scr, W, 1, W, pl, tw);
  for (int e = tid; e < n * W; e += T) {
    int p = e >> lw, w = e & (W - 1);
    if (w < nw) g[(size_t)p * pstride + w] = buf[e];
  }
}

// ------------------------------------------------------------------ pipelined transforms
//
// Persistent forms of the transforms above: each CTA walks work units (row chunks, or
// column tiles) with a stride of the grid size, and copies the next unit's input into a
// second shared buffer with cp.async while it transforms the current one, so that loads
// are in flight during the arithmetic.  Same arithmetic as the one-unit kernels.



// Even nxp only.  Unit u = (grid u / nchunk, rows [c rpc, c rpc + rpc)).
__global__ void __launch_bounds__(512, 2) k_x_r2c_pipe(const __grid_constant__ GridSet gs, int nxp, int rows, int rpc,
                                                     int nchunk, const __grid_constant__ LinePlan pl,
                                                     const float2* __restrict__ twg, const float2* __restrict__ twn) {
  extern __shared__ float2 sm[];
  const int T = blockDim.x, tid = threadIdx.x;
  const int h = nxp / 2, cnxp = h + 1, np = h / 2 + 1;
  const float rh = __frcp_rn((float)h), rnp = __frcp_rn((float)np), rchunk = __frcp_rn((float)nchunk);
  float2* tw = sm;
  float2* twh = tw + h;
  float2* const tile0 = twh + h;
  float2* const tile1 = tile0 + rpc * h;
  float2* scr = tile1 + rpc * h;
  for (int t = tid; t < h; t += T) {
    tw[t] = twg[t];
    twh[t] = twn[t];
  }
  const int units = gs.n * nchunk;
  auto issue = [&](int u, float2* dst) {
    int c;
    const int gi = fdivmod(u, nchunk, rchunk, c);
    const int row0 = c * rpc, nr = min(rpc, rows - row0);
    const float2* src = reinterpret_cast<const float2*>(gs.src[gi]) + (size_t)row0 * cnxp;
    const uint32_t d = smem_addr(dst);
    for (int e = tid; e < nr * h; e += T) {
      int m;
      const int r = fdivmod(e, h, rh, m);
      cp_async8(d + 8u * (uint32_t)e, src + (size_t)r * cnxp + m);
    }
  };
  int i = 0;
  if ((int)blockIdx.x < units) issue(blockIdx.x, tile0);
  cp_async_commit();
  for (int u = blockIdx.x; u < units; u += gridDim.x, i ^= 1) {
    if (u + (int)gridDim.x < units) issue(u + gridDim.x, i ? tile0 : tile1);
    cp_async_commit();
    cp_async_wait_1();
    __syncthreads();
    int c;
    const int gi = fdivmod(u, nchunk, rchunk, c);
    const int row0 = c * rpc, nr = min(rpc, rows - row0);
    float2* buf = i ? tile1 : tile0;
    fft_lines<false, -1, false>(buf, scr, nr, h, 1, pl, tw);
    const float scale = gs.scale[gi];
    float2* dst = reinterpret_cast<float2*>(gs.p[gi]) + (size_t)row0 * cnxp;
    for (int e = tid; e < nr * np; e += T) {
      int k;
      const int r = fdivmod(e, np, rnp, k);
      const float2* Z = buf + r * h;
      float2* X = dst + (size_t)r * cnxp;
      if (k == 0) {
        const float2 z0 = Z[0];
        X[0] = make_float2(scale * (z0.x + z0.y), 0.f);
        X[h] = make_float2(scale * (z0.x - z0.y), 0.f);
        continue;
      }
      const float2 A = Z[k], Bc = Z[h - k];
      const float2 E = make_float2(0.5f * (A.x + Bc.x), 0.5f * (A.y - Bc.y));
      const float2 D = make_float2(A.x - Bc.x, A.y + Bc.y);
      const float2 O = make_float2(0.5f * D.y, -0.5f * D.x);
      const float2 t = cmul(twh[k], O);
      const float2 xk = cadd(E, t);
      X[k] = make_float2(scale * xk.x, scale * xk.y);
      if (2 * k != h) {
        const float2 m = csub(E, t);
        X[h - k] = make_float2(scale * m.x, -scale * m.y);
      }
    }
    __syncthreads();  // the buffer is refilled by the prefetch of the next iteration but one
  }
  cp_async_wait_0();
}

// Even nxp only.  The raw half-spectrum rows land in tile0/tile1; the merge step writes the
// length-h complex input of the inverse into buf.
__global__ void __launch_bounds__(512, 2) k_x_c2r_pipe(const __grid_constant__ GridSet gs, int nxp, int rows, int rpc,
                                                     int nchunk, const __grid_constant__ LinePlan pl,
                                                     const float2* __restrict__ twg, const float2* __restrict__ twn) {
  extern __shared__ float2 sm[];
  const int T = blockDim.x, tid = threadIdx.x;
  const int h = nxp / 2, cnxp = h + 1, np = h / 2 + 1;
  const float rc = __frcp_rn((float)cnxp), rnp = __frcp_rn((float)np), rchunk = __frcp_rn((float)nchunk);
  float2* tw = sm;
  float2* twh = tw + h;
  float2* const tile0 = twh + h;
  float2* const tile1 = tile0 + rpc * cnxp;
  float2* buf = tile1 + rpc * cnxp;
  float2* scr = buf + rpc * h;
  for (int t = tid; t < h; t += T) {
    tw[t] = twg[t];
    twh[t] = twn[t];
  }
  const int units = gs.n * nchunk;
  auto issue = [&](int u, float2* dst) {
    int c;
    const int gi = fdivmod(u, nchunk, rchunk, c);
    const int row0 = c * rpc, nr = min(rpc, rows - row0);
    const float2* src = reinterpret_cast<const float2*>(gs.p[gi]) + (size_t)row0 * cnxp;
    const uint32_t d = smem_addr(dst);
    for (int e = tid; e < nr * cnxp; e += T) cp_async8(d + 8u * (uint32_t)e, src + e);
  };
  int i = 0;
  if ((int)blockIdx.x < units) issue(blockIdx.x, tile0);
  cp_async_commit();
  for (int u = blockIdx.x; u < units; u += gridDim.x, i ^= 1) {
    if (u + (int)gridDim.x < units) issue(u + gridDim.x, i ? tile0 : tile1);
    cp_async_commit();
    cp_async_wait_1();
    __syncthreads();
    int c;
    const int gi = fdivmod(u, nchunk, rchunk, c);
    const int row0 = c * rpc, nr = min(rpc, rows - row0);
    const float2* xin = i ? tile1 : tile0;
    for (int e = tid; e < nr * np; e += T) {
      int k;
      const int r = fdivmod(e, np, rnp, k);
      const float2* X = xin + r * cnxp;
      float2* Z = buf + r * h;
      if (k == 0) {
        const float a = X[0].x, b = X[h].x;
        Z[0] = make_float2(a + b, a - b);
        continue;
      }
      const float2 xk = X[k], xm = X[h - k];
      const float2 P = make_float2(xk.x + xm.x, xk.y - xm.y);
      const float2 M = make_float2(xk.x - xm.x, xk.y + xm.y);
      const float2 w = twh[k];
      const float2 Q = make_float2(M.x * w.x + M.y * w.y, M.y * w.x - M.x * w.y);
      Z[k] = make_float2(P.x - Q.y, P.y + Q.x);
      if (2 * k != h) Z[h - k] = make_float2(P.x + Q.y, -P.y + Q.x);
    }
    __syncthreads();
    fft_lines<false, 1, false>(buf, scr, nr, h, 1, pl, tw);
    const float scale = gs.scale[gi];
    float2* dst = reinterpret_cast<float2*>(gs.p[gi]) + (size_t)row0 * cnxp;
    for (int e = tid; e < nr * cnxp; e += T) {
      int m;
      const int r = fdivmod(e, cnxp, rc, m);
      const float2 v = (m < h) ? buf[r * h + m] : make_float2(0.f, 0.f);
      dst[e] = make_float2(v.x * scale, v.y * scale);
    }
    __syncthreads();
  }
  cp_async_wait_0();
}

// Unit u = (grid, outer index o, column tile it): W consecutive columns i0.. of the
// n points at stride pstride; columns beyond ni are zero-filled and not stored.
template <int DIR>
__global__ void __launch_bounds__(512, 2) k_line_pipe(const __grid_constant__ GridSet gs, int ni, int n, size_t pstride,
                                                    int no, size_t ostride, int W, int nIT,
                                                    const __grid_constant__ LinePlan pl,
                                                    const float2* __restrict__ twg) {
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* const tile0 = sm + n;
  float2* const tile1 = tile0 + W * n;
  float2* scr = tile1 + W * n;
  const int T = blockDim.x, tid = threadIdx.x;
  for (int t = tid; t < n; t += T) tw[t] = twg[t];
  const int lw = 31 - __clz(W);
  const int per_grid = nIT * no;
  const float rpg = __frcp_rn((float)per_grid), rit = __frcp_rn((float)nIT);
  const int units = gs.n * per_grid;
  auto locate = [&](int u, int& gi, int& i0, int& nw) -> float2* {
    int rem, it;
    gi = fdivmod(u, per_grid, rpg, rem);
    const int o = fdivmod(rem, nIT, rit, it);
    i0 = it * W;
    nw = min(W, ni - i0);
    return reinterpret_cast<float2*>(gs.p[gi]) + (size_t)o * ostride + i0;
  };
  auto issue = [&](int u, float2* dst) {
    int gi, i0, nw;
    const float2* g = locate(u, gi, i0, nw);
    const uint32_t d = smem_addr(dst);
    for (int e = tid; e < n * W; e += T) {
      const int p = e >> lw, w = e & (W - 1);
      const bool ok = w < nw;
      cp_async8_zfill(d + 8u * (uint32_t)e, ok ? g + (size_t)p * pstride + w : g, ok);
    }
  };
  int i = 0;
  if ((int)blockIdx.x < units) issue(blockIdx.x, tile0);
  cp_async_commit();
  for (int u = blockIdx.x; u < units; u += gridDim.x, i ^= 1) {
    if (u + (int)gridDim.x < units) issue(u + gridDim.x, i ? tile0 : tile1);
    cp_async_commit();
    cp_async_wait_1();
    __syncthreads();
    float2* buf = i ? tile1 : tile0;
    fft_lines<true, DIR, false>(buf, scr, W, 1, W, pl, tw);
    int gi, i0, nw;
    float2* g = locate(u, gi, i0, nw);
    for (int e = tid; e < n * W; e += T) {
      const int p = e >> lw, w = e & (W - 1);
      if (w < nw) g[(size_t)p * pstride + w] = buf[e];
    }
    __syncthreads();
  }
  cp_async_wait_0();
}

// ------------------------------------------------------------------ launchers

static int round_threads(int t) {
  t = (t + 31) / 32 * 32;
  return t < 64 ? 64 : t;
}

static bool pipe_enabled() { return tuned("pipe", -1, 1) != 0; }

// Persistent grid: resident CTAs of `fn` at (T, smem) on every SM of the current device,
// no more than the work units.
static cudaError_t persistent_grid(const void* fn, int T, size_t smem, int units, int* grid) {
  int dev = 0, nsm = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, T, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  *grid = std::max(1, std::min(units, per_sm * nsm));
  return cudaSuccess;
}

static cudaError_t launch_x(bool fwd, const GridSet& gs, int nxp, int rows, const LinePlan& pl, const float2* tw,
                            const float2* twn, cudaStream_t st, int* nlaunch) {
  const bool even = (nxp & 1) == 0;
  const int n = even ? nxp / 2 : nxp;
  if (even && four_step_supported(n)) return launch_x4(fwd, gs, nxp, rows, tw, twn, st, nlaunch);
  if (even && pipe_enabled()) {
    // rows per unit and threads: about 8 points per thread (schedule keys x_ppt, x_rpc)
    const int ppt = std::max(1, tuned("x_ppt", n, 8));
    const int rpc = std::max(1, tuned("x_rpc", n, std::max(1, std::min(64, 2048 / n))));
    const int T = std::min(512, round_threads((rpc * n + ppt - 1) / ppt));
    const int h = n, cnxp = h + 1;
    const size_t smem = fwd ? sizeof(float2) * (size_t)(2 * h + 3 * rpc * h)
                            : sizeof(float2) * (size_t)(2 * h + 2 * rpc * cnxp + 2 * rpc * h);
    const int nchunk = (rows + rpc - 1) / rpc;
    const void* fn = fwd ? (const void*)k_x_r2c_pipe : (const void*)k_x_c2r_pipe;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int grid = 0;
    if ((e = persistent_grid(fn, T, smem, gs.n * nchunk, &grid)) != cudaSuccess) return e;
    if (fwd) k_x_r2c_pipe<<<grid, T, smem, st>>>(gs, nxp, rows, rpc, nchunk, pl, tw, twn);
    else k_x_c2r_pipe<<<grid, T, smem, st>>>(gs, nxp, rows, rpc, nchunk, pl, tw, twn);
    if (nlaunch) (*nlaunch)++;
    return cudaGetLastError();
  }
  // rows per CTA and threads: about 16 points per thread (schedule key x_ppt1)
  const int ppt = std::max(1, tuned("x_ppt1", n, 16));
  int rpc = std::max(1, std::min(64, 2048 / n));
  int T = std::min(512, round_threads((rpc * n + ppt - 1) / ppt));
  size_t smem = sizeof(float2) * (size_t)(n + (even ? nxp / 2 : 0) + 2 * rpc * n);
  dim3 grid((rows + rpc - 1) / rpc, gs.n);
  const void* fn = fwd ? (const void*)k_x_r2c : (const void*)k_x_c2r;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  if (fwd) k_x_r2c<<<grid, T, smem, st>>>(gs, nxp, rows, rpc, pl, tw, twn);
  else k_x_c2r<<<grid, T, smem, st>>>(gs, nxp, rows, rpc, pl, tw, twn);
  if (nlaunch) (*nlaunch)++;
  return cudaGetLastError();
}

cudaError_t launch_x_r2c(const GridSet& gs, int nxp, int rows, const LinePlan& pl, const float2* tw,
                         const float2* twn, cudaStream_t st, int* nlaunch) {
  return launch_x(true, gs, nxp, rows, pl, tw, twn, st, nlaunch);
}

cudaError_t launch_x_c2r(const GridSet& gs, int nxp, int rows, const LinePlan& pl, const float2* tw,
                         const float2* twn, cudaStream_t st, int* nlaunch) {
  return launch_x(false, gs, nxp, rows, pl, tw, twn, st, nlaunch);
}

cudaError_t launch_line_fft(const GridSet& gs, int ni, int n, size_t pstride, int no, size_t ostride,
                            const LinePlan& pl, const float2* tw, float sign, cudaStream_t st, int* nlaunch) {
  if (four_step_supported(n)) return launch_line4(gs, ni, n, pstride, no, ostride, tw, sign, st, nlaunch);
  int W = std::max(1, tuned("line_w", n, 16));
  while (W > 1 && W * n > 8192) W /= 2;
  while (W > 1 && W / 2 >= ni) W /= 2;  // power of two, not wider than needed
  const int tdiv = std::max(1, tuned("line_tdiv", n, 16));
  int T = std::min(512, round_threads((W * n + tdiv - 1) / tdiv));
  int nIT = (ni + W - 1) / W;
  // the pipelined form measured slower for column tiles (fewer resident CTAs): opt-in
  const bool line_pipe = tuned("line_pipe", n, 0) != 0;
  if (line_pipe) {
    const size_t smem = sizeof(float2) * (size_t)(n + 3 * W * n);
    const void* fn = sign < 0.f ? (const void*)k_line_pipe<-1> : (const void*)k_line_pipe<1>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int grid = 0;
    if ((e = persistent_grid(fn, T, smem, gs.n * nIT * no, &grid)) != cudaSuccess) return e;
    if (sign < 0.f) k_line_pipe<-1><<<grid, T, smem, st>>>(gs, ni, n, pstride, no, ostride, W, nIT, pl, tw);
    else k_line_pipe<1><<<grid, T, smem, st>>>(gs, ni, n, pstride, no, ostride, W, nIT, pl, tw);
    if (nlaunch) (*nlaunch)++;
    return cudaGetLastError();
  }
  size_t smem = sizeof(float2) * (size_t)(n + 2 * W * n);
  dim3 grid((unsigned)(nIT * no), gs.n);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_line_fft, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_line_fft<<<grid, T, smem, st>>>(gs, ni, n, pstride, no, ostride, W, nIT, pl, tw, sign);
  if (nlaunch) (*nlaunch)++;
  return cudaGetLastError();
}

}  // namespace crava
