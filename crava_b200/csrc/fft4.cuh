// Four-step transform kernels and their launch templates for the lengths of the size table
// in fft4.cu (sm_100a): the
// same transforms as k_x_r2c / k_x_c2r / k_line_fft (kernels.cu), with each line done in
// two register-codelet passes (fft2.cuh) instead of one shared-memory stage per radix.
//
//   k_line4<N1,N2,DIR>  W columns of one strided line set: global -> pass 1 -> shared
//                       -> pass 2 -> global
//   k_xr2c4<N1,N2>      rows of even nxp, h = nxp/2 = N1 N2: global -> pass 1 -> shared
//                       -> pass 2 -> shared (natural order) -> split -> global
//   k_xc2r4<N1,N2>      global -> merge -> shared -> pass 1 -> pass 2 -> global
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cooperative_groups.h>

#include <algorithm>
#include <cstdlib>

#include "fft2.cuh"
#include "kernels.cuh"

namespace crava {

// ------------------------------------------------------------------ strided lines
//
// One tile of W columns (nw of them valid) of the lines through g: point p of column w at
// g[p pstride + w], read from src[p spstride + w] (g itself, or a staged copy of the tile in
// shared memory).  Shared layout of the W lines: element (w, p = t + N2 m) at
// p W + w + m SK, with SK chosen so that the pass-2 reads of neighbouring k2 fall on
// disjoint banks.  Needs tw (the length-N table) in shared memory; ends with a barrier.
template <int N1, int N2, int DIR>
__device__ __forceinline__ void line4_tile(const float2* srcb, size_t spstride, float2* g, int nw, size_t pstride,
                                           int W, int lw, int SK, const float2* tw, float2* Y) {
  const int T = blockDim.x, tid = threadIdx.x;
  const size_t mstride = (size_t)N2 * spstride;
  const int mpitch = N2 * W + SK;
  for (int q = tid; q < W * N2; q += T) {
    const int w = q & (W - 1), t = q >> lw;
    const bool ok = w < nw;
    const float2* src = srcb + (size_t)t * spstride + w;
    float2* y = Y + t * W + w;
    four_step_pass1<N1, N2, DIR>(
        t, tw, [&](int, int m) { return ok ? src[m * mstride] : make_float2(0.f, 0.f); },
        [&](int, int k2, float2 v) { y[k2 * mpitch] = v; });
  }
  __syncthreads();
  for (int q = tid; q < W * N1; q += T) {
    const int w = q & (W - 1), k2 = q >> lw;
    const float2* y = Y + k2 * mpitch + w;
    float2 v[N2];
    four_step_pass2<N1, N2, DIR>(k2, [&](int, int t) { return y[t * W]; }, v);
    if (w < nw) {
      float2* dst = g + (size_t)k2 * pstride + w;
#pragma unroll
      for (int k1 = 0; k1 < N2; k1++) dst[(size_t)k1 * N1 * pstride] = v[k1];
    }
  }
  __syncthreads();
}

template <int N1, int N2>
constexpr size_t line4_smem(int W, int SK) {
  return sizeof(float2) * ((size_t)W * N1 * N2 + (size_t)N1 * SK);
}

// Forward instances bounded at 256 threads (the register allocation the forward passes were
// tuned with), inverse ones at 512 (a CTA may take one pass in a single round).
template <int N1, int N2, int DIR>
__global__ void __launch_bounds__(DIR > 0 ? 512 : 256) k_line4(const __grid_constant__ GridSet gs, int ni, size_t pstride,
                                               size_t ostride, int W, int lw, int nIT, int SK,
                                               const float2* __restrict__ twg, int pf) {
  constexpr int N = N1 * N2;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  for (int t = threadIdx.x; t < N; t += blockDim.x) tw[t] = twg[t];
  const int it = blockIdx.x % nIT, o = blockIdx.x / nIT;
  const int i0 = it * W, nw = min(W, ni - i0);
  float2* g = reinterpret_cast<float2*>(gs.p[blockIdx.y]) + (size_t)o * ostride + i0;
  // pf > 0: the cache lines of the tile pf block indices on (x fastest) go to L2
  if (pf > 0) {
    const int tn = blockIdx.y * gridDim.x + blockIdx.x + pf;
    if (tn < (int)(gridDim.x * gridDim.y)) {
      const int gy = tn / gridDim.x, gx = tn - gy * gridDim.x;
      const int itn = gx % nIT, on = gx / nIT;
      const int nwn = min(W, ni - itn * W);
      const float2* gn = reinterpret_cast<const float2*>(gs.p[gy]) + (size_t)on * ostride + itn * W;
      for (int q = threadIdx.x; q < 2 * N; q += blockDim.x) {
        const float2* row = gn + (size_t)(q >> 1) * pstride;
        l2_prefetch_line((q & 1) ? (const void*)(row + nwn - 1) : (const void*)row);
      }
    }
  }
  __syncthreads();
  line4_tile<N1, N2, DIR>(g, pstride, g, nw, pstride, W, lw, SK, tw, sm + N);
}

// ------------------------------------------------------------------ rows, even nxp
//
// Row r of a unit in shared memory at r * PITCH; pass-1 position t + N2 m at
// t + m (N2 + SK) with SK = 1 for even N2 (odd stride for the pass-2 reads).
template <int N1, int N2>
struct RowLayout {
  static constexpr int H = N1 * N2;
  static constexpr int SK = (N2 % 2 == 0) ? 1 : 0;
  static constexpr int PITCH = H + N1 * SK;
  static __device__ __forceinline__ int pad(int t, int m) { return t + m * (N2 + SK); }
};

// nr rows, even nxp: src rows (h complex values x[2m] + i x[2m+1] each, row pitch h + 1) to
// the scaled half spectra in dst (may equal src).  The split step as k_x_r2c (kernels.cu),
// done in registers: output k = k2 + N1 k1 of pass-2 item k2 has its mirror h - k in item
// (N1 - k2) mod N1, so one thread takes both items of a pair (k2 <= N1 / 2) and forms every
// X[k], X[h-k] from the two DFTs it holds.  Needs tw (length h) and twh (e^{-2 pi i k / nxp},
// k < h) in shared memory; Z: rpc * PITCH.  Ends with a barrier.
template <int N1, int N2>
__device__ __forceinline__ void xr2c4_rows(const float2* src, float2* dst, int nr, float scale, const float2* tw,
                                           const float2* twh, float2* Z) {
  using L = RowLayout<N1, N2>;
  constexpr int H = L::H, PITCH = L::PITCH;
  constexpr int CN = H + 1, NPI = N1 / 2 + 1;
  const int T = blockDim.x, tid = threadIdx.x;
  for (int q = tid; q < nr * N2; q += T) {
    const int r = q / N2, t = q - r * N2;
    const float2* x = src + (size_t)r * CN + t;
    float2* z = Z + r * PITCH;
    four_step_pass1<N1, N2, -1>(
        t, tw, [&](int, int m) { return x[m * N2]; }, [&](int, int k2, float2 v) { z[L::pad(t, k2)] = v; });
  }
  __syncthreads();
  for (int q = tid; q < nr * NPI; q += T) {
    const int r = q / NPI, a = q - r * NPI;        // item a and its mirror item b
    const int b = a == 0 ? 0 : N1 - a;
    const float2* z = Z + r * PITCH;
    float2 va[N2], vb[N2];
    four_step_pass2<N1, N2, -1>(a, [&](int k, int t) { return z[L::pad(t, k)]; }, va);
    if (b != a) four_step_pass2<N1, N2, -1>(b, [&](int k, int t) { return z[L::pad(t, k)]; }, vb);
    float2* X = dst + (size_t)r * CN;
#pragma unroll
    for (int k1 = 0; k1 < N2; k1++) {
      const int k = a + N1 * k1;
      if (k == 0) {
        const float2 z0 = va[0];
        X[0] = make_float2(scale * (z0.x + z0.y), 0.f);
        X[H] = make_float2(scale * (z0.x - z0.y), 0.f);
        continue;
      }
      // z[h - k]: item b's output N2 - 1 - k1 (N2 - k1 for item 0, its own mirror)
      const float2 zm = a == 0 ? va[N2 - k1] : (b != a ? vb[N2 - 1 - k1] : va[N2 - 1 - k1]);
      if (b == a && 2 * k > H) continue;           // a self-mirrored item's upper half: done below
      // the pair (k0, h - k0), k0 <= h/2, as the separate split loop forms it
      const bool lo = 2 * k <= H;
      const int k0 = lo ? k : H - k;
      const float2 A = lo ? va[k1] : zm, Bc = lo ? zm : va[k1];
      const float2 E = make_float2(0.5f * (A.x + Bc.x), 0.5f * (A.y - Bc.y));
      const float2 D = make_float2(A.x - Bc.x, A.y + Bc.y);
      const float2 O = make_float2(0.5f * D.y, -0.5f * D.x);
      const float2 tt = cmul(twh[k0], O);
      const float2 xk = cadd(E, tt);
      X[k0] = make_float2(scale * xk.x, scale * xk.y);
      if (2 * k0 != H) {
        const float2 m = csub(E, tt);
        X[H - k0] = make_float2(scale * m.x, -scale * m.y);
      }
    }
  }
  __syncthreads();
}

// nr rows of half spectra in g (pitch h + 1) to scaled real rows in place; the merge step
// as k_x_c2r (kernels.cu).  Z: rpc * PITCH, Xs: rpc * (h + 1).  Ends with a barrier.
// The same from rows already staged in Xs (shared), writing g; COPY: the real rows also go
// to Vc (shared, row r at r * h pairs of samples).
template <int N1, int N2, bool COPY = false>
__device__ __forceinline__ void xc2r4_staged(const float2* Xs, float2* g, int nr, float scale, const float2* tw,
                                             const float2* twh, float2* Z, float2* Vc = nullptr) {
  using L = RowLayout<N1, N2>;
  constexpr int H = L::H, PITCH = L::PITCH;
  constexpr int CN = H + 1;
  const int T = blockDim.x, tid = threadIdx.x;
  // pass 1 reads the half-length sequence z straight from the staged half spectrum: the merge
  // z[k] = (X[k] + conj X[h-k]) + i w^k (X[k] - conj X[h-k]) (w = e^{2 pi i / nxp}) computed
  // where pass 1 loads it, each z[k] with the operations of its pair's lower index k0 <= h/2
  // (z[h - k0] is the mirrored combination of the same terms)
  for (int q = tid; q < nr * N2; q += T) {
    const int r = q / N2, t = q - r * N2;
    const float2* X = Xs + r * CN;
    float2* z = Z + r * PITCH;
    four_step_pass1<N1, N2, 1>(
        t, tw,
        [&](int, int m) {
          const int k = t + N2 * m;
          if (k == 0) {
            const float a = X[0].x, b = X[H].x;
            return make_float2(a + b, a - b);
          }
          const bool lo = 2 * k <= H;
          const int k0 = lo ? k : H - k;
          const float2 xk = X[k0], xm = X[H - k0];
          const float2 P = make_float2(xk.x + xm.x, xk.y - xm.y);
          const float2 M = make_float2(xk.x - xm.x, xk.y + xm.y);
          const float2 w = twh[k0];
          const float2 Q = make_float2(M.x * w.x + M.y * w.y, M.y * w.x - M.x * w.y);
          return lo ? make_float2(P.x - Q.y, P.y + Q.x) : make_float2(P.x + Q.y, -P.y + Q.x);
        },
        [&](int, int k2, float2 v) { z[L::pad(t, k2)] = v; });
  }
  __syncthreads();
  for (int q = tid; q < nr * N1; q += T) {
    const int r = q / N1, k2 = q - r * N1;
    const float2* z = Z + r * PITCH;
    float2 v[N2];
    four_step_pass2<N1, N2, 1>(k2, [&](int k, int t) { return z[L::pad(t, k)]; }, v);
    float2* X = g + (size_t)r * CN;
#pragma unroll
    for (int k1 = 0; k1 < N2; k1++) {
      const float2 o = make_float2(v[k1].x * scale, v[k1].y * scale);
      X[k2 + N1 * k1] = o;
      if (COPY) Vc[r * H + k2 + N1 * k1] = o;
    }
    if (k2 == 0) X[H] = make_float2(0.f, 0.f);
  }
  __syncthreads();
}

template <int N1, int N2>
__device__ __forceinline__ void xc2r4_rows(float2* g, int nr, float scale, const float2* tw, const float2* twh,
                                           float2* Z, float2* Xs) {
  constexpr int CN = N1 * N2 + 1;
  {
    const uint32_t xb = smem_addr(Xs);
    for (int e = threadIdx.x; e < nr * CN; e += blockDim.x) cp_async8(xb + 8u * (uint32_t)e, g + e);
    cp_async_commit();
    cp_async_wait_0();
  }
  __syncthreads();
  xc2r4_staged<N1, N2>(Xs, g, nr, scale, tw, twh, Z);
}

template <int N1, int N2>
constexpr size_t x4_smem(bool fwd, int rpc) {
  using L = RowLayout<N1, N2>;
  return sizeof(float2) * ((size_t)rpc * L::PITCH + (fwd ? 0 : (size_t)rpc * (L::H + 1)));
}

// L2 prefetch of the row chunk pf block indices on (x fastest): rows of (h + 1) complex values,
// chunks of rpc rows, blockIdx.y the grid; from gs.src (FWD) or gs.p.
template <bool FWD>
__device__ __forceinline__ void x4_prefetch(const GridSet& gs, int rows, int rpc, int CN, int pf) {
  const int tn = blockIdx.y * gridDim.x + blockIdx.x + pf;
  if (threadIdx.x != 0 || tn >= (int)(gridDim.x * gridDim.y)) return;
  const int gy = tn / gridDim.x, c = tn - gy * gridDim.x;
  const int row0 = c * rpc, nr = min(rpc, rows - row0);
  const float2* s = reinterpret_cast<const float2*>(FWD ? gs.src[gy] : gs.p[gy]) + (size_t)row0 * CN;
  const size_t n = (size_t)nr * CN;
  // in pieces of 64 KB
  for (size_t o = 0; o < n; o += 8192) l2_prefetch(s + o, 8u * min((size_t)8192, n - o), s, s + n);
}

// stage != 0: the twiddle tables are copied into shared memory first; 0: the passes read
// them from global memory (L1-resident: every CTA of the launch reads the same 2 h values),
// and the CTA's first barrier and the table copy go away.
template <int N1, int N2>
__global__ void __launch_bounds__(256) k_xr2c4(const __grid_constant__ GridSet gs, int rows, int rpc,
                                               const float2* __restrict__ twg, const float2* __restrict__ twn,
                                               int stage, int pf) {
  constexpr int H = N1 * N2;
  extern __shared__ float2 sm[];
  const float2 *tw = twg, *twh = twn;
  float2* Z = sm;
  if (pf > 0) x4_prefetch<true>(gs, rows, rpc, H + 1, pf);
  if (stage) {
    float2* t1 = sm;
    float2* t2 = t1 + H;
    for (int t = threadIdx.x; t < H; t += blockDim.x) {
      t1[t] = twg[t];
      t2[t] = twn[t];
    }
    tw = t1;
    twh = t2;
    Z = t2 + H;
    __syncthreads();
  }
  const int row0 = blockIdx.x * rpc, nr = min(rpc, rows - row0);
  const float2* src = reinterpret_cast<const float2*>(gs.src[blockIdx.y]) + (size_t)row0 * (H + 1);
  float2* dst = reinterpret_cast<float2*>(gs.p[blockIdx.y]) + (size_t)row0 * (H + 1);
  xr2c4_rows<N1, N2>(src, dst, nr, gs.scale[blockIdx.y], tw, twh, Z);
}

template <int N1, int N2>
__global__ void __launch_bounds__(256) k_xc2r4(const __grid_constant__ GridSet gs, int rows, int rpc,
                                               const float2* __restrict__ twg, const float2* __restrict__ twn,
                                               int stage, int pf) {
  using L = RowLayout<N1, N2>;
  constexpr int H = N1 * N2, CN = H + 1;
  extern __shared__ float2 sm[];
  const float2 *tw = twg, *twh = twn;
  float2* Z = sm;
  const int row0 = blockIdx.x * rpc, nr = min(rpc, rows - row0);
  float2* g = reinterpret_cast<float2*>(gs.p[blockIdx.y]) + (size_t)row0 * CN;
  if (pf > 0) x4_prefetch<false>(gs, rows, rpc, CN, pf);
  if (stage) {
    float2* t1 = sm;
    float2* t2 = t1 + H;
    Z = t2 + H;
    // the rows' copies go out before the tables are staged
    float2* Xs = Z + rpc * L::PITCH;
    const uint32_t xb = smem_addr(Xs);
    for (int e = threadIdx.x; e < nr * CN; e += blockDim.x) cp_async8(xb + 8u * (uint32_t)e, g + e);
    cp_async_commit();
    for (int t = threadIdx.x; t < H; t += blockDim.x) {
      t1[t] = twg[t];
      t2[t] = twn[t];
    }
    cp_async_wait_0();
    __syncthreads();
    xc2r4_staged<N1, N2>(Xs, g, nr, gs.scale[blockIdx.y], t1, t2, Z);
    return;
  }
  xc2r4_rows<N1, N2>(g, nr, gs.scale[blockIdx.y], tw, twh, Z, Z + rpc * L::PITCH);
}

// ------------------------------------------------------------------ persistent, pipelined
//
// The same row and column transforms as persistent CTAs that stage the next unit's input
// in shared memory with cp.async while the current unit is transformed: every CTA keeps one
// unit of loads in flight during its arithmetic.  Units are disjoint row chunks or column
// tiles, each read and written by the one CTA that owns it, so in-place grids are safe.

template <int N1, int N2, bool FWD>
__global__ void __launch_bounds__(256) k_x4p(const __grid_constant__ GridSet gs, int rows, int rpc, int nchunk,
                                             const float2* __restrict__ twg, const float2* __restrict__ twn) {
  using L = RowLayout<N1, N2>;
  constexpr int H = N1 * N2, CN = H + 1;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* twh = tw + H;
  float2* const X0 = twh + H;
  float2* const X1 = X0 + rpc * CN;
  float2* Z = X1 + rpc * CN;
  for (int t = threadIdx.x; t < H; t += blockDim.x) {
    tw[t] = twg[t];
    twh[t] = twn[t];
  }
  const int units = gs.n * nchunk;
  auto issue = [&](int u, float2* buf) {
    const int gi = u / nchunk, c = u - gi * nchunk;
    const int row0 = c * rpc, nr = min(rpc, rows - row0);
    const float2* src = reinterpret_cast<const float2*>(FWD ? gs.src[gi] : gs.p[gi]) + (size_t)row0 * CN;
    const uint32_t b = smem_addr(buf);
    for (int e = threadIdx.x; e < nr * CN; e += blockDim.x) cp_async8(b + 8u * (uint32_t)e, src + e);
  };
  if ((int)blockIdx.x < units) issue(blockIdx.x, X0);
  cp_async_commit();
  int i = 0;
  for (int u = blockIdx.x; u < units; u += gridDim.x, i ^= 1) {
    if (u + (int)gridDim.x < units) issue(u + gridDim.x, i ? X0 : X1);
    cp_async_commit();
    cp_async_wait_1();
    __syncthreads();
    const int gi = u / nchunk, c = u - gi * nchunk;
    const int row0 = c * rpc, nr = min(rpc, rows - row0);
    float2* dst = reinterpret_cast<float2*>(gs.p[gi]) + (size_t)row0 * CN;
    const float2* cur = i ? X1 : X0;
    if (FWD) xr2c4_rows<N1, N2>(cur, dst, nr, gs.scale[gi], tw, twh, Z);
    else xc2r4_staged<N1, N2>(cur, dst, nr, gs.scale[gi], tw, twh, Z);
  }
  cp_async_wait_0();
  (void)L::PITCH;
}

template <int N1, int N2, int DIR>
__global__ void __launch_bounds__(256) k_line4p(const __grid_constant__ GridSet gs, int ni, size_t pstride, int no,
                                                size_t ostride, int W, int lw, int nIT, int SK,
                                                const float2* __restrict__ twg) {
  constexpr int N = N1 * N2;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* const T0 = sm + N;
  float2* const T1 = T0 + W * N;
  float2* Y = T1 + W * N;
  for (int t = threadIdx.x; t < N; t += blockDim.x) tw[t] = twg[t];
  const int per_grid = nIT * no, units = gs.n * per_grid;
  auto locate = [&](int u, int& nw) -> float2* {
    const int gi = u / per_grid, rem = u - gi * per_grid;
    const int o = rem / nIT, it = rem - o * nIT;
    nw = min(W, ni - it * W);
    return reinterpret_cast<float2*>(gs.p[gi]) + (size_t)o * ostride + (size_t)it * W;
  };
  auto issue = [&](int u, float2* buf) {
    int nw;
    const float2* g = locate(u, nw);
    const uint32_t b = smem_addr(buf);
    for (int e = threadIdx.x; e < N * W; e += blockDim.x) {
      const int p = e >> lw, w = e & (W - 1);
      const bool ok = w < nw;
      cp_async8_zfill(b + 8u * (uint32_t)e, ok ? g + (size_t)p * pstride + w : g, ok);
    }
  };
  if ((int)blockIdx.x < units) issue(blockIdx.x, T0);
  cp_async_commit();
  int i = 0;
  for (int u = blockIdx.x; u < units; u += gridDim.x, i ^= 1) {
    if (u + (int)gridDim.x < units) issue(u + gridDim.x, i ? T0 : T1);
    cp_async_commit();
    cp_async_wait_1();
    __syncthreads();
    int nw;
    float2* g = locate(u, nw);
    line4_tile<N1, N2, DIR>(i ? T1 : T0, (size_t)W, g, nw, pstride, W, lw, SK, tw, Y);
  }
  cp_async_wait_0();
}

// Opt-in (schedule key pipe4): measured slower than the one-unit kernels for the column
// transforms (staging a W-column tile costs more than it hides) and mixed for the rows.
static inline bool pipe4_enabled(int n) { return tuned("pipe4", n, 0) != 0; }

static inline cudaError_t resident_grid(const void* fn, int T, size_t smem, int units, int* grid) {
  int dev = 0, nsm = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, T, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  *grid = std::max(1, std::min(units, per_sm * nsm));
  return cudaSuccess;
}

// ------------------------------------------------------------------ fused xy passes
//
// One z-plane of one grid at a time per cluster of C CTAs: the rows of the plane (x
// transform, split across the cluster), a cluster barrier, then the columns (y transform,
// split across the cluster), in place in the destination grid.  The plane (nyp half-
// spectrum rows, 1-2.4 MB) is written by the first phase and read back by the second while
// it sits in L2, so each grid crosses HBM once each way per xy pass.  Persistent clusters
// walk the planes of every grid in the set.  The inverse runs the phases the other way.
template <int HX1, int HX2, int NY1, int NY2, bool FWD>
__global__ void __launch_bounds__(256, 2) k_xy4(const __grid_constant__ GridSet gs, int nzp, int rpc, int W, int lw,
                                             int SK, const float2* __restrict__ twx, const float2* __restrict__ twn,
                                             const float2* __restrict__ twy) {
  namespace cg = cooperative_groups;
  constexpr int H = HX1 * HX2, NY = NY1 * NY2, CN = H + 1;
  using L = RowLayout<HX1, HX2>;
  extern __shared__ float2 sm[];
  float2* tx = sm;
  float2* th = tx + H;
  float2* ty = th + H;
  float2* work = ty + NY;
  for (int t = threadIdx.x; t < H; t += blockDim.x) {
    tx[t] = twx[t];
    th[t] = twn[t];
  }
  for (int t = threadIdx.x; t < NY; t += blockDim.x) ty[t] = twy[t];
  __syncthreads();
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  const int ncl = gridDim.x / C, cid = blockIdx.x / C;
  const int planes = gs.n * nzp;
  const int nchunk = (NY + rpc - 1) / rpc, ntile = (CN + W - 1) / W;
  const size_t plane = (size_t)NY * CN;
  for (int p = cid; p < planes; p += ncl) {
    const int gi = p / nzp, z = p - gi * nzp;
    float2* dst = reinterpret_cast<float2*>(gs.p[gi]) + (size_t)z * plane;
    const float scale = gs.scale[gi];
    if (FWD) {
      const float2* src = reinterpret_cast<const float2*>(gs.src[gi]) + (size_t)z * plane;
      for (int c = rank; c < nchunk; c += C) {
        const int row0 = c * rpc, nr = min(rpc, NY - row0);
        xr2c4_rows<HX1, HX2>(src + (size_t)row0 * CN, dst + (size_t)row0 * CN, nr, scale, tx, th, work);
      }
      __threadfence();
      cl.sync();
      __threadfence();  // acquire side: no line of this plane cached before the barrier is reused
      for (int it = rank; it < ntile; it += C) {
        const int i0 = it * W;
        line4_tile<NY1, NY2, -1>(dst + i0, (size_t)CN, dst + i0, min(W, CN - i0), (size_t)CN, W, lw, SK, ty, work);
      }
    } else {
      for (int it = rank; it < ntile; it += C) {
        const int i0 = it * W;
        line4_tile<NY1, NY2, 1>(dst + i0, (size_t)CN, dst + i0, min(W, CN - i0), (size_t)CN, W, lw, SK, ty, work);
      }
      __threadfence();
      cl.sync();
      __threadfence();
      for (int c = rank; c < nchunk; c += C) {
        const int row0 = c * rpc, nr = min(rpc, NY - row0);
        xc2r4_rows<HX1, HX2>(dst + (size_t)row0 * CN, nr, scale, tx, th, work, work + rpc * L::PITCH);
      }
    }
    // a plane's two phases touch only that plane: the next plane needs no cluster barrier
  }
}

// ------------------------------------------------------------------ launch templates

static inline bool four_step_enabled(int n) { return tuned("four_step", n, 1) != 0; }

static inline int round_up32(int t) { return std::max(64, (t + 31) / 32 * 32); }

template <int N1, int N2>
static cudaError_t line4(const GridSet& gs, int ni, size_t pstride, int no, size_t ostride, const float2* tw,
                         float sign, cudaStream_t st) {
  constexpr int N = N1 * N2;
  // 8-column tiles; 16 for inverse transforms up to 540 points (measured faster there,
  // slower at 768)
  int W = std::max(1, tuned(sign < 0.f ? "line4_w_fwd" : "line4_w_inv", N, (sign > 0.f && N <= 540) ? 16 : 8));
  while (W > 1 && W / 2 >= ni) W /= 2;
  int lw = 0;
  while ((1 << lw) < W) lw++;
  W = 1 << lw;
  const int SK = W < 16 ? (((W - N2 * W) % 16) + 16) % 16 : 0;
  // threads per CTA: by default one item per thread of the longer pass up to 256; the
  // schedule may set up to 512 (a whole number of warps), e.g. so that one pass runs in a
  // single round
  int T = std::min(256, round_up32(W * std::max(N1, N2)));
  T = std::max(64, std::min(sign < 0.f ? 256 : 512,
                            tuned(sign < 0.f ? "line4_threads_fwd" : "line4_threads_inv", N, T) / 32 * 32));
  const int nIT = (ni + W - 1) / W;
  if (pipe4_enabled(N)) {
    // two staged tiles and the work tile: narrower tiles for the longest lines
    int Wp = W;
    while (Wp > 1 && sizeof(float2) * (2 * (size_t)Wp * N) + line4_smem<N1, N2>(Wp, SK) > 104 * 1024) Wp /= 2;
    int lwp = 0;
    while ((1 << lwp) < Wp) lwp++;
    const int SKp = Wp < 16 ? (((Wp - N2 * Wp) % 16) + 16) % 16 : 0;
    const int Tp = std::min(256, round_up32(Wp * std::max(N1, N2)));   // k_line4p is bounded at 256
    const int nITp = (ni + Wp - 1) / Wp;
    const size_t smem = sizeof(float2) * ((size_t)N + 2 * (size_t)Wp * N) + line4_smem<N1, N2>(Wp, SKp);
    const void* fn = sign < 0.f ? (const void*)k_line4p<N1, N2, -1> : (const void*)k_line4p<N1, N2, 1>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int grid = 0;
    if ((e = resident_grid(fn, Tp, smem, gs.n * nITp * no, &grid)) != cudaSuccess) return e;
    if (sign < 0.f)
      k_line4p<N1, N2, -1><<<grid, Tp, smem, st>>>(gs, ni, pstride, no, ostride, Wp, lwp, nITp, SKp, tw);
    else
      k_line4p<N1, N2, 1><<<grid, Tp, smem, st>>>(gs, ni, pstride, no, ostride, Wp, lwp, nITp, SKp, tw);
    return cudaGetLastError();
  }
  const size_t smem = sizeof(float2) * (size_t)N + line4_smem<N1, N2>(W, SK);
  const void* fn = sign < 0.f ? (const void*)k_line4<N1, N2, -1> : (const void*)k_line4<N1, N2, 1>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)(nIT * no), gs.n);
  // L2 line prefetch ahead of the tiles: schedule keys line4_pf_fwd / line4_pf_inv, the distance in
  // quarters of the resident tiles (0 = off)
  int pf = 0;
  if (const int q = tuned(sign < 0.f ? "line4_pf_fwd" : "line4_pf_inv", N, 0)) {
    int res = 0;
    if ((e = resident_grid(fn, T, smem, 1 << 30, &res)) != cudaSuccess) return e;
    pf = std::max(1, res * q / 4);
  }
  if (sign < 0.f) k_line4<N1, N2, -1><<<grid, T, smem, st>>>(gs, ni, pstride, ostride, W, lw, nIT, SK, tw, pf);
  else k_line4<N1, N2, 1><<<grid, T, smem, st>>>(gs, ni, pstride, ostride, W, lw, nIT, SK, tw, pf);
  return cudaGetLastError();
}

template <int N1, int N2>
static cudaError_t x4(bool fwd, const GridSet& gs, int rows, const float2* tw, const float2* twn, cudaStream_t st) {
  using L = RowLayout<N1, N2>;
  // 128-thread blocks: more CTAs per SM and cheaper barriers than 256 (measured 15 % faster);
  // the inverse rows up to h = 270 are faster still at 64 (3.53 vs 3.66 ms at 540x540x256)
  const int T = std::max(64, std::min(256, tuned(fwd ? "x4_threads_fwd" : "x4_threads_inv", L::H,
                                                   (!fwd && L::H <= 270) ? 64 : 128) / 32 * 32));
  // rows per CTA: by default a whole number of pass-2 items per thread (N1 items per row
  // inverse, N1 / 2 + 1 item pairs forward); the schedule entry may set up to 64
  int rpc = std::max(1, fwd ? T / (N1 / 2 + 1) : T / N1);
  rpc = std::max(1, std::min(64, tuned(fwd ? "x4_rpc_fwd" : "x4_rpc_inv", L::H, rpc)));
  if (pipe4_enabled(L::H)) {
    const int nchunk = (rows + rpc - 1) / rpc;
    const size_t smem = sizeof(float2) * (2 * (size_t)L::H + 2 * (size_t)rpc * (L::H + 1) + (size_t)rpc * L::PITCH);
    const void* fn = fwd ? (const void*)k_x4p<N1, N2, true> : (const void*)k_x4p<N1, N2, false>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int grid = 0;
    if ((e = resident_grid(fn, T, smem, gs.n * nchunk, &grid)) != cudaSuccess) return e;
    if (fwd) k_x4p<N1, N2, true><<<grid, T, smem, st>>>(gs, rows, rpc, nchunk, tw, twn);
    else k_x4p<N1, N2, false><<<grid, T, smem, st>>>(gs, rows, rpc, nchunk, tw, twn);
    return cudaGetLastError();
  }
  // twiddle tables staged in shared memory (schedule key x4_stage, default 1) or read from
  // global memory
  const int stage = tuned(fwd ? "x4_stage_fwd" : "x4_stage_inv", L::H, 1) != 0 ? 1 : 0;
  const size_t smem = sizeof(float2) * 2 * (size_t)L::H * stage + x4_smem<N1, N2>(fwd, rpc);
  const void* fn = fwd ? (const void*)k_xr2c4<N1, N2> : (const void*)k_xc2r4<N1, N2>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((rows + rpc - 1) / rpc), gs.n);
  // L2 prefetch of the row chunk ahead of the CTAs (schedule keys x4_pf_fwd / x4_pf_inv: the
  // distance in quarters of the resident CTAs, 0 = off; one wave, 4, measured faster for the
  // forward rows at h = 270, slower for the inverse ones)
  int pf = 0;
  if (const int q = tuned(fwd ? "x4_pf_fwd" : "x4_pf_inv", L::H, fwd ? 4 : 0)) {
    int res = 0;
    if ((e = resident_grid(fn, T, smem, 1 << 30, &res)) != cudaSuccess) return e;
    pf = std::max(1, res * q / 4);
  }
  if (fwd) k_xr2c4<N1, N2><<<grid, T, smem, st>>>(gs, rows, rpc, tw, twn, stage, pf);
  else k_xc2r4<N1, N2><<<grid, T, smem, st>>>(gs, rows, rpc, tw, twn, stage, pf);
  return cudaGetLastError();
}

// Fused xy pass for (h, nyp) pairs; cluster size from CRAVA_XY_CLUSTER (default 8).

}  // namespace crava
