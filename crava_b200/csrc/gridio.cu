// CRAVA binary grid files staged directly between the file and a device grid (sm_100a):
// FFTGrid::writeCravaFile / readCravaFile (src/fftgrid.cpp:2183-2270).
//
// The file is the tag line "crava_fftgrid_binary", the simbox geometry and the padded
// dimensions (big-endian doubles and 4-byte integers, NRLib::WriteBinaryDouble / Int), then
// the rnxp x nyp x nzp real values of the FFTGrid layout as big-endian IEEE floats.  The
// values cross the host in chunks through two pinned buffers: while one chunk is read from
// (or written to) the file, the other is copied to (or from) the device, and the byte order
// is swapped on the device, in place after an upload, into a device staging chunk before a
// download.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/crava_gpu.h"
#include "kernels.cuh"

namespace crava {

__global__ void k_bswap32(uint32_t* __restrict__ dst, const uint32_t* __restrict__ src, size_t n) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    dst[e] = __byte_perm(src[e], 0u, 0x0123);
}

cudaError_t launch_bswap32(uint32_t* dst, const uint32_t* src, size_t n, cudaStream_t st) {
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  if (blocks < 1) return cudaSuccess;
  k_bswap32<<<blocks, 256, 0, st>>>(dst, src, n);
  return cudaGetLastError();
}

// Elements e0 .. e0+n-1 of the dense (i fastest, then j, then k) ordering of the nx x ny x nz
// region of a padded real grid (row pitch rnxp, nyp rows per slice) as big-endian words,
// and back.
__global__ void k_storm_pack(uint32_t* __restrict__ dst, const float* __restrict__ grid, int nx, int ny, size_t e0,
                             size_t n, int rnxp, int nyp) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t a = e0 + e;
    const int i = (int)(a % nx);
    const size_t r = a / nx;
    const int j = (int)(r % ny);
    const size_t k = r / ny;
    dst[e] = __byte_perm(__float_as_uint(grid[(k * nyp + j) * rnxp + i]), 0u, 0x0123);
  }
}

__global__ void k_storm_unpack(float* __restrict__ grid, const uint32_t* __restrict__ src, int nx, int ny, size_t e0,
                               size_t n, int rnxp, int nyp) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t a = e0 + e;
    const int i = (int)(a % nx);
    const size_t r = a / nx;
    const int j = (int)(r % ny);
    const size_t k = r / ny;
    grid[(k * nyp + j) * rnxp + i] = __uint_as_float(__byte_perm(src[e], 0u, 0x0123));
  }
}

// FFTGrid(const StormContGrid*, nxp, nyp, nzp) padding (src/fftgrid.cpp:242-302): a padded
// voxel is the float blend c1 w1 + c2 w2 of the grid's two edge values along one axis, z
// padding first (from the x- and y-padded slices 0 and nz-1), then y (from rows 0 and ny-1,
// x padding included), then x (from columns 0 and nx-1); the columns beyond nxp are zero.
// Phase 0: x padding of the interior rows; 1: y padding of the interior slices; 2: z padding.
__global__ void k_pad_fill(float* __restrict__ g, int nx, int ny, int nz, int nxp, int nyp, int nzp, int rnxp,
                           int phase) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y + (phase == 1 ? ny : 0), k = blockIdx.z + (phase == 2 ? nz : 0);
  if (i >= rnxp) return;
  const size_t slice = (size_t)nyp * rnxp;
  float* row = g + (size_t)k * slice + (size_t)j * rnxp;
  if (phase == 0) {   // j < ny, k < nz
    if (i < nx) return;
    if (i >= nxp) { row[i] = 0.f; return; }
    const float sa = 1.0f / static_cast<float>(nxp - nx + 1);
    const float w1 = __fmul_rn(sa, (float)(i - nx + 1)), w2 = __fmul_rn(sa, (float)(nxp - i));
    row[i] = __fadd_rn(__fmul_rn(row[0], w1), __fmul_rn(row[nx - 1], w2));
  } else if (phase == 1) {   // ny <= j < nyp, k < nz
    if (i >= nxp) { row[i] = 0.f; return; }
    const float sb = 1.0f / static_cast<float>(nyp - ny + 1);
    const float w1 = __fmul_rn(sb, (float)(j - ny + 1)), w2 = __fmul_rn(sb, (float)(nyp - j));
    const float* s0 = g + (size_t)k * slice;
    row[i] = __fadd_rn(__fmul_rn(s0[i], w1), __fmul_rn(s0[(size_t)(ny - 1) * rnxp + i], w2));
  } else {   // nz <= k < nzp, all j
    if (i >= nxp) { row[i] = 0.f; return; }
    const float sc = 1.0f / static_cast<float>(nzp - nz + 1);
    const float w1 = __fmul_rn(sc, (float)(k - nz + 1)), w2 = __fmul_rn(sc, (float)(nzp - k));
    const size_t o = (size_t)j * rnxp + i;
    row[i] = __fadd_rn(__fmul_rn(g[o], w1), __fmul_rn(g[(size_t)(nz - 1) * slice + o], w2));
  }
}

static int stream_blocks(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

cudaError_t launch_storm_pack(uint32_t* dst, const float* grid, int nx, int ny, size_t e0, size_t n, int rnxp,
                              int nyp, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_storm_pack<<<stream_blocks(n), 256, 0, st>>>(dst, grid, nx, ny, e0, n, rnxp, nyp);
  return cudaGetLastError();
}

cudaError_t launch_storm_unpack(float* grid, const uint32_t* src, int nx, int ny, size_t e0, size_t n, int rnxp,
                                int nyp, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_storm_unpack<<<stream_blocks(n), 256, 0, st>>>(grid, src, nx, ny, e0, n, rnxp, nyp);
  return cudaGetLastError();
}

cudaError_t launch_pad_fill(float* grid, int nx, int ny, int nz, int nxp, int nyp, int nzp, int rnxp, cudaStream_t st,
                            int* nlaunch) {
  const unsigned bx = (unsigned)((rnxp + 127) / 128);
  if (rnxp > nx) {
    k_pad_fill<<<dim3(bx, ny, nz), 128, 0, st>>>(grid, nx, ny, nz, nxp, nyp, nzp, rnxp, 0);
    if (nlaunch) (*nlaunch)++;
  }
  if (nyp > ny) {
    // rows ny .. nyp-1 of the interior slices (blockIdx.y counts from ny)
    k_pad_fill<<<dim3(bx, nyp - ny, nz), 128, 0, st>>>(grid, nx, ny, nz, nxp, nyp, nzp, rnxp, 1);
    if (nlaunch) (*nlaunch)++;
  }
  if (nzp > nz) {
    // slices nz .. nzp-1 (blockIdx.z counts from nz)
    k_pad_fill<<<dim3(bx, nyp, nzp - nz), 128, 0, st>>>(grid, nx, ny, nz, nxp, nyp, nzp, rnxp, 2);
    if (nlaunch) (*nlaunch)++;
  }
  return cudaGetLastError();
}

}  // namespace crava
