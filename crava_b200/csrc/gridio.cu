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

}  // namespace crava
