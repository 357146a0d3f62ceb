// SegY trace records of a device grid (sm_100a): FFTGrid::writeSegyFile's regular-z resampling
// (src/fftgrid.cpp:2001-2037 with getRegularZInterpolatedRealValue, :2275-2306) and NRLib's
// trace layout (a 240-byte header, then big-endian IBM floats,
// libs/nrlib/segy/segy.cpp:1397-1430), packed on the device for a chunk of records.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "ibm_float.h"
#include "kernels.cuh"

namespace crava {

constexpr float kSegyMissing = -99999.0f;   // RMISSING of the grid's interpolation

__device__ __forceinline__ uint32_t bswap32(uint32_t v) { return __byte_perm(v, 0u, 0x0123); }

// Sample k of one trace on the regular axis z0 + k dz: the float value the reference's
// interpolation returns, its operations rounded one by one in its order (double products and
// sums as on the host, no fused multiply-adds).
__device__ __forceinline__ float segy_sample(const float* __restrict__ g, size_t col, size_t plane, int nz, float z0,
                                             float dz, int k, double ztop, double gdz) {
  const float z = (float)__dadd_rn((double)z0, __dmul_rn((double)dz, (double)k));
  float t = (float)__ddiv_rn(__dsub_rn((double)z, ztop), gdz);
  int kg = (int)t;
  t = __fsub_rn(t, (float)kg);
  if (kg < 0) {
    if (kg < -1) return kSegyMissing;
    kg = 0;
    t = 0.f;
  } else if (kg > nz - 2) {
    if (kg > nz - 1) return kSegyMissing;
    kg = nz - 2;
    t = 1.f;
  }
  const float v1 = g[col + plane * (size_t)kg];
  const float v2 = g[col + plane * (size_t)(kg + 1)];
  return __fadd_rn(__fmul_rn(__fsub_rn(1.f, t), v1), __fmul_rn(t, v2));
}

// Records r0 .. r0 + nr - 1 into out (nr records of 60 + ns words): word w < 60 of record r
// is header word w of hdr (record order), word 60 + k the big-endian IBM float of sample k.
__global__ void k_segy_pack(const __grid_constant__ SegyPack P, size_t r0, int nr, uint32_t* __restrict__ out) {
  const size_t words = (size_t)60 + P.ns;
  const size_t n = words * nr;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t rl = e / words;
    const int w = (int)(e - rl * words);
    const size_t r = r0 + rl;
    if (w < 60) {
      out[e] = P.hdr[r * 60 + w];
      continue;
    }
    const int k = w - 60;
    const SegyTrace tr = P.tr[r];
    float v = 0.f;
    if (k >= tr.first && k < tr.end)
      v = segy_sample(P.grid, (size_t)tr.i + (size_t)P.rnxp * tr.j, (size_t)P.rnxp * P.nyp, P.nz, P.z0, P.dz, k,
                      tr.ztop, tr.gdz);
    out[e] = bswap32(ibm_from_ieee(__float_as_uint(v)));
  }
}

cudaError_t launch_segy_pack(const SegyPack& P, size_t r0, int nr, uint32_t* out, cudaStream_t st) {
  const size_t n = ((size_t)60 + P.ns) * nr;
  if (n == 0) return cudaSuccess;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_segy_pack<<<blocks, 256, 0, st>>>(P, r0, nr, out);
  return cudaGetLastError();
}

}  // namespace crava
