// IEEE single to IBM System/360 single-precision hexadecimal float (the SEG-Y sample format
// code 1), as NRLib's WriteBinaryIbmFloatArray writes CRAVA's SegY traces
// (libs/nrlib/iotools/fileio.hpp:796-817): the fraction truncated, not rounded.
//
// An IBM single is sign | 7-bit exponent X (base 16, bias 64) | 24-bit fraction F with
// value 0.F * 16^(X - 64).  A normal IEEE float 1.m * 2^e is written with q = floor(e / 4) + 1
// (so that the value's hex fraction lies in [1/16, 1)), X = q + 64 and
// F = (2^23 | m) >> (3 - r), r = e - 4 q + 4 in 0..3; +-0 gives 0.  Usable on host and device.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define CRAVA_HD __host__ __device__ __forceinline__
#else
#define CRAVA_HD inline
#endif

namespace crava {

// IBM bits of the IEEE bits u.  Inputs whose IBM exponent leaves 0..127 (IEEE exponents below
// 2^-260 or above 2^252: subnormals, Inf and NaN among them) keep the reference's bit
// arithmetic: the biased exponent wraps modulo 128 into the neighbouring fields, which
// ibm_from_ieee reproduces by forming the same sum.
CRAVA_HD uint32_t ibm_from_ieee(uint32_t u) {
  if ((u & 0x7fffffffu) == 0u) return 0u;
  const uint32_t sign = u & 0x80000000u;
  const int E = (int)((u >> 23) & 0xffu);      // biased binary exponent
  const uint32_t m = u & 0x007fffffu;
  const int e = E - 127;
  // floor(e / 4) for negative e as well
  const int q = (e >= 0 ? e / 4 : -((-e + 3) / 4)) + 1;
  const int r = e - 4 * q + 4;                  // 0..3
  const uint32_t F = (0x00800000u | m) >> (3 - r);
  // exponent field and fraction added as integers (the fraction never reaches bit 24; an
  // exponent outside 0..127 carries into the sign bit position, which the sign OR masks)
  const uint32_t X = (uint32_t)(q + 64);
  return ((X << 24) + F) | sign;
}

}  // namespace crava
