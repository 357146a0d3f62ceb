// Checker (test infrastructure): crava::ibm_from_ieee (crava_b200/csrc/ibm_float.h) against
// the reference's own Ieee2Ibm (libs/nrlib/iotools/fileio.hpp:1128-1140, compiled from the
// reference tree) over every stride-th 32-bit pattern.  Prints the mismatch count.
#include <cstdio>
#include <cstdlib>

#include "iotools/fileio.hpp"
#include "ibm_float.h"

int main(int argc, char** argv) {
  const unsigned long long stride = argc > 1 ? std::strtoull(argv[1], nullptr, 10) : 1;
  unsigned long long bad = 0, n = 0;
  for (unsigned long long v = 0; v <= 0xffffffffull; v += stride, n++) {
    unsigned int a = (unsigned int)v, b = a;
    Ieee2Ibm(b);
    if (b != crava::ibm_from_ieee(a)) bad++;
  }
  std::printf("%llu %llu\n", n, bad);
  return bad != 0;
}
