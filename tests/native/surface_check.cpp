// Reads a float surface and query points from a binary file and prints NRLib's
// RegularSurface<float>::GetZ at every point (one value per line, %.9g), for the test that
// pins the oracle's restatement of the bilinear lookup to NRLib's own template code.
// File layout: int32 ni, nj; double x0, y0, dx, dy; float z[ni*nj] (i + ni*j);
// int32 npts; double xy[2*npts].
#include <cstdio>
#include <vector>

#include "nrlib/surface/regularsurface.hpp"

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  int ni = 0, nj = 0, np = 0;
  double g[4];
  if (std::fread(&ni, 4, 1, f) != 1 || std::fread(&nj, 4, 1, f) != 1 || std::fread(g, 8, 4, f) != 4) return 3;
  std::vector<float> z((size_t)ni * nj);
  if (std::fread(z.data(), 4, z.size(), f) != z.size() || std::fread(&np, 4, 1, f) != 1) return 3;
  std::vector<double> xy(2 * (size_t)np);
  if (std::fread(xy.data(), 8, xy.size(), f) != xy.size()) return 3;
  std::fclose(f);
  // RegularSurface(x0, y0, lx, ly, ni, nj, value) with dx = lx / (ni - 1)
  NRLib::RegularSurface<float> s(g[0], g[1], g[2] * (ni - 1), g[3] * (nj - 1), ni, nj, 0.0f);
  for (int j = 0; j < nj; j++)
    for (int i = 0; i < ni; i++) s(i, j) = z[i + (size_t)ni * j];
  for (int p = 0; p < np; p++) std::printf("%.9g\n", (double)s.GetZ(xy[2 * p], xy[2 * p + 1]));
  return 0;
}
