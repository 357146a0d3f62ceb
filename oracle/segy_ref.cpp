// Test infrastructure (oracle): a SegY file of a host grid written the reference's way.
// FFTGrid::writeSegyFile (src/fftgrid.cpp:1960-2050) with getRegularZInterpolatedRealValue
// (:2275-2306) and Simbox::getXYCoord (src/simbox.cpp:821-827) are restated here (they sit in
// classes that need the FLENS/CBLAS headers); SegY::StoreTrace and WriteAllTracesToFile
// (libs/nrlib/segy/segy.cpp:1218-1272, 1364-1430) are restated around NRLib's own
// TextualHeader, BinaryHeader, TraceHeader, TraceHeaderFormat, SegyGeometry and
// WriteBinaryIbmFloatArray, compiled from the reference tree (oracle/Makefile).
#include <algorithm>
#include <cmath>
#include <fstream>
#include <vector>

#include "iotools/fileio.hpp"
#include "segy/commonheaders.hpp"
#include "segy/segygeometry.hpp"
#include "segy/traceheader.hpp"

#include "crava_gpu.h"

namespace {

const double kRMissing = -99999.000;
const double kWellMissing = -999.00000;

// FFTGrid::getRegularZInterpolatedRealValue on the real grid g (FFTGrid layout)
float regular_z_value(const float* g, int rnxp, int nyp, int nz, int i, int j, double z0Reg, double dzReg,
                      int kReg, double z0Grid, double dzGrid) {
  float z = static_cast<float>(z0Reg + dzReg * kReg);
  float t = static_cast<float>((z - z0Grid) / dzGrid);
  int kGrid = int(t);
  t -= kGrid;
  if (kGrid < 0) {
    if (kGrid < -1) return static_cast<float>(kRMissing);
    kGrid = 0;
    t = 0;
  } else if (kGrid > nz - 2) {
    if (kGrid > nz - 1) return static_cast<float>(kRMissing);
    kGrid = nz - 2;
    t = 1;
  }
  const size_t col = static_cast<size_t>(i) + static_cast<size_t>(rnxp) * j;
  const size_t plane = static_cast<size_t>(rnxp) * nyp;
  float v1 = g[col + plane * kGrid];
  float v2 = g[col + plane * (kGrid + 1)];
  float v = (1 - t) * v1 + t * v2;
  return v;
}

struct Trace {
  std::vector<float> data;
  double x, y;
  int il, xl;
  size_t index;
};

}  // namespace

extern "C" int segy_ref_write(const char* path, const float* grid, int rnxp, int nyp, const crava_segy_desc* d) {
  NRLib::TextualHeader header;
  if (!d->text) {
    header = NRLib::TextualHeader::standardHeader();
  } else {
    for (int i = 0; i < d->ntext; i++) header.SetLine(i + 1, d->text[i]);
  }
  float dz = float(std::floor(d->dz + 0.5));
  if (dz == 0) dz = 1.0;
  const int segynz = int(std::ceil((d->zmax - d->z0) / dz));
  // SegY::SegY -> WriteMainHeader (no geometry yet)
  std::ofstream file(path, std::ios::out | std::ios::binary);
  if (!file) return 1;
  header.Write(file);
  NRLib::BinaryHeader bh;
  bh.Write(file, NULL, dz, static_cast<size_t>(segynz));
  NRLib::SegyGeometry geometry(d->x0, d->y0, d->dx, d->dy, d->nx, d->ny, d->il0, d->xl0, d->il_step_x,
                               d->il_step_y, d->xl_step_x, d->xl_step_y, d->angle);
  std::vector<Trace*> traces(static_cast<size_t>(d->nx) * d->ny, nullptr);
  const double cosrot = std::cos(d->angle), sinrot = std::sin(d->angle);
  std::vector<float> trace(segynz);
  for (int j = 0; j < d->ny; j++) {
    for (int i = 0; i < d->nx; i++) {
      double rx = (static_cast<double>(i) + 0.5) * d->dx;
      double ry = (static_cast<double>(j) + 0.5) * d->dy;
      double x = rx * cosrot - ry * sinrot + d->x0;
      double y = rx * sinrot + ry * cosrot + d->y0;
      double z = d->top ? d->top[i + static_cast<size_t>(d->nx) * j] : d->top_z;
      if (z == kRMissing || z == kWellMissing) continue;
      double gdz = d->dz * (d->rel_thick ? d->rel_thick[i + static_cast<size_t>(d->nx) * j] : 1.0);
      int firstData = static_cast<int>(std::floor(0.5 + (z - d->z0) / dz));
      int endData = static_cast<int>(std::floor(0.5 + ((z - d->z0) + d->nz * gdz) / dz));
      if (endData > segynz) endData = segynz;
      int k;
      for (k = 0; k < firstData && k < segynz; k++) trace[k] = 0;
      for (; k < endData; k++) trace[k] = regular_z_value(grid, rnxp, nyp, d->nz, i, j, d->z0, dz, k, z, gdz);
      for (; k < segynz; k++) trace[k] = 0;
      float xx = static_cast<float>(x);
      float yy = static_cast<float>(y);
      // SegY::StoreTrace(double x, double y, ...)
      const double xd = xx, yd = yy;
      if (!geometry.IsInside(xd, yd)) return 2;
      Trace* t = new Trace;
      geometry.FindILXL(xd, yd, t->il, t->xl);
      size_t ii, jj;
      geometry.FindIndex(xd, yd, ii, jj);
      t->index = ii + geometry.GetNx() * jj;
      t->x = xd;
      t->y = yd;
      t->data = trace;
      delete traces[t->index];
      traces[t->index] = t;
    }
  }
  std::sort(traces.begin(), traces.end(), [](const Trace* a, const Trace* b) {
    if (a == nullptr) return false;
    if (b == nullptr) return true;
    if (a->il != b->il) return a->il < b->il;
    if (a->xl != b->xl) return a->xl < b->xl;
    return a->index < b->index;
  });
  NRLib::TraceHeaderFormat thf(d->header_format);
  for (Trace* t : traces) {
    if (!t) continue;
    NRLib::TraceHeader th(thf);
    th.SetNSamples(static_cast<size_t>(segynz));
    th.SetDt(static_cast<unsigned short>(dz * 1000));
    th.SetScalCo(1);
    th.SetUtmx(t->x);
    th.SetUtmy(t->y);
    th.SetInline(t->il);
    th.SetCrossline(t->xl);
    th.SetStartTime(static_cast<short>(d->z0));
    th.SetOffset(0);
    th.Write(file);
    NRLib::WriteBinaryIbmFloatArray(file, t->data.begin(), t->data.end());
    delete t;
  }
  return file.good() ? 0 : 3;
}
