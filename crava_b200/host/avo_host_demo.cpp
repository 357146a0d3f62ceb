// Runs one inversion block through the C++ host layer (crava_host.h) the way the
// reference's AVOInversion constructor does: DATA and PARAMETER grids in, then
// computePostMeanResidAndFFTCov and simulate, results read back from the same grids.
//
//   avo_host_demo <block.bin> <out.bin> [device]
//
// block.bin (little endian, written by tests/test_gpu_host_layer.py):
//   int32  nx ny nz nxp nyp nzp ntheta nsim prior_mode(0 separable, 1 grids) host_noise
//   uint64 seed
//   f64    lz min_rel_thick low_cut high_cut wnc
//   f64    A[ntheta*3] errThetaCov[ntheta*ntheta] priorVar0[9]
//   f32    wavelet[ntheta*nzp] waveletNorm[ntheta]
//   f32    corrXY[nxp*nyp] circCorrT[nzp]                      (separable)
//   f32    cov[6][rsize] errCorr[rsize]                        (grids)
//   f32    data[ntheta][rsize] mean[3][rsize]
//   f32    noise[3*nsim][rsize]                                (host_noise)
//   then optional sections, each after an int32 flag: non-constant thickness, correlation
//   gradients, 3D wavelets (see the reads below)
// out.bin: f32 mean[3][rsize] cov[6][rsize] sims[3*nsim][rsize] resid[ntheta][rsize],
//          int64 inverted_bins chol_fallbacks sim_chol_zero fp64_bins, f32 postVar0[9],
//          f32 fft round-trip max abs error of one DATA grid (FFTGrid::fftInPlace +
//          invFFTInPlace on the GPU)
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#include "crava_host.h"

using crava_b200::AVOInversion;
using crava_b200::AVOInversionSettings;
using crava_b200::Context;
using crava_b200::FFTGrid;
using crava_b200::SeismicParametersHolder;

namespace {

struct Reader {
  FILE* f;
  template <class T>
  void read(T* p, size_t n) {
    if (fread(p, sizeof(T), n, f) != n) {
      fprintf(stderr, "short read\n");
      exit(2);
    }
  }
  template <class T>
  T one() {
    T v;
    read(&v, 1);
    return v;
  }
};

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s block.bin out.bin [device]\n", argv[0]);
    return 2;
  }
  FILE* fi = fopen(argv[1], "rb");
  if (!fi) {
    perror(argv[1]);
    return 2;
  }
  Reader rd{fi};
  int h[10];
  rd.read(h, 10);
  const int nx = h[0], ny = h[1], nz = h[2], nxp = h[3], nyp = h[4], nzp = h[5], nth = h[6], nsim = h[7];
  const bool separable = h[8] == 0, host_noise = h[9] != 0;
  const uint64_t seed = rd.one<uint64_t>();
  double sc[5];
  rd.read(sc, 5);
  AVOInversionSettings set;
  set.ntheta = nth;
  set.lz = sc[0];
  set.minRelThick = sc[1];
  set.lowCut = (float)sc[2];
  set.highCut = (float)sc[3];
  set.wnc = (float)sc[4];
  set.nSimulations = nsim;
  set.seed = seed;
  std::vector<double> A(nth * 3), etc(nth * nth), pv(9);
  rd.read(A.data(), A.size());
  rd.read(etc.data(), etc.size());
  rd.read(pv.data(), 9);
  set.A.assign(A.begin(), A.end());
  set.errThetaCov = etc;
  set.wavelet.assign(nth, std::vector<float>(nzp));
  for (int l = 0; l < nth; l++) rd.read(set.wavelet[l].data(), nzp);
  set.waveletNorm.resize(nth);
  rd.read(set.waveletNorm.data(), nth);

  try {
    Context ctx(argc > 3 ? atoi(argv[3]) : 0);
    auto grid = [&](int type) {
      auto g = std::make_unique<FFTGrid>(&ctx, nx, ny, nz, nxp, nyp, nzp);
      g->setType(type);
      g->createRealGrid();
      return g;
    };
    SeismicParametersHolder sp;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) sp.priorVar0[a][b] = pv[a * 3 + b];
    std::vector<float> corrXY, circCorrT;
    std::vector<std::unique_ptr<FFTGrid>> own;
    FFTGrid* cov[6] = {};
    for (int q = 0; q < 6; q++) {
      own.push_back(grid(FFTGrid::COVARIANCE));
      cov[q] = own.back().get();
    }
    sp.covVp = cov[0];
    sp.covVs = cov[1];
    sp.covRho = cov[2];
    sp.crCovVpVs = cov[3];
    sp.crCovVpRho = cov[4];
    sp.crCovVsRho = cov[5];
    if (separable) {
      corrXY.resize((size_t)nxp * nyp);
      circCorrT.resize(nzp);
      rd.read(corrXY.data(), corrXY.size());
      rd.read(circCorrT.data(), circCorrT.size());
    } else {
      for (int q = 0; q < 6; q++) rd.read(cov[q]->getRealData(), cov[q]->getrsize());
      own.push_back(grid(FFTGrid::COVARIANCE));
      sp.errCorr = own.back().get();
      rd.read(sp.errCorr->getRealData(), sp.errCorr->getrsize());
    }
    std::vector<FFTGrid*> seis;
    for (int l = 0; l < nth; l++) {
      own.push_back(grid(FFTGrid::DATA));
      rd.read(own.back()->getRealData(), own.back()->getrsize());
      seis.push_back(own.back().get());
    }
    FFTGrid* mean[3];
    for (int a = 0; a < 3; a++) {
      own.push_back(grid(FFTGrid::PARAMETER));
      mean[a] = own.back().get();
      rd.read(mean[a]->getRealData(), mean[a]->getrsize());
    }
    sp.meanVp = mean[0];
    sp.meanVs = mean[1];
    sp.meanRho = mean[2];
    std::vector<FFTGrid*> noise;
    if (host_noise) {
      for (int q = 0; q < 3 * nsim; q++) {
        own.push_back(grid(FFTGrid::PARAMETER));
        own.back()->createComplexGrid();
        rd.read(own.back()->getRealData(), own.back()->getrsize());
        noise.push_back(own.back().get());
      }
    }
    // optional trailing section: non-constant thickness (relThick nxp*nyp doubles, then the
    // energy threshold)
    int nonconst = 0;
    if (fread(&nonconst, sizeof(int), 1, fi) == 1 && nonconst) {
      set.relThick.resize((size_t)nxp * nyp);
      rd.read(set.relThick.data(), set.relThick.size());
      set.energyThreshold = rd.one<float>();
    }
    // optional trailing section after it: correlation gradients (two floats)
    int grads = 0;
    if (fread(&grads, sizeof(int), 1, fi) == 1 && grads) {
      set.corrGradI = rd.one<float>();
      set.corrGradJ = rd.one<float>();
    }
    // optional trailing section after it: 3D wavelets (int32 ni nj has_grad has_halpha, f64 x0 y0
    // dx dy, f32 theta[ntheta], gradX/gradY[nx*ny] if has_grad, alpha1[ntheta*ni*nj],
    // halpha[ntheta*ni*nj] if has_halpha, global wavelets[ntheta*nzp], their norms[ntheta])
    int w3 = 0;
    if (fread(&w3, sizeof(int), 1, fi) == 1 && w3) {
      set.waveletDim = 3;
      set.filterNI = rd.one<int>();
      set.filterNJ = rd.one<int>();
      const int has_grad = rd.one<int>(), has_halpha = rd.one<int>();
      set.filterX0 = rd.one<double>();
      set.filterY0 = rd.one<double>();
      set.filterDX = rd.one<double>();
      set.filterDY = rd.one<double>();
      set.theta.resize(nth);
      rd.read(set.theta.data(), nth);
      if (has_grad) {
        set.depthGradX.resize((size_t)nx * ny);
        set.depthGradY.resize((size_t)nx * ny);
        rd.read(set.depthGradX.data(), set.depthGradX.size());
        rd.read(set.depthGradY.data(), set.depthGradY.size());
      }
      const size_t nij = (size_t)set.filterNI * set.filterNJ;
      set.filterAlpha1.resize(nth * nij);
      rd.read(set.filterAlpha1.data(), set.filterAlpha1.size());
      if (has_halpha) {
        set.filterHalpha.resize(nth * nij);
        rd.read(set.filterHalpha.data(), set.filterHalpha.size());
      }
      set.globalWavelet.assign(nth, std::vector<float>(nzp));
      for (int l = 0; l < nth; l++) rd.read(set.globalWavelet[l].data(), nzp);
      set.globalWaveletNorm.resize(nth);
      rd.read(set.globalWaveletNorm.data(), nth);
    }
    fclose(fi);

    // FFTGrid round trip on a copy of the first DATA grid
    FFTGrid probe(*seis[0]);
    probe.fftInPlace();
    probe.invFFTInPlace();
    float rt = 0.f;
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
          rt = std::fmax(rt, std::fabs(probe.getRealValue(i, j, k) - seis[0]->getRealValue(i, j, k)));

    AVOInversion inv(&ctx, set, seis, sp, separable ? &corrXY : nullptr, separable ? &circCorrT : nullptr);
    if (host_noise) inv.simulate(&noise);
    inv.computePostMeanResidAndFFTCov();
    if (!host_noise) inv.simulate();

    FILE* fo = fopen(argv[2], "wb");
    if (!fo) {
      perror(argv[2]);
      return 2;
    }
    auto put = [&](const FFTGrid* g) { fwrite(g->getRealData(), sizeof(float), g->getrsize(), fo); };
    put(inv.getPostVp());
    put(inv.getPostVs());
    put(inv.getPostRho());
    for (int q = 0; q < 6; q++) put(cov[q]);
    for (auto& g : sp.simulations) put(g.get());
    for (int l = 0; l < nth; l++) put(seis[l]);
    const crava_counters c = inv.counters();
    const long long cnt[4] = {c.inverted_bins, c.chol_fallbacks, c.sim_chol_zero, c.fp64_bins};
    fwrite(cnt, sizeof(long long), 4, fo);
    float pv0[9];
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) pv0[a * 3 + b] = (float)sp.postVar0[a][b];
    fwrite(pv0, sizeof(float), 9, fo);
    fwrite(&rt, sizeof(float), 1, fo);
    fclose(fo);
    printf("ok: %lld inverted bins, %lld Cholesky fallbacks, fft round trip %.3e\n", cnt[0], cnt[1], rt);
  } catch (const crava_b200::Error& e) {
    fprintf(stderr, "crava error %d: %s\n", (int)e.status, e.what());
    return 1;
  }
  return 0;
}
