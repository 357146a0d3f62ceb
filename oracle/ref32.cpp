// FP32 reference harness: the reference's own CPU inversion path.
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline).  Nothing in the
// product links this file.  It is compiled by oracle/Makefile together with the
// reference's unmodified numerics, taken from the reference tree where they lie:
//   libs/fft/{fftw,rfftw}/*.c   FFTW 2.1.2 single precision (rfftw3d / rfftwnd)
//   libs/lib/lib_matr.c         lib_matrCholCpx, lib_matrAXeqBMatCpx, products
//   libs/lib/random.cpp         RandomGen (LCG + Marsaglia-Bray normals)
// and restates, in float and in the reference's call order, the loops that call them:
//   FFTGrid::fftInPlace / invFFTInPlace           src/fftgrid.cpp:1587-1643
//   FFTGrid::fillInComplexNoise                    src/fftgrid.cpp:997-1055
//   SeismicParametersHolder::getNextParameterCovariance
//                                                 src/seismicparametersholder.cpp:485-557
//   Wavelet::getCAmp, Wavelet::findNorm            src/wavelet.cpp:318-334, 882-900
//   Wavelet1D diff constructors                    src/wavelet1D.cpp:389-500
//   AVOInversion::computePostMeanResidAndFFTCov    src/avoinversion.cpp:794-1114
//   AVOInversion::getNextErrorVariance, fillkW, fillkWNorm  :1236-1300
//   AVOInversion::simulate                         src/avoinversion.cpp:1354-1511
//   SeismicParametersHolder::invFFTCovGrids        src/seismicparametersholder.cpp:432-456
//   AVOInversion::divideDataByScaleWavelet, the trace transform   src/avoinversion.cpp:537-588
//   FaciesProb::findDensity + calculateFaciesProb (local-noise corners)
//                                                 src/faciesprob.cpp:1307-1423, 1909-2075
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

extern "C" {
#include "fftw.h"
#include "rfftw.h"
}
#include "lib/lib_matr.h"
#include "lib/random.h"

// random.cpp references NRLib::OpenRead only for its seed-file constructor, which this
// harness never calls; this definition satisfies the linker.
namespace NRLib {
void OpenRead(std::ifstream& stream, const std::string& filename, std::ios_base::openmode mode) {
  stream.open(filename.c_str(), mode);
}
}  // namespace NRLib

namespace {

struct Grid {
  // FFTGrid storage: rnxp*nyp*nzp floats, complex view cnxp*nyp*nzp
  int nxp, nyp, nzp, cnxp, rnxp;
  float* r;
  fftw_complex* c() { return reinterpret_cast<fftw_complex*>(r); }
  size_t rsize() const { return size_t(rnxp) * nyp * nzp; }
  size_t csize() const { return size_t(cnxp) * nyp * nzp; }
};

Grid make_grid(float* p, int nxp, int nyp, int nzp) {
  Grid g;
  g.nxp = nxp; g.nyp = nyp; g.nzp = nzp;
  g.cnxp = nxp / 2 + 1; g.rnxp = 2 * g.cnxp; g.r = p;
  return g;
}

// FFTGrid::fftInPlace (src/fftgrid.cpp:1587-1612)
void fft_in_place(Grid& g, bool covariance) {
  if (!covariance) {
    float s = 1.0f / std::sqrt(static_cast<float>(size_t(g.nxp) * g.nyp * g.nzp));
    for (size_t i = 0; i < g.rsize(); i++) g.r[i] *= s;
  }
  rfftwnd_plan plan = rfftw3d_create_plan(g.nzp, g.nyp, g.nxp, FFTW_REAL_TO_COMPLEX,
                                          FFTW_ESTIMATE | FFTW_IN_PLACE);
  rfftwnd_one_real_to_complex(plan, g.r, g.c());
  rfftwnd_destroy_plan(plan);
}

// FFTGrid::invFFTInPlace (src/fftgrid.cpp:1615-1643)
void inv_fft_in_place(Grid& g, bool covariance) {
  float scale;
  size_t N = size_t(g.nxp) * g.nyp * g.nzp;
  if (covariance) scale = float(1.0 / N);
  else scale = float(1.0 / std::sqrt(float(N)));
  rfftwnd_plan plan = rfftw3d_create_plan(g.nzp, g.nyp, g.nxp, FFTW_COMPLEX_TO_REAL,
                                          FFTW_ESTIMATE | FFTW_IN_PLACE);
  rfftwnd_one_complex_to_real(plan, g.c(), g.r);
  rfftwnd_destroy_plan(plan);
  for (size_t i = 0; i < g.rsize(); i++) g.r[i] *= scale;
}

// A 1D operator vector in FFT order with FFTW's in-place half spectrum
// (Wavelet / Wavelet1D storage, src/wavelet.cpp:255-270).
struct Vec1D {
  int nzp, cnzp;
  std::vector<float> a;  // rnzp floats
  float norm;
  explicit Vec1D(int n) : nzp(n), cnzp(n / 2 + 1), a(2 * (n / 2 + 1), 0.0f), norm(0.0f) {}
  void fft() {
    rfftwnd_plan plan = rfftwnd_create_plan(1, &nzp, FFTW_REAL_TO_COMPLEX, FFTW_ESTIMATE | FFTW_IN_PLACE);
    rfftwnd_one_real_to_complex(plan, a.data(), reinterpret_cast<fftw_complex*>(a.data()));
    rfftwnd_destroy_plan(plan);
  }
  // Wavelet::getCAmp(k) (src/wavelet.cpp:318-334)
  fftw_complex camp(int k) const {
    const fftw_complex* c = reinterpret_cast<const fftw_complex*>(a.data());
    fftw_complex v;
    if (k < cnzp) { v.re = c[k].re; v.im = c[k].im; }
    else { v.re = c[nzp - k].re; v.im = -c[nzp - k].im; }
    return v;
  }
  // Wavelet::getCAmp(k, scale) (src/wavelet.cpp:336-393): the stretched wavelet's spectrum by
  // linear interpolation at k / scale, divided by scale
  fftw_complex camp_scaled(int k, float scale) const {
    const fftw_complex* c = reinterpret_cast<const fftw_complex*>(a.data());
    fftw_complex value;
    float omega, dOmega;
    int omU, omL;
    const bool lo = k < cnzp;
    omega = float(lo ? k : nzp - k) / scale;
    if (omega >= cnzp) {
      value.re = 0.0f;
      value.im = 0.0f;
    } else {
      omL = int(std::floor(omega));
      omU = int(std::floor(omega)) + 1;
      if (omU >= cnzp) omU -= 1;
      dOmega = omega - float(omL);
      value.re = c[omL].re * (1.0f - dOmega) + c[omU].re * dOmega;
      value.im = lo ? (c[omL].im * (1.0f - dOmega) + c[omU].im * dOmega)
                    : (-c[omL].im * (1.0f - dOmega) - c[omU].im * dOmega);
    }
    value.re /= scale;
    value.im /= scale;
    return value;
  }
  // Wavelet::findNorm, real branch (src/wavelet.cpp:882-889)
  float find_norm() const {
    double n2 = 0.0;
    for (int i = 0; i < nzp; i++) n2 += static_cast<double>(a[i] * a[i]);
    return static_cast<float>(std::sqrt(n2));
  }
};

enum { FWD = 0, BWD = 1, CEN = 2 };
// Wavelet1D(Wavelet*, difftype) (src/wavelet1D.cpp:438-500), real branch
Vec1D diff_of(const Vec1D& w, int type) {
  Vec1D o(w.nzp);
  int n = w.nzp;
  for (int i = 0; i < n; i++) {
    switch (type) {
      case FWD: o.a[i] = (i == n - 1) ? w.a[0] - w.a[i] : w.a[i + 1] - w.a[i]; break;
      case BWD: o.a[i] = (i == 0) ? w.a[0] - w.a[n - 1] : w.a[i] - w.a[i - 1]; break;
      default:
        if (i == 0) o.a[i] = static_cast<float>(0.5 * (w.a[i + 1] - w.a[n - 1]));
        else if (i == n - 1) o.a[i] = static_cast<float>(0.5 * (w.a[0] - w.a[i - 1]));
        else o.a[i] = static_cast<float>(0.5 * (w.a[i + 1] - w.a[i - 1]));
    }
  }
  o.norm = o.find_norm();
  return o;
}

fftw_complex** cmat(int n, int m) {
  fftw_complex** x = new fftw_complex*[n];
  for (int i = 0; i < n; i++) x[i] = new fftw_complex[m];
  return x;
}
void free_cmat(fftw_complex** x, int n) {
  for (int i = 0; i < n; i++) delete[] x[i];
  delete[] x;
}

// FFTGrid::fillInComplexNoise (src/fftgrid.cpp:997-1055) with the reference RandomGen
void fill_complex_noise(fftw_complex* cv, int nxp, int nyp, int nzp) {
  size_t cnxp = nxp / 2 + 1;
  size_t csize = cnxp * nyp * nzp;
  float sd = float(1 / std::sqrt(2.0));
  for (size_t i = 0; i < csize; i++) {
    if (((i % cnxp) == 0) || (((i % cnxp) == cnxp - 1) && ((i % 2) == 1))) {
      int xshift = int(i % cnxp);
      int jkind = int((i - xshift) / cnxp);
      int jind = jkind % nyp;
      int kind = jkind / nyp;
      int jcc = (jind == 0) ? 0 : nyp - jind;
      int kcc = (kind == 0) ? 0 : nzp - kind;
      int jkcc = jcc + kcc * nyp;
      if (jkcc == jkind) {
        cv[i].re = float(RandomGen::rnorm01());
        cv[i].im = 0;
      } else if (jkcc > jkind) {
        cv[i].re = float(sd * RandomGen::rnorm01());
        cv[i].im = float(sd * RandomGen::rnorm01());
      } else {
        size_t cci = size_t(jkcc) * cnxp + xshift;
        cv[i].re = cv[cci].re;
        cv[i].im = -cv[cci].im;
      }
    } else {
      cv[i].re = float(sd * RandomGen::rnorm01());
      cv[i].im = float(sd * RandomGen::rnorm01());
    }
  }
}

}  // namespace

extern "C" {

// Block description in the reference's terms.  Grids are FFTGrid-padded float arrays.
typedef struct {
  int nx, ny, nz, nxp, nyp, nzp, ntheta;
  double lz, min_rel_thick;
  float low_cut, high_cut, wnc;
  const double* A;              // ntheta x 3
  const double* err_theta_cov;  // ntheta x ntheta
  const float* wavelet;         // ntheta x nzp, FFT order
  const float* wavelet_norm;    // ntheta
  const double* prior_var0;     // 3 x 3
  int nonconst;                 // 1: the non-constant-thickness branch (K = kD A,
                                // src/avoinversion.cpp:976-1014) on data already divided
} ref32_block;

// In-place 3D transforms with FFTGrid's scaling.
void ref32_fft(float* grid, int nxp, int nyp, int nzp, int covariance) {
  Grid g = make_grid(grid, nxp, nyp, nzp);
  fft_in_place(g, covariance != 0);
}
void ref32_ifft(float* grid, int nxp, int nyp, int nzp, int covariance) {
  Grid g = make_grid(grid, nxp, nyp, nzp);
  inv_fft_in_place(g, covariance != 0);
}

// The whole inversion of one block in the reference's order:
//   constructor FFTs (data, mean), FFTCovGrids + errCorr FFT, the per-bin loop,
//   simulate (nsim realisations from RandomGen(seed)), inverse mean transforms,
//   invFFTCovGrids.
// grids: mean[3] (in prior mean, out posterior mean, real), cov[6] (in prior covariance
// grids, out posterior covariance, real), errcorr (in; consumed), data[ntheta] (in seismic,
// out residual spectra, complex), sims (out, 3*nsim real grids) or NULL.
// counters: [0] inverted bins, [1] Cholesky fallbacks.
int ref32_invert(const ref32_block* b, float** mean, float** cov, float* errcorr,
                 float** data, int nsim, unsigned int seed, float** sims,
                 const float* noise_in, long long* counters) {
  const int nth = b->ntheta, nxp = b->nxp, nyp = b->nyp, nzp = b->nzp;
  const int cnxp = nxp / 2 + 1;
  std::vector<Grid> G_mean, G_cov, G_data;
  for (int a = 0; a < 3; a++) G_mean.push_back(make_grid(mean[a], nxp, nyp, nzp));
  for (int a = 0; a < 6; a++) G_cov.push_back(make_grid(cov[a], nxp, nyp, nzp));
  for (int l = 0; l < nth; l++) G_data.push_back(make_grid(data[l], nxp, nyp, nzp));
  Grid G_err = make_grid(errcorr, nxp, nyp, nzp);

  // AVOInversion constructor (src/avoinversion.cpp:229-244)
  for (int l = 0; l < nth; l++) fft_in_place(G_data[l], false);
  for (int a = 0; a < 3; a++) fft_in_place(G_mean[a], false);
  // computePostMeanResidAndFFTCov setup (:845-934)
  Vec1D diff1(nzp);
  diff1.a[0] = -1.0f;
  diff1.a[nzp - 1] = 1.0f;
  // diff3Operator: the backward then central difference of diff1's samples (:846-851)
  Vec1D diff3 = diff_of(diff_of(diff1, BWD), CEN);
  diff3.fft();
  diff1.fft();
  std::vector<Vec1D> w_seis, w_norm, es3;
  std::vector<float> norm_seis(nth), norm_es3(nth);
  for (int l = 0; l < nth; l++) {
    Vec1D w(nzp);
    for (int k = 0; k < nzp; k++) w.a[k] = b->wavelet[size_t(l) * nzp + k];
    w.norm = b->wavelet_norm[l];
    Vec1D e1 = diff_of(w, FWD), e2 = diff_of(e1, BWD), e3 = diff_of(e2, CEN);
    norm_es3[l] = e3.norm;
    e3.fft();
    es3.push_back(e3);
    Vec1D wn = w;
    wn.fft();
    w_norm.push_back(wn);
    norm_seis[l] = w.norm;
    Vec1D ws = w;
    ws.fft();
    w_seis.push_back(ws);
  }
  for (int a = 0; a < 6; a++) fft_in_place(G_cov[a], true);
  fft_in_place(G_err, true);

  fftw_complex* kW = new fftw_complex[nth];
  fftw_complex* m1 = new fftw_complex[nth];
  fftw_complex* m2 = new fftw_complex[nth];
  fftw_complex* m3 = new fftw_complex[nth];
  fftw_complex* d = new fftw_complex[nth];
  fftw_complex* dmean = new fftw_complex[nth];
  fftw_complex* res = new fftw_complex[nth];
  fftw_complex mu[3], ans[3];
  fftw_complex** K = cmat(nth, 3);
  fftw_complex** KS = cmat(nth, 3);
  fftw_complex** KScc = cmat(3, nth);
  fftw_complex** par = cmat(3, 3);
  fftw_complex** marg = cmat(nth, nth);
  fftw_complex** err = cmat(nth, nth);
  fftw_complex** red = cmat(3, 3);
  float** Af = new float*[nth];
  for (int l = 0; l < nth; l++) {
    Af[l] = new float[3];
    for (int j = 0; j < 3; j++) Af[l][j] = static_cast<float>(b->A[l * 3 + j]);
  }
  const double* pv = b->prior_var0;
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  long long n_inv = 0, n_fail = 0;
  size_t idx = 0;
  for (int k = 0; k < nzp; k++) {
    float realFrequency = static_cast<float>((b->nz * 1000.0f) / (b->lz * nzp) * std::min(k, nzp - k));
    fftw_complex kD = diff1.camp(k);
    if (!b->nonconst) {
      for (int l = 0; l < nth; l++) {           // fillkW
        fftw_complex c = w_seis[l].camp(k);
        kW[l].re = c.re;
        kW[l].im = -c.im;
      }
      lib_matrProdScalVecCpx(kD, kW, nth);
      lib_matrProdDiagCpxR(kW, Af, nth, 3, K);
      for (int l = 0; l < nth; l++) {           // fillkWNorm x2, ones
        fftw_complex c = w_norm[l].camp(k);
        m1[l].re = c.re / norm_seis[l];
        m1[l].im = -(c.im / norm_seis[l]);
        fftw_complex e = es3[l].camp(k);
        m2[l].re = e.re / norm_es3[l];
        m2[l].im = -(e.im / norm_es3[l]);
      }
      lib_matrFillOnesVecCpx(m3, nth);
    } else {
      // K = D A, errMult1 = 1 / norm, errMult2 = kD3 / norm(errorSmooth3),
      // errMult3 = fillInverseAbskWRobust (:976-1014, :1296-1322)
      fftw_complex kD3 = diff3.camp(k);
      lib_matrFillValueVecCpx(kD, m1, nth);
      lib_matrProdDiagCpxR(m1, Af, nth, 3, K);
      lib_matrFillOnesVecCpx(m1, nth);
      for (int l = 0; l < nth; l++) m1[l].re /= norm_seis[l];
      lib_matrFillValueVecCpx(kD3, m2, nth);
      for (int l = 0; l < nth; l++) {
        float errorSmoothMult = 1.0f / norm_es3[l];
        m2[l].re *= errorSmoothMult;
        m2[l].im *= errorSmoothMult;
      }
      for (int l = 0; l < nth; l++) {
        fftw_complex value = w_norm[l].camp(k);
        fftw_complex valueFine = w_norm[l].camp_scaled(k, 0.999f);
        float modulus = value.re * value.re + value.im * value.im;
        float modulusFine = valueFine.re * valueFine.re + valueFine.im * valueFine.im;
        float maxMod = std::max(modulus, modulusFine);
        if (maxMod > 0.0) {
          m3[l].re = float(1.0 / std::sqrt(maxMod));
          m3[l].im = 0.0f;
        } else {
          m3[l].re = w_norm[l].norm * nzp * nzp * 100.0f;
          m3[l].im = 0.0;
        }
      }
    }
    bool inv = realFrequency > b->low_cut * b->min_rel_thick && realFrequency < b->high_cut;
    for (int j = 0; j < nyp; j++) {
      for (int i = 0; i < cnxp; i++, idx++) {
        for (int a = 0; a < 3; a++) mu[a] = G_mean[a].c()[idx];
        for (int l = 0; l < nth; l++) { d[l] = G_data[l].c()[idx]; res[l] = d[l]; }
        // getNextParameterCovariance
        for (int q = 0; q < 6; q++) {
          fftw_complex t = G_cov[q].c()[idx];
          float p = static_cast<float>(pv[pa[q] * 3 + pb[q]]);
          if (pv[pa[q] * 3 + pb[q]] != 0) t.re = t.re / p;
          float v = float(std::sqrt(t.re * t.re));
          par[pa[q]][pb[q]].re = v * p;
          par[pa[q]][pb[q]].im = 0.0f;
          par[pb[q]][pa[q]].re = v * p;
          par[pb[q]][pa[q]].im = -0.0f;
        }
        // getNextErrorVariance
        fftw_complex et = G_err.c()[idx];
        float lam = float(std::sqrt(et.re * et.re));
        if (inv) {
          for (int l = 0; l < nth; l++) {
            for (int m = 0; m < nth; m++) {
              double ec = b->err_theta_cov[l * nth + m];
              err[l][m].re = float(0.5 * (1.0 - b->wnc) * ec * lam * (m1[l].re * m1[m].re + m1[l].im * m1[m].im));
              err[l][m].re += float(0.5 * (1.0 - b->wnc) * ec * lam * (m2[l].re * m2[m].re + m2[l].im * m2[m].im));
              if (l == m) {
                err[l][m].re += float(b->wnc * ec * m3[l].re * m3[l].re);
                err[l][m].im = 0.0;
              } else {
                err[l][m].im = float(0.5 * (1.0 - b->wnc) * ec * lam * (-m1[l].re * m1[m].im + m1[l].im * m1[m].re));
                err[l][m].im += float(0.5 * (1.0 - b->wnc) * ec * lam * (-m2[l].re * m2[m].im + m2[l].im * m2[m].re));
              }
            }
          }
          n_inv++;
          lib_matrProdCpx(K, par, nth, 3, 3, KS);
          lib_matrProdAdjointCpx(KS, K, nth, 3, nth, marg);
          lib_matrAddMatCpx(err, nth, nth, marg);
          int flag = lib_matrCholCpx(nth, marg);
          if (flag == 0) {
            lib_matrAdjoint(KS, nth, 3, KScc);
            lib_matrAXeqBMatCpx(nth, marg, KS, 3);
            lib_matrProdCpx(KScc, KS, 3, nth, 3, red);
            lib_matrSubtMatCpx(red, 3, 3, par);
            lib_matrProdMatVecCpx(K, mu, nth, 3, dmean);
            lib_matrSubtVecCpx(dmean, nth, d);
            lib_matrProdAdjointMatVecCpx(KS, d, 3, nth, ans);
            lib_matrAddVecCpx(ans, 3, mu);
            lib_matrProdMatVecCpx(K, mu, nth, 3, d);
            lib_matrSubtVecCpx(d, nth, res);
          } else {
            n_fail++;
          }
        }
        for (int a = 0; a < 3; a++) G_mean[a].c()[idx] = mu[a];
        for (int q = 0; q < 6; q++) G_cov[q].c()[idx] = par[pa[q]][pb[q]];
        for (int l = 0; l < nth; l++) G_data[l].c()[idx] = res[l];
      }
    }
  }
  for (int a = 0; a < 3; a++) inv_fft_in_place(G_mean[a], false);

  // simulate (src/avoinversion.cpp:1354-1511)
  if (nsim > 0 && sims) {
    RandomGen rg(seed);
    size_t csize = size_t(cnxp) * nyp * nzp;
    fftw_complex** pc = cmat(3, 3);
    fftw_complex sd[3];
    for (int s = 0; s < nsim; s++) {
      Grid sg[3];
      for (int a = 0; a < 3; a++) {
        sg[a] = make_grid(sims[s * 3 + a], nxp, nyp, nzp);
        if (noise_in)
          std::memcpy(sg[a].r, noise_in + (size_t(s) * 3 + a) * 2 * csize, 2 * csize * sizeof(float));
        else
          fill_complex_noise(sg[a].c(), nxp, nyp, nzp);
      }
      for (size_t q = 0; q < csize; q++) {
        pc[0][0] = G_cov[0].c()[q];
        pc[1][1] = G_cov[1].c()[q];
        pc[2][2] = G_cov[2].c()[q];
        pc[0][1] = G_cov[3].c()[q];
        pc[0][2] = G_cov[4].c()[q];
        pc[1][2] = G_cov[5].c()[q];
        pc[1][0].re = pc[0][1].re; pc[1][0].im = -pc[0][1].im;
        pc[2][0].re = pc[0][2].re; pc[2][0].im = -pc[0][2].im;
        pc[2][1].re = pc[1][2].re; pc[2][1].im = -pc[1][2].im;
        for (int a = 0; a < 3; a++) sd[a] = sg[a].c()[q];
        if (lib_matrCholCpx(3, pc) == 0) {
          lib_matrProdCholVec(3, pc, sd);
        } else {
          for (int a = 0; a < 3; a++) { sd[a].re = 0.0; sd[a].im = 0.0; }
        }
        for (int a = 0; a < 3; a++) sg[a].c()[q] = sd[a];
      }
      for (int a = 0; a < 3; a++) {
        inv_fft_in_place(sg[a], false);
        for (size_t q = 0; q < sg[a].rsize(); q++) sg[a].r[q] += G_mean[a].r[q];
      }
    }
    free_cmat(pc, 3);
  }
  // invFFTCovGrids (src/seismicparametersholder.cpp:432-456)
  for (int a = 0; a < 6; a++) inv_fft_in_place(G_cov[a], true);

  if (counters) { counters[0] = n_inv; counters[1] = n_fail; }
  delete[] kW; delete[] m1; delete[] m2; delete[] m3; delete[] d; delete[] dmean; delete[] res;
  free_cmat(K, nth); free_cmat(KS, nth); free_cmat(KScc, 3); free_cmat(par, 3);
  free_cmat(marg, nth); free_cmat(err, nth); free_cmat(red, 3);
  for (int l = 0; l < nth; l++) delete[] Af[l];
  delete[] Af;
  return 0;
}

// The trace transform of AVOInversion::divideDataByScaleWavelet (src/avoinversion.cpp:
// 537-588) with the reference's FFTW: ntr traces of nzp floats (traces[t*nzp + k]), each
// divided by float(sqrt(float(nzp))), tapered (taper[k], 1 up to nz), transformed by a
// 1D in-place rfftwnd plan, multiplied by factor[t*cnzp + k] (complex) where band[t*cnzp + k]
// and zeroed elsewhere, transformed back and divided by float(sqrt(float(nzp))), in place.
void ref32_divide_traces(float* traces, int ntr, int nzp, const float* taper, const float* factor,
                         const unsigned char* band) {
  const int cn = nzp / 2 + 1;
  std::vector<float> r(2 * cn);
  fftw_complex* c = reinterpret_cast<fftw_complex*>(r.data());
  int n = nzp;
  rfftwnd_plan p1 = rfftwnd_create_plan(1, &n, FFTW_REAL_TO_COMPLEX, FFTW_ESTIMATE | FFTW_IN_PLACE);
  rfftwnd_plan p2 = rfftwnd_create_plan(1, &n, FFTW_COMPLEX_TO_REAL, FFTW_ESTIMATE | FFTW_IN_PLACE);
  const float rsq = static_cast<float>(std::sqrt(static_cast<float>(nzp)));
  for (int t = 0; t < ntr; t++) {
    float* tr = traces + (size_t)t * nzp;
    for (int k = 0; k < nzp; k++) r[k] = tr[k] / rsq * taper[k];
    rfftwnd_one_real_to_complex(p1, r.data(), c);
    const float* f = factor + 2 * (size_t)t * cn;
    const unsigned char* b = band + (size_t)t * cn;
    for (int k = 0; k < cn; k++) {
      if (b[k]) {
        const float fr = f[2 * k], fi = f[2 * k + 1];
        const float tmp = c[k].re * fr - c[k].im * fi;
        c[k].im = c[k].im * fr + c[k].re * fi;
        c[k].re = tmp;
      } else {
        c[k].re = 0.0f;
        c[k].im = 0.0f;
      }
    }
    rfftwnd_one_complex_to_real(p2, c, r.data());
    for (int k = 0; k < nzp; k++) tr[k] = r[k] / rsq;
  }
  rfftwnd_destroy_plan(p1);
  rfftwnd_destroy_plan(p2);
}

// Noise grids of nsim realisations exactly as simulate draws them from RandomGen(seed):
// out holds (nsim*3) complex grids of cnxp*nyp*nzp values each.
void ref32_sim_noise(unsigned int seed, int nsim, int nxp, int nyp, int nzp, float* out) {
  RandomGen rg(seed);
  size_t csize = size_t(nxp / 2 + 1) * nyp * nzp;
  for (int g = 0; g < nsim * 3; g++)
    fill_complex_noise(reinterpret_cast<fftw_complex*>(out + size_t(g) * 2 * csize), nxp, nyp, nzp);
}


// FaciesProb::calculateFaciesProb with findDensity (src/faciesprob.cpp:1909-2075, 1307-1423)
// in the reference's float arithmetic: per voxel, for every corner volume c (2^nang of them,
// the single-volume case nang = 0) Simbox::getInterpolationIndexes of a flat, unrotated box
// (src/simbox.cpp:745-760: (x - xmin) / dx - 0.5 in double), the clamped trilinear sum in float
// with the reference's term order, the corner weights prod (t or 1 - t) by the bits of c, the
// prior weighting and the normalisation with undefSum.  post: 3 arrays of nx*ny*nz (index
// i + nx (j + ny k)); dens[c]: nf cubes of nb0*nb1*nb2 (index j + nb0 (k + nb1 l)); box[c]:
// 9 doubles (vmin[3], dv[3], nb[3]); t: nang x nx*ny; out: (nf + 1) x nx*ny*nz.
void ref32_facies_prob(const float* const* post, int nx, int ny, int nz, int nang, const float* const* dens,
                       const double* box, int nf, const float* prior, float p_undefined, const float* t,
                       float* out) {
  const int nc = 1 << nang;
  const size_t nvox = (size_t)nx * ny * nz;
  const float undefSum = p_undefined / (float)((int)box[6] * (int)box[7] * (int)box[8]);
  std::vector<float> value(nc), val(nf);
  for (size_t e = 0; e < nvox; e++) {
    const size_t tr = e % ((size_t)nx * ny);
    const float vp = post[0][e], vs = post[1][e], rho = post[2][e];
    float sum = undefSum;
    for (int l = 0; l < nf; l++) {
      for (int c = 0; c < nc; c++) {
        const double* b = box + 9 * c;
        const int nb[3] = {(int)b[6], (int)b[7], (int)b[8]};
        const double full[3] = {((double)vp - b[0]) / b[3] - 0.5, ((double)vs - b[1]) / b[4] - 0.5,
                                ((double)rho - b[2]) / b[5] - 0.5};
        int i1[3], i2[3];
        float w[3];
        for (int d = 0; d < 3; d++) {
          i1[d] = static_cast<int>(floor(full[d]));
          if (i1[d] < 0) { i1[d] = 0; i2[d] = 0; w[d] = 0; }
          else if (i1[d] >= nb[d] - 1) { i1[d] = nb[d] - 1; i2[d] = i1[d]; w[d] = 0; }
          else { i2[d] = i1[d] + 1; w[d] = static_cast<float>(full[d] - i1[d]); }
        }
        const float* D = dens[c] + (size_t)l * nb[0] * nb[1] * nb[2];
        auto at = [&](int j, int k, int m) { return std::max<float>(0, D[j + (size_t)nb[0] * (k + (size_t)nb[1] * m)]); };
        const float wj = w[0], wk = w[1], wl = w[2];
        float v = 0;
        v += (1.0f - wj) * (1.0f - wk) * (1.0f - wl) * at(i1[0], i1[1], i1[2]);
        v += (1.0f - wj) * (1.0f - wk) * (wl) * at(i1[0], i1[1], i2[2]);
        v += (1.0f - wj) * (wk) * (1.0f - wl) * at(i1[0], i2[1], i1[2]);
        v += (1.0f - wj) * (wk) * (wl) * at(i1[0], i2[1], i2[2]);
        v += (wj) * (1.0f - wk) * (1.0f - wl) * at(i2[0], i1[1], i1[2]);
        v += (wj) * (1.0f - wk) * (wl) * at(i2[0], i1[1], i2[2]);
        v += (wj) * (wk) * (1.0f - wl) * at(i2[0], i2[1], i1[2]);
        v += (wj) * (wk) * (wl) * at(i2[0], i2[1], i2[2]);
        value[c] = v;
      }
      float valuesum = 0;
      for (int c = 0; c < nc; c++) {
        int factor = 1;
        for (int a = 0; a < nang; a++) {
          if (a > 0) factor *= 2;
          const float ta = t[(size_t)a * nx * ny + tr];
          if ((c & factor) > 0) value[c] *= ta;
          else value[c] *= (1 - ta);
        }
        valuesum += value[c];
      }
      const float dns = valuesum > 0.0 ? valuesum : 0.0f;
      val[l] = prior[l] * dns;
      sum = sum + val[l];
    }
    for (int l = 0; l < nf; l++) out[(size_t)l * nvox + e] = val[l] / sum;
    out[(size_t)nf * nvox + e] = undefSum / sum;
  }
}

}  // extern "C"
