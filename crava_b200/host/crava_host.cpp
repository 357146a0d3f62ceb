// C++ host layer over the C ABI; see crava_host.h.
#include "crava_host.h"

#include <algorithm>
#include <cstring>

namespace crava_b200 {

namespace {

void check(crava_status s) {
  if (s != CRAVA_OK) {
    const char* m = crava_last_error();
    throw Error(s, std::string(crava_status_string(s)) + ": " + (m ? m : ""));
  }
}

}  // namespace

// ------------------------------------------------------------------ Context

Context::Context(int device, size_t hbm_budget) { check(crava_ctx_create(&ctx_, device, hbm_budget)); }

Context::~Context() {
  if (ctx_) crava_ctx_destroy(ctx_);
}

// ------------------------------------------------------------------ FFTGrid
// FFTGrid::FFTGrid (src/fftgrid.cpp:40-70): padded sizes cnxp = nxp/2 + 1, rnxp = 2 cnxp,
// element (i, j, k) of the real grid at i + rnxp (j + nyp k).

FFTGrid::FFTGrid(Context* ctx, int nx, int ny, int nz, int nxp, int nyp, int nzp)
    : ctx_(ctx), nx_(nx), ny_(ny), nz_(nz), nxp_(nxp), nyp_(nyp), nzp_(nzp) {
  cnxp_ = nxp_ / 2 + 1;
  rnxp_ = 2 * cnxp_;
  csize_ = (size_t)cnxp_ * nyp_ * nzp_;
  rsize_ = (size_t)rnxp_ * nyp_ * nzp_;
}

FFTGrid::FFTGrid(const FFTGrid& o)
    : ctx_(o.ctx_), cubetype_(o.cubetype_), nx_(o.nx_), ny_(o.ny_), nz_(o.nz_), nxp_(o.nxp_), nyp_(o.nyp_),
      nzp_(o.nzp_), cnxp_(o.cnxp_), rnxp_(o.rnxp_), csize_(o.csize_), rsize_(o.rsize_),
      istransformed_(o.istransformed_), rvalue_(o.rvalue_) {}

void FFTGrid::createRealGrid() {
  rvalue_.assign(rsize_, 0.f);
  istransformed_ = false;
  counterForGet_ = counterForSet_ = 0;
}

void FFTGrid::createComplexGrid() {
  rvalue_.assign(rsize_, 0.f);
  istransformed_ = true;
  counterForGet_ = counterForSet_ = 0;
}

// FFTGrid::fftInPlace / invFFTInPlace (src/fftgrid.cpp:1587-1643)
void FFTGrid::fftInPlace() {
  if (rvalue_.empty()) createRealGrid();
  check(crava_fft_r2c_host(ctx_->get(), rvalue_.data(), nxp_, nyp_, nzp_, cubetype_ == COVARIANCE));
  istransformed_ = true;
}

void FFTGrid::invFFTInPlace() {
  if (rvalue_.empty()) createComplexGrid();
  check(crava_fft_c2r_host(ctx_->get(), rvalue_.data(), nxp_, nyp_, nzp_, cubetype_ == COVARIANCE));
  istransformed_ = false;
}

// Sequential access (src/fftgrid.cpp:1203-1235, 1392-1443): the counter walks the whole
// padded buffer and wraps to zero after the last element.
float FFTGrid::getNextReal() {
  if (istransformed_ || counterForGet_ >= rsize_) return RMISSING;
  float r = rvalue_[counterForGet_++];
  if (counterForGet_ == rsize_) counterForGet_ = 0;
  return r;
}

int FFTGrid::setNextReal(float value) {
  if (istransformed_ || counterForSet_ >= rsize_) return 1;
  rvalue_[counterForSet_++] = value;
  if (counterForSet_ == rsize_) counterForSet_ = 0;
  return 0;
}

std::complex<float> FFTGrid::getNextComplex() {
  if (!istransformed_ || counterForGet_ >= csize_) return {RMISSING, RMISSING};
  const size_t c = counterForGet_++;
  if (counterForGet_ == csize_) counterForGet_ = 0;
  return {rvalue_[2 * c], rvalue_[2 * c + 1]};
}

int FFTGrid::setNextComplex(std::complex<float> value) {
  if (!istransformed_ || counterForSet_ >= csize_) return 1;
  const size_t c = counterForSet_++;
  rvalue_[2 * c] = value.real();
  rvalue_[2 * c + 1] = value.imag();
  if (counterForSet_ == csize_) counterForSet_ = 0;
  return 0;
}

// Random access (src/fftgrid.cpp:1237-1283, 1335-1390, 1445-1500): RMISSING (and a
// non-zero return for the setters) outside the simbox, or outside the padded grid when
// extSimbox is set.
float FFTGrid::getRealValue(int i, int j, int k, bool extSimbox) const {
  const bool in = extSimbox ? (i < nxp_ && j < nyp_ && k < nzp_) : (i < nx_ && j < ny_ && k < nz_);
  if (istransformed_ || !in || i < 0 || j < 0 || k < 0 || rvalue_.empty()) return RMISSING;
  return rvalue_[(size_t)i + (size_t)rnxp_ * ((size_t)j + (size_t)nyp_ * k)];
}

int FFTGrid::setRealValue(int i, int j, int k, float value, bool extSimbox) {
  const bool in = extSimbox ? (i < nxp_ && j < nyp_ && k < nzp_) : (i < nx_ && j < ny_ && k < nz_);
  if (istransformed_ || !in || i < 0 || j < 0 || k < 0 || rvalue_.empty()) return 1;
  rvalue_[(size_t)i + (size_t)rnxp_ * ((size_t)j + (size_t)nyp_ * k)] = value;
  return 0;
}

std::complex<float> FFTGrid::getComplexValue(int i, int j, int k, bool extSimbox) const {
  const bool in = extSimbox ? (i < cnxp_ && j < nyp_ && k < nzp_) : (i < nx_ && j < ny_ && k < nz_);
  if (!istransformed_ || !in || i < 0 || j < 0 || k < 0 || rvalue_.empty()) return {RMISSING, RMISSING};
  const size_t c = (size_t)i + (size_t)cnxp_ * ((size_t)j + (size_t)nyp_ * k);
  return {rvalue_[2 * c], rvalue_[2 * c + 1]};
}

int FFTGrid::setComplexValue(int i, int j, int k, std::complex<float> value, bool extSimbox) {
  const bool in = extSimbox ? (i < cnxp_ && j < nyp_ && k < nzp_) : (i < nx_ && j < ny_ && k < nz_);
  if (!istransformed_ || !in || i < 0 || j < 0 || k < 0 || rvalue_.empty()) return 1;
  const size_t c = (size_t)i + (size_t)cnxp_ * ((size_t)j + (size_t)nyp_ * k);
  rvalue_[2 * c] = value.real();
  rvalue_[2 * c + 1] = value.imag();
  return 0;
}

// FFTGrid::fillInConstant (src/fftgrid.cpp:634-652): the padded real grid.
void FFTGrid::fillInConstant(float value) {
  createRealGrid();
  for (int k = 0; k < nzp_; k++)
    for (int j = 0; j < nyp_; j++)
      for (int i = 0; i < nxp_; i++) rvalue_[(size_t)i + (size_t)rnxp_ * ((size_t)j + (size_t)nyp_ * k)] = value;
}

// ------------------------------------------------------------------ AVOInversion

AVOInversion::AVOInversion(Context* ctx, const AVOInversionSettings& settings, std::vector<FFTGrid*>& seisData,
                           SeismicParametersHolder& sp, const std::vector<float>* corrXY,
                           const std::vector<float>* circCorrT)
    : ctx_(ctx), set_(settings), seis_(seisData), sp_(sp) {
  if (corrXY && circCorrT) {
    corrXY_ = *corrXY;
    circCorrT_ = *circCorrT;
    separable_ = true;
  }
  if ((int)seis_.size() != set_.ntheta || set_.ntheta < 1)
    throw Error(CRAVA_EINVAL, "AVOInversion: one DATA grid per angle is needed");
}

AVOInversion::~AVOInversion() = default;

int AVOInversion::simulate(const std::vector<FFTGrid*>* noise) {
  noise_ = noise;
  if (done_) {
    // the realisations were produced with the posterior; with new noise, run again
    if (noise) {
      done_ = false;
      run();
    }
  }
  return 0;
}

int AVOInversion::computePostMeanResidAndFFTCov() {
  if (!done_) run();
  return 0;
}

// One job: the forward transforms of AVOInversion::AVOInversion (src/avoinversion.cpp:
// 229-244), computePostMeanResidAndFFTCov (:794-1231), simulate (:1354-1540) and the
// inverse transforms of the posterior (:1112-1114, :274-282) in one fused pass.
void AVOInversion::run() {
  FFTGrid* g0 = seis_[0];
  const int nth = set_.ntheta;
  const int nsim = set_.nSimulations;
  crava_job_desc d;
  std::memset(&d, 0, sizeof(d));
  d.nx = g0->getNx();
  d.ny = g0->getNy();
  d.nz = g0->getNz();
  d.nxp = g0->getNxp();
  d.nyp = g0->getNyp();
  d.nzp = g0->getNzp();
  d.ntheta = nth;
  d.lz = set_.lz;
  d.min_rel_thick = set_.minRelThick;
  d.low_cut = set_.lowCut;
  d.high_cut = set_.highCut;
  d.wnc = set_.wnc;
  std::vector<double> A(set_.A.begin(), set_.A.end());
  std::vector<float> wav((size_t)nth * d.nzp);
  const std::vector<float>& wn = set_.waveletNorm;
  for (int l = 0; l < nth; l++)
    for (int k = 0; k < d.nzp; k++) wav[(size_t)l * d.nzp + k] = set_.wavelet[l][k];
  std::vector<double> pv(9);
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) pv[a * 3 + b] = sp_.priorVar0[a][b];
  d.A = A.data();
  d.err_theta_cov = set_.errThetaCov.data();
  d.wavelet = wav.data();
  d.wavelet_norm = wn.data();
  d.prior_var0 = pv.data();
  // factors with nonzero correlation gradients: InitializeCorrelations' grids are generated
  // on the device (crava_job_fill_prior) and inverted in GRIDS mode
  const bool gradients = separable_ && (set_.corrGradI != 0.f || set_.corrGradJ != 0.f);
  if (separable_) {
    d.prior_mode = gradients ? CRAVA_PRIOR_GRIDS : CRAVA_PRIOR_SEPARABLE;
    d.corr_xy = corrXY_.data();
    d.circ_corr_t = circCorrT_.data();
  } else {
    d.prior_mode = CRAVA_PRIOR_GRIDS;
  }
  d.nsim = nsim;
  d.seed = set_.seed;
  d.flags = CRAVA_FLAG_KEEP_RESIDUAL | (noise_ ? CRAVA_FLAG_HOST_NOISE : 0);
  d.fp64_threshold = set_.fp64Threshold;
  // non-constant thickness: the temporal correlation the adjustment factor needs is the
  // covVp column at (0, 0) (SeismicParametersHolder::extractParamCorrFromCovVp,
  // src/seismicparametersholder.cpp:1008-1028) unless the separable factor is given
  std::vector<float> corrCol;
  if (!set_.relThick.empty()) {
    if (set_.relThick.size() != (size_t)d.nxp * d.nyp)
      throw Error(CRAVA_EINVAL, "AVOInversion: relThick needs nxp*nyp values");
    d.flags |= CRAVA_FLAG_NONCONST_THICK;
    d.rel_thick = set_.relThick.data();
    d.energy_threshold = set_.energyThreshold;
    if (!separable_) {
      if (!sp_.covVp) throw Error(CRAVA_EINVAL, "AVOInversion: covVp is missing");
      const float* cv = sp_.covVp->getRealData();
      const size_t rnxp = 2 * (size_t)(d.nxp / 2 + 1);
      corrCol.resize(d.nzp);
      for (int k = 0; k < d.nzp; k++) corrCol[k] = cv[(size_t)k * rnxp * d.nyp];
      d.circ_corr_t = corrCol.data();
    }
  }

  crava_job* job = nullptr;
  check(crava_job_create(ctx_->get(), &d, &job));
  struct Guard {
    crava_job* j;
    ~Guard() { crava_job_destroy(j); }
  } guard{job};
  auto up = [&](crava_role role, int index, FFTGrid* g) {
    if (!g) throw Error(CRAVA_EINVAL, "AVOInversion: a grid the inversion needs is missing");
    check(crava_job_upload(job, role, index, g->getRealData(), nullptr));
  };
  for (int l = 0; l < nth; l++) up(CRAVA_ROLE_DATA, l, seis_[l]);
  up(CRAVA_ROLE_MEAN, 0, sp_.meanVp);
  up(CRAVA_ROLE_MEAN, 1, sp_.meanVs);
  up(CRAVA_ROLE_MEAN, 2, sp_.meanRho);
  FFTGrid* cov[6] = {sp_.covVp, sp_.covVs, sp_.covRho, sp_.crCovVpVs, sp_.crCovVpRho, sp_.crCovVsRho};
  if (!separable_) {
    for (int q = 0; q < 6; q++) up(CRAVA_ROLE_PRIOR_COV, q, cov[q]);
    up(CRAVA_ROLE_ERR_CORR, 0, sp_.errCorr);
  } else if (gradients) {
    check(crava_job_fill_prior(job, set_.corrGradI, set_.corrGradJ, nullptr));
  }
  if (noise_) {
    if ((int)noise_->size() != 3 * nsim) throw Error(CRAVA_EINVAL, "simulate: 3 noise grids per realisation");
    for (int q = 0; q < 3 * nsim; q++) up(CRAVA_ROLE_NOISE, q, (*noise_)[q]);
  }
  // the wavelets' local shift and gain grids, and 3D wavelets (used by the division)
  const size_t nxy = (size_t)d.nx * d.ny;
  for (int l = 0; l < nth; l++) {
    const float* sh = (size_t)l < set_.waveletShift.size() && !set_.waveletShift[l].empty()
                          ? set_.waveletShift[l].data() : nullptr;
    const float* gn = (size_t)l < set_.waveletGain.size() && !set_.waveletGain[l].empty()
                          ? set_.waveletGain[l].data() : nullptr;
    if ((sh && set_.waveletShift[l].size() != nxy) || (gn && set_.waveletGain[l].size() != nxy))
      throw Error(CRAVA_EINVAL, "AVOInversion: wavelet shift and gain grids need nx*ny values");
    if (sh || gn) check(crava_job_set_wavelet_grids(job, l, sh, gn));
  }
  std::vector<float> gw;
  if (set_.waveletDim == 3) {
    const size_t nij = (size_t)set_.filterNI * set_.filterNJ;
    if ((int)set_.theta.size() != nth || set_.filterAlpha1.size() != nth * nij ||
        (!set_.filterHalpha.empty() && set_.filterHalpha.size() != nth * nij) ||
        (int)set_.globalWavelet.size() != nth || (int)set_.globalWaveletNorm.size() != nth ||
        (!set_.depthGradX.empty() && set_.depthGradX.size() != nxy) ||
        (!set_.depthGradY.empty() && set_.depthGradY.size() != nxy))
      throw Error(CRAVA_EINVAL, "AVOInversion: 3D wavelet settings have the wrong sizes");
    for (int l = 0; l < nth; l++) {
      if ((int)set_.globalWavelet[l].size() != d.nzp) throw Error(CRAVA_EINVAL, "AVOInversion: global wavelet needs nzp samples");
      gw.insert(gw.end(), set_.globalWavelet[l].begin(), set_.globalWavelet[l].end());
    }
    crava_wavelet3d_desc w{};
    w.grad_x = set_.depthGradX.empty() ? nullptr : set_.depthGradX.data();
    w.grad_y = set_.depthGradY.empty() ? nullptr : set_.depthGradY.data();
    w.theta = set_.theta.data();
    w.filter_ni = set_.filterNI;
    w.filter_nj = set_.filterNJ;
    w.filter_x0 = set_.filterX0;
    w.filter_y0 = set_.filterY0;
    w.filter_dx = set_.filterDX;
    w.filter_dy = set_.filterDY;
    w.alpha1 = set_.filterAlpha1.data();
    w.halpha = set_.filterHalpha.empty() ? nullptr : set_.filterHalpha.data();
    w.global_wavelet = gw.data();
    w.global_wavelet_norm = set_.globalWaveletNorm.data();
    check(crava_job_set_wavelet_3d(job, &w));
  }
  // the constructor's divideDataByScaleWavelet (src/avoinversion.cpp:226-227)
  if (d.flags & CRAVA_FLAG_NONCONST_THICK) check(crava_job_divide_data(job, nullptr));
  check(crava_job_run(job, nullptr));
  // outputs in place of the inputs, as the reference overwrites them
  FFTGrid* mean[3] = {sp_.meanVp, sp_.meanVs, sp_.meanRho};
  for (int a = 0; a < 3; a++) {
    check(crava_job_download(job, CRAVA_ROLE_POST_MEAN, a, mean[a]->getRealData(), nullptr));
    mean[a]->setTransformedStatus(false);
  }
  for (int q = 0; q < 6; q++) {
    if (!cov[q]) continue;
    check(crava_job_download(job, CRAVA_ROLE_POST_COV, q, cov[q]->getRealData(), nullptr));
    cov[q]->setTransformedStatus(false);
  }
  for (int l = 0; l < nth; l++) {
    check(crava_job_download(job, CRAVA_ROLE_RESIDUAL, l, seis_[l]->getRealData(), nullptr));
    seis_[l]->setTransformedStatus(true);
  }
  sp_.simulations.clear();
  for (int q = 0; q < 3 * nsim; q++) {
    auto g = std::make_unique<FFTGrid>(*sp_.meanVp);
    g->createRealGrid();
    check(crava_job_download(job, CRAVA_ROLE_SIM, q, g->getRealData(), nullptr));
    sp_.simulations.push_back(std::move(g));
  }
  check(crava_job_counters(job, &counters_));
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) sp_.postVar0[a][b] = counters_.post_var0[a * 3 + b];
  done_ = true;
}

}  // namespace crava_b200
