// C++ host layer over the C ABI (include/crava_gpu.h): the reference's hot-path classes
// with their names, argument meaning and error behaviour, backed by the B200 library.
//
//   crava_b200::FFTGrid        FFTGrid (src/fftgrid.h:22-285): padded real/complex grid in
//                              host memory, fftInPlace / invFFTInPlace on the GPU
//   crava_b200::AVOInversion   AVOInversion (src/avoinversion.h:33-120):
//                              computePostMeanResidAndFFTCov and simulate on the GPU
//   crava_b200::SeismicParametersHolder  the grids of SeismicParametersHolder that the
//                              inversion reads and overwrites (src/seismicparametersholder.h)
//
// Error behaviour follows the reference: the int-returning calls return 0, grid accessors
// return RMISSING outside the grid, the per-bin Cholesky fallbacks are silent (counted in
// AVOInversion::counters()).  Library failures (no GPU, out of memory) throw
// crava_b200::Error, where the reference would have stopped with exit(1).
#pragma once

#include <complex>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "crava_gpu.h"

namespace crava_b200 {

constexpr float RMISSING = -99999.000f;

class Error : public std::runtime_error {
 public:
  Error(crava_status s, const std::string& what) : std::runtime_error(what), status(s) {}
  crava_status status;
};

// One GPU: the library context every grid and inversion on that device uses.
class Context {
 public:
  explicit Context(int device = 0, size_t hbm_budget = 0);
  ~Context();
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  crava_ctx* get() const { return ctx_; }

 private:
  crava_ctx* ctx_ = nullptr;
};

class FFTGrid {
 public:
  enum gridTypes { CTMISSING, DATA, PARAMETER, COVARIANCE, VELOCITY };
  enum accessMode { NONE, READ, WRITE, READANDWRITE, RANDOMACCESS };

  FFTGrid(Context* ctx, int nx, int ny, int nz, int nxp, int nyp, int nzp);
  FFTGrid(const FFTGrid& other);   // deep copy, like FFTGrid(FFTGrid*)
  virtual ~FFTGrid() = default;

  void setType(int cubeType) { cubetype_ = cubeType; }
  int getType() const { return cubetype_; }
  void createRealGrid();           // zeroed, real state
  void createComplexGrid();        // zeroed, Fourier state
  // 3D transforms with FFTGrid's scalings: PARAMETER/DATA 1/sqrt(N) both ways,
  // COVARIANCE none forward and 1/N inverse.
  virtual void fftInPlace();
  virtual void invFFTInPlace();

  virtual void setAccessMode(int mode) { accessMode_ = mode; }
  virtual void endAccess() { counterForGet_ = counterForSet_ = 0; }
  float getNextReal();
  int setNextReal(float value);
  std::complex<float> getNextComplex();
  int setNextComplex(std::complex<float> value);
  float getRealValue(int i, int j, int k, bool extSimbox = false) const;
  int setRealValue(int i, int j, int k, float value, bool extSimbox = false);
  std::complex<float> getComplexValue(int i, int j, int k, bool extSimbox = false) const;
  int setComplexValue(int i, int j, int k, std::complex<float> value, bool extSimbox = false);
  void fillInConstant(float value);

  int getNx() const { return nx_; }
  int getNy() const { return ny_; }
  int getNz() const { return nz_; }
  int getNxp() const { return nxp_; }
  int getNyp() const { return nyp_; }
  int getNzp() const { return nzp_; }
  int getRNxp() const { return rnxp_; }
  int getCNxp() const { return cnxp_; }
  size_t getrsize() const { return rsize_; }
  size_t getcsize() const { return csize_; }
  bool getIsTransformed() const { return istransformed_; }
  void setTransformedStatus(bool status) { istransformed_ = status; }
  // The padded buffer (rsize floats; the spectrum as csize complex in the same bytes).
  float* getRealData() { return rvalue_.data(); }
  const float* getRealData() const { return rvalue_.data(); }
  Context* context() const { return ctx_; }

 protected:
  Context* ctx_;
  int cubetype_ = CTMISSING;
  int nx_, ny_, nz_, nxp_, nyp_, nzp_, cnxp_, rnxp_;
  size_t csize_, rsize_;
  size_t counterForGet_ = 0, counterForSet_ = 0;
  int accessMode_ = NONE;
  bool istransformed_ = false;
  std::vector<float> rvalue_;
};

// The grids AVOInversion reads from and writes to SeismicParametersHolder: prior mean
// (overwritten by the posterior mean, as postVp_ = meanVp_ aliases it), the six prior
// covariance grids (overwritten by the posterior covariance) and the error correlation,
// plus the realisations simulate() adds.
struct SeismicParametersHolder {
  FFTGrid* meanVp = nullptr;
  FFTGrid* meanVs = nullptr;
  FFTGrid* meanRho = nullptr;
  FFTGrid* covVp = nullptr;      // COVARIANCE grids, order Vp, Vs, Rho, VpVs, VpRho, VsRho
  FFTGrid* covVs = nullptr;
  FFTGrid* covRho = nullptr;
  FFTGrid* crCovVpVs = nullptr;
  FFTGrid* crCovVpRho = nullptr;
  FFTGrid* crCovVsRho = nullptr;
  FFTGrid* errCorr = nullptr;    // COVARIANCE
  std::vector<std::unique_ptr<FFTGrid>> simulations;  // 3 per realisation: Vp, Vs, Rho
  double priorVar0[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  double postVar0[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
};

// What AVOInversion takes from ModelSettings, ModelGeneral and ModelAVODynamic for the
// constant-thickness inversion.
struct AVOInversionSettings {
  int ntheta = 0;
  std::vector<float> A;                    // ntheta x 3 reflection coefficients, row major
  std::vector<double> errThetaCov;         // ntheta x ntheta
  std::vector<std::vector<float>> wavelet; // ntheta x nzp, resampled, FFT order
  std::vector<float> waveletNorm;          // ntheta
  double lz = 0, minRelThick = 1;
  float lowCut = 5, highCut = 55, wnc = 0.1f;
  int nSimulations = 0;
  uint64_t seed = 1;                       // device noise (product mode)
  float fp64Threshold = 0;                 // 0: FP32 only
  // Simbox::getIsConstantThick() == false: Simbox::getRelThick(i, j) at every padded trace
  // (nxp*nyp, index i+nxp*j); the data are then divided by the scale wavelet first
  // (divideDataByScaleWavelet + interpolateSeismic).  Empty: constant thickness.
  std::vector<double> relThick;
  float energyThreshold = 0;               // ModelSettings::getEnergyThreshold
  // Local wavelets of the division (Wavelet::shiftGrid_ / gainGrid_ in ms and as factors,
  // nx*ny per angle, index i+nx*j; an empty angle or an empty vector: none)
  std::vector<std::vector<float>> waveletShift, waveletGain;
  // 3D wavelets (Wavelet3D, getDim() == 3): the wavelets above are their own pulses; the
  // filter surfaces, depth gradients, angles and global (average) wavelets as in
  // crava_wavelet3d_desc.  waveletDim 1: none of these is used.
  int waveletDim = 1;
  std::vector<float> depthGradX, depthGradY;                 // nx*ny each, or empty
  std::vector<float> theta;                                  // ntheta radians
  int filterNI = 0, filterNJ = 0;
  double filterX0 = 0, filterY0 = 0, filterDX = 1, filterDY = 1;
  std::vector<float> filterAlpha1, filterHalpha;             // ntheta x ni*nj; Halpha may be empty
  std::vector<std::vector<float>> globalWavelet;             // ntheta x nzp
  std::vector<float> globalWaveletNorm;                      // ntheta
  // lateral correlation gradients of InitializeCorrelations (samples per index); with the
  // separable factors and a nonzero gradient the prior grids are generated on the device
  float corrGradI = 0, corrGradJ = 0;
};

class AVOInversion {
 public:
  // seisData: ntheta DATA grids in the real state.  The prior in `sp` is either the six
  // covariance grids and errCorr (any correlation gradients), or, with corrXY (nxp*nyp)
  // and circCorrT (nzp) given, the separable factors of InitializeCorrelations.
  AVOInversion(Context* ctx, const AVOInversionSettings& settings, std::vector<FFTGrid*>& seisData,
               SeismicParametersHolder& sp, const std::vector<float>* corrXY = nullptr,
               const std::vector<float>* circCorrT = nullptr);
  ~AVOInversion();

  // Posterior mean into sp.meanVp/Vs/Rho, posterior covariance into the six covariance
  // grids, residual spectra into seisData (Fourier state), postVar0.  The realisations of
  // simulate() are produced in the same pass.  Returns 0.
  int computePostMeanResidAndFFTCov();
  // nSimulations realisations into sp.simulations.  With noise (3 complex grids per
  // realisation, FFTGrid::fillInComplexNoise order) the given noise is used, as the
  // reference's RandomGen would; otherwise the device generator with settings.seed.
  // Call before computePostMeanResidAndFFTCov to give noise.  Returns 0.
  int simulate(const std::vector<FFTGrid*>* noise = nullptr);

  FFTGrid* getPostVp() { return sp_.meanVp; }
  FFTGrid* getPostVs() { return sp_.meanVs; }
  FFTGrid* getPostRho() { return sp_.meanRho; }
  crava_counters counters() const { return counters_; }

 private:
  void run();
  Context* ctx_;
  AVOInversionSettings set_;
  std::vector<FFTGrid*>& seis_;
  SeismicParametersHolder& sp_;
  std::vector<float> corrXY_, circCorrT_;
  bool separable_ = false;
  const std::vector<FFTGrid*>* noise_ = nullptr;
  bool done_ = false;
  crava_counters counters_{};
};

}  // namespace crava_b200
