// Kernel parameter blocks and launch helpers shared by the host API and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "fft_core.cuh"

namespace crava {

// Schedule table: tile shapes and kernel choices by name and size (n), from the schedule
// file the library loads at first use (schedules.txt beside the library, written by
// crava_b200/autotune.py; CRAVA_SCHEDULES names another file) or set through
// crava_tuning_set.  An entry for n, else one for n = -1 (any size), else `fallback`.
int tuned(const char* key, int n, int fallback);

constexpr int kMaxGrids = 64;   // grids per batched transform launch
constexpr int kMaxTheta = 8;    // angle stacks per block
constexpr int kMaxSim = 16;     // realisations per job launch

// Grids of one batched transform launch.  p[] are the grids transformed in place;
// for the forward x pass src[] are the real inputs it reads (src[q] == p[q] is in place).
struct GridSet {
  float* p[kMaxGrids];
  const float* src[kMaxGrids];
  float scale[kMaxGrids];
  int n;
};

// Per-kz operator tables of one block (device pointers), see the host-side builder.
struct KzTables {
  const float2* kw;     // nzp x nth : conj(W_l(k)) kD(k)
  const float2* e1;     // nzp x nth : conj(W_l(k)) / |w_l|
  const float2* e2;     // nzp x nth : conj(E3_l(k)) / |e3_l|
  const uint8_t* inv;   // nzp       : invert_frequency
  const double2* kwd;   // the same three tables in double, read by the FP64
  const double2* e1d;   //   re-factorisation of flagged bins
  const double2* e2d;
  const float* ed;      // nzp x nth : wnc errThetaCov_ll |e3_l(k)|^2 (e3 = 1 for constant
  const double* edd;    //   thickness); edd in double, null: the per-angle constants edd
};

struct ZParams {
  int nxp, nyp, nzp, cnxp;
  int W, logW, nIT;            // tile width in x-bins (power of two), log2 W, tiles per x-row
  int GT, SB;                  // slots per z-transform call, realisations per batch (3 SB <= GT)
  int zsplit;                  // four-step z transform: 0 none, 1 16x16, 2 20x16, 3 16x8
  int nth, nsim;
  int separable;               // 1: prior from cxy/ct factors, 0: from spectral grids
  int base_prior;              // grids: the six prior spectra are pv x one base spectrum, only
                               // cov[0] (= pv[0] x base) transformed
  int host_noise;              // 1: noise from `noise` grids
  int keep_resid;              // 1: write residual spectra into data grids
  int cov_spectral;            // 1: posterior covariance left as per-bin spectra
  int nxp_even;
  float2* data[kMaxTheta];
  float2* mean[3];
  float2* cov[6];              // out; in GRIDS mode also the prior spectra (in)
  const float2* errspec;       // GRIDS mode: error correlation spectrum
  float2* sim[3 * kMaxSim];
  const float2* noise[3 * kMaxSim];
  const float2* cxy;           // SEPARABLE: nyp x cnxp spectrum of corrXY
  const float2* ct;            // SEPARABLE: nzp spectrum of circCorrT
  const float2* septab;        // SEPARABLE: per-kz lower triangle of M2 (or null)
  float pv[6];                 // priorVar0: 00 11 22 01 02 12
  float A[kMaxTheta][3];
  float ec[kMaxTheta][kMaxTheta];  // 0.5 (1 - wnc) errThetaCov
  float ed[kMaxTheta];             // wnc errThetaCov_ll |e3_l|^2
  float G0[kMaxTheta][kMaxTheta];  // SEPARABLE: A P0 A^T
  float AP[kMaxTheta][3];          // SEPARABLE: A P0
  KzTables kz;
  LinePlan zp;
  const float2* twz;
  uint64_t seed;
  float fp64_threshold;            // > 0: re-factorise flagged bins in FP64
  double Ad[kMaxTheta][3];         // A, ec, ed in double for that path
  double ecd[kMaxTheta][kMaxTheta];
  double edd[kMaxTheta];
  // eigen form of the separable posterior (pencil.cu): per-position rows of the per-kz
  // tables, float4 group g of position p at eig[g * nzp + p]; null for the general kernel
  const float4* eig;
  int n_inv_rows;                  // inverted kz (counted per tile, not per bin)
  int dense;                       // 1: the 80-register instantiation (two CTAs per SM)
  int nb2;                         // 1: two bins of one z position per thread in the per-bin step
  unsigned long long* counters;    // [0] inverted bins [1] chol fallbacks [2] zero sim bins
                                   // [3] bins re-factorised in FP64 [4] pencil tiles whose
                                   // input spectra are not finite
};
constexpr int kNumCounters = 5;

// Local-noise shrinkage (localnoise.cu): per-trace maps of the posterior and realisations
// from the local noise scales; the matrices are job constants computed on the host.
struct LocalNoiseParams {
  int nx, ny, nz, nyp, rnxp, nth, nsim;
  const float* scale;                 // nth x ny x nx local noise scales, index i + nx (j + ny l)
  float* maps;                        // ny x nx x 18 floats: every trace's S and Msim (scratch)
  double inv_min[kMaxTheta];          // 1 / (smallest scale of angle l)
  double gsg[kMaxTheta][kMaxTheta];   // G Sm G^T
  double sth[kMaxTheta][kMaxTheta];   // SigmaTheta (errThetaCov)
  double b[kMaxTheta][3];             // G Sm
  double sm[3][3];                    // priorVar0
  double sdel[3][3];                  // (Sm - Smd)^-1/2, eigenvalues <= 1e-7 dropped
  double smdi[3][3];                  // Smd^-1/2, eigenvalues <= 0 dropped
  const float* prior_mean[3];         // real grids (FFTGrid layout)
  float* post[3];                     // posterior mean, corrected in place
  float* sim[3 * kMaxSim];            // realisations, corrected in place
};
cudaError_t launch_local_noise(const LocalNoiseParams& P, cudaStream_t st, int* nlaunch);

constexpr int kMaxFacies = 16;
constexpr int kMaxFaciesAngles = 4;   // local-noise angles of the facies densities (16 corners)
struct FaciesPrior { float p[kMaxFacies]; };
struct FaciesOut { float* p[kMaxFacies + 1]; };
struct FaciesBoxHost {
  int nb[3];
  double vmin[3];
  double dv[3];
  int rs;
  size_t fstride;
};

// Non-constant-thickness data pre-processing (thick.cu).  Per-angle tables of
// computeAdjustmentFactor over kz < cnzp: wamp the wavelet spectrum (cAmp), es3 the
// band-normalised spectrum of the third difference of the wavelet, tau2 |Re| of the
// reflection-coefficient covariance spectrum.
struct ThickParams {
  int nx, ny, nz, nxp, nyp, nzp, rnxp, cnzp;
  int W, logW, nIT;            // W complex lines (2W traces) per CTA, log2 W, tiles per row
  float* grid[kMaxTheta];      // the data grids, processed in place
  const double* rel_thick;     // nxp x nyp, Simbox::getRelThick(i, j)
  const float2* wamp;          // nth x cnzp
  const float2* es3;           // nth x cnzp
  const float* tau2;           // nth x cnzp
  const float2* glob;          // nth x cnzp: {0.05 wGlob2Adj, wGlob2Adj / (tau2 wGlob2 + sigma2Glob)}
  const float* ztaper;         // nzp: 1, or max(1 - dist^2, 0) for kz > nz
  const int* fillx;            // nxp, nyp: getFillNumber of every padded index
  const int* filly;
  const float* distx;          // nxp, nyp, nzp: getDistToBoundary of every padded index
  const float* disty;
  const float* distz;
  float wn2[kMaxTheta];        // (wavelet norm)^2
  float modW[kMaxTheta];       // norm^2 * maxfrequency / highCut
  float err_var[kMaxTheta];    // errThetaCov_ll
  float wnc, low_cut, high_cut;
  float rsq;                   // float(sqrt(float(nzp)))
  float inv_rsq;               // 1/rsq when rsq is a power of two (x/rsq == x*inv_rsq exactly),
                               // else 0: the kernel divides
  double lz;
  LinePlan zp;
  const float2* twz;
  // local wavelets (Wavelet1D with shift and gain grids): per angle and trace i + nx j the
  // shift in samples (shift / dz) and the gain; null: every local wavelet is the global one
  const float* wshift;
  const float* wgain;
  float2 es3_last[kMaxTheta];  // es3 at cnzp - 1 before the RMISSING that the table carries
  // 0: divideDataByScaleWavelet on every padded trace; 1: the wavelet convolution of
  // multiplyDataByScaleWaveletAndWriteToFile on the traces i < nx, j < ny
  int mode;
  float rsq_out;               // mode 1: float(sqrt(double(nzp))), its final divisor
  // 3D wavelets (Wavelet3D, src/wavelet3D.cpp:328-459): per angle and unpadded trace
  // i + nx j the dip adjustment of the trace's local wavelet (Wavelet3DFill), or null for
  // 1D wavelets
  const double* w3_mult;       // multiplyer = alpha1(phi, psi) cos(psi) cos(theta)
  const float4* w3_par;        // {Halpha, local stretch, norm^2 of the adjusted wavelet, gamma}
  const float2* wglob;         // nth x cnzp: the global (average) wavelets' half spectra
  double w3_den;               // double(nzp * dz * 1e-3): the bin spacing's reciprocal, 1/Hz
};
// Per-trace dip adjustment of 3D wavelets (Wavelet3D::getLocalStretch and
// createLocalWavelet1D -> extractLocalWaveletByDip1D -> dipAdjustWavelet, src/wavelet3D.cpp:
// 328-459; the filter surfaces are NRLib::RegularSurface<float> read by WaveletFilter,
// src/waveletfilter.cpp:60-75): for every angle and unpadded trace, from the structure depth
// gradients, phi, psi, the filter values alpha1 and Halpha, multiplyer and the stretch, then
// the norm^2 of the adjusted wavelet (Parseval over its half spectrum) and gamma, the factor
// that band-normalises the adjusted errorSmooth3 given the job's normalised table.
struct Wavelet3DFill {
  const float* gx;             // nx*ny depth gradients (i + nx j), or null: flat
  const float* gy;
  const float* alpha1;         // nth x ni*nj (i + ni j): phi (degrees) along i, psi along j
  const float* halpha;         // nth x ni*nj, or null: no damping
  int ni, nj;
  double x0, y0, dx, dy;       // surface origin and spacing (degrees)
  float theta[kMaxTheta];      // Wavelet::getTheta (radians)
  const float2* wamp;          // nth x cnzp: the 3D wavelets' own half spectra
  const float2* es3;           // nth x cnzp: band-normalised errorSmooth3 (RMISSING last), or null
  float2 es3_last[kMaxTheta];  // es3 at cnzp - 1 before the RMISSING
  int nx, ny, nzp, cnzp, loI, hiI;
  double den;                  // double(nzp * dz * 1e-3)
  double* mult;                // out: nth x nx*ny
  float4* par;                 // out: nth x nx*ny
};
// Prior grids of a GRIDS-mode job generated on the device (prior.cu): the six covariance
// grids fillInParamCorr x priorVar0 and the error-correlation grid fillInErrCorr.
struct PriorFill {
  float* cov[6];               // order Vp, Vs, Rho, VpVs, VpRho, VsRho
  float* err;
  const float* cxy;            // nxp x nyp corrXY
  const float* ct;             // nzp circCorrT
  float pv[6];                 // float(priorVar0(a, b)) in the grid order
  const float* act;            // estimated covariance: 6 x nzp circular auto-covariances in the
                               // grid order (FFTGrid::FillInLateralCorr; pv unused), or null
  float gi, gj;                // correlation gradients (samples per lateral index)
  int nxp, nyp, nzp, rnxp;
};
cudaError_t launch_fill_prior(const PriorFill& P, cudaStream_t st, int* nlaunch);

// One interpolateTrace: trace t (i + nx j) <- mean of nb[] (left, right, up, down; -1 absent)
struct TraceOp {
  int t;
  int nb[4];
  int nt;
};
size_t thick_smem_bytes(int W, int nzp);
int thick_tile_width(int nzp);
cudaError_t launch_thick_divide(const ThickParams& P, int nth, cudaStream_t st, int* nlaunch);
cudaError_t launch_wavelet3d_fill(const Wavelet3DFill& F, int nth, cudaStream_t st, int* nlaunch);
cudaError_t launch_trace_energy(const ThickParams& P, int nth, float* energy, int* nzero, cudaStream_t st,
                                int* nlaunch);
cudaError_t launch_trace_interp(float* g, int rnxp, int nyp, int nzp, int nx, const TraceOp* ops, int nops,
                                cudaStream_t st, int* nlaunch);
cudaError_t launch_extrapolate(const ThickParams& P, int l, const int box[4], cudaStream_t st, int* nlaunch);
float dist_to_boundary(int i, int n, int np);
int fill_number(int i, int n, int np);
void plan_trace_interpolation(const float* energy, int nx, int ny, float threshold, std::vector<TraceOp>& ops,
                              std::vector<int>& level_start, int box[4]);

// four-step launchers (fft4.cu): lengths of its size table only
bool four_step_supported(int n);
cudaError_t launch_line4(const GridSet& gs, int ni, int n, size_t pstride, int no, size_t ostride, const float2* tw,
                         float sign, cudaStream_t st, int* nlaunch);
cudaError_t launch_x4(bool fwd, const GridSet& gs, int nxp, int rows, const float2* tw, const float2* twn,
                      cudaStream_t st, int* nlaunch);
// fused xy pass (fft4.cu) for the (nxp, nyp) pairs of its table: x then y forward (src ->
// p), or y then x inverse (in place in p); twx/twn as launch_x4, twy the length-nyp table
bool xy_fused_supported(int nxp, int nyp);
cudaError_t launch_xy4(bool fwd, const GridSet& gs, int nxp, int nyp, int nzp, const float2* twx, const float2* twn,
                       const float2* twy, cudaStream_t st, int* nlaunch);

// launchers (kernels.cu)
// x transforms: pl/tw are the plan and table of length nxp/2 (even nxp) or nxp (odd);
// twn is the length-nxp table (its first nxp/2 entries are read; unused for odd nxp).
cudaError_t launch_x_r2c(const GridSet& gs, int nxp, int rows, const LinePlan& pl, const float2* tw,
                         const float2* twn, cudaStream_t st, int* nlaunch);
cudaError_t launch_x_c2r(const GridSet& gs, int nxp, int rows, const LinePlan& pl, const float2* tw,
                         const float2* twn, cudaStream_t st, int* nlaunch);
// Complex transform along a strided axis, in place, for all grids of gs:
//   element (i, p, o) at ((size_t)o * ostride + (size_t)p * pstride + i) complex,
//   0 <= i < ni (contiguous), 0 <= p < n (the transform axis), 0 <= o < no.
cudaError_t launch_line_fft(const GridSet& gs, int ni, int n, size_t pstride, int no, size_t ostride,
                            const LinePlan& pl, const float2* tw, float sign, cudaStream_t st, int* nlaunch);
cudaError_t launch_zpass(const ZParams& zp, int threads, cudaStream_t st, int* nlaunch);
// pencil.cu: the separable-prior pencil pass in its eigen form, for the four-step z lengths
// (zp.zsplit 1..3); zp.eig from build_eig_tables
cudaError_t launch_pencil(const ZParams& zp, int threads, cudaStream_t st, int* nlaunch);
size_t pencil_smem_bytes(int W, int nzp, int nth, int SB);
// Float layout of one position's row of the eigen tables: kw (2n floats), Lam (n), then per
// angle l a row of V (2n floats) and Q_l (6) + H_l (9); sections padded to 4 floats so the
// kernel reads them as float4 groups and streams one angle's row at a time.
struct EigLayout {
  int kw, lam, rows, vpad, rs, floats;
  explicit EigLayout(int n) {
    auto pad = [](int x) { return (x + 3) / 4 * 4; };
    kw = 0;
    lam = pad(2 * n);
    rows = lam + pad(n);
    vpad = pad(2 * n);
    rs = vpad + 16;
    floats = rows + n * rs;
  }
};
size_t zpass_smem_bytes(int W, int nzp, int nth);                  // GT = 3, SB = 1
size_t zpass_smem_bytes(int W, int nzp, int nth, int GT, int SB);
// facies.cu: prior[] and out[] are host arrays (copied into the launch parameters)
cudaError_t launch_spec_mul(float2* a, const float2* b, size_t n, cudaStream_t st);
// gridio.cu: dst[e] = src[e] with the byte order of every 4-byte word reversed (dst == src
// allowed)
cudaError_t launch_bswap32(uint32_t* dst, const uint32_t* src, size_t n, cudaStream_t st);
// STORM grid files (gridio.cu): elements e0 .. e0+n-1 of the dense ordering (i fastest) of
// the nx x ny x nz region of a padded real grid (row pitch rnxp, nyp rows per slice) to
// big-endian words and back, and the linear padding fill of FFTGrid's StormContGrid
// constructor.
cudaError_t launch_storm_pack(uint32_t* dst, const float* grid, int nx, int ny, size_t e0, size_t n, int rnxp,
                              int nyp, cudaStream_t st);
cudaError_t launch_storm_unpack(float* grid, const uint32_t* src, int nx, int ny, size_t e0, size_t n, int rnxp,
                                int nyp, cudaStream_t st);
cudaError_t launch_pad_fill(float* grid, int nx, int ny, int nz, int nxp, int nyp, int nzp, int rnxp, cudaStream_t st,
                            int* nlaunch);
// SegY records (segy.cu): per record (inline/crossline order) the trace's grid column, its
// first and end regular samples with data, its top and grid sample spacing; hdr holds the 240-byte
// trace headers (60 words per record, already big-endian).
struct SegyTrace {
  int i, j, first, end;
  double ztop, gdz;
};
struct SegyPack {
  const float* grid;
  int rnxp, nyp, nz;
  int ns;
  float z0, dz;
  const SegyTrace* tr;
  const uint32_t* hdr;
};
cudaError_t launch_segy_pack(const SegyPack& P, size_t r0, int nr, uint32_t* out, cudaStream_t st);
struct FaciesCornersHost {
  int nang;
  const float* t;                                 // device, nang x ny x nx
  FaciesBoxHost box[1 << kMaxFaciesAngles];
  const float* dens[1 << kMaxFaciesAngles];       // device density volume of each corner
  float4* packed[1 << kMaxFaciesAngles];          // device scratch of facies_packed_bytes each
};
size_t facies_packed_bytes(const FaciesBoxHost& b, int nf);
// the probabilities from volumes already packed (launch_facies_prob_corners = pack + eval)
cudaError_t launch_facies_eval(const float* vp, const float* vs, const float* rho, int nx, int ny, int nz, int rnxp_in,
                               int nyp_in, int rnxp_out, const FaciesCornersHost& hc, int nf, const float* prior,
                               float undef_sum, float* const* out, float* seis_lh, cudaStream_t st);
// the facies-interleaved copies of every corner volume (hc.dens -> hc.packed)
cudaError_t launch_facies_pack(const FaciesCornersHost& hc, int nf, cudaStream_t st);
// What the inverse x transform of the posterior mean needs to evaluate the facies
// probabilities in the same pass (fft4_facies.cuh).
struct FaciesFuse {
  float* mean[3];        // the posterior-mean grids: half spectra in, real rows out, in place
  float scale;           // their FFTGrid inverse scale
  int nx, ny, nz, nyp;   // voxels evaluated; the grids' padded y size (rows j + nyp k)
  int rnxp_out;          // floats per row of the probability grids, 2 (nx / 2 + 1)
  int nf;
  float undef_sum;
  FaciesPrior pr;
  FaciesOut out;         // nf + 1 probability grids (the last the undefined class)
  float* seis_lh;        // the seismic likelihood, or null
};
// The fused pass for even nxp whose half length has a four-step split (four_step_supported);
// rows = nyp nzp.  The corner volumes must be packed already.
cudaError_t launch_x4_facies(const FaciesFuse& F, const FaciesCornersHost& hc, int nxp, int rows, const float2* tw,
                             const float2* twn, cudaStream_t st, int* nlaunch);
cudaError_t launch_facies_prob_corners(const float* vp, const float* vs, const float* rho, int nx, int ny, int nz,
                                       int rnxp_in, int nyp_in, int rnxp_out, const FaciesCornersHost& hc, int nf,
                                       const float* prior, float undef_sum, float* const* out, float* seis_lh,
                                       cudaStream_t st);

}  // namespace crava
