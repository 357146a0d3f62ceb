/* crava_gpu.h -- C ABI of the B200 implementation of CRAVA's FFT-domain AVO inversion.
 *
 * The reference has no FFI for this path: its boundary is in-process C++ classes.  Each
 * entry point below replaces one of those calls, so a C++ shim (a DeviceFFTGrid subclass
 * of FFTGrid and an AVOInversion that calls crava_job_run) can route the reference's own
 * call sites here.  Plain C types only; `stream` arguments are cudaStream_t passed as
 * void* (NULL = the legacy default stream).
 *
 * Conventions shared with the reference:
 *   - grids are FFTGrid-padded float arrays of rnxp*nyp*nzp values, x fastest,
 *     rnxp = 2*(nxp/2+1), index i + rnxp*j + rnxp*nyp*k          (src/fftgrid.cpp:34-47)
 *   - spectra occupy the same buffer as cnxp*nyp*nzp interleaved complex values,
 *     cnxp = nxp/2+1, index i + cnxp*j + cnxp*nyp*k               (src/fftgrid.h:256-259)
 *   - forward transforms are unnormalised e^{-2 pi i}; PARAMETER/DATA grids are scaled
 *     by 1/sqrt(N) before the forward and after the inverse transform, COVARIANCE grids
 *     by nothing before and 1/N after                             (src/fftgrid.cpp:1587-1643)
 *
 * Every call returns a crava_status; nothing aborts the process.
 */
#ifndef CRAVA_GPU_H
#define CRAVA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CRAVA_OK = 0,
  CRAVA_EINVAL = 1,     /* bad argument: size, role, index, null pointer          */
  CRAVA_ENOMEM = 2,     /* device allocation failed or the HBM budget is exceeded */
  CRAVA_ECUDA = 3,      /* a CUDA runtime call failed (message in crava_last_error) */
  CRAVA_ETIMEDOUT = 4,  /* a bounded wait gave up                                  */
  CRAVA_ENUMERIC = 5,   /* non-finite input detected: a NaN or Inf in the job description
                           (at crava_job_create) or in the data / prior-mean grids (reported
                           by crava_job_counters after the run)                     */
  CRAVA_ENOTSUP = 6,    /* size or configuration outside what the kernels handle   */
  CRAVA_ESTATE = 7,     /* call out of order (e.g. download before run)            */
  CRAVA_EBUSY = 8,      /* the server's queue is at its limit: submit again later  */
  CRAVA_ECANCELED = 9   /* the request was cancelled before it started             */
} crava_status;

typedef struct crava_ctx crava_ctx;
typedef struct crava_job crava_job;

/* Grid roles of one inversion block.  Inputs are never modified by crava_job_run, so a
 * job can be run again on the same resident inputs; the reference's in-place aliasing
 * (posterior mean over prior mean, residual over data, posterior covariance over the
 * holder's covariance grids) is a matter of where the caller downloads the outputs. */
typedef enum {
  CRAVA_ROLE_DATA = 0,       /* seismic angle stack l (in, real)                          */
  CRAVA_ROLE_MEAN = 1,       /* prior mean a=0..2, order Vp, Vs, Rho (in, real)           */
  CRAVA_ROLE_PRIOR_COV = 2,  /* prior covariance grid q=0..5 (in, real, COVARIANCE) in the
                                order Vp, Vs, Rho, VpVs, VpRho, VsRho; CRAVA_PRIOR_GRIDS only */
  CRAVA_ROLE_ERR_CORR = 3,   /* error correlation grid (in, real, COVARIANCE);
                                CRAVA_PRIOR_GRIDS only                                     */
  CRAVA_ROLE_POST_COV = 4,   /* posterior covariance q=0..5 (out, real, after
                                invFFTCovGrids, src/seismicparametersholder.cpp:432-456)  */
  CRAVA_ROLE_SIM = 5,        /* realisation s, parameter a: index 3*s+a (out, real)       */
  CRAVA_ROLE_NOISE = 6,      /* complex noise of realisation s, parameter a, index 3*s+a
                                (in, complex cnxp*nyp*nzp); CRAVA_FLAG_HOST_NOISE only    */
  CRAVA_ROLE_RESIDUAL = 7,   /* residual spectrum l (out, complex), the reference's
                                seisData_ after the loop (src/avoinversion.cpp:1080-1081);
                                CRAVA_FLAG_KEEP_RESIDUAL only                              */
  CRAVA_ROLE_POST_MEAN = 8   /* posterior mean a (out, real), postVp_/postVs_/postRho_
                                after invFFTInPlace (src/avoinversion.cpp:1112-1114)      */
} crava_role;

enum {
  CRAVA_PRIOR_SEPARABLE = 0, /* prior and error correlation given as the separable
                                factors corr_xy (nxp*nyp) and circ_corr_t (nzp) with zero
                                correlation gradients: the covariance grids of
                                InitializeCorrelations are never materialised             */
  CRAVA_PRIOR_GRIDS = 1      /* six prior covariance grids and the error correlation grid
                                uploaded as real grids (any gradients)                     */
};

enum {
  CRAVA_FLAG_HOST_NOISE = 1,   /* realisation noise uploaded by the caller (parity with a
                                  sequential generator such as the reference RandomGen)   */
  CRAVA_FLAG_KEEP_RESIDUAL = 2, /* keep the residual spectra for CRAVA_ROLE_RESIDUAL         */
  CRAVA_FLAG_SPECTRAL_COV = 4,  /* leave the posterior covariance in the Fourier domain, as
                                   the reference holds it between computePostMeanResidAndFFTCov
                                   and invFFTCovGrids (src/avoinversion.cpp:1071-1077,
                                   src/seismicparametersholder.cpp:432-456): CRAVA_ROLE_POST_COV
                                   then reads complex cnxp*nyp*nzp per-bin S_post           */
  CRAVA_FLAG_NONCONST_THICK = 8 /* Simbox with non-constant thickness: the data are divided
                                   by the per-trace scale wavelet first (crava_job_divide_data)
                                   and the per-bin posterior uses K = kD A with the
                                   wavelet-normalised error multipliers of the reference's
                                   non-constant branch (src/avoinversion.cpp:976-1014);
                                   needs rel_thick and circ_corr_t                          */
};

/* One inversion block: the scalars and small arrays AVOInversion reads from ModelSettings,
 * ModelAVODynamic, Simbox and SeismicParametersHolder (src/avoinversion.cpp:72-111). */
typedef struct {
  int nx, ny, nz;              /* simbox dims                                  */
  int nxp, nyp, nzp;           /* padded dims (2,3,5,7-smooth)                 */
  int ntheta;                  /* angle stacks, 1..8                           */
  double lz;                   /* Simbox::getlz (ms)                           */
  double min_rel_thick;        /* Simbox::getMinRelThick                       */
  float low_cut, high_cut;     /* ModelSettings::getLowCut/getHighCut (Hz)     */
  float wnc;                   /* white-noise component                        */
  const double* A;             /* ntheta x 3 reflection matrix, row-major      */
  const double* err_theta_cov; /* ntheta x ntheta                              */
  const float* wavelet;        /* ntheta x nzp, resampled wavelets, FFT order  */
  const float* wavelet_norm;   /* ntheta, Wavelet::getNorm                     */
  const double* prior_var0;    /* 3 x 3, SeismicParametersHolder::priorVar0_  */
  int prior_mode;              /* CRAVA_PRIOR_SEPARABLE or CRAVA_PRIOR_GRIDS   */
  const float* corr_xy;        /* nxp*nyp lateral correlation, index i+nxp*j   */
  const float* circ_corr_t;    /* nzp circular temporal correlation            */
  int nsim;                    /* realisations                                 */
  uint64_t seed;               /* device noise seed (ignored with HOST_NOISE)  */
  int flags;                   /* CRAVA_FLAG_*                                 */
  float fp64_threshold;        /* 0: FP32 only.  t > 0: a bin whose FP32 factorisation has
                                  (max/min pivot)^2 of Sd > t, or S_post/S < 1/t on a
                                  diagonal entry, is re-factorised in FP64 with one
                                  iterative-refinement step of the data solve         */
  /* CRAVA_FLAG_NONCONST_THICK only (ignored otherwise): */
  const double* rel_thick;     /* nxp*nyp, Simbox::getRelThick(i, j) at every padded trace
                                  (index i+nxp*j), all > 0                              */
  float energy_threshold;      /* ModelSettings::getEnergyThreshold (interpolateSeismic) */
} crava_job_desc;

typedef struct {
  long long inverted_bins;     /* bins inside (lowCut*minRelThick, highCut)    */
  long long chol_fallbacks;    /* inverted bins whose Cholesky failed: prior kept */
  long long sim_chol_zero;     /* realisation bins left at zero (simulate fallback) */
  long long fp64_bins;         /* bins re-factorised in FP64 (fp64_threshold > 0)   */
  float post_var0[9];          /* SeismicParametersHolder::updatePriorVar after the run */
  long long nonfinite_tiles;   /* pencil tiles whose input spectra held a NaN or Inf: the
                                  data or prior-mean grids were not finite; then
                                  crava_job_counters returns CRAVA_ENUMERIC              */
} crava_counters;

/* Context on one device; hbm_budget = 0 means no limit beyond the device's memory. */
crava_status crava_ctx_create(crava_ctx** ctx, int device, size_t hbm_budget);
crava_status crava_ctx_destroy(crava_ctx* ctx);
const char* crava_last_error(void);
const char* crava_status_string(crava_status s);

/* Resident table cache (no counterpart in the reference, which builds every interval's
 * operators anew, src/avoinversion.cpp:845-934): with max_bytes > 0, jobs of this context
 * keep their per-kz tables (wavelet and prior-model operators, separable factors, eigen
 * tables) and their lateral correlation spectrum in device entries shared by every job with
 * the same model, built on first use and evicted least recently used beyond max_bytes or
 * under the context's HBM budget; 0 turns it off (the tables then sit in each job's pool).
 * crava_serve_start turns it on (256 MiB) when it is off.  Stats: hits and misses of entry
 * lookups, bytes and number of resident entries. */
crava_status crava_ctx_set_table_cache(crava_ctx* ctx, size_t max_bytes);
crava_status crava_ctx_table_cache_stats(crava_ctx* ctx, long long* hits, long long* misses, size_t* bytes,
                                         int* entries);

/* Job = one AVOInversion on one block.  Allocates the device grids for the block.
 * Replaces the AVOInversion constructor's set-up (src/avoinversion.cpp:53-111). */
crava_status crava_job_create(crava_ctx* ctx, const crava_job_desc* desc, crava_job** job);
crava_status crava_job_destroy(crava_job* job);
/* Bytes of device memory crava_job_create would allocate for desc. */
crava_status crava_job_footprint(const crava_job_desc* desc, size_t* bytes);

/* Host <-> device copies of one grid (rnxp*nyp*nzp floats; NOISE/RESIDUAL are
 * cnxp*nyp*nzp complex = the same number of floats).  Asynchronous on `stream`. */
crava_status crava_job_upload(crava_job* job, crava_role role, int index, const float* host, void* stream);
crava_status crava_job_download(crava_job* job, crava_role role, int index, float* host, void* stream);
/* Device pointer of one grid (for callers that keep data resident). */
crava_status crava_job_device_ptr(crava_job* job, crava_role role, int index, float** dptr);

/* The whole hot path of one block on `stream`:
 *   forward transforms of data and prior mean     (src/avoinversion.cpp:229-244)
 *   FFTCovGrids + errCorr transform, GRIDS mode   (:908, :917)
 *   computePostMeanResidAndFFTCov per-bin loop    (:944-1091)
 *   simulate, nsim realisations                   (:1354-1511)
 *   inverse transforms of mean, covariance, realisations (:1112-1114, :1476-1483,
 *   src/seismicparametersholder.cpp:432-456)
 * Counters are available after the stream reaches the end of the call. */
crava_status crava_job_run(crava_job* job, void* stream);
crava_status crava_job_counters(crava_job* job, crava_counters* out);

/* CRAVA_FLAG_NONCONST_THICK jobs: AVOInversion::divideDataByScaleWavelet
 * (src/avoinversion.cpp:484-612, with computeAdjustmentFactor :630-719) followed by
 * FFTGrid::interpolateSeismic (src/fftgrid.cpp:2349-2516) on every DATA grid, in place,
 * as the reference's constructor does before the data transform (:226-227).  Call it
 * after the DATA uploads and before crava_job_run.  The trace-interpolation plan is made
 * on the host from the trace energies, so the call returns after `stream` has finished
 * the work.  Wavelets are 1D: the local wavelet of every trace is the global one stretched
 * by rel_thick, shifted and scaled by the trace's entries of the grids that
 * crava_job_set_wavelet_grids gave (none: no shift, unit gain).  Returns CRAVA_ESTATE for a
 * job without the flag. */
crava_status crava_job_divide_data(crava_job* job, void* stream);

/* Local wavelet grids of angle stack `angle` (Wavelet::getLocalTimeshift /
 * getLocalGainFactor, src/wavelet.cpp:1251-1278, applied by Wavelet1D::shiftAndScale,
 * src/wavelet1D.cpp:580-602, when createLocalWavelet1D builds a trace's wavelet): shift_ms
 * (time shift in ms) and gain, nx*ny floats each (index i + nx*j), host memory; NULL for
 * either means none; WELLMISSING (-999) entries mean no shift / unit gain.  Padded traces use
 * the wavelet of the unpadded trace the reference maps them to (src/avoinversion.cpp:525-543).
 * Used by crava_job_divide_data and crava_job_residual_synthetics from the next call on.  The
 * first call allocates 2*ntheta*nx*ny floats of device memory outside the job's footprint
 * (crava_job_footprint) and is synchronous.  The reference re-transforms each local wavelet
 * before taking its errorSmooth3 spectrum (the difference constructors work on samples); this
 * library turns the global spectra directly, which differs by the rounding of that round trip. */
crava_status crava_job_set_wavelet_grids(crava_job* job, int angle, const float* shift_ms, const float* gain);

/* 3D wavelets (Wavelet3D, src/wavelet3D.cpp): the job's wavelets (crava_job_desc.wavelet) are
 * the 3D wavelets' own pulses, and every trace's local wavelet is its angle's pulse adjusted
 * for the local dip (createLocalWavelet1D -> extractLocalWaveletByDip1D -> dipAdjustWavelet,
 * :347-373, :436-459: multiplyer = alpha1(phi, psi) cos(psi) cos(theta) and the damping
 * exp(-pi f Halpha(phi, psi)) of Wavelet1D::adjustForAmplitudeEffect,
 * src/wavelet1D.cpp:605-636), then shifted and scaled by the wavelet grids; its stretch is
 * rel_thick * cos(psi) cos(theta) (getLocalStretch, :328-344), and the adjustment factor's
 * global wavelet is the average wavelet (getGlobalWavelet), src/avoinversion.cpp:508-566.
 * phi and psi come from the structure depth gradients of the trace (findPhi / findPsi,
 * :819-851); alpha1 and Halpha are the wavelet filter surfaces (WaveletFilter,
 * src/waveletfilter.cpp:27-75), read by bilinear interpolation as
 * NRLib::RegularSurface<float>::GetZ at (phi, psi) in degrees. */
typedef struct crava_wavelet3d_desc {
  const float* grad_x;         /* nx*ny structure depth gradients (i + nx*j), or NULL: flat */
  const float* grad_y;
  const float* theta;          /* ntheta angles (radians, Wavelet::getTheta)   */
  int filter_ni, filter_nj;    /* filter surface nodes: phi along i, psi along j */
  double filter_x0, filter_y0; /* surface origin (degrees)                     */
  double filter_dx, filter_dy; /* node spacing (degrees), > 0                  */
  const float* alpha1;         /* ntheta x ni*nj (i + ni*j); -999 marks missing */
  const float* halpha;         /* ntheta x ni*nj, or NULL: no Halpha surface   */
  const float* global_wavelet; /* ntheta x nzp samples of the average wavelets, FFT order */
  const float* global_wavelet_norm; /* ntheta, their Wavelet::getNorm          */
} crava_wavelet3d_desc;

/* Sets the job's wavelets to 3D wavelets (all angles) for crava_job_divide_data and
 * crava_job_residual_synthetics from the next call on.  The dip adjustment of every angle and
 * trace is evaluated on the device once, here: phi, psi, the filter values, the norm of the
 * adjusted wavelet and the band normalisation of its errorSmooth3.  The first call allocates
 * 12*ntheta*nx*ny bytes (plus the global wavelets' spectra) of device memory outside the job's
 * footprint; the call is synchronous.  As with the wavelet grids, the reference re-transforms
 * each local wavelet to samples between the adjustment steps; this library works on the
 * spectra, which differs by the rounding of those round trips. */
crava_status crava_job_set_wavelet_3d(crava_job* job, const crava_wavelet3d_desc* w);

/* AVOInversion::multiplyDataByScaleWaveletAndWriteToFile (src/avoinversion.cpp:721-790), the
 * wavelet-convolved residuals the reference writes after the inversion (:1123): for a job
 * with CRAVA_FLAG_KEEP_RESIDUAL after crava_job_run, every residual spectrum is transformed
 * back (FFTGrid::invFFTInPlace) and every trace i < nx, j < ny is convolved along z with its
 * local wavelet (1/sqrt(nzp), r2c, times the conjugate of the wavelet spectrum stretched by
 * rel_thick (1 for constant thickness), shifted and scaled by the wavelet grids, c2r,
 * 1/sqrt(nzp)); the padding traces keep the transformed-back residual.  CRAVA_ROLE_RESIDUAL
 * then reads real rnxp*nyp*nzp grids.  Once per run (CRAVA_ESTATE otherwise).  A job without
 * CRAVA_FLAG_NONCONST_THICK allocates its wavelet spectra (ntheta*(nzp/2+1) complex) on the
 * first call, outside its footprint. */
crava_status crava_job_residual_synthetics(crava_job* job, void* stream);

/* Local noise (ModelAVODynamic::GetUseLocalNoise): AVOInversion::correctVpVsRho with
 * newPosteriorCovPointwise (src/avoinversion.cpp:2028-2302) and the local-noise mixing of
 * the realisations in simulate (:1485-1504), applied after crava_job_run to the posterior
 * mean and realisation grids in place.  scales: ntheta host maps of the local noise scale,
 * nx*ny floats each (index i + nx*j), all finite and > 0.  Per trace the 3x3 maps come from
 * G (AVOInversion::computeG, :1943-2026, computed on the host: its eigenvectors are taken
 * with the largest-magnitude component positive), the posterior lag-0 covariance
 * (updatePriorVar) and the trace's scales; the prior mean is the job's prior-mean input.
 * Returns after `stream` has finished the work. */
crava_status crava_job_local_noise(crava_job* job, const float* scales, void* stream);

/* CRAVA_PRIOR_GRIDS jobs whose description also carries corr_xy and circ_corr_t: the six
 * prior covariance grids and the error-correlation grid are generated on the device, in
 * place of their uploads, as SeismicParametersHolder::InitializeCorrelations
 * (src/seismicparametersholder.cpp:333-348: FFTGrid::fillInParamCorr x priorVar0,
 * src/fftgrid.cpp:878-928) and FFTGrid::fillInErrCorr (src/fftgrid.cpp:777-828) fill them,
 * with the lateral correlation gradients corr_grad_i, corr_grad_j (samples per index) and
 * the reference's float arithmetic (the grids are equal bit for bit).  Call before
 * crava_job_run; returns after `stream` has finished the work.  The six grids are then
 * priorVar0 multiples of one correlation grid, so the next runs transform only the first
 * (FFTCovGrids forms one spectrum, not six; getNextParameterCovariance scales its |Re/pv|
 * by each pair's priorVar0, equal to the six-spectrum form up to the float rounding of the
 * six grids' products), until a prior grid is uploaded or its device pointer taken. */
crava_status crava_job_fill_prior(crava_job* job, float corr_grad_i, float corr_grad_j, void* stream);

/* CRAVA_PRIOR_GRIDS jobs with estimated covariance (InitializeCorrelations with
 * cov_estimated, src/seismicparametersholder.cpp:247-325): the six prior covariance grids
 * FFTGrid::FillInLateralCorr(corrXY, circAutoCov_ab, gradI, gradJ) (src/fftgrid.cpp:830-876)
 * and the error-correlation grid, generated on the device.  circ_auto_cov: 6 x nzp floats,
 * the circular auto-covariances of the pairs Vp, Vs, Rho, VpVs, VpRho, VsRho (from
 * crava_circ_auto_cov).  Returns after `stream` has finished the work. */
crava_status crava_job_fill_prior_auto_cov(crava_job* job, const float* circ_auto_cov, float corr_grad_i,
                                           float corr_grad_j, void* stream);

/* CRAVA binary grid files (FFTGrid::writeCravaFile / readCravaFile, src/fftgrid.cpp:2183-2270):
 * the tag line "crava_fftgrid_binary", the simbox geometry below and rnxp, nyp, nzp as
 * big-endian doubles and 4-byte integers, then the rnxp*nyp*nzp floats of the FFTGrid layout,
 * big-endian.  The grid is staged straight between the file and the device grid d_grid in
 * 32 MiB chunks through two pinned buffers of the context, the byte order reversed on the
 * device; both calls return when the file and the device grid are complete.  The reader
 * fails with CRAVA_EINVAL when the file's padded dimensions differ from the target's, as the
 * reference does. */
typedef struct {
  double x0, y0, dx, dy;       /* Simbox::getx0, gety0, getdx, getdy            */
  int nx, ny;                  /* Simbox::getnx, getny                          */
  double il0, xl0;             /* Simbox::getIL0, getXL0                        */
  double il_step_x, il_step_y; /* Simbox::getILStepX, getILStepY               */
  double xl_step_x, xl_step_y; /* Simbox::getXLStepX, getXLStepY               */
  double angle;                /* Simbox::getAngle                              */
} crava_simbox_geom;
crava_status crava_grid_write_crava(crava_ctx* ctx, const char* path, const float* d_grid, int rnxp, int nyp, int nzp,
                                    const crava_simbox_geom* geom, void* stream);
crava_status crava_grid_read_crava(crava_ctx* ctx, const char* path, float* d_grid, int rnxp, int nyp, int nzp,
                                   crava_simbox_geom* geom, void* stream);

/* STORM grid files.
 * crava_grid_write_storm: FFTGrid::writeStormFile (src/fftgrid.cpp:1889-1930), binary form:
 * the header of Simbox::getStormHeader (src/simbox.cpp:1012-1034; numbers in fixed notation
 * with six decimals, the angle in degrees), then the nx*ny*nz values (padding = 0) or the
 * nxp*nyp*nzp values (padding = 1) of the padded real device grid, i fastest then j then k, as
 * big-endian floats, then "0\n".  Staged through the context's pinned chunks as the CRAVA
 * format.
 * crava_grid_read_storm: a STORM binary grid of that layout (storm_petro_binary, nx ny nz on
 * the header's last line, which must equal the given ones) into the interior of a padded real
 * device grid, whose padding is then filled as FFTGrid's StormContGrid constructor does
 * (src/fftgrid.cpp:215-302: linear blends of the two edge values, z padding first, then y,
 * then x, zero beyond nxp).  geom receives the header's numbers (top_name and bot_name NULL;
 * flat when the surface fields read 0.0).  Both return after the work is done. */
typedef struct {
  double xmin, lx, ymin, ly;   /* Simbox::GetXMin, GetLX, GetYMin, GetLY        */
  double lz;                   /* Simbox::GetLZ                                 */
  double angle;                /* Simbox::GetAngle (radians)                    */
  int cubetype;                /* FFTGrid cube type written into the header     */
  int flat;                    /* 1: flat header (0.0 and lz in place of the surface names) */
  const char* top_name;        /* flat == 0: the top and base surface names     */
  const char* bot_name;
} crava_storm_geom;
crava_status crava_grid_write_storm(crava_ctx* ctx, const char* path, const float* d_grid, int nx, int ny, int nz,
                                    int nxp, int nyp, int nzp, int padding, const crava_storm_geom* geom,
                                    void* stream);
crava_status crava_grid_read_storm(crava_ctx* ctx, const char* path, float* d_grid, int nx, int ny, int nz, int nxp,
                                   int nyp, int nzp, crava_storm_geom* geom, void* stream);

/* SegY file of a device grid: FFTGrid::writeSegyFile (src/fftgrid.cpp:1960-2050) with NRLib's
 * SegY writer (libs/nrlib/segy/segy.cpp:294-320, 1218-1272, 1397-1430): the 3200-byte EBCDIC
 * textual header (the standard CRAVA banner; or, with text, the empty header with text[t] in
 * line t + 2 from column 6, at most 75 characters, t < 39, as TextualHeader::SetLine(t + 1)), the
 * 400-byte binary header (sample interval 1000 dz, ns, format 1), then one record per trace
 * whose top is not missing, in inline/crossline order: a 240-byte trace header (scalco 1, x, y,
 * ns, dt, inline, crossline, start time z0, offset 0 at the locations of header_format) and ns
 * IBM floats, big-endian.  Samples lie on the regular axis z0 + k dz, dz = round(simbox dz)
 * (1 if that is 0), ns = ceil((zmax - z0) / dz); each trace's grid values (top + (k' + 1/2) of
 * its simbox dz times rel_thick) are interpolated linearly onto it between the trace's first and
 * last regular sample (FFTGrid::getRegularZInterpolatedRealValue, :2275-2306), zero outside.
 * The trace resampling, the IBM conversion and the record packing run on the device; files are
 * staged through two pinned chunks as crava_grid_write_crava. */
typedef struct {
  double x0, y0, dx, dy, angle;   /* simbox: GetXMin, GetYMin, cell size, rotation (radians)   */
  int nx, ny, nz;                 /* simbox cells (the grid's nx_, ny_, nz_)                     */
  double dz;                      /* simbox getdz()                                              */
  const double* top;              /* nx*ny top z per trace (i + nx*j), -99999 = missing; or NULL */
  double top_z;                   /*   constant top when top is NULL                             */
  const double* rel_thick;        /* nx*ny relative thickness (i + nx*j), or NULL for 1          */
  double zmin, zmax;              /* simbox getMinMaxZ                                           */
  double il0, xl0, il_step_x, il_step_y, xl_step_x, xl_step_y;   /* simbox IL/XL geometry      */
  float z0;                       /* time of the first regular sample                            */
  int header_format;              /* 0 SeisWorks, 1 IESX, 2 SIP, 3 Charisma, 4 SIPX, 5 HESS      */
  const char* const* text;        /* ntext textual header lines (line 1 first), or NULL          */
  int ntext;
} crava_segy_desc;
crava_status crava_grid_write_segy(crava_ctx* ctx, const char* path, const float* d_grid, int rnxp, int nyp, int nzp,
                                   const crava_segy_desc* desc, void* stream);

/* Host-side temporal prior functions (no device needed).
 * crava_circ_corr_t: SeismicParametersHolder::computeCircCorrT with makeCircCorrTPosDef
 * (src/seismicparametersholder.cpp:624-660, 805-840): the circular temporal correlation of
 * nzp samples from the lags 0..n-1 of prior_corr_t, its spectrum zeroed at k <= min_int_fq
 * and made non-negative, normalised to 1 at lag 0 (CRAVA_EINVAL where the reference aborts:
 * a lag-0 value below 1e-5).
 * crava_circ_auto_cov: ComputeCircAutoCov, MakeCircAutoCovPosDef and
 * TaperCircAutoCovFunction (:559-757) of estimated auto-covariances auto_cov (nlag 3x3
 * matrices, lag-major, row-major each; lag k of pair (i, j) is the forward lag, (j, i) the
 * backward one), sampling dz ms: out = 6 x nzp floats in the order Vp, Vs, Rho, VpVs, VpRho,
 * VsRho.  Both evaluate their transforms in double; the reference's FFTW float path agrees
 * to float rounding. */
crava_status crava_circ_corr_t(const double* prior_corr_t, int n, int min_int_fq, int nzp, float* out);
crava_status crava_circ_auto_cov(const double* auto_cov, int nlag, int nzp, double dz, float* out);

/* FFTGrid drop-ins on a device grid (src/fftgrid.cpp:1587-1612 / 1615-1643).
 * covariance != 0 selects the COVARIANCE scaling. */
crava_status crava_fft_r2c(crava_ctx* ctx, float* dgrid, int nxp, int nyp, int nzp, int covariance, void* stream);
crava_status crava_fft_c2r(crava_ctx* ctx, float* dgrid, int nxp, int nyp, int nzp, int covariance, void* stream);
/* The same on a host-resident grid (the FFTGrid's own buffer, rnxp*nyp*nzp floats): the
 * grid is staged through a device grid the context keeps, transformed, and copied back
 * before the call returns.  Calls on one context serialise on that staging grid. */
crava_status crava_fft_r2c_host(crava_ctx* ctx, float* hgrid, int nxp, int nyp, int nzp, int covariance);
crava_status crava_fft_c2r_host(crava_ctx* ctx, float* hgrid, int nxp, int nyp, int nzp, int covariance);

/* Schedules (no counterpart in the reference, whose FFTW plans pick their own codelets):
 * tile shapes and kernel choices of the transform and pencil kernels, looked up by key and
 * size n.  The library loads them once per process from the file CRAVA_SCHEDULES names, or
 * else schedules.txt beside the library (written by crava_b200/autotune.py; lines
 * "key n value", n = -1 for every size); built-in defaults apply where the table has no
 * entry.  crava_tuning_set overrides one entry for this process (value < 0 removes it),
 * crava_tuning_get returns the value a launch would use (-1: the built-in default),
 * crava_tuning_load replaces the table from another file, and crava_tuning_path names the
 * file in use ("" when none was found).  Keys: see crava_b200/autotune.py. */
crava_status crava_tuning_set(const char* key, int n, int value);
crava_status crava_tuning_get(const char* key, int n, int* value);
crava_status crava_tuning_load(const char* path);
const char* crava_tuning_path(void);

/* Kernels launched by this library since the context was created (all entry points). */
long long crava_ctx_kernel_launches(crava_ctx* ctx);

/* Per-kernel-class device time (no reference counterpart: the reference's TimeKit records
 * wall/CPU time per phase, libs/lib/timekit.cpp:9-27, src/avoinversion.cpp:1229).
 * With profiling on, every launch is bracketed by CUDA events on its stream.
 * crava_ctx_kernel_times waits for the recorded launches and returns, per class
 *   0 forward x transform, 1 forward line transforms, 2 fused pencil pass,
 *   3 inverse line transforms, 4 inverse x transform, 5/6 fused xy pass forward/inverse,
 *   7 trace division (crava_job_divide_data), 8 trace energies, interpolation, extrapolation,
 *   9 local-noise correction, 10 facies probabilities, 11 prior-grid generation,
 * the summed milliseconds and launch counts (n entries), then clears them if reset. */
crava_status crava_ctx_set_profiling(crava_ctx* ctx, int enable);
crava_status crava_ctx_kernel_times(crava_ctx* ctx, double* ms, long long* launches, int n, int reset);

/* Facies probabilities from the posterior (FaciesProb, src/faciesprob.cpp).  A density
 * volume per facies over (ln Vp, ln Vs, ln rho) with nbins (100, 100, 50 in the reference),
 * lower edges vmin and bin widths dv (the Simbox makeFaciesDens builds, :428-441). */
typedef struct {
  int nfacies;            /* 1..16                                        */
  int nbins[3];
  double vmin[3];
  double dv[3];
  const float* prior;     /* nfacies prior probabilities (host)           */
  float p_undefined;      /* probability mass of the undefined class       */
} crava_facies_desc;
/* Gaussian smoothing of the facies histograms in place (makeFaciesDens, :440-522):
 * d_hist holds nfacies device grids in the FFTGrid layout of the density volume
 * (2*(nbins[0]/2+1) floats per row); sigma_inv is the 3x3 inverse smoothing covariance. */
crava_status crava_facies_smooth(crava_ctx* ctx, const crava_facies_desc* fd, const double* sigma_inv, float* d_hist,
                                 void* stream);
/* Per voxel, calculateFaciesProb / findDensity (:1909-2075, :1307-1423): trilinear density
 * lookups at the posterior parameters d_post[3] (real grids, padded nxp x nyp), prior-
 * weighted and normalised.  Outputs d_prob[nfacies+1] (the last is the undefined class) and
 * optionally the seismic likelihood, each in the FFTGrid(nx,ny,nz) layout (2*(nx/2+1)
 * floats per row, RMISSING in the padding).  density_row: floats per density row. */
crava_status crava_facies_prob(crava_ctx* ctx, const crava_facies_desc* fd, const float* d_density, int density_row,
                               const float* const* d_post, int nx, int ny, int nz, int nxp, int nyp,
                               float* const* d_prob, float* d_seis_lh, void* stream);

/* The same with local noise (calculateFaciesProb with noiseScale, findDensity's corners,
 * src/faciesprob.cpp:1307-1423, 1961-1977): 2^nang density volumes (nang <= 4 angles with a
 * local noise scale), corner c built for the angles' extreme scales (bit a of c: the largest
 * scale of angle a), each with its own box corners[c] (nfacies, prior and p_undefined are
 * read from corners[0]) and device volume d_density[c]; noise_scale: nang host maps of nx*ny
 * floats (index i + nx*j).  A voxel's density is the corner densities weighted by
 * prod_a (t_a or 1 - t_a), t_a = (scale_a - min_a) / (max_a - min_a) of its trace (0 when the
 * map is constant).  nang = 0 is the single-volume case.  Returns after `stream` has
 * finished the work when nang > 0. */
crava_status crava_facies_prob_local_noise(crava_ctx* ctx, const crava_facies_desc* corners, int nang,
                                           const float* const* d_density, int density_row, const float* noise_scale,
                                           const float* const* d_post, int nx, int ny, int nz, int nxp, int nyp,
                                           float* const* d_prob, float* d_seis_lh, void* stream);

/* Facies probabilities computed by crava_job_run itself (AVOInversion's constructor calls
 * FaciesProb on the posterior right after the inversion, src/avoinversion.cpp:299-302 with
 * src/faciesprob.cpp:1909-2075): the arguments of crava_facies_prob_local_noise for this job's
 * lateral size and nz; every later crava_job_run writes d_prob[nfacies+1] (and d_seis_lh if
 * not null, FFTGrid(nx,ny,nz) layout) from its posterior mean: a pass after the inverse x
 * transform of the mean, or, where nxp/2 has a four-step split and the schedule entry
 * facies_fused is 1, inside that transform (the mean is not read back; measured slower on
 * B200, the density gathers then run at the transform kernel's occupancy).  The
 * volumes are packed (and the noise scales tabulated) here into the job's own device memory;
 * d_density may be freed afterwards, d_prob and d_seis_lh must stay valid while set.
 * corners = NULL clears the evaluation.  Results are identical to crava_facies_prob_local_noise
 * on the job's downloaded posterior mean. */
crava_status crava_job_set_facies(crava_job* job, const crava_facies_desc* corners, int nang,
                                  const float* const* d_density, int density_row, const float* noise_scale,
                                  float* const* d_prob, float* d_seis_lh);

/* Batches (no counterpart in the reference, which inverts one interval at a time,
 * main.cpp:217-353): the runs of n created jobs, of any sizes and angle counts, captured
 * once into a CUDA graph with `branches` concurrent branches; every crava_batch_run
 * replays the whole batch on `stream`.  Inputs are uploaded to the jobs beforehand. */
typedef struct crava_batch crava_batch;
crava_status crava_batch_create(crava_ctx* ctx, crava_job* const* jobs, int n, int branches, crava_batch** out);
crava_status crava_batch_run(crava_batch* b, void* stream);
crava_status crava_batch_destroy(crava_batch* b);

/* Serving (no counterpart in the reference): a request loop on a native thread.  Jobs
 * are admitted first come first served while the in-flight count is below max_inflight
 * and their footprint fits the context's HBM budget; each runs on its own stream (inputs
 * host->device, the inversion, outputs device->host) and overlaps with the others; its
 * device memory is released, stream-ordered, when it completes.  The per-kz and lateral
 * tables of requests stay resident in the context's table cache, so requests that share
 * a prior and wavelet model (or a lateral grid and correlation) skip their set-up.  host_in: ntheta data
 * grids then 3 prior mean grids; host_out: 3 posterior mean, 6 covariance, 3*nsim
 * realisation grids (NULL entries are not downloaded).  Host buffers stay owned by the
 * caller and must stay valid until the request is done (pinned buffers keep the copies
 * asynchronous).  Served jobs take the separable prior and device noise. */
typedef struct crava_server crava_server;
enum { CRAVA_REQ_QUEUED = 0, CRAVA_REQ_RUNNING = 1, CRAVA_REQ_DONE = 2, CRAVA_REQ_FAILED = 3 };
typedef struct {
  int state;           /* CRAVA_REQ_*                                     */
  crava_status status; /* failure reason                                  */
  double queue_ms;     /* submit -> admission                             */
  double latency_ms;   /* submit -> completion seen by the loop (-1 if not done) */
} crava_request_info;
crava_status crava_serve_start(crava_ctx* ctx, int max_inflight, crava_server** out);
crava_status crava_serve_submit(crava_server* sv, const crava_job_desc* desc, const float* const* host_in,
                                float* const* host_out, uint64_t* ticket);
/* Poll and wait report a request's state; once they have reported its final state (done or
 * failed) the request's record is released and its ticket is no longer known.  A request
 * whose data or prior-mean grids hold a NaN or Inf fails with CRAVA_ENUMERIC; one that
 * cannot fit the device memory even with nothing else in flight fails with CRAVA_ENOMEM
 * (a job larger than the context budget is refused at submit). */
crava_status crava_serve_poll(crava_server* sv, uint64_t ticket, crava_request_info* info);
/* Waits at most timeout_ms; CRAVA_ETIMEDOUT when the request is still queued or running. */
crava_status crava_serve_wait(crava_server* sv, uint64_t ticket, double timeout_ms, crava_request_info* info);
/* Finishes the running requests, fails the queued ones, joins the loop thread. */
crava_status crava_serve_stop(crava_server* sv);
/* At most max_queued requests wait for admission (0 = no limit, the default); a submit beyond
 * it returns CRAVA_EBUSY and queues nothing. */
crava_status crava_serve_set_queue_limit(crava_server* sv, int max_queued);
/* Removes a request that is still queued: it fails with CRAVA_ECANCELED (poll and wait report
 * that once).  A request already admitted runs to completion: CRAVA_ESTATE. */
crava_status crava_serve_cancel(crava_server* sv, uint64_t ticket);

/* Fault injection for callers' recovery paths (no counterpart in the reference): the next n
 * device allocations of jobs created in ctx (crava_job_create, the served jobs) fail as if
 * the device were out of memory (CRAVA_ENOMEM); nothing reaches the GPU. */
crava_status crava_ctx_fail_next_allocs(crava_ctx* ctx, int n);

/* One block, end to end, with no device allocation (no counterpart in the reference).
 *
 * For callers that cannot allocate device memory: plugins hosted by an application that
 * owns the device memory pool and admits no other allocator, and loops that cannot afford
 * the implicit device synchronisation of an allocation.  All intermediates live in a fixed
 * array of CRAVA_NOALLOC_SCRATCH_BYTES inside the library, which every GPU that loads the
 * library keeps until the process exits.  The caller passes device grids:
 *   d_in  : ntheta data grids, then the 3 prior mean grids (real, read only);
 *   d_out : 3 posterior mean, 6 posterior covariance, 3*nsim realisations (real).
 * Separable prior only, FP32 only (fp64_threshold 0); no host noise, no residual or
 * spectral covariance output; the per-job counters are not reported.  Blocks whose
 * intermediates exceed the array return CRAVA_ENOTSUP.  The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress).  The small per-kz and twiddle
 * tables are built on the host and copied into the array on `stream` from pageable host
 * memory, so the call returns after those copies have left the host buffers.  Every call
 * shares the array: calls whose work overlaps on the GPU (other streams, other threads)
 * race; serialise them on one stream. */
#define CRAVA_NOALLOC_SCRATCH_BYTES (64u << 20)
crava_status crava_invert_noalloc(const crava_job_desc* desc, const float* const* d_in, float* const* d_out,
                                  void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CRAVA_GPU_H */
