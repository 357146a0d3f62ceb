// C ABI of the B200 AVO-inversion path (declared in include/crava_gpu.h).
//
// Host side of one inversion block: device grid allocation, per-kz operator tables
// (AVOInversion's fillkW / fillkWNorm / diff operators, src/avoinversion.cpp:845-975 and
// :1275-1300), transform plans with double-precision twiddles, and the launch sequence
// that replaces the reference's call chain
//   AVOInversion::AVOInversion -> computePostMeanResidAndFFTCov -> simulate ->
//   invFFTCovGrids (src/avoinversion.cpp:229-282).
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/crava_gpu.h"
#include "kernels.cuh"

using namespace crava;
typedef std::complex<double> cd;

namespace {

thread_local std::string g_last_error;

crava_status fail(crava_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

crava_status cuda_fail(cudaError_t e, const char* where) {
  g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
  return CRAVA_ECUDA;
}

#define CUDA_TRY(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

bool smooth(int n) {
  if (n < 1) return false;
  for (int p : {2, 3, 5, 7})
    while (n % p == 0) n /= p;
  return n == 1;
}

// Stage radices for a length-n transform, fewest stages first: radix 16 while four
// factors of two remain, then 8, 4 or 2 (a lone 2 pairs with a 3 into radix 6); pairs of
// threes become radix 9; then 3, 5, 7.
bool make_plan(int n, LinePlan& pl, bool allow16) {
  if (!smooth(n)) return false;
  pl.n = n;
  pl.nst = 0;
  int a = 0, b = 0, c = 0, e = 0, m = n;
  while (m % 2 == 0) { a++; m /= 2; }
  while (m % 3 == 0) { b++; m /= 3; }
  while (m % 5 == 0) { c++; m /= 5; }
  while (m % 7 == 0) { e++; m /= 7; }
  auto push = [&](int r) { if (pl.nst < kMaxStages) pl.radix[pl.nst++] = (int8_t)r; };
  while (allow16 && a >= 4) { push(16); a -= 4; }
  while (a >= 3) { push(8); a -= 3; }
  if (a == 3) { push(8); a = 0; }
  if (a == 2) { push(4); a = 0; }
  if (a == 1) {
    if (b > 0 && b % 2 == 1) { push(6); b--; }
    else push(2);
    a = 0;
  }
  while (b >= 2) { push(9); b -= 2; }
  if (b == 1) push(3);
  while (c-- > 0) push(5);
  while (e-- > 0) push(7);
  return pl.nst < kMaxStages;  // n == 1: no stages (identity)
}

struct Plan {
  LinePlan lp;
  float2* tw = nullptr;  // device, e^{-2 pi i t/n}
};

}  // namespace

// ---------------------------------------------------------------------------------------
// Schedule table (kernels.cuh `tuned`): "key n value" lines of the schedule file, loaded
// once per process from CRAVA_SCHEDULES or else schedules.txt beside this library, and
// entries set through crava_tuning_set.

#include <dlfcn.h>
#include <fstream>
#include <sstream>

namespace {
std::mutex g_tune_mu;
std::map<std::pair<std::string, int>, int> g_tune;
bool g_tune_loaded = false;
std::string g_tune_path;

bool tune_parse(const std::string& path, std::map<std::pair<std::string, int>, int>& out) {
  std::ifstream f(path);
  if (!f) return false;
  std::string line;
  while (std::getline(f, line)) {
    const size_t h = line.find('#');
    if (h != std::string::npos) line.resize(h);
    std::istringstream is(line);
    std::string key;
    long long n, v;
    if (is >> key >> n >> v) out[{key, (int)n}] = (int)v;
  }
  return true;
}

void tune_load_default_locked() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  std::string path;
  if (const char* ev = getenv("CRAVA_SCHEDULES")) path = ev;
  else {
    Dl_info info;
    if (dladdr((void*)&tune_parse, &info) && info.dli_fname) {
      path = info.dli_fname;
      const size_t sl = path.rfind('/');
      path = (sl == std::string::npos ? std::string(".") : path.substr(0, sl)) + "/schedules.txt";
    }
  }
  if (!path.empty() && tune_parse(path, g_tune)) g_tune_path = path;
}
}  // namespace

namespace crava {
int tuned(const char* key, int n, int fallback) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  tune_load_default_locked();
  auto it = g_tune.find({key, n});
  if (it != g_tune.end()) return it->second;
  it = g_tune.find({key, -1});
  return it != g_tune.end() ? it->second : fallback;
}
}  // namespace crava

// Per-kernel-class CUDA-event timing (off unless crava_ctx_set_profiling enables it).
enum { KT_X_R2C = 0, KT_LINE_FWD = 1, KT_ZPASS = 2, KT_LINE_INV = 3, KT_X_C2R = 4, KT_XY_FWD = 5, KT_XY_INV = 6,
       KT_THICK_DIVIDE = 7, KT_THICK_FILL = 8, KT_LOCAL_NOISE = 9, KT_FACIES = 10, KT_FILL_PRIOR = 11,
       KT_COUNT = 12 };
// NVTX range names of the kernel classes (one range per pass, visible in Nsight Systems)
const char* const kKtName[KT_COUNT] = {"x_r2c",        "line_fwd",   "pencil",      "line_inv",
                                       "x_c2r",        "xy_fwd",     "xy_inv",      "thick_divide",
                                       "thick_fill",   "local_noise", "facies",     "fill_prior"};

struct ProfRec {
  int cat;
  cudaEvent_t a, b;
};

namespace {
// Per-block device tables: the per-kz operator tables of the prior and wavelet model (with
// the separable factors and the eigen tables of pencil.cu) and the lateral correlation
// spectrum.  They sit in the job's pool, or in an entry of the context's resident cache
// shared by every job with the same model (crava_ctx_set_table_cache).
struct KzSet {
  float2 *kw = nullptr, *e1 = nullptr, *e2 = nullptr, *septab = nullptr, *ct = nullptr;
  double2 *kwd = nullptr, *e1d = nullptr, *e2d = nullptr;
  uint8_t* inv = nullptr;
  float* edk = nullptr;
  double* eddk = nullptr;
  float4* eig = nullptr;
  bool eig_base = false;     // eigen tables built; a job applies them when its largest
  double lam_limit = 0;      //   lateral factor is below lam_limit
  int n_inv_rows = 0;
  std::string eig_why;
};

struct LatSet {
  float2* cxy = nullptr;     // nyp x cnxp spectrum of corrXY
  float* grid = nullptr;     // its real staging grid
};

struct CacheEntry {
  std::string key;
  char* mem = nullptr;
  size_t bytes = 0;
  int refs = 0;
  uint64_t tick = 0;
  cudaEvent_t ready = nullptr;   // recorded after the tables were built, on the building stream
  KzSet k;
  LatSet l;
};
}  // namespace

struct crava_ctx {
  int device = 0;
  size_t budget = 0;
  size_t allocated = 0;
  long long launches = 0;
  std::mutex mu;
  std::map<int, Plan> plans;
  bool profiling = false;
  std::vector<ProfRec> prof;
  int fail_allocs = 0;   // crava_ctx_fail_next_allocs: job allocations still to fail
  double kt_ms[KT_COUNT] = {};
  long long kt_n[KT_COUNT] = {};
  std::mutex stage_mu;         // device staging grid of the host-grid transforms
  float* stage = nullptr;
  size_t stage_bytes = 0;
  // CRAVA grid file staging: two pinned chunks, a device chunk and their events
  std::mutex io_mu;
  char* io_host[2] = {nullptr, nullptr};
  char* io_dev = nullptr;
  cudaEvent_t io_ev[2] = {nullptr, nullptr};
  // resident table cache: key (model bytes) -> device tables, least recently used evicted
  std::mutex cache_mu;
  std::map<std::string, CacheEntry*> cache;
  size_t cache_max = 0, cache_bytes = 0;
  long long cache_hits = 0, cache_misses = 0;
  uint64_t cache_tick = 0;
};

namespace {
void cache_evict_locked(crava_ctx* ctx, size_t want, cudaStream_t st);

// Brackets one launch with events on its stream when profiling is on.
struct ProfScope {
  crava_ctx* ctx;
  int cat;
  cudaStream_t st;
  cudaEvent_t a = nullptr;
  ProfScope(crava_ctx* c, int k, cudaStream_t s) : ctx(c), cat(k), st(s) {
    nvtxRangePushA(kKtName[k]);
    if (ctx->profiling && cudaEventCreate(&a) == cudaSuccess) cudaEventRecord(a, st);
  }
  ~ProfScope() {
    nvtxRangePop();
    if (!a) return;
    cudaEvent_t b;
    if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); return; }
    cudaEventRecord(b, st);
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->prof.push_back({cat, a, b});
  }
};
}  // namespace

struct crava_job {
  crava_ctx* ctx = nullptr;
  crava_job_desc d{};
  int cnxp = 0, rnxp = 0;
  size_t rsize = 0;          // floats per grid
  size_t N = 0;              // nxp*nyp*nzp
  char* pool = nullptr;      // one allocation for everything below
  size_t pool_bytes = 0;
  float* in_data[kMaxTheta] = {};  // caller inputs (preserved)
  float* in_mean[3] = {};
  float* in_cov[6] = {};
  float* in_err = nullptr;
  float* data[kMaxTheta] = {};     // work: data spectra, then residual spectra
  float* mean[3] = {};             // work: mean spectra, then posterior mean
  float* cov[6] = {};              // work: prior spectra (GRIDS), then posterior covariance
  float* err = nullptr;            // work: error correlation spectrum (GRIDS)
  float* sim[3 * kMaxSim] = {};
  float* noise[3 * kMaxSim] = {};
  float2* kw = nullptr;
  double2* kwd = nullptr;
  float2* septab = nullptr;   // SEPARABLE: per-kz error part of Sd (lower triangle)
  double2* e1d = nullptr;
  double2* e2d = nullptr;
  float2* e1 = nullptr;
  float2* e2 = nullptr;
  uint8_t* inv = nullptr;
  float2* cxy = nullptr;     // SEPARABLE
  float2* ct = nullptr;
  float4* eig = nullptr;     // SEPARABLE: eigen tables of the in-place pencil kernel (pencil.cu)
  bool eig_ok = false;       //   built and applicable: crava_job_run launches k_pencil
  int n_inv_rows = 0;        //   inverted kz
  std::string eig_why;       //   why the general kernel runs instead
  float* cxy_grid = nullptr; // staging for the corr_xy transform
  float* fill_xy = nullptr;  // GRIDS: corrXY and circCorrT for crava_job_fill_prior
  float* fill_t = nullptr;
  CacheEntry* kz_entry = nullptr;   // tables held in the context's cache (referenced)
  CacheEntry* lat_entry = nullptr;
  unsigned long long* counters = nullptr;
  // CRAVA_FLAG_NONCONST_THICK: per-kz diagonal error terms, the data pre-processing
  // parameters (device tables inside) and its work buffers
  float* edk = nullptr;
  double* eddk = nullptr;
  ThickParams tp{};
  float* energy = nullptr;
  int* nzero = nullptr;            // zero-energy traces per angle
  TraceOp* ops = nullptr;
  // host copies of the small inputs
  std::vector<double> A, etc, pv, relt;
  std::vector<float> wav, wnorm, corr_xy, circ;
  bool ran = false;
  // GRIDS: the prior grids are the last crava_job_fill_prior's (priorVar0 x one correlation
  // grid, pv00 > 0), so the run transforms one of them; any upload of a prior grid clears it
  bool base_prior = false;
  bool resid_real = false;        // the residual grids hold the wavelet-convolved residuals
  // local wavelet grids (crava_job_set_wavelet_grids) and the wavelet half spectra of a job
  // without the non-constant tables (crava_job_residual_synthetics): own allocations
  float* wgrid = nullptr;         // ntheta x nx*ny shifts (samples), then ntheta x nx*ny gains
  float2* wspec = nullptr;        // ntheta x cnzp
  // 3D wavelets (crava_job_set_wavelet_3d), one own allocation: per angle and trace the dip
  // adjustment (w3mult, w3par) and the global wavelets' half spectra (w3glob); the global
  // wavelets' modW
  void* w3mem = nullptr;
  double* w3mult = nullptr;
  float4* w3par = nullptr;
  float2* w3glob = nullptr;
  double w3den = 0.0;
  float w3modW[kMaxTheta] = {};
  bool async = false;             // pool from cudaMallocAsync on alloc_stream
  cudaStream_t alloc_stream = nullptr;
  // facies probabilities evaluated by crava_job_run (crava_job_set_facies): the corner boxes
  // with their packed volumes and trace noise scales in fac_mem (own allocation), the
  // caller's probability grids
  bool fac_on = false;
  FaciesCornersHost fac_hc{};
  int fac_nf = 0;
  float fac_prior[kMaxFacies] = {};
  float fac_undef = 0.f;
  float* fac_prob[kMaxFacies + 1] = {};
  float* fac_lh = nullptr;
  char* fac_mem = nullptr;
};

namespace {

crava_status get_plan(crava_ctx* ctx, int n, Plan** out, bool allow16 = false);

// Plans of the x transform: the transform length (nxp/2 for even nxp, nxp for odd) and
// the length-nxp table used to split the half-length transform.
crava_status get_xplans(crava_ctx* ctx, int nxp, Plan** px, Plan** pn) {
  crava_status s = get_plan(ctx, (nxp % 2 == 0) ? nxp / 2 : nxp, px);
  if (s) return s;
  return get_plan(ctx, nxp, pn);
}

// Plans are cached per (length, radix-16 allowed): the pencil pass has the register room
// for radix-16 butterflies, the row and column passes run capped at 64 registers.
crava_status get_plan(crava_ctx* ctx, int n, Plan** out, bool allow16) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  const int key = 2 * n + (allow16 ? 1 : 0);
  auto it = ctx->plans.find(key);
  if (it != ctx->plans.end()) { *out = &it->second; return CRAVA_OK; }
  Plan p;
  if (!make_plan(n, p.lp, allow16)) return fail(CRAVA_ENOTSUP, "transform length " + std::to_string(n) + " is not 2,3,5,7-smooth");
  std::vector<float2> tw(n);
  for (int t = 0; t < n; t++) {
    double ang = 2.0 * M_PI * (double)t / (double)n;
    tw[t] = make_float2((float)std::cos(ang), (float)(-std::sin(ang)));
  }
  CUDA_TRY(cudaMalloc(&p.tw, sizeof(float2) * n));
  CUDA_TRY(cudaMemcpy(p.tw, tw.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
  auto res = ctx->plans.emplace(key, p);
  *out = &res.first->second;
  return CRAVA_OK;
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

struct Layout {
  size_t grid_bytes, total;
  size_t off_tables;
};

crava_status validate(const crava_job_desc* d) {
  if (!d) return fail(CRAVA_EINVAL, "null job description");
  if (d->nx < 1 || d->ny < 1 || d->nz < 1 || d->nxp < d->nx || d->nyp < d->ny || d->nzp < d->nz)
    return fail(CRAVA_EINVAL, "inconsistent grid dimensions");
  if (d->nxp < 2 || d->nyp < 2 || d->nzp < 2) return fail(CRAVA_ENOTSUP, "padded dimensions must be >= 2");
  if (!smooth(d->nxp) || !smooth(d->nyp) || !smooth(d->nzp))
    return fail(CRAVA_ENOTSUP, "padded dimensions must be 2,3,5,7-smooth");
  if (d->nxp > 4096 || d->nyp > 4096 || d->nzp > 4096) return fail(CRAVA_ENOTSUP, "transform length above 4096");
  if (d->nzp * 4 > 16 * 256) return fail(CRAVA_ENOTSUP, "nzp above 1024 is not supported by the pencil pass");
  if (d->ntheta < 1 || d->ntheta > kMaxTheta) return fail(CRAVA_ENOTSUP, "ntheta must be 1..8");
  if (d->nsim < 0 || d->nsim > kMaxSim) return fail(CRAVA_ENOTSUP, "nsim must be 0..16");
  if (!d->A || !d->err_theta_cov || !d->wavelet || !d->wavelet_norm || !d->prior_var0)
    return fail(CRAVA_EINVAL, "null pointer in job description");
  if (d->prior_mode == CRAVA_PRIOR_SEPARABLE) {
    if (!d->corr_xy || !d->circ_corr_t) return fail(CRAVA_EINVAL, "separable prior needs corr_xy and circ_corr_t");
  } else if (d->prior_mode != CRAVA_PRIOR_GRIDS) {
    return fail(CRAVA_EINVAL, "unknown prior mode");
  }
  if (!(d->lz > 0)) return fail(CRAVA_EINVAL, "lz must be positive");
  if (d->flags & ~(CRAVA_FLAG_HOST_NOISE | CRAVA_FLAG_KEEP_RESIDUAL | CRAVA_FLAG_SPECTRAL_COV |
                   CRAVA_FLAG_NONCONST_THICK))
    return fail(CRAVA_EINVAL, "unknown flag");
  if (d->flags & CRAVA_FLAG_NONCONST_THICK) {
    if (!d->rel_thick || !d->circ_corr_t)
      return fail(CRAVA_EINVAL, "non-constant thickness needs rel_thick and circ_corr_t");
    for (size_t q = 0; q < (size_t)d->nxp * d->nyp; q++)
      if (!(d->rel_thick[q] > 0) || !(d->rel_thick[q] < INFINITY))
        return fail(CRAVA_EINVAL, "rel_thick must be finite and positive");
    if (!(d->energy_threshold >= 0.f) || !(d->energy_threshold < INFINITY))
      return fail(CRAVA_EINVAL, "energy_threshold must be finite and >= 0");
    if (!(d->circ_corr_t[0] != 0.f)) return fail(CRAVA_EINVAL, "circ_corr_t[0] must be nonzero");
    if (thick_tile_width(d->nzp) < 1) return fail(CRAVA_ENOTSUP, "nzp too long for the trace transform");
  }
  if (!(d->fp64_threshold >= 0.f) || !(d->fp64_threshold < INFINITY))
    return fail(CRAVA_EINVAL, "fp64_threshold must be finite and >= 0");
  {
    // the small inputs of the description are read on the host: a NaN or Inf there is
    // rejected before anything reaches the device
    auto finite = [](const auto* p, size_t n) {
      for (size_t q = 0; q < n; q++)
        if (!std::isfinite((double)p[q])) return false;
      return true;
    };
    const size_t nth = (size_t)d->ntheta;
    if (!finite(d->A, 3 * nth) || !finite(d->err_theta_cov, nth * nth) || !finite(d->prior_var0, 9) ||
        !finite(d->wavelet, nth * d->nzp) || !finite(d->wavelet_norm, nth) || !std::isfinite(d->lz) ||
        !std::isfinite(d->min_rel_thick) || !std::isfinite(d->low_cut) || !std::isfinite(d->high_cut) ||
        !std::isfinite(d->wnc))
      return fail(CRAVA_ENUMERIC, "non-finite value in the job description (A, err_theta_cov, prior_var0, "
                                  "wavelets or scalars)");
    if (d->corr_xy && !finite(d->corr_xy, (size_t)d->nxp * d->nyp))
      return fail(CRAVA_ENUMERIC, "non-finite value in corr_xy");
    if (d->circ_corr_t && !finite(d->circ_corr_t, (size_t)d->nzp))
      return fail(CRAVA_ENUMERIC, "non-finite value in circ_corr_t");
  }
  for (int l = 0; l < d->ntheta; l++)
    if (!(d->wavelet_norm[l] > 0)) return fail(CRAVA_EINVAL, "wavelet norm must be positive");
  return CRAVA_OK;
}

// Device bytes of the non-constant-thickness tables and work buffers (0 without the flag):
// per-angle adjustment tables, the taper,
// fill and distance tables, rel_thick, the trace energies and the interpolation plan.
size_t thick_bytes(const crava_job_desc* d) {
  if (!(d->flags & CRAVA_FLAG_NONCONST_THICK)) return 0;
  const size_t nth = d->ntheta, cnzp = d->nzp / 2 + 1, nxy = (size_t)d->nx * d->ny;
  return 3 * align256(sizeof(float2) * nth * cnzp) + align256(sizeof(float) * nth * cnzp) +
         2 * align256(sizeof(float) * d->nzp) + align256(sizeof(int) * d->nxp) + align256(sizeof(int) * d->nyp) +
         align256(sizeof(float) * d->nxp) + align256(sizeof(float) * d->nyp) +
         align256(sizeof(double) * d->nxp * d->nyp) + align256(sizeof(float) * nth * nxy) +
         align256(sizeof(TraceOp) * nth * nxy) + align256(sizeof(int) * kMaxTheta);
}

size_t eig_table_bytes(const crava_job_desc* d);

// Device bytes of one job, in three parts: the grids (caller inputs, work grids, counters,
// non-constant-thickness buffers), the per-kz tables of its prior and wavelet model, and its
// lateral correlation factor.  The last two live in the job's pool, or in the context's
// resident table cache when that is on (crava_ctx_set_table_cache).
size_t grid_part_bytes(const crava_job_desc* d) {
  size_t cnxp = d->nxp / 2 + 1;
  size_t gb = align256(sizeof(float) * 2 * cnxp * d->nyp * d->nzp);
  size_t ngrids = 2 * ((size_t)d->ntheta + 3) + 6 + 3 * (size_t)d->nsim;
  if (d->prior_mode == CRAVA_PRIOR_GRIDS) ngrids += 6 + 2;
  if (d->flags & CRAVA_FLAG_HOST_NOISE) ngrids += 3 * (size_t)d->nsim;
  const size_t fill = d->prior_mode == CRAVA_PRIOR_GRIDS
                          ? align256(sizeof(float) * 2 * cnxp * d->nyp) + align256(sizeof(float) * d->nzp)
                          : 0;
  return ngrids * gb + 256 + thick_bytes(d) + fill;
}

size_t kz_set_bytes(const crava_job_desc* d) {
  const size_t sep_stride = (size_t)d->ntheta * (d->ntheta + 1) / 2;
  return 3 * align256(sizeof(float2) * d->nzp * d->ntheta) + align256(sizeof(float2) * d->nzp * sep_stride) +
         3 * align256(sizeof(double2) * d->nzp * d->ntheta) + align256(d->nzp) + align256(sizeof(float2) * d->nzp) +
         align256(sizeof(float) * d->nzp * d->ntheta) + align256(sizeof(double) * d->nzp * d->ntheta) +
         eig_table_bytes(d);
}

size_t lat_set_bytes(const crava_job_desc* d) {
  if (d->prior_mode != CRAVA_PRIOR_SEPARABLE) return 0;
  const size_t cnxp = d->nxp / 2 + 1;
  return align256(sizeof(float2) * cnxp * d->nyp) + align256(sizeof(float) * 2 * cnxp * d->nyp);
}

size_t footprint(const crava_job_desc* d) { return grid_part_bytes(d) + kz_set_bytes(d) + lat_set_bytes(d); }

// DFT of a real vector in double precision, e^{-2 pi i k t / n}.
std::vector<cd> dft(const std::vector<double>& x) {
  size_t n = x.size();
  std::vector<double> c(n), s(n);
  for (size_t q = 0; q < n; q++) {
    double ang = 2.0 * M_PI * (double)q / (double)n;
    c[q] = std::cos(ang);
    s[q] = std::sin(ang);
  }
  std::vector<cd> X(n);
  for (size_t k = 0; k < n; k++) {
    double re = 0, im = 0;
    size_t q = 0;
    for (size_t t = 0; t < n; t++) {
      re += x[t] * c[q];
      im -= x[t] * s[q];
      q += k;
      if (q >= n) q -= n;
    }
    X[k] = cd(re, im);
  }
  return X;
}

// Per-kz operator tables, constant-thickness branch of computePostMeanResidAndFFTCov.
// With kwd/e1d/e2d given, the same three tables are also written in double.
double j_etc(const crava_job_desc& d, int l) { return d.err_theta_cov[l * d.ntheta + l]; }

// Wavelet::getCAmp(k, scale) (src/wavelet.cpp:337-382) on a float spectrum c[0..cnzp),
// in float as the reference evaluates it.
std::complex<float> camp_scaled_host(const std::vector<std::complex<float>>& c, int nzp, int k, float scale) {
  const int cn = nzp / 2 + 1;
  const bool mirror = k >= cn;
  const float om = float(mirror ? nzp - k : k) / scale;
  if (om >= cn) return {0.f, 0.f};
  const int lo = int(std::floor(om));
  int hi = lo + 1;
  if (hi >= cn) hi -= 1;
  const float dO = om - float(lo);
  float re = c[lo].real() * (1.0f - dO) + c[hi].real() * dO;
  float im = c[lo].imag() * (1.0f - dO) + c[hi].imag() * dO;
  if (mirror) im = -im;
  return {re / scale, im / scale};
}

// fillInverseAbskWRobust (src/avoinversion.cpp:1296-1322): 1/|W(k)| from the larger of the
// spectrum and the spectrum sampled at 0.999 stretch, per kz; a large number where both vanish.
std::vector<double> inverse_abs_kw_robust(const std::vector<cd>& W, int n, float wnorm) {
  const int cn = n / 2 + 1;
  std::vector<std::complex<float>> c(cn);
  for (int k = 0; k < cn; k++) c[k] = {(float)W[k].real(), (float)W[k].imag()};
  std::vector<double> out(n);
  for (int k = 0; k < n; k++) {
    const std::complex<float> v = k < cn ? c[k] : std::conj(c[n - k]);
    const std::complex<float> vf = camp_scaled_host(c, n, k, 0.999f);
    const float m = v.real() * v.real() + v.imag() * v.imag();
    const float mf = vf.real() * vf.real() + vf.imag() * vf.imag();
    const float mx = std::max(m, mf);
    out[k] = mx > 0.0f ? (double)float(1.0 / std::sqrt(mx)) : (double)(wnorm * n * n * 100.0f);
  }
  return out;
}

void build_kz_tables(const crava_job_desc& d, std::vector<float2>& kw, std::vector<float2>& e1,
                     std::vector<float2>& e2, std::vector<uint8_t>& inv, std::vector<double2>* kwd,
                     std::vector<double2>* e1d,std::vector<double2>* e2d, std::vector<float>& edk,
                     std::vector<double>* eddk) {
  int n = d.nzp, nth = d.ntheta;
  kw.assign((size_t)n * nth, make_float2(0, 0));
  e1 = kw;
  e2 = kw;
  inv.assign(n, 0);
  if (kwd) {
    kwd->assign((size_t)n * nth, make_double2(0, 0));
    *e1d = *kwd;
    *e2d = *kwd;
  }
  // diff1Operator: FIRSTORDERFORWARDDIFF, -1 at 0 and +1 at nzp-1 (src/wavelet1D.cpp:407-411)
  std::vector<double> d1(n, 0.0);
  d1[0] = -1.0;
  d1[n - 1] = 1.0;
  std::vector<cd> kD = dft(d1);
  // diff3Operator = central(backward(diff1Operator)) (src/avoinversion.cpp:842-848)
  // diagonal error term wnc errThetaCov_ll |e3_l(k)|^2; e3 = 1 for constant thickness
  edk.assign((size_t)n * nth, 0.f);
  if (eddk) eddk->assign((size_t)n * nth, 0.0);
  for (int k = 0; k < n; k++)
    for (int l = 0; l < nth; l++) {
      edk[(size_t)k * nth + l] = float(d.wnc * j_etc(d, l));
      if (eddk) (*eddk)[(size_t)k * nth + l] = d.wnc * j_etc(d, l);
    }
  std::vector<cd> kD3;
  if (d.flags & CRAVA_FLAG_NONCONST_THICK) {
    std::vector<double> f2(n), f3(n);
    for (int i = 0; i < n; i++) f2[i] = (i == 0) ? d1[0] - d1[n - 1] : d1[i] - d1[i - 1];
    for (int i = 0; i < n; i++) f3[i] = 0.5 * (f2[(i + 1) % n] - f2[(i + n - 1) % n]);
    kD3 = dft(f3);
  }
  for (int l = 0; l < nth; l++) {
    std::vector<float> wf(d.wavelet + (size_t)l * n, d.wavelet + (size_t)(l + 1) * n);
    std::vector<double> w(wf.begin(), wf.end());
    std::vector<cd> W = dft(w);
    // errorSmooth3 = central(backward(forward(w))) in float (src/wavelet1D.cpp:438-500)
    std::vector<float> f1(n), f2(n), f3(n);
    for (int i = 0; i < n; i++) f1[i] = (i == n - 1) ? wf[0] - wf[i] : wf[i + 1] - wf[i];
    for (int i = 0; i < n; i++) f2[i] = (i == 0) ? f1[0] - f1[n - 1] : f1[i] - f1[i - 1];
    for (int i = 0; i < n; i++) {
      if (i == 0) f3[i] = (float)(0.5 * (f2[i + 1] - f2[n - 1]));
      else if (i == n - 1) f3[i] = (float)(0.5 * (f2[0] - f2[i - 1]));
      else f3[i] = (float)(0.5 * (f2[i + 1] - f2[i - 1]));
    }
    double n3 = 0;
    for (int i = 0; i < n; i++) n3 += (double)(f3[i] * f3[i]);
    float norm3 = (float)std::sqrt(n3);
    std::vector<double> e3(f3.begin(), f3.end());
    std::vector<cd> E3 = dft(e3);
    double wn = d.wavelet_norm[l];
    const bool nonconst = (d.flags & CRAVA_FLAG_NONCONST_THICK) != 0;
    std::vector<double> e3r;
    if (nonconst) e3r = inverse_abs_kw_robust(W, n, d.wavelet_norm[l]);
    for (int k = 0; k < n; k++) {
      cd kwv = std::conj(W[k]) * kD[k];
      cd a = std::conj(W[k]) / wn;
      cd b = norm3 > 0 ? std::conj(E3[k]) / (double)norm3 : cd(0, 0);
      if (nonconst) {
        // K = kD A, errMult1 = 1/|w|, errMult2 = kD3/|errorSmooth3|, errMult3 = robust
        // 1/|W| (src/avoinversion.cpp:976-1014, fillInverseAbskWRobust :1296-1322)
        kwv = kD[k];
        a = cd(1.0f / d.wavelet_norm[l], 0.0);
        b = norm3 > 0 ? kD3[k] * (double)(1.0f / norm3) : cd(0, 0);
        const double ev = (double)d.wnc * j_etc(d, l) * e3r[k] * e3r[k];
        edk[(size_t)k * nth + l] = (float)ev;
        if (eddk) (*eddk)[(size_t)k * nth + l] = ev;
      }
      kw[(size_t)k * nth + l] = make_float2((float)kwv.real(), (float)kwv.imag());
      e1[(size_t)k * nth + l] = make_float2((float)a.real(), (float)a.imag());
      e2[(size_t)k * nth + l] = make_float2((float)b.real(), (float)b.imag());
      if (kwd) {
        (*kwd)[(size_t)k * nth + l] = make_double2(kwv.real(), kwv.imag());
        (*e1d)[(size_t)k * nth + l] = make_double2(a.real(), a.imag());
        (*e2d)[(size_t)k * nth + l] = make_double2(b.real(), b.imag());
      }
    }
  }
  // realFrequency and the inversion band (src/avoinversion.cpp:946, :1029)
  for (int k = 0; k < n; k++) {
    int kk = std::min(k, n - k);
    float rf = static_cast<float>((d.nz * 1000.0f) / (d.lz * n) * kk);
    inv[k] = (rf > d.low_cut * d.min_rel_thick && rf < d.high_cut) ? 1 : 0;
  }
}

// Four-step split of a z length that the in-place pencil kernels handle (kernels.cuh
// ZParams.zsplit): 1 16x16, 2 20x16, 3 16x8; 0 for the other lengths.
int zsplit_of(int nzp) { return nzp == 256 ? 1 : nzp == 320 ? 2 : nzp == 128 ? 3 : 0; }
int zsplit_n1(int zs) { return zs == 1 ? 16 : zs == 2 ? 20 : zs == 3 ? 16 : 0; }
int zsplit_n2(int zs) { return zs == 1 ? 16 : zs == 2 ? 16 : zs == 3 ? 8 : 0; }

// Eigen tables of a separable-prior job: bytes on the device (0 for other priors).
size_t eig_table_bytes(const crava_job_desc* d) {
  if (d->prior_mode != CRAVA_PRIOR_SEPARABLE) return 0;
  return align256(sizeof(float) * (size_t)EigLayout(d->ntheta).floats * d->nzp);
}

// Hermitian eigen-decomposition A = U diag(lam) U^H of a small matrix (n <= 8) by cyclic
// Jacobi rotations in double (Jacobi's method with a phase per rotation that makes the
// pivot real).  A is overwritten; the columns of U are the eigenvectors.
void herm_eig(int n, cd (&A)[kMaxTheta][kMaxTheta], double (&lam)[kMaxTheta], cd (&U)[kMaxTheta][kMaxTheta]) {
  for (int i = 0; i < n; i++)
    for (int k = 0; k < n; k++) U[i][k] = i == k ? cd(1, 0) : cd(0, 0);
  for (int sweep = 0; sweep < 64; sweep++) {
    double off = 0, diag = 0;
    for (int i = 0; i < n; i++) {
      diag += std::norm(A[i][i]);
      for (int k = i + 1; k < n; k++) off += std::norm(A[i][k]);
    }
    if (off <= 1e-32 * diag || off == 0.0) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = std::abs(A[p][q]);
        if (apq == 0.0) continue;
        const cd ph = A[p][q] / apq;                   // A_pq = |A_pq| ph
        const double theta = (A[q][q].real() - A[p][p].real()) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        // G = D R: D = diag(.., conj(ph) at q) makes the pivot real, R the real rotation
        const cd gpp = c, gpq = sn, gqp = -sn * std::conj(ph), gqq = c * std::conj(ph);
        for (int k = 0; k < n; k++) {   // A G, U G
          const cd akp = A[k][p], akq = A[k][q];
          A[k][p] = akp * gpp + akq * gqp;
          A[k][q] = akp * gpq + akq * gqq;
          const cd ukp = U[k][p], ukq = U[k][q];
          U[k][p] = ukp * gpp + ukq * gqp;
          U[k][q] = ukp * gpq + ukq * gqq;
        }
        for (int k = 0; k < n; k++) {   // G^H (A G)
          const cd apk = A[p][k], aqk = A[q][k];
          A[p][k] = std::conj(gpp) * apk + std::conj(gqp) * aqk;
          A[q][k] = std::conj(gpq) * apk + std::conj(gqq) * aqk;
        }
        A[p][q] = A[q][p] = cd(0, 0);
        A[p][p] = cd(A[p][p].real(), 0);
        A[q][q] = cd(A[q][q].real(), 0);
      }
  }
  for (int i = 0; i < n; i++) lam[i] = A[i][i].real();
}

// Job constants of the separable posterior in the float values the pencil kernels use:
// AP = A P0 (ntheta x 3) and G0 = A P0 A^T.
void sep_constants(const std::vector<double>& A, const std::vector<double>& pv, int nth,
                   float (&G0)[kMaxTheta][kMaxTheta], float (&AP)[kMaxTheta][3]) {
  for (int l = 0; l < nth; l++) {
    double ap[3] = {0, 0, 0};
    for (int c = 0; c < 3; c++)
      for (int b = 0; b < 3; b++) ap[c] += A[l * 3 + b] * pv[b * 3 + c];
    for (int c = 0; c < 3; c++) AP[l][c] = (float)ap[c];
    for (int m = 0; m < nth; m++) {
      double g = 0;
      for (int c = 0; c < 3; c++) g += ap[c] * A[m * 3 + c];
      G0[l][m] = (float)g;
    }
  }
}

// Tables of the eigen form of the separable posterior (pencil.cu), one row per z position
// in the order the in-place four-step transform leaves the spectrum in (position
// k1 + N2 k2 holds kz = k2 + N1 k1), float4 group g of position p at rows[4 (g nzp + p)].
// Per inverted kz, from the float values the general kernel uses (kw, M2 = the septab
// lower triangle, ed, |ct|, G0 = A P0 A^T, AP = A P0):
//   M = |ct| (kw kw^H) o G0 + M2,  E = diag(ed),  E^-1/2 M E^-1/2 = U diag(Lam) U^H,
//   V = U^H E^-1/2,  Q = |ct| V diag(kw) AP,  H_l = conj(Q_la) Q_lb.
// Rows of kz outside the inversion band are zero (prior kept, residual = data).  Returns
// false with the reason when the form does not apply: some ed <= 0 or an eigenvalue of M
// clearly negative.  lam_limit: the largest lateral factor lam for which no reference
// Cholesky of Sd could reach its 1e-20 pivot test (pivots of Sd >= min ed, Sd_00 <=
// lam M_00 + ed_0); a job applies the form when max lam (<= sum |corrXY|) is below it.
bool build_eig_tables(const crava_job_desc& d, const std::vector<float2>& kw, const std::vector<float2>& sep,
                      const std::vector<float>& edk, const std::vector<uint8_t>& inv, const std::vector<float2>& ct,
                      const float (&G0)[kMaxTheta][kMaxTheta], const float (&AP)[kMaxTheta][3], double& lam_limit,
                      std::vector<float>& rows, int& n_inv_rows, std::string& why) {
  lam_limit = INFINITY;
  const int n = d.ntheta, nzp = d.nzp, zs = zsplit_of(nzp);
  const int N1 = zsplit_n1(zs), N2 = zsplit_n2(zs);
  const EigLayout L(n);
  const int G4 = L.floats / 4;
  rows.assign((size_t)L.floats * nzp, 0.f);
  n_inv_rows = 0;
  const int tri = n * (n + 1) / 2;
  for (int p = 0; p < nzp; p++) {
    // the in-place four-step order of k_pencil at its lengths, natural kz order otherwise
    // (k_zpass)
    const int kz = zs ? p / N2 + N1 * (p % N2) : p;
    if (!inv[kz]) continue;
    n_inv_rows++;
    double row[4 * 96] = {};
    const double cta = std::fabs((double)ct[kz].x);
    cd kwv[kMaxTheta];
    double e[kMaxTheta];
    for (int l = 0; l < n; l++) {
      kwv[l] = cd(kw[(size_t)kz * n + l].x, kw[(size_t)kz * n + l].y);
      e[l] = edk[(size_t)kz * n + l];
      if (!(e[l] > 0)) { why = "white-noise error term not positive"; return false; }
    }
    cd M[kMaxTheta][kMaxTheta], U[kMaxTheta][kMaxTheta];
    for (int l = 0; l < n; l++)
      for (int m = 0; m <= l; m++) {
        const float2 b = sep[(size_t)kz * tri + l * (l + 1) / 2 + m];
        const cd v = cta * (double)G0[l][m] * kwv[l] * std::conj(kwv[m]) + cd(b.x, b.y);
        M[l][m] = v;
        M[m][l] = std::conj(v);
      }
    const double m00 = M[0][0].real();
    double emin = e[0];
    for (int l = 1; l < n; l++) emin = std::min(emin, e[l]);
    if (m00 > 0) lam_limit = std::min(lam_limit, (emin * 1e18 - e[0]) / m00);
    for (int l = 0; l < n; l++)
      for (int m = 0; m < n; m++) M[l][m] /= std::sqrt(e[l] * e[m]);
    double lam[kMaxTheta];
    herm_eig(n, M, lam, U);
    double lmax = 0;
    for (int l = 0; l < n; l++) lmax = std::max(lmax, std::fabs(lam[l]));
    for (int l = 0; l < n; l++) {
      // float rounding of the rank-deficient parts leaves eigenvalues of order -1e-7 lmax:
      // those are zero; a clearly negative one means M is not a covariance
      if (lam[l] < -1e-4 * lmax) { why = "prior part of the data covariance not positive semidefinite"; return false; }
      lam[l] = std::max(lam[l], 0.0);
    }
    cd V[kMaxTheta][kMaxTheta], Q[kMaxTheta][3];
    for (int l = 0; l < n; l++)
      for (int m = 0; m < n; m++) V[l][m] = std::conj(U[m][l]) / std::sqrt(e[m]);
    for (int l = 0; l < n; l++)
      for (int a = 0; a < 3; a++) {
        cd acc = 0;
        for (int m = 0; m < n; m++) acc += V[l][m] * kwv[m] * (double)AP[m][a];
        Q[l][a] = cta * acc;
      }
    for (int l = 0; l < n; l++) {
      row[L.kw + 2 * l] = kwv[l].real();
      row[L.kw + 2 * l + 1] = kwv[l].imag();
      row[L.lam + l] = lam[l];
      double* r = row + L.rows + l * L.rs;   // V row l, then Q_l (6) and H_l (9)
      for (int m = 0; m < n; m++) {
        r[2 * m] = V[l][m].real();
        r[2 * m + 1] = V[l][m].imag();
      }
      for (int a = 0; a < 3; a++) {
        r[L.vpad + 2 * a] = Q[l][a].real();
        r[L.vpad + 2 * a + 1] = Q[l][a].imag();
      }
      const cd h01 = std::conj(Q[l][0]) * Q[l][1], h02 = std::conj(Q[l][0]) * Q[l][2],
               h12 = std::conj(Q[l][1]) * Q[l][2];
      const double h[9] = {std::norm(Q[l][0]), std::norm(Q[l][1]), std::norm(Q[l][2]), h01.real(), h01.imag(),
                           h02.real(), h02.imag(), h12.real(), h12.imag()};
      for (int c = 0; c < 9; c++) r[L.vpad + 6 + c] = h[c];
    }
    for (int g = 0; g < G4; g++)
      for (int c = 0; c < 4; c++) rows[4 * ((size_t)g * nzp + p) + c] = (float)row[4 * g + c];
  }
  return true;
}

// Host tables of the data pre-processing of one job (computeAdjustmentFactor,
// src/avoinversion.cpp:630-719, and the taper/fill helpers of FFTGrid), in the float
// arithmetic of the reference wherever it computes in float.
struct ThickTables {
  std::vector<float2> wamp, es3, glob;
  std::vector<float> tau2, ztaper, distx, disty, distz;
  std::vector<int> fillx, filly;
  float wn2[kMaxTheta], modW[kMaxTheta], err_var[kMaxTheta];
  float2 es3_last[kMaxTheta];   // es3 at cnzp - 1 before the RMISSING
};

// The half spectra of the wavelets (FFT order, Wavelet1D::fft1DInPlace) in float:
// ntheta x cnzp.
std::vector<float2> wavelet_spectra(const crava_job_desc& d) {
  const int n = d.nzp, cn = n / 2 + 1;
  std::vector<float2> w((size_t)d.ntheta * cn);
  for (int l = 0; l < d.ntheta; l++) {
    const float* wf = d.wavelet + (size_t)l * n;
    std::vector<cd> W = dft(std::vector<double>(wf, wf + n));
    for (int k = 0; k < cn; k++) w[(size_t)l * cn + k] = make_float2((float)W[k].real(), (float)W[k].imag());
  }
  return w;
}

void build_thick_tables(const crava_job_desc& d, ThickTables& t) {
  const int n = d.nzp, cn = n / 2 + 1, nth = d.ntheta;
  t.wamp.assign((size_t)nth * cn, make_float2(0, 0));
  t.es3 = t.wamp;
  t.glob = t.wamp;
  t.tau2.assign((size_t)nth * cn, 0.f);
  // Wavelet::findNormWithinFrequencyBand (src/wavelet.cpp:903-925) with the wavelet's dz
  const float dz = (float)(d.lz / d.nz);
  const float dOmega = static_cast<float>(1.0 / (n * dz * 0.001));
  const int loI = std::max(0, (int)std::floor(d.low_cut / dOmega));
  const int hiI = std::min(cn, (int)std::ceil(d.high_cut / dOmega));
  const float maxfreq = static_cast<float>((n / 2) * 1000.0 * d.nz) / static_cast<float>(d.lz * n);
  // getPriorCorrTFiltered (src/seismicparametersholder.cpp:842-868) of the temporal
  // correlation circCorrT / circCorrT[0] (extractParamCorrFromCovVp, :1008-1028)
  std::vector<float> corrT(n);
  for (int i = 0; i < n; i++) {
    const int refk = i < n / 2 + 1 ? i : n - i;
    corrT[i] = refk < d.nz ? d.circ_corr_t[refk] / d.circ_corr_t[0] : 0.f;
  }
  for (int l = 0; l < nth; l++) {
    const float* wf = d.wavelet + (size_t)l * n;
    std::vector<cd> W = dft(std::vector<double>(wf, wf + n));
    // errorSmooth3 = central(backward(forward(w))) in float (src/wavelet1D.cpp:441-500)
    std::vector<float> f1(n), f2(n), f3(n);
    for (int i = 0; i < n; i++) f1[i] = (i == n - 1) ? wf[0] - wf[i] : wf[i + 1] - wf[i];
    for (int i = 0; i < n; i++) f2[i] = (i == 0) ? f1[0] - f1[n - 1] : f1[i] - f1[i - 1];
    for (int i = 0; i < n; i++) f3[i] = (float)(0.5 * (f2[(i + 1) % n] - f2[(i + n - 1) % n]));
    std::vector<cd> E3 = dft(std::vector<double>(f3.begin(), f3.end()));
    std::vector<std::complex<float>> e3f(cn);
    for (int k = 0; k < cn; k++) e3f[k] = {(float)E3[k].real(), (float)E3[k].imag()};
    const double fac = 1.0 / double(n);
    double norm2 = 0.0;
    for (int i = loI; i < hiI; i++)
      norm2 += static_cast<double>(2.0 * fac * (e3f[i].real() * e3f[i].real() + e3f[i].imag() * e3f[i].imag()));
    if (loI == 0) norm2 -= fac * (e3f[0].real() * e3f[0].real() + e3f[0].imag() * e3f[0].imag());
    const float c3 = 1.0f / static_cast<float>(std::sqrt(norm2));
    for (int k = 0; k < cn; k++) {
      t.wamp[(size_t)l * cn + k] = make_float2((float)W[k].real(), (float)W[k].imag());
      float2 v = make_float2(e3f[k].real() * c3, e3f[k].imag() * c3);
      // multiplyRAmpByConstant (src/wavelet.cpp:507-515) writes RMISSING into the floats
      // at index >= nzp of the complex array: the last entry's imaginary part, and its
      // real part too when nzp is even
      if (k == cn - 1) {
        t.es3_last[l] = v;
        v.y = -99999.0f;
        if (n % 2 == 0) v.x = -99999.0f;
      }
      t.es3[(size_t)l * cn + k] = v;
    }
    // reflection-coefficient time covariance (computeElasticImpedanceTimeCovariance +
    // computeReflectionCoefficientTimeCovariance, src/avoinversion.cpp:369-401), then |Re|
    // of its transform
    const float Al[3] = {(float)d.A[l * 3 + 0], (float)d.A[l * 3 + 1], (float)d.A[l * 3 + 2]};
    double eiVar = 0.0;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) eiVar += Al[a] * static_cast<float>(d.prior_var0[a * 3 + b]) * Al[b];
    std::vector<float> rc(n);
    for (int k = 0; k < n; k++) rc[k] = static_cast<float>(eiVar * corrT[k]);
    {
      const float first = rc[0];
      float prev = rc[n - 1];
      for (int i = 0; i < n - 1; i++) {
        const float curr = rc[i], next = rc[i + 1];
        rc[i] = 2 * curr - next - prev;
        prev = curr;
      }
      rc[n - 1] = 2 * rc[n - 1] - first - prev;
    }
    std::vector<cd> RC = dft(std::vector<double>(rc.begin(), rc.end()));
    for (int k = 0; k < cn; k++) t.tau2[(size_t)l * cn + k] = std::fabs((float)RC[k].real());
    const float norm = d.wavelet_norm[l];
    t.wn2[l] = norm * norm;
    float modW = norm;
    modW *= modW;
    modW *= maxfreq / static_cast<float>(d.high_cut);
    t.modW[l] = modW;
    t.err_var[l] = static_cast<float>(j_etc(d, l));
    // the trace-independent part of computeAdjustmentFactor (src/avoinversion.cpp:679-712),
    // float operations in the reference's order
    const float wn2 = t.wn2[l], wnc = d.wnc, ev = t.err_var[l];
    const float c = (1.0f - wnc) * 0.5f;
    const float tm = 0.05f * modW;
    for (int k = 0; k < cn; k++) {
      const float2 wg = t.wamp[(size_t)l * cn + k], es = t.es3[(size_t)l * cn + k];
      const float wGlob2 = wg.x * wg.x + wg.y * wg.y;
      const float sG = wGlob2 / wn2 + (es.x * es.x + es.y * es.y);
      const float s2G = ev * (wnc + c * sG);
      const float wG2A = wGlob2 < tm ? 0.5f * (wGlob2 + tm) : wGlob2;
      const float tau2 = t.tau2[(size_t)l * cn + k];
      t.glob[(size_t)l * cn + k] = make_float2(0.05f * wG2A, wG2A / (tau2 * wGlob2 + s2G));
    }
  }
  t.ztaper.assign(n, 1.f);
  t.distz.assign(n, 0.f);
  for (int k = 0; k < n; k++) {
    const float dk = dist_to_boundary(k, d.nz, n);
    t.distz[k] = dk;
    if (k > d.nz) t.ztaper[k] = std::max<float>(1 - dk * dk, 0);
  }
  t.distx.resize(d.nxp);
  t.fillx.resize(d.nxp);
  for (int i = 0; i < d.nxp; i++) {
    t.distx[i] = dist_to_boundary(i, d.nx, d.nxp);
    t.fillx[i] = fill_number(i, d.nx, d.nxp);
  }
  t.disty.resize(d.nyp);
  t.filly.resize(d.nyp);
  for (int i = 0; i < d.nyp; i++) {
    t.disty[i] = dist_to_boundary(i, d.ny, d.nyp);
    t.filly[i] = fill_number(i, d.ny, d.nyp);
  }
}

float* grid_ptr(crava_job* j, crava_role role, int index, crava_status* st) {
  *st = CRAVA_OK;
  const crava_job_desc& d = j->d;
  switch ((int)role) {
    case CRAVA_ROLE_DATA:
      if (index >= 0 && index < d.ntheta) return j->in_data[index];
      break;
    case CRAVA_ROLE_RESIDUAL:
      if ((d.flags & CRAVA_FLAG_KEEP_RESIDUAL) && index >= 0 && index < d.ntheta) return j->data[index];
      break;
    case CRAVA_ROLE_MEAN:
      if (index >= 0 && index < 3) return j->in_mean[index];
      break;
    case CRAVA_ROLE_POST_MEAN:
      if (index >= 0 && index < 3) return j->mean[index];
      break;
    case CRAVA_ROLE_PRIOR_COV:
      if (d.prior_mode == CRAVA_PRIOR_GRIDS && index >= 0 && index < 6) return j->in_cov[index];
      break;
    case CRAVA_ROLE_POST_COV:
      if (index >= 0 && index < 6) return j->cov[index];
      break;
    case CRAVA_ROLE_ERR_CORR:
      if (d.prior_mode == CRAVA_PRIOR_GRIDS && index == 0) return j->in_err;
      break;
    case CRAVA_ROLE_SIM:
      if (index >= 0 && index < 3 * d.nsim) return j->sim[index];
      break;
    case CRAVA_ROLE_NOISE:
      if ((d.flags & CRAVA_FLAG_HOST_NOISE) && index >= 0 && index < 3 * d.nsim) return j->noise[index];
      break;
  }
  *st = fail(CRAVA_EINVAL, "role/index not valid for this job");
  return nullptr;
}

float fwd_scale(size_t N) { return 1.0f / std::sqrt(static_cast<float>(N)); }
float inv_scale(size_t N, bool cov) {
  if (cov) return float(1.0 / (double)N);
  return float(1.0 / std::sqrt(float(N)));
}

// 3D transforms of a list of grids (x, y[, z]) -- the FFTGrid::fftInPlace work split over
// batched launches.
crava_status fwd_xy(crava_ctx* ctx, const std::vector<const float*>& src, const std::vector<float*>& g,
                    const std::vector<float>& sc, int nxp, int nyp, int nzp, bool with_z, cudaStream_t st) {
  if (g.empty()) return CRAVA_OK;
  Plan *px, *pn, *py, *pz;
  crava_status s;
  if ((s = get_xplans(ctx, nxp, &px, &pn)) || (s = get_plan(ctx, nyp, &py)) || (s = get_plan(ctx, nzp, &pz))) return s;
  int cnxp = nxp / 2 + 1;
  int nl = 0;
  for (size_t b = 0; b < g.size(); b += kMaxGrids) {
    GridSet gs;
    gs.n = (int)std::min(g.size() - b, (size_t)kMaxGrids);
    for (int q = 0; q < gs.n; q++) { gs.p[q] = g[b + q]; gs.src[q] = src[b + q]; gs.scale[q] = sc[b + q]; }
    if (xy_fused_supported(nxp, nyp)) {
      ProfScope ps(ctx, KT_XY_FWD, st);
      CUDA_TRY(launch_xy4(true, gs, nxp, nyp, nzp, px->tw, pn->tw, py->tw, st, &nl));
    } else {
      {
        ProfScope ps(ctx, KT_X_R2C, st);
        CUDA_TRY(launch_x_r2c(gs, nxp, nyp * nzp, px->lp, px->tw, pn->tw, st, &nl));
      }
      {
        ProfScope ps(ctx, KT_LINE_FWD, st);
        CUDA_TRY(launch_line_fft(gs, cnxp, nyp, (size_t)cnxp, nzp, (size_t)cnxp * nyp, py->lp, py->tw, -1.f, st, &nl));
      }
    }
    if (with_z) {
      ProfScope ps(ctx, KT_LINE_FWD, st);
      CUDA_TRY(launch_line_fft(gs, cnxp, nzp, (size_t)cnxp * nyp, nyp, (size_t)cnxp, pz->lp, pz->tw, -1.f, st, &nl));
    }
  }
  ctx->launches += nl;
  return CRAVA_OK;
}

crava_status inv_xy(crava_ctx* ctx, const std::vector<float*>& g, const std::vector<float>& sc, int nxp, int nyp,
                    int nzp, bool with_z, cudaStream_t st) {
  if (g.empty()) return CRAVA_OK;
  Plan *px, *pn, *py, *pz;
  crava_status s;
  if ((s = get_xplans(ctx, nxp, &px, &pn)) || (s = get_plan(ctx, nyp, &py)) || (s = get_plan(ctx, nzp, &pz))) return s;
  int cnxp = nxp / 2 + 1;
  int nl = 0;
  for (size_t b = 0; b < g.size(); b += kMaxGrids) {
    GridSet gs;
    gs.n = (int)std::min(g.size() - b, (size_t)kMaxGrids);
    for (int q = 0; q < gs.n; q++) { gs.p[q] = g[b + q]; gs.src[q] = g[b + q]; gs.scale[q] = sc[b + q]; }
    if (with_z) {
      ProfScope ps(ctx, KT_LINE_INV, st);
      CUDA_TRY(launch_line_fft(gs, cnxp, nzp, (size_t)cnxp * nyp, nyp, (size_t)cnxp, pz->lp, pz->tw, 1.f, st, &nl));
    }
    if (xy_fused_supported(nxp, nyp)) {
      ProfScope ps(ctx, KT_XY_INV, st);
      CUDA_TRY(launch_xy4(false, gs, nxp, nyp, nzp, px->tw, pn->tw, py->tw, st, &nl));
    } else {
      {
        ProfScope ps(ctx, KT_LINE_INV, st);
        CUDA_TRY(launch_line_fft(gs, cnxp, nyp, (size_t)cnxp, nzp, (size_t)cnxp * nyp, py->lp, py->tw, 1.f, st, &nl));
      }
      {
        ProfScope ps(ctx, KT_X_C2R, st);
        CUDA_TRY(launch_x_c2r(gs, nxp, nyp * nzp, px->lp, px->tw, pn->tw, st, &nl));
      }
    }
  }
  ctx->launches += nl;
  return CRAVA_OK;
}

}  // namespace

extern "C" {

const char* crava_last_error(void) { return g_last_error.c_str(); }

const char* crava_status_string(crava_status s) {
  switch (s) {
    case CRAVA_OK: return "ok";
    case CRAVA_EINVAL: return "invalid argument";
    case CRAVA_ENOMEM: return "out of device memory or over budget";
    case CRAVA_ECUDA: return "CUDA error";
    case CRAVA_ETIMEDOUT: return "timed out";
    case CRAVA_ENUMERIC: return "numeric error";
    case CRAVA_ENOTSUP: return "not supported";
    case CRAVA_ESTATE: return "call out of order";
    case CRAVA_EBUSY: return "queue full";
    case CRAVA_ECANCELED: return "cancelled";
  }
  return "unknown status";
}

}  // extern "C"

namespace {

constexpr size_t kIoChunk = (size_t)32 << 20;   // bytes per staging chunk

crava_status io_buffers(crava_ctx* ctx) {
  for (int b = 0; b < 2; b++) {
    if (!ctx->io_host[b]) CUDA_TRY(cudaHostAlloc((void**)&ctx->io_host[b], kIoChunk, cudaHostAllocDefault));
    if (!ctx->io_ev[b]) CUDA_TRY(cudaEventCreateWithFlags(&ctx->io_ev[b], cudaEventDisableTiming));
  }
  if (!ctx->io_dev) CUDA_TRY(cudaMalloc(&ctx->io_dev, 2 * kIoChunk));
  return CRAVA_OK;
}

void put_be(std::string& h, const void* p, size_t n) {
  const unsigned char* c = (const unsigned char*)p;
  for (size_t q = 0; q < n; q++) h.push_back((char)c[n - 1 - q]);   // little-endian host to big-endian
}
template <class T>
T get_be(const unsigned char* c) {
  unsigned char r[sizeof(T)];
  for (size_t q = 0; q < sizeof(T); q++) r[q] = c[sizeof(T) - 1 - q];
  T v;
  std::memcpy(&v, r, sizeof(T));
  return v;
}

const char kCravaTag[] = "crava_fftgrid_binary";

}  // namespace

extern "C" {

crava_status crava_grid_write_crava(crava_ctx* ctx, const char* path, const float* d_grid, int rnxp, int nyp, int nzp,
                                    const crava_simbox_geom* geom, void* stream) {
  if (!ctx || !path || !d_grid || !geom || rnxp < 2 || nyp < 1 || nzp < 1) return fail(CRAVA_EINVAL, "bad arguments");
  std::lock_guard<std::mutex> lk(ctx->io_mu);
  CUDA_TRY(cudaSetDevice(ctx->device));
  crava_status s = io_buffers(ctx);
  if (s) return s;
  cudaStream_t st = (cudaStream_t)stream;
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(CRAVA_EINVAL, std::string("cannot open ") + path + " for writing");
  std::string h = std::string(kCravaTag) + "\n";
  const double d1[4] = {geom->x0, geom->y0, geom->dx, geom->dy};
  for (double v : d1) put_be(h, &v, 8);
  put_be(h, &geom->nx, 4);
  put_be(h, &geom->ny, 4);
  const double d2[7] = {geom->il0, geom->xl0, geom->il_step_x, geom->il_step_y, geom->xl_step_x, geom->xl_step_y,
                        geom->angle};
  for (double v : d2) put_be(h, &v, 8);
  const int dims[3] = {rnxp, nyp, nzp};
  for (int v : dims) put_be(h, &v, 4);
  bool ok = std::fwrite(h.data(), 1, h.size(), f) == h.size();
  const size_t total = sizeof(float) * (size_t)rnxp * nyp * nzp;
  size_t pending_bytes[2] = {0, 0};
  int nl = 0;
  cudaError_t e = cudaSuccess;
  // chunk c: swap into device staging half c%2, download into pinned half c%2; the file write
  // of chunk c-1 runs while chunk c is in flight
  for (size_t off = 0, c = 0; ok && e == cudaSuccess && off < total; off += kIoChunk, c++) {
    const int b = (int)(c % 2);
    const size_t n = std::min(kIoChunk, total - off);
    if (pending_bytes[b]) {   // the chunk this half held is downloaded: write it out first
      e = cudaEventSynchronize(ctx->io_ev[b]);
      if (e == cudaSuccess) ok = std::fwrite(ctx->io_host[b], 1, pending_bytes[b], f) == pending_bytes[b];
      pending_bytes[b] = 0;
    }
    uint32_t* dst = (uint32_t*)(ctx->io_dev + b * kIoChunk);
    if (e == cudaSuccess) e = launch_bswap32(dst, (const uint32_t*)((const char*)d_grid + off), n / 4, st);
    nl++;
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->io_host[b], dst, n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->io_ev[b], st);
    pending_bytes[b] = n;
    // the other half, if it holds the previous chunk, goes to the file now
    const int o = 1 - b;
    if (e == cudaSuccess && ok && pending_bytes[o]) {
      e = cudaEventSynchronize(ctx->io_ev[o]);
      if (e == cudaSuccess) ok = std::fwrite(ctx->io_host[o], 1, pending_bytes[o], f) == pending_bytes[o];
      pending_bytes[o] = 0;
    }
  }
  for (int b = 0; b < 2 && e == cudaSuccess && ok; b++)
    if (pending_bytes[b]) {
      e = cudaEventSynchronize(ctx->io_ev[b]);
      if (e == cudaSuccess) ok = std::fwrite(ctx->io_host[b], 1, pending_bytes[b], f) == pending_bytes[b];
    }
  ok = (std::fclose(f) == 0) && ok;
  if (e != cudaSuccess) return cuda_fail(e, "crava_grid_write_crava");
  if (!ok) return fail(CRAVA_EINVAL, std::string("write error on ") + path);
  std::lock_guard<std::mutex> lk2(ctx->mu);
  ctx->launches += nl;
  return CRAVA_OK;
}

crava_status crava_grid_read_crava(crava_ctx* ctx, const char* path, float* d_grid, int rnxp, int nyp, int nzp,
                                   crava_simbox_geom* geom, void* stream) {
  if (!ctx || !path || !d_grid || rnxp < 2 || nyp < 1 || nzp < 1) return fail(CRAVA_EINVAL, "bad arguments");
  std::lock_guard<std::mutex> lk(ctx->io_mu);
  CUDA_TRY(cudaSetDevice(ctx->device));
  crava_status s = io_buffers(ctx);
  if (s) return s;
  cudaStream_t st = (cudaStream_t)stream;
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(CRAVA_EINVAL, std::string("cannot open ") + path);
  char tag[64] = {0};
  size_t t = 0;
  int ch;
  while (t < sizeof(tag) - 1 && (ch = std::fgetc(f)) != EOF && ch != '\n') tag[t++] = (char)ch;
  unsigned char hb[11 * 8 + 5 * 4];
  if (std::strcmp(tag, kCravaTag) != 0 || std::fread(hb, 1, sizeof(hb), f) != sizeof(hb)) {
    std::fclose(f);
    return fail(CRAVA_EINVAL, std::string(path) + " is not a CRAVA binary grid");
  }
  const unsigned char* q = hb;
  crava_simbox_geom g;
  g.x0 = get_be<double>(q); q += 8;
  g.y0 = get_be<double>(q); q += 8;
  g.dx = get_be<double>(q); q += 8;
  g.dy = get_be<double>(q); q += 8;
  g.nx = get_be<int>(q); q += 4;
  g.ny = get_be<int>(q); q += 4;
  g.il0 = get_be<double>(q); q += 8;
  g.xl0 = get_be<double>(q); q += 8;
  g.il_step_x = get_be<double>(q); q += 8;
  g.il_step_y = get_be<double>(q); q += 8;
  g.xl_step_x = get_be<double>(q); q += 8;
  g.xl_step_y = get_be<double>(q); q += 8;
  g.angle = get_be<double>(q); q += 8;
  const int frnxp = get_be<int>(q), fnyp = get_be<int>(q + 4), fnzp = get_be<int>(q + 8);
  if (frnxp != rnxp || fnyp != nyp || fnzp != nzp) {
    std::fclose(f);
    return fail(CRAVA_EINVAL, std::string("grid on file ") + path + " is " + std::to_string(frnxp) + "x" +
                                  std::to_string(fnyp) + "x" + std::to_string(fnzp) + ", the target " +
                                  std::to_string(rnxp) + "x" + std::to_string(nyp) + "x" + std::to_string(nzp) +
                                  " (readCravaFile: check the padding)");
  }
  if (geom) *geom = g;
  const size_t total = sizeof(float) * (size_t)rnxp * nyp * nzp;
  bool ok = true, used[2] = {false, false};
  int nl = 0;
  cudaError_t e = cudaSuccess;
  // chunk c: read into pinned half c%2 once its previous upload finished, upload, swap in place
  for (size_t off = 0, c = 0; ok && e == cudaSuccess && off < total; off += kIoChunk, c++) {
    const int b = (int)(c % 2);
    const size_t n = std::min(kIoChunk, total - off);
    if (used[b]) e = cudaEventSynchronize(ctx->io_ev[b]);
    if (e != cudaSuccess) break;
    ok = std::fread(ctx->io_host[b], 1, n, f) == n;
    if (!ok) break;
    uint32_t* dst = (uint32_t*)((char*)d_grid + off);
    e = cudaMemcpyAsync(dst, ctx->io_host[b], n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->io_ev[b], st);
    if (e == cudaSuccess) e = launch_bswap32(dst, dst, n / 4, st);
    nl++;
    used[b] = true;
  }
  std::fclose(f);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "crava_grid_read_crava");
  if (!ok) return fail(CRAVA_EINVAL, std::string(path) + " ends before its grid");
  std::lock_guard<std::mutex> lk2(ctx->mu);
  ctx->launches += nl;
  return CRAVA_OK;
}

}  // extern "C"

namespace {

// NRLib::ToString(x, 6): fixed notation with six decimals.
std::string fixed6(double x) {
  char b[64];
  std::snprintf(b, sizeof(b), "%.6f", x);
  return b;
}

std::string storm_header(const crava_storm_geom& g, int nx, int ny, int nz) {
  std::string h = "storm_petro_binary\n";
  h += "0 " + std::to_string(g.cubetype) + " " + fixed6(-99999.0) + "\n";
  h += "FFTGrid\n";
  h += fixed6(g.xmin) + " " + fixed6(g.lx) + " " + fixed6(g.ymin) + " " + fixed6(g.ly) + " ";
  if (g.flat) h += "0.0 " + fixed6(g.lz) + " 0.0 0.0\n";
  else h += std::string(g.top_name ? g.top_name : "") + " " + (g.bot_name ? g.bot_name : "") + " 0.0 0.0\n";
  h += fixed6(g.lz) + " " + fixed6(g.angle * 180.0 / 3.14159265358979323846) + "\n\n";
  h += std::to_string(nx) + " " + std::to_string(ny) + " " + std::to_string(nz) + "\n";
  return h;
}

bool read_line(FILE* f, std::string& line) {
  line.clear();
  int ch;
  while ((ch = std::fgetc(f)) != EOF && ch != '\n') line.push_back((char)ch);
  return ch != EOF || !line.empty();
}

}  // namespace

extern "C" {

crava_status crava_grid_write_storm(crava_ctx* ctx, const char* path, const float* d_grid, int nx, int ny, int nz,
                                    int nxp, int nyp, int nzp, int padding, const crava_storm_geom* geom,
                                    void* stream) {
  if (!ctx || !path || !d_grid || !geom || nx < 1 || ny < 1 || nz < 1 || nxp < nx || nyp < ny || nzp < nz)
    return fail(CRAVA_EINVAL, "bad arguments");
  if (!geom->flat && (!geom->top_name || !geom->bot_name || !*geom->top_name || !*geom->bot_name))
    return fail(CRAVA_EINVAL, "a STORM header that is not flat names its top and base surfaces");
  std::lock_guard<std::mutex> lk(ctx->io_mu);
  CUDA_TRY(cudaSetDevice(ctx->device));
  crava_status s = io_buffers(ctx);
  if (s) return s;
  cudaStream_t st = (cudaStream_t)stream;
  const int rnxp = 2 * (nxp / 2 + 1);
  const int wx = padding ? nxp : nx, wy = padding ? nyp : ny, wz = padding ? nzp : nz;
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(CRAVA_EINVAL, std::string("cannot open ") + path + " for writing");
  const std::string h = storm_header(*geom, wx, wy, wz);
  bool ok = std::fwrite(h.data(), 1, h.size(), f) == h.size();
  const size_t total = (size_t)wx * wy * wz, per = kIoChunk / 4;
  size_t pending[2] = {0, 0};
  int nl = 0;
  cudaError_t e = cudaSuccess;
  auto flush = [&](int b) {
    if (!pending[b]) return;
    e = cudaEventSynchronize(ctx->io_ev[b]);
    if (e == cudaSuccess) ok = ok && std::fwrite(ctx->io_host[b], 4, pending[b], f) == pending[b];
    pending[b] = 0;
  };
  // chunk c: gather and swap into device staging half c%2, download into pinned half c%2;
  // the file write of the previous chunk runs while this one is in flight
  for (size_t e0 = 0, c = 0; ok && e == cudaSuccess && e0 < total; e0 += per, c++) {
    const int b = (int)(c % 2);
    const size_t n = std::min(per, total - e0);
    flush(b);
    if (e != cudaSuccess || !ok) break;
    uint32_t* dst = (uint32_t*)(ctx->io_dev + b * kIoChunk);
    e = launch_storm_pack(dst, d_grid, wx, wy, e0, n, rnxp, nyp, st);
    nl++;
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->io_host[b], dst, 4 * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->io_ev[b], st);
    pending[b] = n;
    if (e == cudaSuccess) flush(1 - b);
  }
  for (int b = 0; b < 2 && e == cudaSuccess; b++) flush(b);
  ok = ok && std::fwrite("0\n", 1, 2, f) == 2;
  ok = (std::fclose(f) == 0) && ok;
  if (e != cudaSuccess) return cuda_fail(e, "crava_grid_write_storm");
  if (!ok) return fail(CRAVA_EINVAL, std::string("write error on ") + path);
  std::lock_guard<std::mutex> lk2(ctx->mu);
  ctx->launches += nl;
  return CRAVA_OK;
}

crava_status crava_grid_read_storm(crava_ctx* ctx, const char* path, float* d_grid, int nx, int ny, int nz, int nxp,
                                   int nyp, int nzp, crava_storm_geom* geom, void* stream) {
  if (!ctx || !path || !d_grid || nx < 1 || ny < 1 || nz < 1 || nxp < nx || nyp < ny || nzp < nz)
    return fail(CRAVA_EINVAL, "bad arguments");
  std::lock_guard<std::mutex> lk(ctx->io_mu);
  CUDA_TRY(cudaSetDevice(ctx->device));
  crava_status s = io_buffers(ctx);
  if (s) return s;
  cudaStream_t st = (cudaStream_t)stream;
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(CRAVA_EINVAL, std::string("cannot open ") + path);
  std::string l[7];
  bool hok = true;
  for (int q = 0; q < 7 && hok; q++) hok = read_line(f, l[q]);
  crava_storm_geom g{};
  int fnx = 0, fny = 0, fnz = 0, zero = -1;
  double missing = 0.0;
  char top[256] = {0}, bot[256] = {0};
  double lzf = 0.0, deg = 0.0;
  hok = hok && l[0] == "storm_petro_binary" &&
        std::sscanf(l[1].c_str(), "%d %d %lf", &zero, &g.cubetype, &missing) == 3 &&
        std::sscanf(l[4].c_str(), "%lf %lf", &lzf, &deg) == 2 && l[5].empty() &&
        std::sscanf(l[6].c_str(), "%d %d %d", &fnx, &fny, &fnz) == 3 &&
        std::sscanf(l[3].c_str(), "%lf %lf %lf %lf %255s %255s", &g.xmin, &g.lx, &g.ymin, &g.ly, top, bot) == 6;
  if (!hok) {
    std::fclose(f);
    return fail(CRAVA_EINVAL, std::string(path) + " is not a STORM binary grid");
  }
  if (fnx != nx || fny != ny || fnz != nz) {
    std::fclose(f);
    return fail(CRAVA_EINVAL, std::string("grid on file ") + path + " is " + std::to_string(fnx) + "x" +
                                  std::to_string(fny) + "x" + std::to_string(fnz) + ", expected " +
                                  std::to_string(nx) + "x" + std::to_string(ny) + "x" + std::to_string(nz));
  }
  g.flat = std::strcmp(top, "0.0") == 0 ? 1 : 0;
  g.lz = lzf;
  g.angle = deg * 3.14159265358979323846 / 180.0;
  g.top_name = g.bot_name = nullptr;
  if (geom) *geom = g;
  const int rnxp = 2 * (nxp / 2 + 1);
  const size_t total = (size_t)nx * ny * nz, per = kIoChunk / 4;
  bool ok = true, used[2] = {false, false};
  int nl = 0;
  cudaError_t e = cudaSuccess;
  // chunk c: read into pinned half c%2 once its previous upload has finished, upload into
  // device staging half c%2, scatter and swap into the grid
  for (size_t e0 = 0, c = 0; ok && e == cudaSuccess && e0 < total; e0 += per, c++) {
    const int b = (int)(c % 2);
    const size_t n = std::min(per, total - e0);
    if (used[b]) e = cudaEventSynchronize(ctx->io_ev[b]);
    if (e != cudaSuccess) break;
    ok = std::fread(ctx->io_host[b], 4, n, f) == n;
    if (!ok) break;
    uint32_t* src = (uint32_t*)(ctx->io_dev + b * kIoChunk);
    e = cudaMemcpyAsync(src, ctx->io_host[b], 4 * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = launch_storm_unpack(d_grid, src, nx, ny, e0, n, rnxp, nyp, st);
    nl++;
    if (e == cudaSuccess) e = cudaEventRecord(ctx->io_ev[b], st);
    used[b] = true;
  }
  std::fclose(f);
  if (e == cudaSuccess && ok) e = launch_pad_fill(d_grid, nx, ny, nz, nxp, nyp, nzp, rnxp, st, &nl);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "crava_grid_read_storm");
  if (!ok) return fail(CRAVA_EINVAL, std::string(path) + " ends before its grid");
  std::lock_guard<std::mutex> lk2(ctx->mu);
  ctx->launches += nl;
  return CRAVA_OK;
}

}  // extern "C"

namespace {

// ASCII to EBCDIC as the SEG-Y rev 1 textual header uses it (code page 037 for the printable
// characters; '[', ']', '^' and the controls 14, 15, 25, which the standard's table leaves out,
// map to 0), the same table as NRLib's transtab (libs/nrlib/segy/commonheaders.cpp:29-48).
const unsigned char kEbcdic[128] = {
    0x00, 0x01, 0x02, 0x03, 0x37, 0x2d, 0x2e, 0x2f, 0x16, 0x05, 0x25, 0x0b, 0x0c, 0x0d, 0x00, 0x00,
    0x10, 0x11, 0x12, 0x13, 0x3c, 0x3d, 0x32, 0x26, 0x18, 0x00, 0x3f, 0x27, 0x1c, 0x1d, 0x1e, 0x1f,
    0x40, 0x5a, 0x7f, 0x7b, 0x5b, 0x6c, 0x50, 0x7d, 0x4d, 0x5d, 0x5c, 0x4e, 0x6b, 0x60, 0x4b, 0x61,
    0xf0, 0xf1, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0x7a, 0x5e, 0x4c, 0x7e, 0x6e, 0x6f,
    0x7c, 0xc1, 0xc2, 0xc3, 0xc4, 0xc5, 0xc6, 0xc7, 0xc8, 0xc9, 0xd1, 0xd2, 0xd3, 0xd4, 0xd5, 0xd6,
    0xd7, 0xd8, 0xd9, 0xe2, 0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9, 0x00, 0xe0, 0x00, 0x00, 0x6d,
    0x79, 0x81, 0x82, 0x83, 0x84, 0x85, 0x86, 0x87, 0x88, 0x89, 0x91, 0x92, 0x93, 0x94, 0x95, 0x96,
    0x97, 0x98, 0x99, 0xa2, 0xa3, 0xa4, 0xa5, 0xa6, 0xa7, 0xa8, 0xa9, 0xc0, 0x4f, 0xd0, 0xa1, 0x07};

// The 3200-byte textual header: 40 card images "C nn" (the last "C40 END EBCDIC"), with CRAVA's
// banner (TextualHeader::standardHeader) or the caller's lines from column 6 of line t + 2
// (TextualHeader::SetLine(t + 1), 75 characters at most).
std::string segy_text_header(const crava_segy_desc* d) {
  std::string a(3200, ' ');
  for (int l = 0; l < 40; l++) {
    char card[8];
    std::snprintf(card, sizeof(card), "C%2d", l + 1);
    a.replace((size_t)l * 80, 3, card);
  }
  a.replace(39 * 80, 14, "C40 END EBCDIC");
  if (!d->text) {
    static const struct { int line; const char* s; } banner[] = {
        {11, "THIS SEGY FILE WAS WRITTEN BY"}, {13, "THE CRAVA PROGRAM"}, {15, "DEVELOPED BY"},
        {17, "RAGNAR HAUGE"}, {19, "ANNE RANDI SYVERSVEEN           AND"}, {21, "ODD KOLBJORNSEN"},
        {23, "AT"}, {25, "THE NORWEGIAN COMPUTING CENTER"}, {27, "2003"}};
    for (const auto& b : banner) a.replace((size_t)b.line * 80 + 12, std::strlen(b.s), b.s);
  } else {
    for (int t = 0; t < d->ntext && t < 39; t++) {
      std::string s = d->text[t] ? d->text[t] : "";
      s.resize(75, ' ');
      a.replace((size_t)(t + 1) * 80 + 5, 75, s);
    }
  }
  for (auto& c : a) c = (char)((unsigned char)c < 128 ? kEbcdic[(unsigned char)c] : 0);
  return a;
}

void put_be16(unsigned char* p, int v) {
  p[0] = (unsigned char)((v >> 8) & 0xff);
  p[1] = (unsigned char)(v & 0xff);
}
void put_be32(unsigned char* p, int v) {
  for (int q = 0; q < 4; q++) p[q] = (unsigned char)(((unsigned)v >> (24 - 8 * q)) & 0xffu);
}

}  // namespace

extern "C" {

crava_status crava_grid_write_segy(crava_ctx* ctx, const char* path, const float* d_grid, int rnxp, int nyp, int nzp,
                                   const crava_segy_desc* d, void* stream) {
  if (!ctx || !path || !d_grid || !d) return fail(CRAVA_EINVAL, "null argument");
  if (d->nx < 1 || d->ny < 1 || d->nz < 2 || rnxp < d->nx || nyp < d->ny || nzp < d->nz || !(d->dx > 0) ||
      !(d->dy > 0) || d->header_format < 0 || d->header_format > 5 || (d->text && d->ntext < 0))
    return fail(CRAVA_EINVAL, "bad SegY description");
  // the regular axis (FFTGrid::writeSegyFile, src/fftgrid.cpp:1980-1986)
  float dz = static_cast<float>(std::floor(d->dz + 0.5));
  if (dz == 0) dz = 1.0f;
  const double nsd = std::ceil((d->zmax - static_cast<double>(d->z0)) / static_cast<double>(dz));
  if (!(nsd >= 1.0) || nsd > 32767.0) return fail(CRAVA_EINVAL, "SegY sample count outside 1..32767");
  const int ns = static_cast<int>(nsd);
  // trace-header locations (1-based) of the format: x, y, inline, crossline
  // (TraceHeaderFormat::Init, libs/nrlib/segy/traceheader.cpp:150-225)
  static const int loc[6][4] = {{73, 77, 9, 21},    {73, 77, 221, 21},  {181, 185, 189, 193},
                                {73, 77, 5, 21},    {73, 77, 181, 185}, {73, 77, 185, 189}};
  const int* L = loc[d->header_format];
  struct Rec {
    int il, xl, ux, uy;
    size_t idx;
    SegyTrace tr;
  };
  std::vector<Rec> rec;
  rec.reserve((size_t)d->nx * d->ny);
  const double cr = std::cos(d->angle), sr = std::sin(d->angle);
  for (int j = 0; j < d->ny; j++)
    for (int i = 0; i < d->nx; i++) {
      const size_t q = (size_t)i + (size_t)d->nx * j;
      const double top = d->top ? d->top[q] : d->top_z;
      if (top == -99999.0 || top == -999.0) continue;   // RMISSING / WELLMISSING: no record
      // Simbox::getXYCoord (src/simbox.cpp:821-827), the coordinates as float, then double
      const double rx = (static_cast<double>(i) + 0.5) * d->dx, ry = (static_cast<double>(j) + 0.5) * d->dy;
      const double x = static_cast<double>(static_cast<float>(rx * cr - ry * sr + d->x0));
      const double y = static_cast<double>(static_cast<float>(rx * sr + ry * cr + d->y0));
      const double gdz = d->dz * (d->rel_thick ? d->rel_thick[q] : 1.0);
      int first = static_cast<int>(std::floor(0.5 + (top - d->z0) / dz));
      int end = static_cast<int>(std::floor(0.5 + ((top - d->z0) + d->nz * gdz) / dz));
      end = std::min(end, ns);
      first = std::min(first, ns);
      Rec r;
      // SegyGeometry::FindILXL (libs/nrlib/segy/segygeometry.cpp:1044-1049)
      r.il = static_cast<int>(0.5 + d->il0 + (x - d->x0) * d->il_step_x + (y - d->y0) * d->il_step_y);
      r.xl = static_cast<int>(0.5 + d->xl0 + (x - d->x0) * d->xl_step_x + (y - d->y0) * d->xl_step_y);
      r.ux = static_cast<int>(x);
      r.uy = static_cast<int>(y);
      r.idx = q;
      r.tr = SegyTrace{i, j, first, end, top, gdz};
      rec.push_back(r);
    }
  // inline, crossline, then table index (SortILXL, libs/nrlib/segy/segy.cpp:1364-1381)
  std::sort(rec.begin(), rec.end(), [](const Rec& a, const Rec& b) {
    if (a.il != b.il) return a.il < b.il;
    if (a.xl != b.xl) return a.xl < b.xl;
    return a.idx < b.idx;
  });
  const size_t nrec = rec.size();
  // 240-byte trace headers (TraceHeader::Write, traceheader.cpp:527-587), big-endian
  std::vector<unsigned char> hdr(nrec * 240, 0);
  std::vector<SegyTrace> trs(nrec);
  const int dt = static_cast<short>(static_cast<unsigned short>(dz * 1000));
  const int t0 = static_cast<short>(static_cast<float>(static_cast<short>(d->z0)));
  for (size_t r = 0; r < nrec; r++) {
    unsigned char* h = hdr.data() + r * 240;
    put_be32(h + 36, 0);                 // offset
    put_be16(h + 70, 1);                 // scalco
    put_be32(h + L[0] - 1, rec[r].ux);
    put_be32(h + L[1] - 1, rec[r].uy);
    put_be16(h + 108, t0);               // start time
    put_be16(h + 114, ns);
    put_be16(h + 116, dt);
    put_be32(h + L[2] - 1, rec[r].il);
    put_be32(h + L[3] - 1, rec[r].xl);
    trs[r] = rec[r].tr;
  }
  // binary header (BinaryHeader::Write, libs/nrlib/segy/commonheaders.cpp:233-265; written before
  // the geometry is set, so its trace count per line is 0)
  unsigned char bin[400] = {};
  put_be32(bin + 0, 9999);
  put_be32(bin + 4, 1);
  put_be32(bin + 8, 1);
  put_be16(bin + 16, static_cast<short>(1000 * static_cast<double>(dz)));
  put_be16(bin + 20, static_cast<short>(ns));
  put_be16(bin + 24, 1);   // IBM float samples
  put_be16(bin + 26, 1);
  put_be16(bin + 28, 4);
  put_be16(bin + 54, 1);
  put_be16(bin + 302, 1);  // constant trace length
  const std::string text = segy_text_header(d);

  std::lock_guard<std::mutex> lk(ctx->io_mu);
  CUDA_TRY(cudaSetDevice(ctx->device));
  crava_status s = io_buffers(ctx);
  if (s) return s;
  cudaStream_t st = (cudaStream_t)stream;
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(CRAVA_EINVAL, std::string("cannot open ") + path + " for writing");
  bool ok = std::fwrite(text.data(), 1, 3200, f) == 3200 && std::fwrite(bin, 1, 400, f) == 400;
  // headers and per-trace parameters on the device, then chunks of whole records packed into
  // the device staging half c%2 and downloaded into the pinned half c%2; the file write of chunk
  // c-1 runs while chunk c is in flight
  char* dmem = nullptr;
  const size_t hb = align256(nrec * 240), tb = align256(nrec * sizeof(SegyTrace));
  cudaError_t e = cudaSuccess;
  if (nrec) {
    e = cudaMallocAsync((void**)&dmem, hb + tb, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dmem, hdr.data(), nrec * 240, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dmem + hb, trs.data(), nrec * sizeof(SegyTrace), cudaMemcpyHostToDevice, st);
  }
  SegyPack P;
  P.grid = d_grid;
  P.rnxp = rnxp;
  P.nyp = nyp;
  P.nz = d->nz;
  P.ns = ns;
  P.z0 = d->z0;
  P.dz = dz;
  P.hdr = (const uint32_t*)dmem;
  P.tr = (const SegyTrace*)(dmem + hb);
  const size_t recb = 240 + 4 * (size_t)ns;
  const size_t per = std::max<size_t>(1, kIoChunk / recb);
  size_t pending[2] = {0, 0};
  int nl = 0;
  for (size_t r0 = 0, c = 0; ok && e == cudaSuccess && r0 < nrec; r0 += per, c++) {
    const int b = (int)(c % 2);
    const size_t nr = std::min(per, nrec - r0);
    if (pending[b]) {
      e = cudaEventSynchronize(ctx->io_ev[b]);
      if (e == cudaSuccess) ok = std::fwrite(ctx->io_host[b], 1, pending[b], f) == pending[b];
      pending[b] = 0;
    }
    uint32_t* dst = (uint32_t*)(ctx->io_dev + b * kIoChunk);
    if (e == cudaSuccess) e = launch_segy_pack(P, r0, (int)nr, dst, st);
    nl++;
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->io_host[b], dst, nr * recb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->io_ev[b], st);
    pending[b] = nr * recb;
    const int o = 1 - b;
    if (e == cudaSuccess && ok && pending[o]) {
      e = cudaEventSynchronize(ctx->io_ev[o]);
      if (e == cudaSuccess) ok = std::fwrite(ctx->io_host[o], 1, pending[o], f) == pending[o];
      pending[o] = 0;
    }
  }
  for (int b = 0; b < 2 && e == cudaSuccess && ok; b++)
    if (pending[b]) {
      e = cudaEventSynchronize(ctx->io_ev[b]);
      if (e == cudaSuccess) ok = std::fwrite(ctx->io_host[b], 1, pending[b], f) == pending[b];
    }
  if (dmem) {
    cudaFreeAsync(dmem, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  ok = (std::fclose(f) == 0) && ok;
  if (e != cudaSuccess) return cuda_fail(e, "crava_grid_write_segy");
  if (!ok) return fail(CRAVA_EINVAL, std::string("writing ") + path + " failed");
  {
    std::lock_guard<std::mutex> lk2(ctx->mu);
    ctx->launches += nl;
  }
  return CRAVA_OK;
}

crava_status crava_circ_corr_t(const double* prior_corr_t, int n, int min_int_fq, int nzp, float* out) {
  if (!prior_corr_t || !out || n < 1 || nzp < 2) return fail(CRAVA_EINVAL, "bad arguments");
  if (!(prior_corr_t[0] != 0.0)) return fail(CRAVA_EINVAL, "prior_corr_t[0] must be nonzero");
  // circular extension (computeCircCorrT, src/seismicparametersholder.cpp:624-660)
  std::vector<double> c(nzp, 0.0);
  for (int k = 0; k < nzp; k++) {
    const int refk = k < nzp / 2 + 1 ? k : nzp - k;
    c[k] = refk < n ? (double)(float)prior_corr_t[refk] : 0.0;
  }
  // makeCircCorrTPosDef (:805-840): spectrum zero at k <= minIntFq, |.| elsewhere, back
  // transform (unnormalised) and divide by the lag-0 value
  std::vector<cd> C = dft(c);
  std::vector<double> mag(nzp / 2 + 1);
  for (int k = 0; k <= nzp / 2; k++) mag[k] = k <= min_int_fq ? 0.0 : std::abs(C[k]);
  std::vector<double> back(nzp, 0.0);
  for (int t = 0; t < nzp; t++) {
    double acc = mag[0];
    for (int k = 1; k <= nzp / 2; k++) {
      const double w = (2 * k == nzp) ? 1.0 : 2.0;   // Hermitian pairs k, nzp - k
      acc += w * mag[k] * std::cos(2.0 * M_PI * (double)((long long)k * t % nzp) / nzp);
    }
    back[t] = acc;
  }
  if (!(back[0] > 1e-5))
    return fail(CRAVA_EINVAL, "circular temporal correlation undefined: too few layers for the correlation range");
  for (int t = 0; t < nzp; t++) out[t] = (float)(back[t] / back[0]);
  return CRAVA_OK;
}

crava_status crava_circ_auto_cov(const double* auto_cov, int nlag, int nzp, double dz, float* out) {
  if (!auto_cov || !out || nlag < 1 || nzp < 2 || !(dz > 0)) return fail(CRAVA_EINVAL, "bad arguments");
  const double eps = 1e-10;
  // ComputeCircAutoCov per pair (src/seismicparametersholder.cpp:559-620) with the lag-0
  // test of InitializeCorrelations (:247-274): lag k of pair (i, j) forward, (j, i) backward
  std::vector<std::vector<double>> circ(9, std::vector<double>(nzp, 0.0));
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      std::vector<double>& c = circ[3 * i + j];
      const bool zero = !(std::fabs(auto_cov[3 * i + j]) > eps);
      for (int k = 0; k < nlag; k++) {
        if (k < nzp) c[k] = zero ? 0.0 : (double)(float)auto_cov[9 * k + 3 * i + j];
        if (k < nlag - 1 && nzp - k - 1 >= 0 && nzp - k - 1 < nzp)
          c[nzp - k - 1] = zero ? 0.0 : (double)(float)auto_cov[9 * (k + 1) + 3 * j + i];
      }
    }
  // MakeCircAutoCovPosDef (:622-720): per frequency, D^-1 C(f) D^-1 with D the lag-0 standard
  // deviations, its eigenvalues replaced by their absolute values, scaled back, inverse
  // transformed and divided by nzp
  const int nh = nzp / 2 + 1;
  std::vector<std::vector<cd>> F(9);
  for (int q = 0; q < 9; q++) F[q] = dft(circ[q]);
  double dstd[3];
  for (int i = 0; i < 3; i++) {
    if (!(circ[4 * i][0] > 0)) return fail(CRAVA_EINVAL, "auto-covariance with a non-positive lag-0 variance");
    dstd[i] = std::sqrt(circ[4 * i][0]);
  }
  for (int f = 0; f < nh; f++) {
    cd A[kMaxTheta][kMaxTheta], U[kMaxTheta][kMaxTheta];
    double lam[kMaxTheta];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) A[i][j] = F[3 * i + j][f] / (dstd[i] * dstd[j]);
    for (int i = 0; i < 3; i++)   // the Hermitian part (exact for a consistent estimate)
      for (int j = 0; j <= i; j++) {
        const cd h = 0.5 * (A[i][j] + std::conj(A[j][i]));
        A[i][j] = h;
        A[j][i] = std::conj(h);
      }
    herm_eig(3, A, lam, U);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        cd acc = 0;
        for (int m = 0; m < 3; m++) acc += U[i][m] * std::fabs(lam[m]) * std::conj(U[j][m]);
        F[3 * i + j][f] = acc * (dstd[i] * dstd[j]);
      }
  }
  // TaperCircAutoCovFunction (:722-757): Gaussian taper of 50 ms standard deviation (at most
  // nzp / 2 samples), cut below 1e-10
  double sd = 50.0 / dz;
  if (sd > nzp / 2.0) sd = nzp / 2.0;
  const int pairs[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
  for (int g = 0; g < 6; g++) {
    const std::vector<cd>& X = F[3 * pairs[g][0] + pairs[g][1]];
    for (int t = 0; t < nzp; t++) {
      double acc = X[0].real();
      for (int k = 1; k < nh; k++) {
        const double ang = 2.0 * M_PI * (double)((long long)k * t % nzp) / nzp;
        const double w = (2 * k == nzp) ? 1.0 : 2.0;
        acc += w * (X[k].real() * std::cos(ang) - X[k].imag() * std::sin(ang));
      }
      const int m = t < nzp / 2 + 1 ? t : nzp - t;
      const double e = std::exp(-0.5 * std::pow((double)(float)m / sd, 2));
      const double taper = e > 1e-10 ? (double)(float)e : 0.0;
      out[(size_t)g * nzp + t] = (float)(acc / nzp * taper);
    }
  }
  return CRAVA_OK;
}

crava_status crava_tuning_set(const char* key, int n, int value) {
  if (!key || !*key) return fail(CRAVA_EINVAL, "null schedule key");
  std::lock_guard<std::mutex> lk(g_tune_mu);
  tune_load_default_locked();
  if (value < 0) g_tune.erase({key, n});
  else g_tune[{key, n}] = value;
  return CRAVA_OK;
}

crava_status crava_tuning_get(const char* key, int n, int* value) {
  if (!key || !value) return fail(CRAVA_EINVAL, "null argument");
  *value = crava::tuned(key, n, -1);
  return CRAVA_OK;
}

crava_status crava_tuning_load(const char* path) {
  if (!path) return fail(CRAVA_EINVAL, "null path");
  std::map<std::pair<std::string, int>, int> t;
  if (!tune_parse(path, t)) return fail(CRAVA_EINVAL, std::string("cannot read schedule file ") + path);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_loaded = true;
  g_tune.swap(t);
  g_tune_path = path;
  return CRAVA_OK;
}

const char* crava_tuning_path(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  tune_load_default_locked();
  return g_tune_path.c_str();
}

crava_status crava_ctx_create(crava_ctx** ctx, int device, size_t hbm_budget) {
  if (!ctx) return fail(CRAVA_EINVAL, "null ctx");
  int n = 0;
  CUDA_TRY(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(CRAVA_EINVAL, "no such device");
  CUDA_TRY(cudaSetDevice(device));
  crava_ctx* c = new crava_ctx();
  c->device = device;
  c->budget = hbm_budget;
  *ctx = c;
  return CRAVA_OK;
}

crava_status crava_ctx_destroy(crava_ctx* ctx) {
  if (!ctx) return CRAVA_OK;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  for (auto& kv : ctx->plans) cudaFree(kv.second.tw);
  if (ctx->stage) cudaFree(ctx->stage);
  for (auto& kv : ctx->cache) {
    if (kv.second->ready) cudaEventDestroy(kv.second->ready);
    cudaFree(kv.second->mem);
    delete kv.second;
  }
  for (int b = 0; b < 2; b++) {
    if (ctx->io_host[b]) cudaFreeHost(ctx->io_host[b]);
    if (ctx->io_ev[b]) cudaEventDestroy(ctx->io_ev[b]);
  }
  if (ctx->io_dev) cudaFree(ctx->io_dev);
  delete ctx;
  return CRAVA_OK;
}

crava_status crava_ctx_set_table_cache(crava_ctx* ctx, size_t max_bytes) {
  if (!ctx) return fail(CRAVA_EINVAL, "null context");
  CUDA_TRY(cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> lk(ctx->cache_mu);
  ctx->cache_max = max_bytes;
  cache_evict_locked(ctx, 0, 0);   // unreferenced entries above the new limit
  return CRAVA_OK;
}

crava_status crava_ctx_table_cache_stats(crava_ctx* ctx, long long* hits, long long* misses, size_t* bytes,
                                         int* entries) {
  if (!ctx) return fail(CRAVA_EINVAL, "null context");
  std::lock_guard<std::mutex> lk(ctx->cache_mu);
  if (hits) *hits = ctx->cache_hits;
  if (misses) *misses = ctx->cache_misses;
  if (bytes) *bytes = ctx->cache_bytes;
  if (entries) *entries = (int)ctx->cache.size();
  return CRAVA_OK;
}

long long crava_ctx_kernel_launches(crava_ctx* ctx) { return ctx ? ctx->launches : 0; }

crava_status crava_ctx_set_profiling(crava_ctx* ctx, int enable) {
  if (!ctx) return fail(CRAVA_EINVAL, "null ctx");
  ctx->profiling = enable != 0;
  return CRAVA_OK;
}

crava_status crava_ctx_kernel_times(crava_ctx* ctx, double* ms, long long* launches, int n, int reset) {
  if (!ctx || !ms || !launches) return fail(CRAVA_EINVAL, "null argument");
  std::vector<ProfRec> recs;
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    recs.swap(ctx->prof);
  }
  CUDA_TRY(cudaSetDevice(ctx->device));
  for (auto& r : recs) {
    float t = 0.f;
    cudaError_t e = cudaEventSynchronize(r.b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, r.a, r.b);
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
    if (e != cudaSuccess) return cuda_fail(e, "kernel timing");
    ctx->kt_ms[r.cat] += t;
    ctx->kt_n[r.cat] += 1;
  }
  for (int c = 0; c < n && c < KT_COUNT; c++) {
    ms[c] = ctx->kt_ms[c];
    launches[c] = ctx->kt_n[c];
  }
  if (reset)
    for (int c = 0; c < KT_COUNT; c++) { ctx->kt_ms[c] = 0; ctx->kt_n[c] = 0; }
  return CRAVA_OK;
}

crava_status crava_job_footprint(const crava_job_desc* desc, size_t* bytes) {
  crava_status s = validate(desc);
  if (s) return s;
  if (!bytes) return fail(CRAVA_EINVAL, "null output");
  *bytes = footprint(desc);
  return CRAVA_OK;
}

}  // extern "C"

namespace {

void cache_release(crava_ctx* ctx, CacheEntry* e) {
  if (!e) return;
  std::lock_guard<std::mutex> lk(ctx->cache_mu);
  e->refs--;
}

void job_release(crava_job* j) {
  if (!j) return;
  cache_release(j->ctx, j->kz_entry);
  cache_release(j->ctx, j->lat_entry);
  if (j->pool) {
    if (j->async) cudaFreeAsync(j->pool, j->alloc_stream);
    else cudaFree(j->pool);
    std::lock_guard<std::mutex> lk(j->ctx->mu);
    j->ctx->allocated -= j->pool_bytes;
  }
  if (j->wgrid) cudaFree(j->wgrid);
  if (j->wspec) cudaFree(j->wspec);
  if (j->w3mem) cudaFree(j->w3mem);
  if (j->fac_mem) cudaFree(j->fac_mem);
  delete j;
}

// Builds the per-kz tables of model d into mem (kz_set_bytes(d) bytes) on stream st: the
// operator tables of computePostMeanResidAndFFTCov, the separable factors (error part of Sd,
// temporal spectrum) and the eigen tables of the in-place pencil kernel.
crava_status kz_set_build(const crava_job_desc& d, const std::vector<double>& A, const std::vector<double>& etc,
                          const std::vector<double>& pv, const std::vector<float>& circ, char* mem, cudaStream_t st,
                          KzSet& k) {
  char* p = mem;
  auto take = [&](size_t bytes) { char* q = p; p += align256(bytes); return q; };
  const int nth = d.ntheta;
  k.kw = (float2*)take(sizeof(float2) * d.nzp * nth);
  k.e1 = (float2*)take(sizeof(float2) * d.nzp * nth);
  k.e2 = (float2*)take(sizeof(float2) * d.nzp * nth);
  k.kwd = (double2*)take(sizeof(double2) * d.nzp * nth);
  k.e1d = (double2*)take(sizeof(double2) * d.nzp * nth);
  k.e2d = (double2*)take(sizeof(double2) * d.nzp * nth);
  k.septab = (float2*)take(sizeof(float2) * d.nzp * ((size_t)nth * (nth + 1) / 2));
  k.inv = (uint8_t*)take(d.nzp);
  k.ct = (float2*)take(sizeof(float2) * d.nzp);
  k.edk = (float*)take(sizeof(float) * d.nzp * nth);
  k.eddk = (double*)take(sizeof(double) * d.nzp * nth);
  if (eig_table_bytes(&d)) k.eig = (float4*)take(eig_table_bytes(&d));
  std::vector<float2> kw, e1, e2;
  std::vector<double2> kwd, e1d, e2d;
  std::vector<uint8_t> inv;
  std::vector<float> edk;
  std::vector<double> eddk;
  build_kz_tables(d, kw, e1, e2, inv, &kwd, &e1d, &e2d, edk, &eddk);
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
  };
  CUDA_TRY(up(k.edk, edk.data(), sizeof(float) * edk.size()));
  CUDA_TRY(up(k.eddk, eddk.data(), sizeof(double) * eddk.size()));
  CUDA_TRY(up(k.kwd, kwd.data(), sizeof(double2) * kwd.size()));
  CUDA_TRY(up(k.e1d, e1d.data(), sizeof(double2) * e1d.size()));
  CUDA_TRY(up(k.e2d, e2d.data(), sizeof(double2) * e2d.size()));
  CUDA_TRY(up(k.kw, kw.data(), sizeof(float2) * kw.size()));
  CUDA_TRY(up(k.e1, e1.data(), sizeof(float2) * e1.size()));
  CUDA_TRY(up(k.e2, e2.data(), sizeof(float2) * e2.size()));
  CUDA_TRY(up(k.inv, inv.data(), inv.size()));
  if (d.prior_mode != CRAVA_PRIOR_SEPARABLE) {
    k.eig_why = "prior given as grids";
    return CRAVA_OK;
  }
  // Separable prior: the error part of Sd per kz, M2 = ec o (e1 e1^H + e2 e2^H) with
  // ec = (1 - wnc) errThetaCov / 2 (getNextErrorVariance, src/avoinversion.cpp:1236-1272),
  // lower triangle row by row.
  const int tri = nth * (nth + 1) / 2;
  std::vector<float2> sep((size_t)d.nzp * tri);
  for (int kz = 0; kz < d.nzp; kz++) {
    float2* row = sep.data() + (size_t)kz * tri;
    const double2* a1 = e1d.data() + (size_t)kz * nth;
    const double2* a2 = e2d.data() + (size_t)kz * nth;
    for (int l = 0; l < nth; l++)
      for (int m = 0; m <= l; m++) {
        const cd ee = cd(a1[l].x, a1[l].y) * std::conj(cd(a1[m].x, a1[m].y)) +
                      cd(a2[l].x, a2[l].y) * std::conj(cd(a2[m].x, a2[m].y));
        const cd m2 = ee * (0.5 * (1.0 - d.wnc) * etc[l * nth + m]);
        row[l * (l + 1) / 2 + m] = make_float2((float)m2.real(), (float)m2.imag());
      }
  }
  CUDA_TRY(up(k.septab, sep.data(), sizeof(float2) * sep.size()));
  // temporal factor: DFT of circCorrT (1D, double); a symmetric circular correlation (the
  // form computeCircCorrT builds, src/seismicparametersholder.cpp:624-660) has a real
  // spectrum, whose imaginary part is then exactly zero
  std::vector<double> c(circ.begin(), circ.end());
  std::vector<cd> C = dft(c);
  bool sym = true;
  for (int t = 1; t < d.nzp && sym; t++) sym = circ[t] == circ[d.nzp - t];
  std::vector<float2> ct(d.nzp);
  for (int kz = 0; kz < d.nzp; kz++) ct[kz] = make_float2((float)C[kz].real(), sym ? 0.f : (float)C[kz].imag());
  CUDA_TRY(up(k.ct, ct.data(), sizeof(float2) * d.nzp));
  // the eigen form of the per-bin posterior (pencil.cu) where it applies
  if (!k.eig) k.eig_why = "no separable prior";
  else if (!sym) k.eig_why = "circular temporal correlation not symmetric";
  else if (d.fp64_threshold > 0.f) k.eig_why = "FP64 re-factorisation requested";
  else {
    float G0[kMaxTheta][kMaxTheta], AP[kMaxTheta][3];
    sep_constants(A, pv, nth, G0, AP);
    std::vector<float> rows;
    k.eig_base = build_eig_tables(d, kw, sep, edk, inv, ct, G0, AP, k.lam_limit, rows, k.n_inv_rows, k.eig_why);
    if (k.eig_base) CUDA_TRY(up(k.eig, rows.data(), sizeof(float) * rows.size()));
  }
  return CRAVA_OK;
}

// Builds the lateral factor of model d into mem (lat_set_bytes(d) bytes) on stream st: the
// 2D transform of corrXY (x then y) on the device.
crava_status lat_set_build(crava_ctx* ctx, const crava_job_desc& d, const std::vector<float>& corr_xy, char* mem,
                           cudaStream_t st, LatSet& l) {
  const int cnxp = d.nxp / 2 + 1, rnxp = 2 * cnxp;
  l.cxy = (float2*)mem;
  l.grid = (float*)(mem + align256(sizeof(float2) * cnxp * d.nyp));
  std::vector<float> g((size_t)rnxp * d.nyp, 0.f);
  for (int jj = 0; jj < d.nyp; jj++)
    for (int ii = 0; ii < d.nxp; ii++) g[(size_t)jj * rnxp + ii] = corr_xy[(size_t)jj * d.nxp + ii];
  CUDA_TRY(cudaMemcpyAsync(l.grid, g.data(), sizeof(float) * g.size(), cudaMemcpyHostToDevice, st));
  Plan *px, *pn, *py;
  crava_status ps;
  if ((ps = get_xplans(ctx, d.nxp, &px, &pn)) || (ps = get_plan(ctx, d.nyp, &py))) return ps;
  GridSet gs;
  gs.n = 1;
  gs.p[0] = l.grid;
  gs.src[0] = l.grid;
  gs.scale[0] = 1.0f;
  int nl = 0;
  CUDA_TRY(launch_x_r2c(gs, d.nxp, d.nyp, px->lp, px->tw, pn->tw, st, &nl));
  CUDA_TRY(launch_line_fft(gs, cnxp, d.nyp, (size_t)cnxp, 1, 0, py->lp, py->tw, -1.f, st, &nl));
  CUDA_TRY(cudaMemcpyAsync(l.cxy, l.grid, sizeof(float2) * cnxp * d.nyp, cudaMemcpyDeviceToDevice, st));
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->launches += nl;
  return CRAVA_OK;
}

// Cache keys: the bytes every table of the entry depends on.
template <class T>
void key_put(std::string& k, const T* p, size_t n) {
  if (p && n) k.append(reinterpret_cast<const char*>(p), sizeof(T) * n);
}
std::string kz_key(const crava_job_desc& d) {
  std::string k = "K";
  const int iv[6] = {d.nz, d.nzp, d.ntheta, d.prior_mode, d.flags & CRAVA_FLAG_NONCONST_THICK,
                     d.fp64_threshold > 0.f ? 1 : 0};
  key_put(k, iv, 6);
  const double dv[2] = {d.lz, d.min_rel_thick};
  key_put(k, dv, 2);
  const float fv[3] = {d.low_cut, d.high_cut, d.wnc};
  key_put(k, fv, 3);
  key_put(k, d.A, 3 * (size_t)d.ntheta);
  key_put(k, d.err_theta_cov, (size_t)d.ntheta * d.ntheta);
  key_put(k, d.prior_var0, 9);
  key_put(k, d.wavelet, (size_t)d.ntheta * d.nzp);
  key_put(k, d.wavelet_norm, (size_t)d.ntheta);
  if (d.prior_mode == CRAVA_PRIOR_SEPARABLE) key_put(k, d.circ_corr_t, (size_t)d.nzp);
  return k;
}
std::string lat_key(const crava_job_desc& d) {
  std::string k = "L";
  const int iv[2] = {d.nxp, d.nyp};
  key_put(k, iv, 2);
  key_put(k, d.corr_xy, (size_t)d.nxp * d.nyp);
  return k;
}

// Frees unreferenced entries, least recently used first, until `want` more bytes fit under
// both the cache limit and the context budget (or nothing is left to free).  Caller holds
// cache_mu.
void cache_evict_locked(crava_ctx* ctx, size_t want, cudaStream_t st) {
  for (;;) {
    size_t allocated;
    {
      std::lock_guard<std::mutex> lk(ctx->mu);
      allocated = ctx->allocated;
    }
    const bool over_cache = ctx->cache_bytes + want > ctx->cache_max;
    const bool over_budget = ctx->budget && allocated + want > ctx->budget;
    if (!over_cache && !over_budget) return;
    CacheEntry* victim = nullptr;
    for (auto& kv : ctx->cache)
      if (kv.second->refs == 0 && (!victim || kv.second->tick < victim->tick)) victim = kv.second;
    if (!victim) return;
    ctx->cache.erase(victim->key);
    ctx->cache_bytes -= victim->bytes;
    {
      std::lock_guard<std::mutex> lk(ctx->mu);
      ctx->allocated -= victim->bytes;
    }
    if (victim->ready) cudaEventDestroy(victim->ready);
    cudaFreeAsync(victim->mem, st);   // no job references it: its users have completed
    delete victim;
  }
}

// The cached tables of `key`, built on a miss by build(mem, entry) into new device memory
// on stream st; a hit makes st wait for the stream that built them.  The entry stays
// referenced until cache_release.
template <class Build>
crava_status cache_acquire(crava_ctx* ctx, const std::string& key, size_t bytes, cudaStream_t st, Build build,
                           CacheEntry** out) {
  std::lock_guard<std::mutex> lk(ctx->cache_mu);
  auto it = ctx->cache.find(key);
  if (it != ctx->cache.end()) {
    CacheEntry* e = it->second;
    e->refs++;
    e->tick = ++ctx->cache_tick;
    ctx->cache_hits++;
    if (e->ready) CUDA_TRY(cudaStreamWaitEvent(st, e->ready, 0));
    *out = e;
    return CRAVA_OK;
  }
  ctx->cache_misses++;
  cache_evict_locked(ctx, bytes, st);
  {
    std::lock_guard<std::mutex> lk2(ctx->mu);
    if (ctx->budget && ctx->allocated + bytes > ctx->budget)
      return fail(CRAVA_ENOMEM, "table cache entry of " + std::to_string(bytes) + " bytes exceeds the budget");
    ctx->allocated += bytes;
  }
  CacheEntry* e = new CacheEntry();
  e->key = key;
  e->bytes = bytes;
  cudaError_t ce = cudaMallocAsync((void**)&e->mem, bytes, st);
  crava_status s = ce == cudaSuccess ? build(e->mem, *e) : fail(CRAVA_ENOMEM, "table cache allocation");
  if (!s && cudaEventCreateWithFlags(&e->ready, cudaEventDisableTiming) != cudaSuccess) s = CRAVA_ECUDA;
  if (!s && cudaEventRecord(e->ready, st) != cudaSuccess) s = CRAVA_ECUDA;
  if (s) {
    if (e->mem) cudaFreeAsync(e->mem, st);
    if (e->ready) cudaEventDestroy(e->ready);
    std::lock_guard<std::mutex> lk2(ctx->mu);
    ctx->allocated -= bytes;
    delete e;
    return s;
  }
  e->refs = 1;
  e->tick = ++ctx->cache_tick;
  ctx->cache[key] = e;
  ctx->cache_bytes += bytes;
  *out = e;
  return CRAVA_OK;
}

// Job set-up on stream st.  async: the pool comes from the stream-ordered allocator and
// nothing waits for the GPU (the serving loop); otherwise the call returns with the job
// ready (the public crava_job_create).  With the context's table cache on, the per-kz and
// lateral tables are shared entries of the cache instead of parts of the job's pool.
crava_status job_create_impl(crava_ctx* ctx, const crava_job_desc* desc, cudaStream_t st, bool async,
                             crava_job** job) {
  if (!ctx || !job) return fail(CRAVA_EINVAL, "null argument");
  crava_status s = validate(desc);
  if (s) return s;
  CUDA_TRY(cudaSetDevice(ctx->device));
  crava_job* j = new crava_job();
  j->ctx = ctx;
  j->d = *desc;
  const crava_job_desc& d = j->d;
  j->cnxp = d.nxp / 2 + 1;
  j->rnxp = 2 * j->cnxp;
  j->rsize = (size_t)j->rnxp * d.nyp * d.nzp;
  j->N = (size_t)d.nxp * d.nyp * d.nzp;
  j->A.assign(d.A, d.A + 3 * d.ntheta);
  j->etc.assign(d.err_theta_cov, d.err_theta_cov + d.ntheta * d.ntheta);
  j->pv.assign(d.prior_var0, d.prior_var0 + 9);
  j->wav.assign(d.wavelet, d.wavelet + (size_t)d.ntheta * d.nzp);
  j->wnorm.assign(d.wavelet_norm, d.wavelet_norm + d.ntheta);
  // the factors are kept in GRIDS mode too when given: crava_job_fill_prior builds the grids
  if (d.prior_mode == CRAVA_PRIOR_SEPARABLE || (d.corr_xy && d.circ_corr_t)) {
    j->corr_xy.assign(d.corr_xy, d.corr_xy + (size_t)d.nxp * d.nyp);
    j->circ.assign(d.circ_corr_t, d.circ_corr_t + d.nzp);
  }
  j->d.A = j->A.data();
  j->d.err_theta_cov = j->etc.data();
  j->d.prior_var0 = j->pv.data();
  j->d.wavelet = j->wav.data();
  j->d.wavelet_norm = j->wnorm.data();
  if (d.flags & CRAVA_FLAG_NONCONST_THICK) {
    j->relt.assign(d.rel_thick, d.rel_thick + (size_t)d.nxp * d.nyp);
    if (j->circ.empty()) j->circ.assign(d.circ_corr_t, d.circ_corr_t + d.nzp);
  }
  j->d.corr_xy = j->corr_xy.empty() ? nullptr : j->corr_xy.data();
  j->d.circ_corr_t = j->circ.empty() ? nullptr : j->circ.data();
  j->d.rel_thick = j->relt.empty() ? nullptr : j->relt.data();

  bool cached;
  {
    std::lock_guard<std::mutex> lk(ctx->cache_mu);
    cached = ctx->cache_max > 0;
  }
  const size_t need = grid_part_bytes(&d) + (cached ? 0 : kz_set_bytes(&d) + lat_set_bytes(&d));
  for (int attempt = 0;; attempt++) {
    std::unique_lock<std::mutex> lk(ctx->mu);
    if (!ctx->budget || ctx->allocated + need <= ctx->budget) {
      ctx->allocated += need;
      break;
    }
    const size_t left = ctx->budget > ctx->allocated ? ctx->budget - ctx->allocated : 0;
    lk.unlock();
    if (attempt == 0) {   // unreferenced cached tables give way to a job
      std::lock_guard<std::mutex> ck(ctx->cache_mu);
      cache_evict_locked(ctx, need, st);
      continue;
    }
    delete j;
    return fail(CRAVA_ENOMEM, "job needs " + std::to_string(need) + " bytes; budget left " + std::to_string(left));
  }
  j->async = async;
  j->alloc_stream = st;
  j->pool_bytes = need;
  bool injected = false;
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (ctx->fail_allocs > 0) {
      ctx->fail_allocs--;
      injected = true;
    }
  }
  cudaError_t e = injected ? cudaErrorMemoryAllocation
                           : async ? cudaMallocAsync((void**)&j->pool, need, st) : cudaMalloc(&j->pool, need);
  if (e != cudaSuccess) {
    cudaGetLastError();
    j->pool = nullptr;
    {
      std::lock_guard<std::mutex> lk(ctx->mu);
      ctx->allocated -= need;
    }
    delete j;
    return fail(CRAVA_ENOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
  }
  size_t gb = align256(sizeof(float) * j->rsize);
  char* p = j->pool;
  auto take = [&](size_t bytes) { char* q = p; p += align256(bytes); return q; };
  for (int l = 0; l < d.ntheta; l++) j->in_data[l] = (float*)take(gb);
  for (int a = 0; a < 3; a++) j->in_mean[a] = (float*)take(gb);
  for (int l = 0; l < d.ntheta; l++) j->data[l] = (float*)take(gb);
  for (int a = 0; a < 3; a++) j->mean[a] = (float*)take(gb);
  for (int q = 0; q < 6; q++) j->cov[q] = (float*)take(gb);
  if (d.prior_mode == CRAVA_PRIOR_GRIDS) {
    for (int q = 0; q < 6; q++) j->in_cov[q] = (float*)take(gb);
    j->in_err = (float*)take(gb);
    j->err = (float*)take(gb);
    j->fill_xy = (float*)take(sizeof(float) * j->rnxp * d.nyp);
    j->fill_t = (float*)take(sizeof(float) * d.nzp);
  }
  for (int q = 0; q < 3 * d.nsim; q++) j->sim[q] = (float*)take(gb);
  if (d.flags & CRAVA_FLAG_HOST_NOISE)
    for (int q = 0; q < 3 * d.nsim; q++) j->noise[q] = (float*)take(gb);
  j->counters = (unsigned long long*)take(256);
  ThickTables tt;
  const bool nonconst = (d.flags & CRAVA_FLAG_NONCONST_THICK) != 0;
  if (nonconst) {
    const size_t nth = d.ntheta, cn = d.nzp / 2 + 1, nxy = (size_t)d.nx * d.ny;
    ThickParams& tp = j->tp;
    tp.wamp = (const float2*)take(sizeof(float2) * nth * cn);
    tp.es3 = (const float2*)take(sizeof(float2) * nth * cn);
    tp.tau2 = (const float*)take(sizeof(float) * nth * cn);
    tp.glob = (const float2*)take(sizeof(float2) * nth * cn);
    tp.ztaper = (const float*)take(sizeof(float) * d.nzp);
    tp.distz = (const float*)take(sizeof(float) * d.nzp);
    tp.fillx = (const int*)take(sizeof(int) * d.nxp);
    tp.filly = (const int*)take(sizeof(int) * d.nyp);
    tp.distx = (const float*)take(sizeof(float) * d.nxp);
    tp.disty = (const float*)take(sizeof(float) * d.nyp);
    tp.rel_thick = (const double*)take(sizeof(double) * d.nxp * d.nyp);
    j->energy = (float*)take(sizeof(float) * nth * nxy);
    j->ops = (TraceOp*)take(sizeof(TraceOp) * nth * nxy);
    j->nzero = (int*)take(sizeof(int) * kMaxTheta);
    build_thick_tables(d, tt);
    tp.nx = d.nx; tp.ny = d.ny; tp.nz = d.nz;
    tp.nxp = d.nxp; tp.nyp = d.nyp; tp.nzp = d.nzp;
    tp.rnxp = j->rnxp;
    tp.cnzp = (int)cn;
    tp.W = thick_tile_width(d.nzp);
    if (const int tw = tuned("thick_w", d.nzp, 0)) {
      int w = 1;
      while (w * 2 <= std::min(16, tw)) w *= 2;
      if (thick_smem_bytes(w, d.nzp) <= 227 * 1024) tp.W = w;
    }
    tp.logW = 0;
    while ((1 << tp.logW) < tp.W) tp.logW++;
    tp.nIT = ((d.nxp + 1) / 2 + tp.W - 1) / tp.W;
    for (int l = 0; l < d.ntheta; l++) {
      tp.grid[l] = j->in_data[l];
      tp.wn2[l] = tt.wn2[l];
      tp.modW[l] = tt.modW[l];
      tp.err_var[l] = tt.err_var[l];
      tp.es3_last[l] = tt.es3_last[l];
    }
    tp.wnc = d.wnc;
    tp.low_cut = d.low_cut;
    tp.high_cut = d.high_cut;
    tp.rsq = static_cast<float>(std::sqrt(static_cast<float>(d.nzp)));
    {
      int e = 0;
      tp.inv_rsq = std::frexp(tp.rsq, &e) == 0.5f ? 1.0f / tp.rsq : 0.f;   // rsq = 2^(e-1)
    }
    tp.lz = d.lz;
  }
#define JOB_TRY(call)                                          \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) {                                   \
      crava_status st_ = cuda_fail(e_, #call);                 \
      job_release(j);                                          \
      return st_;                                              \
    }                                                          \
  } while (0)
#define JOB_STATUS(call)                                       \
  do {                                                         \
    crava_status s_ = (call);                                  \
    if (s_) {                                                  \
      job_release(j);                                          \
      return s_;                                               \
    }                                                          \
  } while (0)
  auto up = [&](const void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(const_cast<void*>(dst), src, bytes, cudaMemcpyHostToDevice, st);
  };
  if (nonconst) {
    ThickParams& tp = j->tp;
    JOB_TRY(up(tp.wamp, tt.wamp.data(), sizeof(float2) * tt.wamp.size()));
    JOB_TRY(up(tp.es3, tt.es3.data(), sizeof(float2) * tt.es3.size()));
    JOB_TRY(up(tp.tau2, tt.tau2.data(), sizeof(float) * tt.tau2.size()));
    JOB_TRY(up(tp.glob, tt.glob.data(), sizeof(float2) * tt.glob.size()));
    JOB_TRY(up(tp.ztaper, tt.ztaper.data(), sizeof(float) * tt.ztaper.size()));
    JOB_TRY(up(tp.distz, tt.distz.data(), sizeof(float) * tt.distz.size()));
    JOB_TRY(up(tp.fillx, tt.fillx.data(), sizeof(int) * tt.fillx.size()));
    JOB_TRY(up(tp.filly, tt.filly.data(), sizeof(int) * tt.filly.size()));
    JOB_TRY(up(tp.distx, tt.distx.data(), sizeof(float) * tt.distx.size()));
    JOB_TRY(up(tp.disty, tt.disty.data(), sizeof(float) * tt.disty.size()));
    JOB_TRY(up(tp.rel_thick, j->relt.data(), sizeof(double) * j->relt.size()));
  }
  // per-kz and lateral tables: entries of the resident cache, or parts of the pool
  KzSet ks;
  LatSet ls;
  const bool sepmode = d.prior_mode == CRAVA_PRIOR_SEPARABLE;
  if (cached) {
    JOB_STATUS(cache_acquire(ctx, kz_key(d), kz_set_bytes(&d), st,
                             [&](char* mem, CacheEntry& ce) {
                               return kz_set_build(d, j->A, j->etc, j->pv, j->circ, mem, st, ce.k);
                             },
                             &j->kz_entry));
    ks = j->kz_entry->k;
    if (sepmode) {
      JOB_STATUS(cache_acquire(ctx, lat_key(d), lat_set_bytes(&d), st,
                               [&](char* mem, CacheEntry& ce) { return lat_set_build(ctx, d, j->corr_xy, mem, st, ce.l); },
                               &j->lat_entry));
      ls = j->lat_entry->l;
    }
  } else {
    char* km = take(kz_set_bytes(&d));
    JOB_STATUS(kz_set_build(d, j->A, j->etc, j->pv, j->circ, km, st, ks));
    if (sepmode) {
      char* lm = take(lat_set_bytes(&d));
      JOB_STATUS(lat_set_build(ctx, d, j->corr_xy, lm, st, ls));
    }
  }
  j->kw = ks.kw; j->e1 = ks.e1; j->e2 = ks.e2;
  j->kwd = ks.kwd; j->e1d = ks.e1d; j->e2d = ks.e2d;
  j->septab = ks.septab; j->inv = ks.inv; j->ct = ks.ct;
  j->edk = ks.edk; j->eddk = ks.eddk; j->eig = ks.eig;
  j->cxy = ls.cxy; j->cxy_grid = ls.grid;
  j->n_inv_rows = ks.n_inv_rows;
  j->eig_why = ks.eig_why;
  if (ks.eig_base) {
    // the eigen form needs every reference Cholesky of the block clear of its pivot test
    double lam_max = 0;
    for (float v : j->corr_xy) lam_max += std::fabs((double)v);
    j->eig_ok = lam_max < ks.lam_limit;
    if (!j->eig_ok) j->eig_why = "data covariance too close to singular";
  }
  if (!async) JOB_TRY(cudaStreamSynchronize(st));
#undef JOB_TRY
#undef JOB_STATUS
  *job = j;
  return CRAVA_OK;
}

}  // namespace

extern "C" {

crava_status crava_job_create(crava_ctx* ctx, const crava_job_desc* desc, crava_job** job) {
  return job_create_impl(ctx, desc, 0, false, job);
}

crava_status crava_job_destroy(crava_job* job) {
  if (!job) return CRAVA_OK;
  cudaSetDevice(job->ctx->device);
  job_release(job);
  return CRAVA_OK;
}

crava_status crava_job_device_ptr(crava_job* job, crava_role role, int index, float** dptr) {
  if (!job || !dptr) return fail(CRAVA_EINVAL, "null argument");
  crava_status s;
  float* p = grid_ptr(job, role, index, &s);
  if (s) return s;
  if (role == CRAVA_ROLE_PRIOR_COV) job->base_prior = false;   // the caller may write the grid
  *dptr = p;
  return CRAVA_OK;
}

crava_status crava_job_upload(crava_job* job, crava_role role, int index, const float* host, void* stream) {
  if (!job || !host) return fail(CRAVA_EINVAL, "null argument");
  crava_status s;
  float* p = grid_ptr(job, role, index, &s);
  if (s) return s;
  if (role == CRAVA_ROLE_PRIOR_COV) job->base_prior = false;
  CUDA_TRY(cudaMemcpyAsync(p, host, sizeof(float) * job->rsize, cudaMemcpyHostToDevice, (cudaStream_t)stream));
  return CRAVA_OK;
}

crava_status crava_job_download(crava_job* job, crava_role role, int index, float* host, void* stream) {
  if (!job || !host) return fail(CRAVA_EINVAL, "null argument");
  if (!job->ran && (role == CRAVA_ROLE_POST_MEAN || role == CRAVA_ROLE_POST_COV || role == CRAVA_ROLE_SIM ||
                    role == CRAVA_ROLE_RESIDUAL))
    return fail(CRAVA_ESTATE, "outputs are defined only after crava_job_run");
  crava_status s;
  float* p = grid_ptr(job, role, index, &s);
  if (s) return s;
  CUDA_TRY(cudaMemcpyAsync(host, p, sizeof(float) * job->rsize, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  return CRAVA_OK;
}

}  // extern "C"

namespace {

// The inverse y and x transforms of the three posterior-mean grids with the facies
// probabilities of crava_job_set_facies: the x transform and the evaluation in one pass
// (launch_x4_facies) where the x length has a four-step split and the schedule key
// facies_fused (n = nxp/2) is 1, else the x transform and then the facies pass.  The default
// is the two passes: at 540x540x256 the one-pass form took 5.4 ms against 0.5 + 2.3 ms, its
// density gathers (L2-latency bound) running at the transform kernel's occupancy (8 warps
// per SM against about 40 in the facies pass).
crava_status inv_mean_facies(crava_ctx* ctx, crava_job* job, float ps, cudaStream_t st) {
  const crava_job_desc& d = job->d;
  Plan *px, *pn, *py;
  crava_status s;
  if ((s = get_xplans(ctx, d.nxp, &px, &pn)) || (s = get_plan(ctx, d.nyp, &py))) return s;
  GridSet gs;
  gs.n = 3;
  for (int a = 0; a < 3; a++) { gs.p[a] = job->mean[a]; gs.src[a] = job->mean[a]; gs.scale[a] = ps; }
  int nl = 0;
  {
    ProfScope pf(ctx, KT_LINE_INV, st);
    CUDA_TRY(launch_line_fft(gs, job->cnxp, d.nyp, (size_t)job->cnxp, d.nzp, (size_t)job->cnxp * d.nyp, py->lp, py->tw,
                             1.f, st, &nl));
  }
  const bool fused = d.nxp % 2 == 0 && four_step_supported(d.nxp / 2) && tuned("facies_fused", d.nxp / 2, 0) != 0;
  const int rnxp_out = 2 * (d.nx / 2 + 1);
  if (fused) {
    FaciesFuse F;
    for (int a = 0; a < 3; a++) F.mean[a] = job->mean[a];
    F.scale = ps;
    F.nx = d.nx; F.ny = d.ny; F.nz = d.nz; F.nyp = d.nyp;
    F.rnxp_out = rnxp_out;
    F.nf = job->fac_nf;
    F.undef_sum = job->fac_undef;
    for (int f = 0; f < job->fac_nf; f++) F.pr.p[f] = job->fac_prior[f];
    for (int f = 0; f <= job->fac_nf; f++) F.out.p[f] = job->fac_prob[f];
    F.seis_lh = job->fac_lh;
    ProfScope pf(ctx, KT_FACIES, st);
    CUDA_TRY(launch_x4_facies(F, job->fac_hc, d.nxp, d.nyp * d.nzp, px->tw, pn->tw, st, &nl));
  } else {
    {
      ProfScope pf(ctx, KT_X_C2R, st);
      CUDA_TRY(launch_x_c2r(gs, d.nxp, d.nyp * d.nzp, px->lp, px->tw, pn->tw, st, &nl));
    }
    ProfScope pf(ctx, KT_FACIES, st);
    CUDA_TRY(launch_facies_eval(job->mean[0], job->mean[1], job->mean[2], d.nx, d.ny, d.nz, job->rnxp, d.nyp,
                                rnxp_out, job->fac_hc, job->fac_nf, job->fac_prior, job->fac_undef, job->fac_prob,
                                job->fac_lh, st));
    nl++;
  }
  ctx->launches += nl;
  return CRAVA_OK;
}

}  // namespace

extern "C" {

crava_status crava_job_run(crava_job* job, void* stream) {
  if (!job) return fail(CRAVA_EINVAL, "null job");
  crava_ctx* ctx = job->ctx;
  const crava_job_desc& d = job->d;
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(cudaSetDevice(ctx->device));
  CUDA_TRY(cudaMemsetAsync(job->counters, 0, kNumCounters * sizeof(unsigned long long), st));
  const bool grids = d.prior_mode == CRAVA_PRIOR_GRIDS;
  const float fs = fwd_scale(job->N);
  crava_status s;
  // forward transforms: data + mean (x, y); GRIDS mode also the prior grids (x, y, z)
  {
    std::vector<const float*> src;
    std::vector<float*> g;
    std::vector<float> sc;
    for (int l = 0; l < d.ntheta; l++) { src.push_back(job->in_data[l]); g.push_back(job->data[l]); sc.push_back(fs); }
    for (int a = 0; a < 3; a++) { src.push_back(job->in_mean[a]); g.push_back(job->mean[a]); sc.push_back(fs); }
    if ((s = fwd_xy(ctx, src, g, sc, d.nxp, d.nyp, d.nzp, false, st))) return s;
  }
  if (grids) {
    std::vector<const float*> src;
    std::vector<float*> g;
    std::vector<float> sc;
    // SeismicParametersHolder::FFTCovGrids (src/seismicparametersholder.cpp:458-482): with a
    // base prior the six spectra are priorVar0 multiples of one, and only the first is formed
    const int ncov = job->base_prior ? 1 : 6;
    for (int q = 0; q < ncov; q++) { src.push_back(job->in_cov[q]); g.push_back(job->cov[q]); sc.push_back(1.0f); }
    src.push_back(job->in_err);
    g.push_back(job->err);
    sc.push_back(1.0f);
    if ((s = fwd_xy(ctx, src, g, sc, d.nxp, d.nyp, d.nzp, true, st))) return s;
  }
  // the fused pencil pass
  Plan* pz;
  const int skey = d.nzp * 16 + d.ntheta;   // schedule key of the pencil pass
  if ((s = get_plan(ctx, d.nzp, &pz, tuned("zpass_r16", d.nzp, 1) != 0))) return s;
  ZParams zp;
  std::memset(&zp, 0, sizeof(zp));
  zp.nxp = d.nxp; zp.nyp = d.nyp; zp.nzp = d.nzp; zp.cnxp = job->cnxp;
  zp.nxp_even = (d.nxp % 2) == 0;
  // pencil tile: W x-bins (power of two), GT slots per z-transform call, SB realisations
  // per batch and T threads.  Preferred: the widest tile (longest contiguous rows, fewest
  // tiles) with every slot of a phase in one call (GT = G), the first of the candidates
  // that fits; 512 threads when one CTA fills the SM's shared memory, 256 when two fit.
  // CRAVA_ZPASS_{W,T,GT,SB} override.
  const int Gs = std::max(d.ntheta + 3, 9);
  int W = 2, T = 256, GT = Gs, SB = 2;
  {
    const int cand[8][3] = {{4, Gs, 2}, {4, Gs, 1}, {2, Gs, 2}, {2, Gs, 1}, {1, Gs, 2}, {4, 3, 1}, {2, 3, 1}, {1, 3, 1}};
    for (const auto& c : cand) {
      if (zpass_smem_bytes(c[0], d.nzp, d.ntheta, c[1], c[2]) <= 227 * 1024) {
        W = c[0]; GT = c[1]; SB = c[2];
        break;
      }
    }
  }
  W = std::max(1, tuned("zpass_w", skey, W));
  GT = std::max(3, tuned("zpass_gt", skey, GT));
  SB = std::max(1, tuned("zpass_sb", skey, SB));
  SB = std::min(SB, GT / 3);
  T = zpass_smem_bytes(W, d.nzp, d.ntheta, GT, SB) > 113 * 1024 ? 512 : 256;
  T = std::max(64, std::min(512, tuned("zpass_threads", skey, T) / 32 * 32));
  if (zpass_smem_bytes(W, d.nzp, d.ntheta, GT, SB) > 227 * 1024)
    return fail(CRAVA_ENOTSUP, "pencil tile does not fit in shared memory");
  zp.GT = GT;
  zp.SB = SB;
  zp.W = W;
  {
    const bool four = tuned("zpass_four", d.nzp, 1) != 0 && GT >= Gs;
    zp.zsplit = !four ? 0 : d.nzp == 256 ? 1 : d.nzp == 320 ? 2 : d.nzp == 128 ? 3 : 0;
  }
  zp.logW = 0;
  while ((1 << zp.logW) < W) zp.logW++;
  zp.nIT = (job->cnxp + W - 1) / W;
  zp.nth = d.ntheta;
  zp.nsim = d.nsim;
  zp.separable = grids ? 0 : 1;
  zp.base_prior = (grids && job->base_prior) ? 1 : 0;
  zp.host_noise = (d.flags & CRAVA_FLAG_HOST_NOISE) ? 1 : 0;
  zp.keep_resid = (d.flags & CRAVA_FLAG_KEEP_RESIDUAL) ? 1 : 0;
  zp.cov_spectral = (d.flags & CRAVA_FLAG_SPECTRAL_COV) ? 1 : 0;
  for (int l = 0; l < d.ntheta; l++) zp.data[l] = (float2*)job->data[l];
  for (int a = 0; a < 3; a++) zp.mean[a] = (float2*)job->mean[a];
  for (int q = 0; q < 6; q++) zp.cov[q] = (float2*)job->cov[q];
  zp.errspec = (const float2*)job->err;
  for (int q = 0; q < 3 * d.nsim; q++) {
    zp.sim[q] = (float2*)job->sim[q];
    zp.noise[q] = (const float2*)job->noise[q];
  }
  zp.cxy = job->cxy;
  zp.ct = job->ct;
  zp.septab = grids ? nullptr : job->septab;
  sep_constants(job->A, job->pv, d.ntheta, zp.G0, zp.AP);
  const int qa[6] = {0, 1, 2, 0, 0, 1}, qb[6] = {0, 1, 2, 1, 2, 2};
  for (int q = 0; q < 6; q++) zp.pv[q] = static_cast<float>(job->pv[qa[q] * 3 + qb[q]]);
  for (int l = 0; l < d.ntheta; l++) {
    for (int c = 0; c < 3; c++) zp.A[l][c] = static_cast<float>(job->A[l * 3 + c]);
    for (int m = 0; m < d.ntheta; m++) zp.ec[l][m] = float(0.5 * (1.0 - d.wnc) * job->etc[l * d.ntheta + m]);
    zp.ed[l] = float(d.wnc * job->etc[l * d.ntheta + l]);
  }
  zp.kz.kw = job->kw; zp.kz.e1 = job->e1; zp.kz.e2 = job->e2; zp.kz.inv = job->inv;
  zp.kz.kwd = job->kwd; zp.kz.e1d = job->e1d; zp.kz.e2d = job->e2d;
  zp.kz.ed = job->edk;     // always uploaded: wnc errThetaCov_ll per kz, times |e3(k)|^2 with
                           // CRAVA_FLAG_NONCONST_THICK
  zp.kz.edd = job->eddk;
  zp.fp64_threshold = d.fp64_threshold;
  for (int l = 0; l < d.ntheta; l++) {
    for (int c = 0; c < 3; c++) zp.Ad[l][c] = job->A[l * 3 + c];
    for (int m = 0; m < d.ntheta; m++) zp.ecd[l][m] = 0.5 * (1.0 - d.wnc) * job->etc[l * d.ntheta + m];
    zp.edd[l] = d.wnc * job->etc[l * d.ntheta + l];
  }
  zp.zp = pz->lp;
  zp.twz = pz->tw;
  zp.seed = d.seed;
  zp.counters = job->counters;
  int nl = 0;
  if (job->eig_ok && zsplit_of(d.nzp) && tuned("pencil_kernel", skey, 2) == 2) {
    // eigen form: in-place z transforms, W x-bins per tile (schedule keys pencil_w,
    // pencil_threads); by default two CTAs per SM where the tile's shared memory allows
    int Wp = 1;
    while (Wp * 2 <= std::min(16, tuned("pencil_w", skey, 4))) Wp *= 2;
    // realisations per transform batch; 0: no realisation slots (the mean is stored first and
    // added back to each realisation), which lets wider tiles fit
    int SBp = tuned("pencil_sb", skey, 1);
    if (SBp != 0) SBp = std::max(1, std::min(std::max(d.nsim, 1), SBp));
    while (SBp > 1 && pencil_smem_bytes(Wp, d.nzp, d.ntheta, SBp) > 227 * 1024) SBp--;
    while (Wp > 1 && pencil_smem_bytes(Wp, d.nzp, d.ntheta, SBp) > 227 * 1024) Wp /= 2;
    if (pencil_smem_bytes(Wp, d.nzp, d.ntheta, SBp) > 227 * 1024)
      return fail(CRAVA_ENOTSUP, "pencil tile does not fit in shared memory");
    zp.SB = SBp;
    zp.dense = tuned("pencil_dense", skey, 0);
    zp.nb2 = tuned("pencil_nb", skey, 1) == 2;
    zp.eig = job->eig;
    zp.n_inv_rows = job->n_inv_rows;
    zp.zsplit = zsplit_of(d.nzp);
    zp.W = Wp;
    zp.logW = 0;
    while ((1 << zp.logW) < Wp) zp.logW++;
    zp.nIT = (job->cnxp + zp.W - 1) / zp.W;
    const int Tp = std::max(32, std::min(512, tuned("pencil_threads", skey,
                                                    pencil_smem_bytes(Wp, d.nzp, d.ntheta, SBp) <= 113 * 1024 ? 256
                                                                                                         : 512) /
                                                   32 * 32));
    ProfScope ps(ctx, KT_ZPASS, st);
    CUDA_TRY(launch_pencil(zp, Tp, st, &nl));
  } else {
    // the general kernel takes the eigen form of the per-bin step where its tables apply
    // (natural kz order at the lengths without the in-place split; schedule key zpass_eig)
    if (job->eig_ok && !zsplit_of(d.nzp) && tuned("zpass_eig", d.nzp, 1) != 0) {
      zp.eig = job->eig;
      zp.n_inv_rows = job->n_inv_rows;
    }
    ProfScope ps(ctx, KT_ZPASS, st);
    CUDA_TRY(launch_zpass(zp, T, st, &nl));
  }
  ctx->launches += nl;
  // inverse transforms (y, x) of the outputs with FFTGrid::invFFTInPlace scales
  {
    std::vector<float*> g;
    std::vector<float> sc;
    float ps = inv_scale(job->N, false), cs = inv_scale(job->N, true);
    if (!job->fac_on)
      for (int a = 0; a < 3; a++) { g.push_back(job->mean[a]); sc.push_back(ps); }
    if (!(d.flags & CRAVA_FLAG_SPECTRAL_COV))
      for (int q = 0; q < 6; q++) { g.push_back(job->cov[q]); sc.push_back(cs); }
    for (int q = 0; q < 3 * d.nsim; q++) { g.push_back(job->sim[q]); sc.push_back(ps); }
    if ((s = inv_xy(ctx, g, sc, d.nxp, d.nyp, d.nzp, false, st))) return s;
    if (job->fac_on && (s = inv_mean_facies(ctx, job, ps, st))) return s;
  }
  job->ran = true;
  job->resid_real = false;
  return CRAVA_OK;
}

crava_status crava_job_counters(crava_job* job, crava_counters* out) {
  if (!job || !out) return fail(CRAVA_EINVAL, "null argument");
  if (!job->ran) return fail(CRAVA_ESTATE, "counters are defined only after crava_job_run");
  CUDA_TRY(cudaSetDevice(job->ctx->device));
  unsigned long long c[kNumCounters];
  CUDA_TRY(cudaMemcpy(c, job->counters, sizeof(c), cudaMemcpyDeviceToHost));
  out->inverted_bins = (long long)c[0];
  out->chol_fallbacks = (long long)c[1];
  out->sim_chol_zero = (long long)c[2];
  out->fp64_bins = (long long)c[3];
  out->nonfinite_tiles = (long long)c[4];
  float v[6];
  for (int q = 0; q < 6; q++) CUDA_TRY(cudaMemcpy(&v[q], job->cov[q], sizeof(float), cudaMemcpyDeviceToHost));
  float P[9] = {v[0], v[3], v[4], v[3], v[1], v[5], v[4], v[5], v[2]};
  std::memcpy(out->post_var0, P, sizeof(P));
  if (c[4] > 0)
    return fail(CRAVA_ENUMERIC, "the data or prior-mean grids hold non-finite values (" + std::to_string(c[4]) +
                                    " pencil tiles of non-finite spectra)");
  return CRAVA_OK;
}

}  // extern "C"

namespace {

// Real symmetric n x n eigen-decomposition in double (herm_eig on a real matrix keeps its
// eigenvectors real), eigenvalues in descending order, each eigenvector's largest-magnitude
// component positive.
void sym_eig_sorted(int n, const double* a, double* w, double* v /* n x n, column i = vector i */) {
  cd A[kMaxTheta][kMaxTheta], U[kMaxTheta][kMaxTheta];
  double lam[kMaxTheta];
  for (int i = 0; i < n; i++)
    for (int k = 0; k < n; k++) A[i][k] = cd(0.5 * (a[i * n + k] + a[k * n + i]), 0);
  herm_eig(n, A, lam, U);
  std::vector<int> idx(n);
  for (int i = 0; i < n; i++) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return lam[x] > lam[y]; });
  for (int c = 0; c < n; c++) {
    const int src = idx[c];
    w[c] = lam[src];
    int big = 0;
    for (int r = 1; r < n; r++)
      if (std::fabs(U[r][src].real()) > std::fabs(U[big][src].real())) big = r;
    const double sg = U[big][src].real() < 0 ? -1.0 : 1.0;
    for (int r = 0; r < n; r++) v[r * n + c] = sg * U[r][src].real();
  }
}

// f(A) = V diag(f(w)) V^T of a real symmetric n x n matrix.
template <class F>
std::vector<double> sym_fun(int n, const double* a, F f) {
  std::vector<double> w(n), v((size_t)n * n), r((size_t)n * n, 0.0);
  sym_eig_sorted(n, a, w.data(), v.data());
  for (int i = 0; i < n; i++)
    for (int k = 0; k < n; k++)
      for (int c = 0; c < n; c++) r[i * n + k] += v[i * n + c] * f(w[c]) * v[k * n + c];
  return r;
}

}  // namespace

extern "C" {

crava_status crava_job_local_noise(crava_job* job, const float* scales, void* stream) {
  if (!job || !scales) return fail(CRAVA_EINVAL, "null argument");
  if (!job->ran) return fail(CRAVA_ESTATE, "crava_job_local_noise follows crava_job_run");
  const crava_job_desc& d = job->d;
  const int n = d.ntheta;
  const size_t nxy = (size_t)d.nx * d.ny;
  std::vector<double> inv_min(n);
  for (int l = 0; l < n; l++) {
    double mn = INFINITY;
    for (size_t q = 0; q < nxy; q++) {
      const float v = scales[(size_t)l * nxy + q];
      if (!(v > 0.f) || !std::isfinite(v)) return fail(CRAVA_EINVAL, "local noise scales must be finite and > 0");
      mn = std::min(mn, (double)v);
    }
    inv_min[l] = 1.0 / mn;
  }
  crava_ctx* ctx = job->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(cudaSetDevice(ctx->device));
  CUDA_TRY(cudaStreamSynchronize(st));
  crava_counters c;
  crava_status s = crava_job_counters(job, &c);
  if (s) return s;
  // job constants (AVOInversion::computeG, src/avoinversion.cpp:1943-2026, and the
  // trace-independent parts of newPosteriorCovPointwise / correctVpVsRho)
  double Sm[9], Smd[9], Sdel[9];
  for (int q = 0; q < 9; q++) {
    Sm[q] = job->pv[q];
    Smd[q] = c.post_var0[q];
    Sdel[q] = Sm[q] - Smd[q];
  }
  std::vector<double> SdelP = sym_fun(3, Sdel, [](double w) { return w > 0.0 ? w : 0.0; });
  std::vector<double> Sinv = sym_fun(3, Sm, [](double w) { return w > 1e-7 ? 1.0 / std::sqrt(w) : 0.0; });
  double Am[9] = {0};
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++)
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) Am[i * 3 + k] += Sinv[i * 3 + a] * SdelP[a * 3 + b] * Sinv[b * 3 + k];
  double ew[3], ev[9];
  sym_eig_sorted(3, Am, ew, ev);   // NRLib::Sort3x3: descending
  double lg[3] = {0, 0, 0};
  for (int i = 0; i < std::min(n, 3); i++)
    if (ew[i] > 0) lg[i] = std::sqrt(ew[i] / (1.0 - ew[i]));
  std::vector<double> Sth(job->etc.begin(), job->etc.end());
  std::vector<double> S12 = sym_fun(n, Sth.data(), [](double w) { return w > 0.0 ? std::sqrt(w) : 0.0; });
  // G = SigmaTheta^1/2 Lg Evec^T Sinv  (n x 3); Lg is n x 3 with Lg(i, i) = lg_i
  std::vector<double> G((size_t)n * 3, 0.0);
  for (int r = 0; r < n; r++)
    for (int k = 0; k < 3; k++) {
      double t = 0;
      for (int i = 0; i < std::min(n, 3); i++) {
        double et = 0;   // (Evec^T Sinv)_ik
        for (int a = 0; a < 3; a++) et += ev[a * 3 + i] * Sinv[a * 3 + k];
        t += S12[r * n + i] * lg[i] * et;
      }
      G[r * 3 + k] = t;
    }
  LocalNoiseParams P;
  std::memset(&P, 0, sizeof(P));
  P.nx = d.nx; P.ny = d.ny; P.nz = d.nz; P.nyp = d.nyp; P.rnxp = job->rnxp;
  P.nth = n; P.nsim = d.nsim;
  for (int l = 0; l < n; l++) P.inv_min[l] = inv_min[l];
  for (int r = 0; r < n; r++) {
    for (int k = 0; k < 3; k++) {
      double t = 0;
      for (int a = 0; a < 3; a++) t += G[r * 3 + a] * Sm[a * 3 + k];
      P.b[r][k] = t;
    }
    for (int m = 0; m < n; m++) P.sth[r][m] = Sth[r * n + m];
  }
  for (int r = 0; r < n; r++)
    for (int m = 0; m < n; m++) {
      double t = 0;
      for (int k = 0; k < 3; k++) t += P.b[r][k] * G[m * 3 + k];
      P.gsg[r][m] = t;
    }
  std::vector<double> sdel = sym_fun(3, Sdel, [](double w) { return w > 1e-7 ? 1.0 / std::sqrt(w) : 0.0; });
  std::vector<double> smdi = sym_fun(3, Smd, [](double w) { return w > 0.0 ? 1.0 / std::sqrt(w) : 0.0; });
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      P.sm[a][b] = Sm[a * 3 + b];
      P.sdel[a][b] = sdel[a * 3 + b];
      P.smdi[a][b] = smdi[a * 3 + b];
    }
  for (int a = 0; a < 3; a++) {
    P.prior_mean[a] = job->in_mean[a];
    P.post[a] = job->mean[a];
  }
  for (int q = 0; q < 3 * d.nsim; q++) P.sim[q] = job->sim[q];
  float* dscale = nullptr;
  CUDA_TRY(cudaMallocAsync((void**)&dscale, sizeof(float) * (n + 18) * nxy, st));
  P.scale = dscale;
  P.maps = dscale + n * nxy;
  cudaError_t e = cudaMemcpyAsync(dscale, scales, sizeof(float) * n * nxy, cudaMemcpyHostToDevice, st);
  int nl = 0;
  if (e == cudaSuccess) {
    ProfScope ps(ctx, KT_LOCAL_NOISE, st);
    e = launch_local_noise(P, st, &nl);
  }
  cudaFreeAsync(dscale, st);
  if (e != cudaSuccess) return cuda_fail(e, "local noise correction");
  CUDA_TRY(cudaStreamSynchronize(st));
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->launches += nl;
  return CRAVA_OK;
}

static crava_status fill_prior_impl(crava_job* job, const float* act_host, float corr_grad_i, float corr_grad_j,
                                    void* stream);

crava_status crava_job_fill_prior(crava_job* job, float corr_grad_i, float corr_grad_j, void* stream) {
  return fill_prior_impl(job, nullptr, corr_grad_i, corr_grad_j, stream);
}

crava_status crava_job_fill_prior_auto_cov(crava_job* job, const float* circ_auto_cov, float corr_grad_i,
                                           float corr_grad_j, void* stream) {
  if (!circ_auto_cov) return fail(CRAVA_EINVAL, "null auto-covariance");
  return fill_prior_impl(job, circ_auto_cov, corr_grad_i, corr_grad_j, stream);
}

static crava_status fill_prior_impl(crava_job* job, const float* act_host, float corr_grad_i, float corr_grad_j,
                                    void* stream) {
  if (!job) return fail(CRAVA_EINVAL, "null job");
  const crava_job_desc& d = job->d;
  if (d.prior_mode != CRAVA_PRIOR_GRIDS)
    return fail(CRAVA_ESTATE, "crava_job_fill_prior needs a CRAVA_PRIOR_GRIDS job");
  if (job->corr_xy.empty() || job->circ.empty())
    return fail(CRAVA_EINVAL, "crava_job_fill_prior needs corr_xy and circ_corr_t in the job description");
  if (!std::isfinite(corr_grad_i) || !std::isfinite(corr_grad_j))
    return fail(CRAVA_EINVAL, "correlation gradients must be finite");
  crava_ctx* ctx = job->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(cudaSetDevice(ctx->device));
  float* cxy = job->fill_xy;
  float* ct = job->fill_t;
  CUDA_TRY(cudaMemcpyAsync(cxy, job->corr_xy.data(), sizeof(float) * job->corr_xy.size(), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(ct, job->circ.data(), sizeof(float) * job->circ.size(), cudaMemcpyHostToDevice, st));
  PriorFill P;
  const int qa[6] = {0, 1, 2, 0, 0, 1}, qb[6] = {0, 1, 2, 1, 2, 2};
  for (int q = 0; q < 6; q++) {
    P.cov[q] = job->in_cov[q];
    P.pv[q] = static_cast<float>(job->pv[qa[q] * 3 + qb[q]]);
  }
  P.err = job->in_err;
  P.cxy = cxy;
  P.ct = ct;
  P.act = nullptr;
  float* dact = nullptr;
  if (act_host) {
    for (size_t q = 0; q < 6 * (size_t)d.nzp; q++)
      if (!std::isfinite(act_host[q])) return fail(CRAVA_ENUMERIC, "non-finite auto-covariance");
    CUDA_TRY(cudaMallocAsync((void**)&dact, sizeof(float) * 6 * d.nzp, st));
    CUDA_TRY(cudaMemcpyAsync(dact, act_host, sizeof(float) * 6 * d.nzp, cudaMemcpyHostToDevice, st));
    P.act = dact;
  }
  P.gi = corr_grad_i;
  P.gj = corr_grad_j;
  P.nxp = d.nxp;
  P.nyp = d.nyp;
  P.nzp = d.nzp;
  P.rnxp = job->rnxp;
  int nl = 0;
  cudaError_t fe;
  {
    ProfScope ps(ctx, KT_FILL_PRIOR, st);
    fe = launch_fill_prior(P, st, &nl);
  }
  if (dact) cudaFreeAsync(dact, st);
  if (fe != cudaSuccess) return cuda_fail(fe, "launch_fill_prior");
  // fillInParamCorr x priorVar0 (no estimated covariance): one correlation grid behind all six
  job->base_prior = !act_host && job->pv[0] > 0.0;
  // the host vectors stay with the job; wait so that the call has the reference's
  // synchronous semantics like the uploads it replaces
  CUDA_TRY(cudaStreamSynchronize(st));
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->launches += nl;
  return CRAVA_OK;
}

crava_status crava_job_divide_data(crava_job* job, void* stream) {
  if (!job) return fail(CRAVA_EINVAL, "null job");
  const crava_job_desc& d = job->d;
  if (!(d.flags & CRAVA_FLAG_NONCONST_THICK))
    return fail(CRAVA_ESTATE, "crava_job_divide_data needs a job with CRAVA_FLAG_NONCONST_THICK");
  crava_ctx* ctx = job->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(cudaSetDevice(ctx->device));
  Plan* pz;
  crava_status s;
  if ((s = get_plan(ctx, d.nzp, &pz, true))) return s;
  ThickParams& tp = job->tp;
  tp.zp = pz->lp;
  tp.twz = pz->tw;
  tp.mode = 0;
  tp.wshift = job->wgrid;
  tp.wgain = job->wgrid ? job->wgrid + (size_t)d.ntheta * d.nx * d.ny : nullptr;
  const int nth = d.ntheta;
  const size_t nxy = (size_t)d.nx * d.ny;
  int nl = 0;
  // divideDataByScaleWavelet, then the trace energies of interpolateSeismic
  {
    ProfScope ps(ctx, KT_THICK_DIVIDE, st);
    CUDA_TRY(launch_thick_divide(tp, nth, st, &nl));
  }
  {
    ProfScope ps(ctx, KT_THICK_FILL, st);
    CUDA_TRY(launch_trace_energy(tp, nth, job->energy, job->nzero, st, &nl));
  }
  // A zero threshold flags exactly the zero-energy traces: an angle without one needs no
  // plan (no interpolation; the box of good traces is the whole interior), and only the
  // other angles' energy maps come back to the host.
  std::vector<int> nzero(nth);
  CUDA_TRY(cudaMemcpyAsync(nzero.data(), job->nzero, sizeof(int) * nth, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  const bool zero_thr = d.energy_threshold == 0.f;
  std::vector<float> energy(nth * nxy);
  bool need = false;
  for (int l = 0; l < nth; l++) need |= !zero_thr || nzero[l] > 0;
  if (need) {
    CUDA_TRY(cudaMemcpyAsync(energy.data(), job->energy, sizeof(float) * energy.size(), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
  }
  // per angle: the interpolation plan (host), its levels in order, then the extrapolation
  std::vector<std::vector<TraceOp>> ops(nth);
  for (int l = 0; l < nth; l++) {
    std::vector<int> level_start;
    int box[4] = {0, d.nx - 1, 0, d.ny - 1};
    if (!zero_thr || nzero[l] > 0)
      plan_trace_interpolation(energy.data() + l * nxy, d.nx, d.ny, d.energy_threshold, ops[l], level_start, box);
    TraceOp* dops = job->ops + l * nxy;
    if (!ops[l].empty())
      CUDA_TRY(cudaMemcpyAsync(dops, ops[l].data(), sizeof(TraceOp) * ops[l].size(), cudaMemcpyHostToDevice, st));
    ProfScope ps(ctx, KT_THICK_FILL, st);
    for (size_t L = 1; L + 1 < level_start.size(); L++)
      CUDA_TRY(launch_trace_interp(tp.grid[l], job->rnxp, d.nyp, d.nzp, d.nx, dops + level_start[L],
                                   level_start[L + 1] - level_start[L], st, &nl));
    // no good trace at all: the reference would clamp into an empty box; nothing is copied
    if (box[0] <= box[1] && box[2] <= box[3]) CUDA_TRY(launch_extrapolate(tp, l, box, st, &nl));
  }
  CUDA_TRY(cudaStreamSynchronize(st));
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->launches += nl;
  }
  return CRAVA_OK;
}

crava_status crava_job_set_wavelet_grids(crava_job* job, int angle, const float* shift_ms, const float* gain) {
  if (!job) return fail(CRAVA_EINVAL, "null job");
  const crava_job_desc& d = job->d;
  if (angle < 0 || angle >= d.ntheta) return fail(CRAVA_EINVAL, "angle out of range");
  const size_t nxy = (size_t)d.nx * d.ny;
  // Wavelet1D::shiftAndScale takes iShift = shift / dz in float, dz the wavelet's sampling
  // (lz / nz); WELLMISSING (-999) entries are no shift and unit gain
  // (Wavelet::getLocalTimeshift / getLocalGainFactor, src/wavelet.cpp:1251-1278)
  const float dz = (float)(d.lz / d.nz);
  std::vector<float> sh(nxy, 0.f), gn(nxy, 1.f);
  for (size_t t = 0; t < nxy; t++) {
    if (shift_ms) {
      if (!std::isfinite(shift_ms[t])) return fail(CRAVA_EINVAL, "shift grid holds a non-finite value");
      if (shift_ms[t] != -999.0f) sh[t] = shift_ms[t] / dz;
    }
    if (gain) {
      if (!std::isfinite(gain[t])) return fail(CRAVA_EINVAL, "gain grid holds a non-finite value");
      if (gain[t] != -999.0f) gn[t] = gain[t];
    }
  }
  CUDA_TRY(cudaSetDevice(job->ctx->device));
  if (!job->wgrid) {
    CUDA_TRY(cudaMalloc(&job->wgrid, sizeof(float) * 2 * d.ntheta * nxy));
    std::vector<float> init(2 * d.ntheta * nxy, 0.f);
    std::fill(init.begin() + d.ntheta * nxy, init.end(), 1.f);
    CUDA_TRY(cudaMemcpy(job->wgrid, init.data(), sizeof(float) * init.size(), cudaMemcpyHostToDevice));
  }
  CUDA_TRY(cudaMemcpy(job->wgrid + angle * nxy, sh.data(), sizeof(float) * nxy, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(job->wgrid + (d.ntheta + angle) * nxy, gn.data(), sizeof(float) * nxy, cudaMemcpyHostToDevice));
  return CRAVA_OK;
}

namespace {

// The 3D wavelets' tables of a job into the parameters of the trace kernel.
void w3_into(const crava_job* job, ThickParams& tp) {
  if (!job->w3mem) return;
  tp.w3_mult = job->w3mult;
  tp.w3_par = job->w3par;
  tp.wglob = job->w3glob;
  tp.w3_den = job->w3den;
  for (int l = 0; l < job->d.ntheta; l++) tp.modW[l] = job->w3modW[l];
}

}  // namespace

crava_status crava_job_set_wavelet_3d(crava_job* job, const crava_wavelet3d_desc* w) {
  if (!job || !w) return fail(CRAVA_EINVAL, "null job or descriptor");
  const crava_job_desc& d = job->d;
  if (!w->theta || !w->alpha1 || !w->global_wavelet || !w->global_wavelet_norm)
    return fail(CRAVA_EINVAL, "theta, alpha1 and the global wavelets are required");
  if (w->filter_ni < 1 || w->filter_nj < 1) return fail(CRAVA_EINVAL, "filter surface needs ni, nj >= 1");
  if (!(w->filter_dx > 0.0) || !(w->filter_dy > 0.0) || !std::isfinite(w->filter_dx) || !std::isfinite(w->filter_dy) ||
      !std::isfinite(w->filter_x0) || !std::isfinite(w->filter_y0))
    return fail(CRAVA_EINVAL, "filter surface origin and spacing must be finite, spacing > 0");
  const int n = d.nzp, cn = n / 2 + 1, nth = d.ntheta;
  const size_t nxy = (size_t)d.nx * d.ny, nij = (size_t)w->filter_ni * w->filter_nj;
  for (int l = 0; l < nth; l++) {
    if (!std::isfinite(w->theta[l])) return fail(CRAVA_EINVAL, "theta holds a non-finite value");
    if (!(w->global_wavelet_norm[l] > 0.f) || !std::isfinite(w->global_wavelet_norm[l]))
      return fail(CRAVA_EINVAL, "global wavelet norms must be finite and > 0");
  }
  for (size_t t = 0; t < (size_t)nth * n; t++)
    if (!std::isfinite(w->global_wavelet[t])) return fail(CRAVA_EINVAL, "global wavelet holds a non-finite value");
  for (const float* g : {w->grad_x, w->grad_y})
    if (g)
      for (size_t t = 0; t < nxy; t++)
        if (!std::isfinite(g[t])) return fail(CRAVA_EINVAL, "gradient map holds a non-finite value");
  for (const float* g : {w->alpha1, w->halpha})
    if (g)
      for (size_t t = 0; t < (size_t)nth * nij; t++)
        if (!std::isfinite(g[t])) return fail(CRAVA_EINVAL, "filter surface holds a non-finite value");
  // the global wavelets: half spectra (wGlob) and modW (src/avoinversion.cpp:666-672 with
  // wGlobal = Wavelet3D::getGlobalWavelet)
  const float maxfreq = static_cast<float>((n / 2) * 1000.0 * d.nz) / static_cast<float>(d.lz * n);
  std::vector<float2> wg((size_t)nth * cn);
  for (int l = 0; l < nth; l++) {
    const float* wf = w->global_wavelet + (size_t)l * n;
    std::vector<cd> W = dft(std::vector<double>(wf, wf + n));
    for (int k = 0; k < cn; k++) wg[(size_t)l * cn + k] = make_float2((float)W[k].real(), (float)W[k].imag());
    float modW = w->global_wavelet_norm[l];
    modW *= modW;
    modW *= maxfreq / static_cast<float>(d.high_cut);
    job->w3modW[l] = modW;
  }
  CUDA_TRY(cudaSetDevice(job->ctx->device));
  const size_t o_par = align256(sizeof(double) * nth * nxy);
  const size_t o_glob = o_par + align256(sizeof(float4) * nth * nxy);
  if (!job->w3mem) {
    CUDA_TRY(cudaMalloc(&job->w3mem, o_glob + sizeof(float2) * nth * cn));
    job->w3mult = (double*)job->w3mem;
    job->w3par = (float4*)((char*)job->w3mem + o_par);
    job->w3glob = (float2*)((char*)job->w3mem + o_glob);
  }
  CUDA_TRY(cudaMemcpy(job->w3glob, wg.data(), sizeof(float2) * wg.size(), cudaMemcpyHostToDevice));
  // the 3D wavelets' own spectra and normalised errorSmooth3: the job's tables, or (constant
  // thickness: only the convolution of crava_job_residual_synthetics reads the adjustment)
  // the wavelet spectra alone
  Wavelet3DFill F{};
  if (d.flags & CRAVA_FLAG_NONCONST_THICK) {
    F.wamp = job->tp.wamp;
    F.es3 = job->tp.es3;
    for (int l = 0; l < nth; l++) F.es3_last[l] = job->tp.es3_last[l];
  } else {
    if (!job->wspec) {
      const std::vector<float2> ws = wavelet_spectra(d);
      CUDA_TRY(cudaMalloc(&job->wspec, sizeof(float2) * ws.size()));
      CUDA_TRY(cudaMemcpy(job->wspec, ws.data(), sizeof(float2) * ws.size(), cudaMemcpyHostToDevice));
    }
    F.wamp = job->wspec;
  }
  // Wavelet::findNormWithinFrequencyBand's band and adjustForAmplitudeEffect's
  // double(nzp * dz * 1e-3), dz the wavelet's sampling lz / nz in float
  const float dz = (float)(d.lz / d.nz);
  const float dOmega = static_cast<float>(1.0 / (n * dz * 0.001));
  F.loI = std::max(0, (int)std::floor(d.low_cut / dOmega));
  F.hiI = std::min(cn, (int)std::ceil(d.high_cut / dOmega));
  job->w3den = static_cast<double>(static_cast<float>(n) * dz) * 1e-3;
  F.den = job->w3den;
  F.nx = d.nx; F.ny = d.ny; F.nzp = n; F.cnzp = cn;
  F.ni = w->filter_ni; F.nj = w->filter_nj;
  F.x0 = w->filter_x0; F.y0 = w->filter_y0; F.dx = w->filter_dx; F.dy = w->filter_dy;
  for (int l = 0; l < nth; l++) F.theta[l] = w->theta[l];
  F.mult = job->w3mult;
  F.par = job->w3par;
  // the maps and surfaces, staged in one temporary allocation
  const size_t o_gy = align256(sizeof(float) * nxy), o_a = 2 * o_gy, o_h = o_a + align256(sizeof(float) * nth * nij);
  void* tmp = nullptr;
  CUDA_TRY(cudaMalloc(&tmp, o_h + sizeof(float) * nth * nij));
  char* tb = (char*)tmp;
  cudaError_t e = cudaSuccess;
  if (w->grad_x && e == cudaSuccess) e = cudaMemcpy(tb, w->grad_x, sizeof(float) * nxy, cudaMemcpyHostToDevice);
  if (w->grad_y && e == cudaSuccess) e = cudaMemcpy(tb + o_gy, w->grad_y, sizeof(float) * nxy, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(tb + o_a, w->alpha1, sizeof(float) * nth * nij, cudaMemcpyHostToDevice);
  if (w->halpha && e == cudaSuccess) e = cudaMemcpy(tb + o_h, w->halpha, sizeof(float) * nth * nij, cudaMemcpyHostToDevice);
  F.gx = w->grad_x ? (const float*)tb : nullptr;
  F.gy = w->grad_y ? (const float*)(tb + o_gy) : nullptr;
  F.alpha1 = (const float*)(tb + o_a);
  F.halpha = w->halpha ? (const float*)(tb + o_h) : nullptr;
  int nl = 0;
  if (e == cudaSuccess) e = launch_wavelet3d_fill(F, nth, 0, &nl);
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  cudaFree(tmp);
  CUDA_TRY(e);
  if (d.flags & CRAVA_FLAG_NONCONST_THICK) w3_into(job, job->tp);
  {
    std::lock_guard<std::mutex> lk(job->ctx->mu);
    job->ctx->launches += nl;
  }
  return CRAVA_OK;
}

crava_status crava_job_residual_synthetics(crava_job* job, void* stream) {
  if (!job) return fail(CRAVA_EINVAL, "null job");
  const crava_job_desc& d = job->d;
  if (!(d.flags & CRAVA_FLAG_KEEP_RESIDUAL))
    return fail(CRAVA_ESTATE, "crava_job_residual_synthetics needs a job with CRAVA_FLAG_KEEP_RESIDUAL");
  if (!job->ran) return fail(CRAVA_ESTATE, "the residuals are defined only after crava_job_run");
  if (job->resid_real) return fail(CRAVA_ESTATE, "the residuals of this run are already convolved");
  crava_ctx* ctx = job->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(cudaSetDevice(ctx->device));
  Plan* pz;
  crava_status s;
  if ((s = get_plan(ctx, d.nzp, &pz, true))) return s;
  if (thick_tile_width(d.nzp) < 1) return fail(CRAVA_ENOTSUP, "nzp too long for the trace transform");
  const int nth = d.ntheta, cn = d.nzp / 2 + 1;
  ThickParams tp{};
  if (d.flags & CRAVA_FLAG_NONCONST_THICK) {
    tp = job->tp;
  } else {
    if (!job->wspec) {
      const std::vector<float2> w = wavelet_spectra(d);
      CUDA_TRY(cudaMalloc(&job->wspec, sizeof(float2) * w.size()));
      CUDA_TRY(cudaMemcpy(job->wspec, w.data(), sizeof(float2) * w.size(), cudaMemcpyHostToDevice));
    }
    tp.wamp = job->wspec;
    tp.nx = d.nx; tp.ny = d.ny; tp.nz = d.nz;
    tp.nxp = d.nxp; tp.nyp = d.nyp; tp.nzp = d.nzp;
    tp.rnxp = job->rnxp;
    tp.cnzp = cn;
    tp.W = thick_tile_width(d.nzp);
    tp.logW = 0;
    while ((1 << tp.logW) < tp.W) tp.logW++;
    tp.rsq = static_cast<float>(std::sqrt(static_cast<float>(d.nzp)));
    int e = 0;
    tp.inv_rsq = std::frexp(tp.rsq, &e) == 0.5f ? 1.0f / tp.rsq : 0.f;
    tp.lz = d.lz;
    w3_into(job, tp);
  }
  tp.mode = 1;
  tp.nIT = ((d.nx + 1) / 2 + tp.W - 1) / tp.W;
  tp.rsq_out = static_cast<float>(std::sqrt(static_cast<double>(d.nzp)));
  tp.zp = pz->lp;
  tp.twz = pz->tw;
  tp.wshift = job->wgrid;
  tp.wgain = job->wgrid ? job->wgrid + (size_t)nth * d.nx * d.ny : nullptr;
  for (int l = 0; l < nth; l++) tp.grid[l] = job->data[l];
  // FFTGrid::invFFTInPlace of the residual spectra (src/avoinversion.cpp:744), then the
  // per-trace convolution
  std::vector<float*> g(job->data, job->data + nth);
  std::vector<float> sc(nth, inv_scale(job->N, false));
  if ((s = inv_xy(ctx, g, sc, d.nxp, d.nyp, d.nzp, true, st))) return s;
  int nl = 0;
  {
    ProfScope ps(ctx, KT_THICK_DIVIDE, st);
    CUDA_TRY(launch_thick_divide(tp, nth, st, &nl));
  }
  job->resid_real = true;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->launches += nl;
  return CRAVA_OK;
}

crava_status crava_fft_r2c(crava_ctx* ctx, float* dgrid, int nxp, int nyp, int nzp, int covariance, void* stream) {
  if (!ctx || !dgrid) return fail(CRAVA_EINVAL, "null argument");
  if (!smooth(nxp) || !smooth(nyp) || !smooth(nzp) || nxp < 2 || nyp < 2 || nzp < 2)
    return fail(CRAVA_ENOTSUP, "dimensions must be 2,3,5,7-smooth and >= 2");
  CUDA_TRY(cudaSetDevice(ctx->device));
  size_t N = (size_t)nxp * nyp * nzp;
  std::vector<const float*> src{dgrid};
  std::vector<float*> g{dgrid};
  std::vector<float> sc{covariance ? 1.0f : fwd_scale(N)};
  return fwd_xy(ctx, src, g, sc, nxp, nyp, nzp, true, (cudaStream_t)stream);
}

// Host-resident grid: copied to the context's staging grid, transformed, copied back.
static crava_status fft_host(crava_ctx* ctx, float* hgrid, int nxp, int nyp, int nzp, int covariance, bool fwd) {
  if (!ctx || !hgrid) return fail(CRAVA_EINVAL, "null argument");
  if (!smooth(nxp) || !smooth(nyp) || !smooth(nzp) || nxp < 2 || nyp < 2 || nzp < 2)
    return fail(CRAVA_ENOTSUP, "dimensions must be 2,3,5,7-smooth and >= 2");
  CUDA_TRY(cudaSetDevice(ctx->device));
  const size_t bytes = sizeof(float) * 2 * (size_t)(nxp / 2 + 1) * nyp * nzp;
  std::lock_guard<std::mutex> lk(ctx->stage_mu);
  if (ctx->stage_bytes < bytes) {
    if (ctx->stage) CUDA_TRY(cudaFree(ctx->stage));
    ctx->stage = nullptr;
    ctx->stage_bytes = 0;
    CUDA_TRY(cudaMalloc(&ctx->stage, bytes));
    ctx->stage_bytes = bytes;
  }
  CUDA_TRY(cudaMemcpy(ctx->stage, hgrid, bytes, cudaMemcpyHostToDevice));
  crava_status s = fwd ? crava_fft_r2c(ctx, ctx->stage, nxp, nyp, nzp, covariance, nullptr)
                       : crava_fft_c2r(ctx, ctx->stage, nxp, nyp, nzp, covariance, nullptr);
  if (s) return s;
  CUDA_TRY(cudaMemcpy(hgrid, ctx->stage, bytes, cudaMemcpyDeviceToHost));
  return CRAVA_OK;
}

crava_status crava_fft_r2c_host(crava_ctx* ctx, float* hgrid, int nxp, int nyp, int nzp, int covariance) {
  return fft_host(ctx, hgrid, nxp, nyp, nzp, covariance, true);
}

crava_status crava_fft_c2r_host(crava_ctx* ctx, float* hgrid, int nxp, int nyp, int nzp, int covariance) {
  return fft_host(ctx, hgrid, nxp, nyp, nzp, covariance, false);
}

crava_status crava_fft_c2r(crava_ctx* ctx, float* dgrid, int nxp, int nyp, int nzp, int covariance, void* stream) {
  if (!ctx || !dgrid) return fail(CRAVA_EINVAL, "null argument");
  if (!smooth(nxp) || !smooth(nyp) || !smooth(nzp) || nxp < 2 || nyp < 2 || nzp < 2)
    return fail(CRAVA_ENOTSUP, "dimensions must be 2,3,5,7-smooth and >= 2");
  CUDA_TRY(cudaSetDevice(ctx->device));
  size_t N = (size_t)nxp * nyp * nzp;
  std::vector<float*> g{dgrid};
  std::vector<float> sc{inv_scale(N, covariance != 0)};
  return inv_xy(ctx, g, sc, nxp, nyp, nzp, true, (cudaStream_t)stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Inversion without device allocation (crava_invert_noalloc).
//
// Some callers cannot call cudaMalloc: plugins hosted by an application that owns the
// device memory pool and forbids other allocators, or hot loops where an allocation's
// implicit device synchronisation is not acceptable.  For them this entry point runs one small block with
// every intermediate in g_noalloc_scratch, a fixed array in the library's own device image:
// each GPU that loads the library holds its CRAVA_NOALLOC_SCRATCH_BYTES until the process
// exits, every call reuses it (so calls whose work overlaps on the GPU race), and blocks
// whose intermediates do not fit are rejected with CRAVA_ENOTSUP.

static __device__ __align__(256) unsigned char g_noalloc_scratch[CRAVA_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[64] = {};

// Device address of the scratch array on the current device, looked up once per device:
// in host code g_noalloc_scratch names a host-side stand-in, not device memory.
crava_status noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= 64) return fail(CRAVA_ENOTSUP, "device index above 63");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_noalloc_ptr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_noalloc_ptr[device];
  return CRAVA_OK;
}

// Host copy of one transform plan: stage radices and the twiddle table.
struct HostPlan {
  LinePlan lp;
  std::vector<float2> tw;
};

bool host_plan(int n, bool allow16, HostPlan& hp) {
  if (!make_plan(n, hp.lp, allow16)) return false;
  hp.tw.resize(n);
  for (int t = 0; t < n; t++) {
    double ang = 2.0 * M_PI * (double)t / (double)n;
    hp.tw[t] = make_float2((float)std::cos(ang), (float)(-std::sin(ang)));
  }
  return true;
}

}  // namespace

extern "C" crava_status crava_invert_noalloc(const crava_job_desc* desc, const float* const* d_in,
                                             float* const* d_out, void* stream) {
  crava_status s = validate(desc);
  if (s) return s;
  if (!d_in || !d_out) return fail(CRAVA_EINVAL, "null grid pointer array");
  const crava_job_desc& d = *desc;
  if (d.prior_mode != CRAVA_PRIOR_SEPARABLE)
    return fail(CRAVA_ENOTSUP, "crava_invert_noalloc takes the separable prior only");
  if (d.fp64_threshold > 0.f) return fail(CRAVA_ENOTSUP, "crava_invert_noalloc runs FP32 only");
  if (d.flags & (CRAVA_FLAG_HOST_NOISE | CRAVA_FLAG_KEEP_RESIDUAL | CRAVA_FLAG_SPECTRAL_COV |
                 CRAVA_FLAG_NONCONST_THICK))
    return fail(CRAVA_ENOTSUP,
                "crava_invert_noalloc supports neither host noise, residual or spectral output nor non-constant "
                "thickness");
  const int nin = d.ntheta + 3, nout = 9 + 3 * d.nsim;
  for (int q = 0; q < nin; q++)
    if (!d_in[q]) return fail(CRAVA_EINVAL, "null input grid");
  for (int q = 0; q < nout; q++)
    if (!d_out[q]) return fail(CRAVA_EINVAL, "null output grid");
  cudaStream_t st = (cudaStream_t)stream;
  int device = 0;
  CUDA_TRY(cudaGetDevice(&device));

  const int cnxp = d.nxp / 2 + 1, rnxp = 2 * cnxp;
  const size_t rsize = (size_t)rnxp * d.nyp * d.nzp;
  const size_t N = (size_t)d.nxp * d.nyp * d.nzp;
  const bool even = d.nxp % 2 == 0;
  HostPlan px, pn, py, pz;
  if (!host_plan(even ? d.nxp / 2 : d.nxp, false, px) || !host_plan(d.nxp, false, pn) ||
      !host_plan(d.nyp, false, py) || !host_plan(d.nzp, true, pz))
    return fail(CRAVA_ENOTSUP, "transform length is not 2,3,5,7-smooth");

  // scratch layout: data work grids, twiddle tables, per-kz tables, lateral and temporal
  // prior factors, counters
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += align256(bytes); return o; };
  const size_t o_data = take(sizeof(float) * rsize * d.ntheta);
  const size_t o_twx = take(sizeof(float2) * px.tw.size());
  const size_t o_twn = take(sizeof(float2) * pn.tw.size());
  const size_t o_twy = take(sizeof(float2) * py.tw.size());
  const size_t o_twz = take(sizeof(float2) * pz.tw.size());
  const size_t o_kw = take(sizeof(float2) * d.nzp * d.ntheta);
  const size_t o_e1 = take(sizeof(float2) * d.nzp * d.ntheta);
  const size_t o_e2 = take(sizeof(float2) * d.nzp * d.ntheta);
  const size_t o_inv = take(d.nzp);
  const size_t o_ed = take(sizeof(float) * d.nzp * d.ntheta);
  const size_t o_cxy = take(sizeof(float) * rnxp * d.nyp);
  const size_t o_ct = take(sizeof(float2) * d.nzp);
  const size_t o_cnt = take(kNumCounters * sizeof(unsigned long long));
  if (off > (size_t)CRAVA_NOALLOC_SCRATCH_BYTES)
    return fail(CRAVA_ENOTSUP, "block needs " + std::to_string(off) + " bytes of scratch; crava_invert_noalloc has " +
                                   std::to_string((size_t)CRAVA_NOALLOC_SCRATCH_BYTES));
  unsigned char* base = nullptr;
  if ((s = noalloc_scratch(device, &base))) return s;

  // host-built tables, copied into the scratch on the stream
  std::vector<float2> kw, e1, e2;
  std::vector<uint8_t> inv;
  std::vector<float> edk;
  build_kz_tables(d, kw, e1, e2, inv, nullptr, nullptr, nullptr, edk, nullptr);
  std::vector<double> c(d.circ_corr_t, d.circ_corr_t + d.nzp);
  std::vector<cd> C = dft(c);
  std::vector<float2> ct(d.nzp);
  for (int k = 0; k < d.nzp; k++) ct[k] = make_float2((float)C[k].real(), (float)C[k].imag());
  std::vector<float> gxy((size_t)rnxp * d.nyp, 0.f);
  for (int jj = 0; jj < d.nyp; jj++)
    for (int ii = 0; ii < d.nxp; ii++) gxy[(size_t)jj * rnxp + ii] = d.corr_xy[(size_t)jj * d.nxp + ii];
  auto put = [&](size_t o, const void* src, size_t bytes) {
    return cudaMemcpyAsync(base + o, src, bytes, cudaMemcpyHostToDevice, st);
  };
  CUDA_TRY(put(o_twx, px.tw.data(), sizeof(float2) * px.tw.size()));
  CUDA_TRY(put(o_twn, pn.tw.data(), sizeof(float2) * pn.tw.size()));
  CUDA_TRY(put(o_twy, py.tw.data(), sizeof(float2) * py.tw.size()));
  CUDA_TRY(put(o_twz, pz.tw.data(), sizeof(float2) * pz.tw.size()));
  CUDA_TRY(put(o_kw, kw.data(), sizeof(float2) * kw.size()));
  CUDA_TRY(put(o_e1, e1.data(), sizeof(float2) * e1.size()));
  CUDA_TRY(put(o_e2, e2.data(), sizeof(float2) * e2.size()));
  CUDA_TRY(put(o_inv, inv.data(), inv.size()));
  CUDA_TRY(put(o_ed, edk.data(), sizeof(float) * edk.size()));
  CUDA_TRY(put(o_ct, ct.data(), sizeof(float2) * ct.size()));
  CUDA_TRY(put(o_cxy, gxy.data(), sizeof(float) * gxy.size()));
  CUDA_TRY(cudaMemsetAsync(base + o_cnt, 0, kNumCounters * sizeof(unsigned long long), st));
  const float2* twx = (const float2*)(base + o_twx);
  const float2* twn = (const float2*)(base + o_twn);
  const float2* twy = (const float2*)(base + o_twy);
  const float2* twz = (const float2*)(base + o_twz);
  float* data = (float*)(base + o_data);

  // lateral prior factor: 2D transform of corrXY in place
  {
    GridSet gs;
    gs.n = 1;
    gs.p[0] = (float*)(base + o_cxy);
    gs.src[0] = gs.p[0];
    gs.scale[0] = 1.0f;
    CUDA_TRY(launch_x_r2c(gs, d.nxp, d.nyp, px.lp, twx, twn, st, nullptr));
    CUDA_TRY(launch_line_fft(gs, cnxp, d.nyp, (size_t)cnxp, 1, 0, py.lp, twy, -1.f, st, nullptr));
  }
  // forward x, y transforms: data into scratch, prior mean into the posterior-mean outputs
  {
    GridSet gs;
    gs.n = nin;
    const float fs = fwd_scale(N);
    for (int l = 0; l < d.ntheta; l++) { gs.src[l] = d_in[l]; gs.p[l] = data + rsize * l; gs.scale[l] = fs; }
    for (int a = 0; a < 3; a++) { gs.src[d.ntheta + a] = d_in[d.ntheta + a]; gs.p[d.ntheta + a] = d_out[a]; gs.scale[d.ntheta + a] = fs; }
    CUDA_TRY(launch_x_r2c(gs, d.nxp, d.nyp * d.nzp, px.lp, twx, twn, st, nullptr));
    CUDA_TRY(launch_line_fft(gs, cnxp, d.nyp, (size_t)cnxp, d.nzp, (size_t)cnxp * d.nyp, py.lp, twy, -1.f, st, nullptr));
  }
  // pencil pass
  ZParams zp;
  std::memset(&zp, 0, sizeof(zp));
  zp.nxp = d.nxp; zp.nyp = d.nyp; zp.nzp = d.nzp; zp.cnxp = cnxp;
  zp.nxp_even = even;
  int W = 4, T = 256;
  if (zpass_smem_bytes(W, d.nzp, d.ntheta) > 113 * 1024) T = 512;
  while (W > 1 && zpass_smem_bytes(W, d.nzp, d.ntheta) > 227 * 1024) W /= 2;
  if (zpass_smem_bytes(W, d.nzp, d.ntheta) > 227 * 1024) return fail(CRAVA_ENOTSUP, "pencil tile does not fit in shared memory");
  zp.W = W;
  zp.logW = 0;
  while ((1 << zp.logW) < W) zp.logW++;
  zp.nIT = (cnxp + W - 1) / W;
  zp.nth = d.ntheta;
  zp.nsim = d.nsim;
  zp.separable = 1;
  for (int l = 0; l < d.ntheta; l++) zp.data[l] = (float2*)(data + rsize * l);
  for (int a = 0; a < 3; a++) zp.mean[a] = (float2*)d_out[a];
  for (int q = 0; q < 6; q++) zp.cov[q] = (float2*)d_out[3 + q];
  for (int q = 0; q < 3 * d.nsim; q++) zp.sim[q] = (float2*)d_out[9 + q];
  zp.cxy = (const float2*)(base + o_cxy);
  zp.ct = (const float2*)(base + o_ct);
  const int qa[6] = {0, 1, 2, 0, 0, 1}, qb[6] = {0, 1, 2, 1, 2, 2};
  for (int q = 0; q < 6; q++) zp.pv[q] = static_cast<float>(d.prior_var0[qa[q] * 3 + qb[q]]);
  for (int l = 0; l < d.ntheta; l++) {
    for (int c3 = 0; c3 < 3; c3++) zp.A[l][c3] = static_cast<float>(d.A[l * 3 + c3]);
    for (int m = 0; m < d.ntheta; m++) zp.ec[l][m] = float(0.5 * (1.0 - d.wnc) * d.err_theta_cov[l * d.ntheta + m]);
    zp.ed[l] = float(d.wnc * d.err_theta_cov[l * d.ntheta + l]);
  }
  zp.kz.kw = (const float2*)(base + o_kw);
  zp.kz.e1 = (const float2*)(base + o_e1);
  zp.kz.e2 = (const float2*)(base + o_e2);
  zp.kz.inv = (const uint8_t*)(base + o_inv);
  zp.kz.ed = (const float*)(base + o_ed);
  zp.zp = pz.lp;
  zp.twz = twz;
  zp.seed = d.seed;
  zp.counters = (unsigned long long*)(base + o_cnt);
  CUDA_TRY(launch_zpass(zp, T, st, nullptr));
  // inverse y, x transforms of the outputs in place
  {
    GridSet gs;
    gs.n = nout;
    const float ps = inv_scale(N, false), cs = inv_scale(N, true);
    for (int q = 0; q < nout; q++) {
      gs.p[q] = d_out[q];
      gs.src[q] = d_out[q];
      gs.scale[q] = (q >= 3 && q < 9) ? cs : ps;
    }
    CUDA_TRY(launch_line_fft(gs, cnxp, d.nyp, (size_t)cnxp, d.nzp, (size_t)cnxp * d.nyp, py.lp, twy, 1.f, st, nullptr));
    CUDA_TRY(launch_x_c2r(gs, d.nxp, d.nyp * d.nzp, px.lp, twx, twn, st, nullptr));
  }
  return CRAVA_OK;
}

// ---------------------------------------------------------------------------------------
// Batches: many blocks of uneven size and angle count captured into one CUDA graph whose
// branches run concurrently (no reference counterpart: the reference inverts one interval
// at a time, main.cpp:217-353).

#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>

struct crava_batch {
  crava_ctx* ctx = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long kernels = 0;  // kernel launches per replay
};

namespace {

// Plans a job's run needs, created before a capture (plan creation allocates).
crava_status prewarm_plans(crava_ctx* ctx, const crava_job_desc& d) {
  Plan *a, *b;
  crava_status s;
  if ((s = get_xplans(ctx, d.nxp, &a, &b))) return s;
  if ((s = get_plan(ctx, d.nyp, &a))) return s;
  if ((s = get_plan(ctx, d.nzp, &a))) return s;
  return get_plan(ctx, d.nzp, &a, tuned("zpass_r16", d.nzp, 1) != 0);
}

}  // namespace

extern "C" {

crava_status crava_batch_create(crava_ctx* ctx, crava_job* const* jobs, int n, int branches, crava_batch** out) {
  if (!ctx || !jobs || !out || n < 1) return fail(CRAVA_EINVAL, "bad batch arguments");
  if (branches < 1) branches = 1;
  if (branches > n) branches = n;
  CUDA_TRY(cudaSetDevice(ctx->device));
  for (int i = 0; i < n; i++) {
    if (!jobs[i] || jobs[i]->ctx != ctx) return fail(CRAVA_EINVAL, "job of another context");
    crava_status s = prewarm_plans(ctx, jobs[i]->d);
    if (s) return s;
  }
  const bool prof = ctx->profiling;
  ctx->profiling = false;
  std::vector<cudaStream_t> br(branches);
  cudaStream_t cap;
  CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  for (auto& b : br) CUDA_TRY(cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking));
  cudaEvent_t fork;
  std::vector<cudaEvent_t> join(branches);
  CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  for (auto& e : join) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  long long l0 = ctx->launches;
  crava_status st = CRAVA_OK;
  cudaGraph_t graph = nullptr;
  cudaError_t ce = cudaStreamBeginCapture(cap, cudaStreamCaptureModeRelaxed);
  if (ce == cudaSuccess) {
    cudaEventRecord(fork, cap);
    for (int b = 0; b < branches; b++) cudaStreamWaitEvent(br[b], fork, 0);
    for (int i = 0; i < n && !st; i++) st = crava_job_run(jobs[i], br[i % branches]);
    for (int b = 0; b < branches; b++) {
      cudaEventRecord(join[b], br[b]);
      cudaStreamWaitEvent(cap, join[b], 0);
    }
    ce = cudaStreamEndCapture(cap, &graph);
  }
  ctx->profiling = prof;
  crava_batch* bt = nullptr;
  if (!st && ce == cudaSuccess) {
    bt = new crava_batch();
    bt->ctx = ctx;
    bt->graph = graph;
    bt->kernels = ctx->launches - l0;
    ce = cudaGraphInstantiate(&bt->exec, graph, 0);
  }
  ctx->launches = l0;  // the capture launched nothing
  cudaEventDestroy(fork);
  for (auto& e : join) cudaEventDestroy(e);
  for (auto& b : br) cudaStreamDestroy(b);
  cudaStreamDestroy(cap);
  if (st) {
    if (graph) cudaGraphDestroy(graph);
    delete bt;
    return st;
  }
  if (ce != cudaSuccess) {
    if (bt) {
      if (bt->graph) cudaGraphDestroy(bt->graph);
      delete bt;
    }
    return cuda_fail(ce, "batch graph capture");
  }
  *out = bt;
  return CRAVA_OK;
}

crava_status crava_batch_run(crava_batch* b, void* stream) {
  if (!b) return fail(CRAVA_EINVAL, "null batch");
  CUDA_TRY(cudaSetDevice(b->ctx->device));
  CUDA_TRY(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  b->ctx->launches += b->kernels;
  return CRAVA_OK;
}

crava_status crava_batch_destroy(crava_batch* b) {
  if (!b) return CRAVA_OK;
  cudaSetDevice(b->ctx->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  delete b;
  return CRAVA_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Serving: a native request loop that admits jobs by their HBM footprint against the
// context's budget and an in-flight limit, runs each admitted job on its own stream
// (host->device inputs, the whole inversion, device->host outputs) so that jobs that
// arrive while others run overlap on the device, and releases each job's memory
// (stream-ordered) when its completion event fires.

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct ServeReq {
  uint64_t id = 0;
  crava_job_desc d{};
  std::vector<double> A, etc, pv;
  std::vector<float> wav, wn, cxy, circ;
  std::vector<const float*> in;
  std::vector<float*> out;
  double t_submit = 0, t_start = 0, t_done = 0;
  int state = CRAVA_REQ_QUEUED;
  crava_status status = CRAVA_OK;
  std::string err;
  crava_job* job = nullptr;
  int slot = -1;
  cudaEvent_t done = nullptr;
  unsigned long long* nonfinite = nullptr;  // pinned host word the job's counter is copied to
};

}  // namespace

struct crava_server {
  crava_ctx* ctx = nullptr;
  int max_inflight = 1;
  std::vector<cudaStream_t> streams;
  std::vector<char> busy;
  std::thread th;
  std::mutex mu;
  std::condition_variable cv;
  bool stopping = false;
  uint64_t next_id = 1;
  std::deque<ServeReq*> pending;
  int max_queued = 0;                 // 0: no limit
  std::vector<ServeReq*> inflight;
  std::map<uint64_t, ServeReq*> reqs;
  long long completed = 0;
  unsigned long long* nf = nullptr;   // pinned, one word per stream: the job's non-finite counter
};

namespace {

// Starts request r on stream slot `slot`: job creation (tables from the resident cache),
// uploads, the inversion, downloads and the completion event.  Runs on the loop thread
// without the server lock; touches only r's job fields, which no other thread reads.
// CRAVA_ENOMEM: the job does not fit now, nothing was allocated.
crava_status serve_admit(crava_server* sv, ServeReq* r, int slot) {
  cudaStream_t st = sv->streams[slot];
  crava_job* job = nullptr;
  crava_status s = job_create_impl(sv->ctx, &r->d, st, true, &job);
  if (s) {
    if (s != CRAVA_ENOMEM) r->err = crava_last_error();
    return s;
  }
  // the job holds its own copies of the description's arrays now
  r->A = {}; r->etc = {}; r->pv = {}; r->wav = {}; r->wn = {}; r->cxy = {}; r->circ = {};
  r->job = job;
  r->slot = slot;
  const int nth = r->d.ntheta;
  for (int l = 0; l < nth && !s; l++) s = crava_job_upload(job, CRAVA_ROLE_DATA, l, r->in[l], st);
  for (int a = 0; a < 3 && !s; a++) s = crava_job_upload(job, CRAVA_ROLE_MEAN, a, r->in[nth + a], st);
  if (!s) s = crava_job_run(job, st);
  if (!s) {
    sv->nf[slot] = 0;
    r->nonfinite = sv->nf + slot;
    if (cudaMemcpyAsync(r->nonfinite, job->counters + 4, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st) !=
        cudaSuccess)
      s = CRAVA_ECUDA;
  }
  for (size_t q = 0; q < r->out.size() && !s; q++) {
    if (!r->out[q]) continue;
    if (q < 3) s = crava_job_download(job, CRAVA_ROLE_POST_MEAN, (int)q, r->out[q], st);
    else if (q < 9) s = crava_job_download(job, CRAVA_ROLE_POST_COV, (int)q - 3, r->out[q], st);
    else s = crava_job_download(job, CRAVA_ROLE_SIM, (int)q - 9, r->out[q], st);
  }
  if (!s && cudaEventCreateWithFlags(&r->done, cudaEventDisableTiming) != cudaSuccess) s = CRAVA_ECUDA;
  if (!s && cudaEventRecord(r->done, st) != cudaSuccess) s = CRAVA_ECUDA;
  if (s) {
    r->err = crava_last_error();
    cudaStreamSynchronize(st);
    if (r->done) cudaEventDestroy(r->done);
    r->done = nullptr;
    job_release(job);
    r->job = nullptr;
    if (s == CRAVA_ENOMEM) s = CRAVA_ECUDA;   // a failure after admission is not a retry
  }
  return s;
}

void serve_loop(crava_server* sv) {
  cudaSetDevice(sv->ctx->device);
  std::unique_lock<std::mutex> lk(sv->mu);
  for (;;) {
    bool progressed = false;
    // completions
    for (size_t i = 0; i < sv->inflight.size();) {
      ServeReq* r = sv->inflight[i];
      cudaError_t q = cudaEventQuery(r->done);
      if (q == cudaErrorNotReady) { i++; continue; }
      r->t_done = now_ms();
      cudaEventDestroy(r->done);
      r->done = nullptr;
      job_release(r->job);
      r->job = nullptr;
      // a job whose data or prior-mean grids were not finite fails with CRAVA_ENUMERIC
      if (q == cudaSuccess) {
        r->state = CRAVA_REQ_DONE;
        if (r->nonfinite && *r->nonfinite) {
          r->state = CRAVA_REQ_FAILED;
          r->status = CRAVA_ENUMERIC;
          r->err = "the data or prior-mean grids hold non-finite values";
        }
      } else {
        r->status = CRAVA_ECUDA;
        r->err = cudaGetErrorString(q);
        r->state = CRAVA_REQ_FAILED;
      }
      sv->busy[r->slot] = 0;
      sv->inflight.erase(sv->inflight.begin() + i);
      sv->completed++;
      progressed = true;
    }
    // admissions, first come first served; the set-up runs without the lock
    while (!sv->pending.empty() && (int)sv->inflight.size() < sv->max_inflight && !sv->stopping) {
      int slot = -1;
      for (int k = 0; k < (int)sv->busy.size(); k++)
        if (!sv->busy[k]) { slot = k; break; }
      if (slot < 0) break;
      ServeReq* r = sv->pending.front();
      sv->pending.pop_front();
      sv->busy[slot] = 1;
      const bool idle = sv->inflight.empty();
      lk.unlock();
      crava_status s = serve_admit(sv, r, slot);
      lk.lock();
      progressed = true;
      if (s == CRAVA_ENOMEM && !idle) {
        // waits at the head of the queue for memory that running jobs will release
        sv->busy[slot] = 0;
        sv->pending.push_front(r);
        break;
      }
      if (s) {
        // out of memory with nothing in flight can never succeed: fail it, keep serving
        sv->busy[slot] = 0;
        r->state = CRAVA_REQ_FAILED;
        r->status = s;
        if (s == CRAVA_ENOMEM) r->err = "job does not fit the device memory even with nothing else in flight";
        r->t_start = r->t_done = now_ms();
        continue;
      }
      r->t_start = now_ms();
      r->state = CRAVA_REQ_RUNNING;
      sv->inflight.push_back(r);
    }
    if (sv->stopping) {
      for (ServeReq* r : sv->pending) {
        r->state = CRAVA_REQ_FAILED;
        r->status = CRAVA_ESTATE;
        r->err = "server stopped before the request started";
      }
      sv->pending.clear();
      if (sv->inflight.empty()) break;
    }
    if (progressed) sv->cv.notify_all();
    sv->cv.wait_for(lk, std::chrono::microseconds(progressed ? 0 : 100));
  }
  sv->cv.notify_all();
}

// Fills info from r (caller holds the lock); a request in a final state is released.
void serve_report(crava_server* sv, ServeReq* r, crava_request_info* info) {
  if (info) {
    info->state = r->state;
    info->status = r->status;
    info->queue_ms = (r->t_start > 0 ? r->t_start : now_ms()) - r->t_submit;
    info->latency_ms = r->t_done > 0 ? r->t_done - r->t_submit : -1.0;
  }
  if (r->state == CRAVA_REQ_DONE || r->state == CRAVA_REQ_FAILED) {
    sv->reqs.erase(r->id);
    delete r;
  }
}

}  // namespace

extern "C" {

crava_status crava_serve_start(crava_ctx* ctx, int max_inflight, crava_server** out) {
  if (!ctx || !out) return fail(CRAVA_EINVAL, "null argument");
  if (max_inflight < 1 || max_inflight > 256) return fail(CRAVA_EINVAL, "max_inflight must be 1..256");
  CUDA_TRY(cudaSetDevice(ctx->device));
  // keep freed job memory in the stream-ordered pool instead of returning it to the driver
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  {
    // served jobs keep their tables resident: on by default for a serving context
    std::lock_guard<std::mutex> lk(ctx->cache_mu);
    if (ctx->cache_max == 0) ctx->cache_max = (size_t)256 << 20;
  }
  crava_server* sv = new crava_server();
  sv->ctx = ctx;
  sv->max_inflight = max_inflight;
  if (cudaHostAlloc((void**)&sv->nf, sizeof(unsigned long long) * max_inflight, cudaHostAllocDefault) != cudaSuccess) {
    delete sv;
    return fail(CRAVA_ENOMEM, "pinned host words of the server");
  }
  sv->streams.resize(max_inflight);
  sv->busy.assign(max_inflight, 0);
  for (auto& s : sv->streams) {
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
  }
  sv->th = std::thread(serve_loop, sv);
  *out = sv;
  return CRAVA_OK;
}

crava_status crava_serve_submit(crava_server* sv, const crava_job_desc* desc, const float* const* host_in,
                                float* const* host_out, uint64_t* ticket) {
  if (!sv || !desc || !host_in || !ticket) return fail(CRAVA_EINVAL, "null argument");
  crava_status s = validate(desc);
  if (s) return s;
  if (desc->prior_mode != CRAVA_PRIOR_SEPARABLE || (desc->flags & (CRAVA_FLAG_HOST_NOISE | CRAVA_FLAG_NONCONST_THICK)))
    return fail(CRAVA_ENOTSUP, "served jobs take the separable prior, device noise and constant thickness");
  if (sv->ctx->budget > 0 && footprint(desc) > sv->ctx->budget)
    return fail(CRAVA_ENOMEM, "job footprint " + std::to_string(footprint(desc)) + " bytes exceeds the context budget " +
                                  std::to_string(sv->ctx->budget));
  ServeReq* r = new ServeReq();
  r->d = *desc;
  const int nth = desc->ntheta;
  r->A.assign(desc->A, desc->A + 3 * nth);
  r->etc.assign(desc->err_theta_cov, desc->err_theta_cov + nth * nth);
  r->pv.assign(desc->prior_var0, desc->prior_var0 + 9);
  r->wav.assign(desc->wavelet, desc->wavelet + (size_t)nth * desc->nzp);
  r->wn.assign(desc->wavelet_norm, desc->wavelet_norm + nth);
  r->cxy.assign(desc->corr_xy, desc->corr_xy + (size_t)desc->nxp * desc->nyp);
  r->circ.assign(desc->circ_corr_t, desc->circ_corr_t + desc->nzp);
  r->d.A = r->A.data();
  r->d.err_theta_cov = r->etc.data();
  r->d.prior_var0 = r->pv.data();
  r->d.wavelet = r->wav.data();
  r->d.wavelet_norm = r->wn.data();
  r->d.corr_xy = r->cxy.data();
  r->d.circ_corr_t = r->circ.data();
  r->d.flags &= ~CRAVA_FLAG_KEEP_RESIDUAL;
  r->in.assign(host_in, host_in + nth + 3);
  const int nout = 9 + 3 * desc->nsim;
  if (host_out) r->out.assign(host_out, host_out + nout);
  else r->out.assign(nout, nullptr);
  std::lock_guard<std::mutex> lk(sv->mu);
  if (sv->stopping) {
    delete r;
    return fail(CRAVA_ESTATE, "server is stopping");
  }
  if (sv->max_queued > 0 && (int)sv->pending.size() >= sv->max_queued) {
    delete r;
    return fail(CRAVA_EBUSY, "server queue holds " + std::to_string(sv->max_queued) + " requests");
  }
  r->id = sv->next_id++;
  r->t_submit = now_ms();
  sv->reqs[r->id] = r;
  sv->pending.push_back(r);
  *ticket = r->id;
  sv->cv.notify_all();
  return CRAVA_OK;
}

crava_status crava_ctx_fail_next_allocs(crava_ctx* ctx, int n) {
  if (!ctx || n < 0) return fail(CRAVA_EINVAL, "bad argument");
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->fail_allocs = n;
  return CRAVA_OK;
}

crava_status crava_serve_set_queue_limit(crava_server* sv, int max_queued) {
  if (!sv || max_queued < 0) return fail(CRAVA_EINVAL, "bad argument");
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->max_queued = max_queued;
  return CRAVA_OK;
}

crava_status crava_serve_cancel(crava_server* sv, uint64_t ticket) {
  if (!sv) return fail(CRAVA_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) return fail(CRAVA_EINVAL, "unknown ticket (or its final state was already reported)");
  ServeReq* r = it->second;
  auto q = std::find(sv->pending.begin(), sv->pending.end(), r);
  if (r->state != CRAVA_REQ_QUEUED || q == sv->pending.end())
    return fail(CRAVA_ESTATE, "the request is no longer queued");
  sv->pending.erase(q);
  r->state = CRAVA_REQ_FAILED;
  r->status = CRAVA_ECANCELED;
  r->err = "request cancelled";
  r->t_done = now_ms();
  sv->cv.notify_all();
  return CRAVA_OK;
}

crava_status crava_serve_poll(crava_server* sv, uint64_t ticket, crava_request_info* info) {
  if (!sv || !info) return fail(CRAVA_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) return fail(CRAVA_EINVAL, "unknown ticket (or its final state was already reported)");
  serve_report(sv, it->second, info);
  return CRAVA_OK;
}

crava_status crava_serve_wait(crava_server* sv, uint64_t ticket, double timeout_ms, crava_request_info* info) {
  if (!sv) return fail(CRAVA_EINVAL, "null server");
  const double t_end = now_ms() + timeout_ms;
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) return fail(CRAVA_EINVAL, "unknown ticket (or its final state was already reported)");
  ServeReq* r = it->second;
  while (r->state == CRAVA_REQ_QUEUED || r->state == CRAVA_REQ_RUNNING) {
    double left = t_end - now_ms();
    if (left <= 0) return fail(CRAVA_ETIMEDOUT, "request not finished within the timeout");
    sv->cv.wait_for(lk, std::chrono::microseconds((long long)std::min(left * 1000.0, 10000.0)));
  }
  const crava_status st = r->state == CRAVA_REQ_FAILED ? (r->status ? r->status : CRAVA_ECUDA) : CRAVA_OK;
  const std::string err = r->err;
  serve_report(sv, r, info);
  if (st) return fail(st, err);
  return CRAVA_OK;
}

crava_status crava_serve_stop(crava_server* sv) {
  if (!sv) return CRAVA_OK;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stopping = true;
    sv->cv.notify_all();
  }
  if (sv->th.joinable()) sv->th.join();
  cudaSetDevice(sv->ctx->device);
  for (auto& s : sv->streams) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  for (auto& kv : sv->reqs) delete kv.second;
  if (sv->nf) cudaFreeHost(sv->nf);
  delete sv;
  return CRAVA_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Facies probabilities (FaciesProb::makeFaciesDens smoothing and calculateFaciesProb).

extern "C" {

crava_status crava_facies_smooth(crava_ctx* ctx, const crava_facies_desc* fd, const double* sigma_inv, float* d_hist,
                                 void* stream) {
  if (!ctx || !fd || !sigma_inv || !d_hist) return fail(CRAVA_EINVAL, "null argument");
  const int na = fd->nbins[0], nb = fd->nbins[1], nr = fd->nbins[2];
  if (fd->nfacies < 1 || fd->nfacies > kMaxFacies) return fail(CRAVA_EINVAL, "nfacies must be 1..16");
  if (!smooth(na) || !smooth(nb) || !smooth(nr) || na < 2 || nb < 1 || nr < 2)
    return fail(CRAVA_ENOTSUP, "density bins must be 2,3,5,7-smooth");
  if (nb < 2) return fail(CRAVA_ENOTSUP, "a single Vs bin is not supported by the smoothing transform");
  CUDA_TRY(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int rna = 2 * (na / 2 + 1);
  const size_t gsize = (size_t)rna * nb * nr;
  // Gaussian smoother with cyclic bin offsets, exp in float, normalised to unit sum
  // (src/faciesprob.cpp:447-496)
  std::vector<float> sm((size_t)na * nb * nr);
  float sum = 0.0f;
  const double dv0 = fd->dv[0], dv1 = fd->dv[1], dv2 = fd->dv[2];
  const double* S = sigma_inv;
  for (int l = 0; l < nr; l++) {
    int ll = l <= nr / 2 ? l : l - nr;
    for (int k = 0; k < nb; k++) {
      int kk = k <= nb / 2 ? k : k - nb;
      for (int j = 0; j < na; j++) {
        int jj = j <= na / 2 ? j : j - na;
        float factor = static_cast<float>(jj * dv0 * jj * dv0 * S[0] + kk * dv1 * kk * dv1 * S[4] +
                                          ll * dv2 * ll * dv2 * S[8] + 2 * jj * dv0 * kk * dv1 * S[3] +
                                          2 * jj * dv0 * ll * dv2 * S[6] + 2 * kk * dv1 * ll * dv2 * S[7]);
        float v = std::exp(-0.5f * factor);
        sm[j + (size_t)k * na + (size_t)l * na * nb] = v;
        sum += v;
      }
    }
  }
  std::vector<float> g(gsize, 0.f);
  for (int l = 0; l < nr; l++)
    for (int k = 0; k < nb; k++)
      for (int j = 0; j < na; j++) g[j + (size_t)rna * (k + (size_t)nb * l)] = sm[j + (size_t)k * na + (size_t)l * na * nb] / sum;
  float* d_sm = nullptr;
  CUDA_TRY(cudaMalloc(&d_sm, sizeof(float) * gsize));
  crava_status s = CRAVA_OK;
  cudaError_t e = cudaMemcpyAsync(d_sm, g.data(), sizeof(float) * gsize, cudaMemcpyHostToDevice, st);
  // PARAMETER-scaled transforms: smoothed = IFFT(FFT(h)/sqrt(N) * FFT(s)/sqrt(N))/sqrt(N) * sqrt(N)
  const size_t N = (size_t)na * nb * nr;
  const float fs = fwd_scale(N);
  std::vector<const float*> src;
  std::vector<float*> gr;
  std::vector<float> sc;
  src.push_back(d_sm);
  gr.push_back(d_sm);
  sc.push_back(fs);
  for (int f = 0; f < fd->nfacies; f++) {
    src.push_back(d_hist + gsize * f);
    gr.push_back(d_hist + gsize * f);
    sc.push_back(fs);
  }
  if (e == cudaSuccess) s = fwd_xy(ctx, src, gr, sc, na, nb, nr, true, st);
  else s = cuda_fail(e, "cudaMemcpyAsync");
  const size_t nbins = (size_t)(na / 2 + 1) * nb * nr;
  for (int f = 0; f < fd->nfacies && !s; f++) {
    e = launch_spec_mul((float2*)(d_hist + gsize * f), (const float2*)d_sm, nbins, st);
    if (e != cudaSuccess) s = cuda_fail(e, "spectrum product");
  }
  if (!s) {
    std::vector<float*> out(gr.begin() + 1, gr.end());
    const float is = inv_scale(N, false) * std::sqrt(static_cast<float>(N));
    std::vector<float> osc(out.size(), is);
    s = inv_xy(ctx, out, osc, na, nb, nr, true, st);
  }
  cudaStreamSynchronize(st);
  cudaFree(d_sm);
  return s;
}

}  // extern "C"

namespace {

// Checks of a facies description (corner boxes, volumes, probability grids) and the relative
// noise scale of every trace per angle (calculateFaciesProb, src/faciesprob.cpp:1961-1977):
// fills hc (without t and the packed volumes) and t (nang x ny x nx).
crava_status facies_setup(const crava_facies_desc* corners, int nang, const float* const* d_density, int density_row,
                          const float* noise_scale, int nx, int ny, float* const* d_prob, FaciesCornersHost& hc,
                          std::vector<float>& t) {
  if (nang < 0 || nang > kMaxFaciesAngles) return fail(CRAVA_ENOTSUP, "local-noise angles must be 0..4");
  const crava_facies_desc* fd = corners;
  if (fd->nfacies < 1 || fd->nfacies > kMaxFacies) return fail(CRAVA_EINVAL, "nfacies must be 1..16");
  if (!fd->prior) return fail(CRAVA_EINVAL, "null facies prior");
  for (int f = 0; f <= fd->nfacies; f++)
    if (!d_prob[f]) return fail(CRAVA_EINVAL, "null probability grid");
  const int nc = 1 << nang;
  hc = FaciesCornersHost{};
  hc.nang = nang;
  for (int c = 0; c < nc; c++) {
    for (int d = 0; d < 3; d++) {
      if (corners[c].nbins[d] < 1 || !(corners[c].dv[d] > 0)) return fail(CRAVA_EINVAL, "bad density box");
      hc.box[c].nb[d] = corners[c].nbins[d];
      hc.box[c].vmin[d] = corners[c].vmin[d];
      hc.box[c].dv[d] = corners[c].dv[d];
    }
    if (density_row < corners[c].nbins[0]) return fail(CRAVA_EINVAL, "density row stride below the vp bin count");
    if (!d_density[c]) return fail(CRAVA_EINVAL, "null density volume");
    hc.box[c].rs = density_row;
    hc.box[c].fstride = (size_t)density_row * corners[c].nbins[1] * corners[c].nbins[2];
    hc.dens[c] = d_density[c];
  }
  const size_t nxy = (size_t)nx * ny;
  t.assign((size_t)nang * nxy, 0.f);
  for (int a = 0; a < nang; a++) {
    double mn = INFINITY, mx = -INFINITY;
    for (size_t q = 0; q < nxy; q++) {
      const double v = noise_scale[(size_t)a * nxy + q];
      if (!std::isfinite(v)) return fail(CRAVA_ENUMERIC, "non-finite noise scale");
      mn = std::min(mn, v);
      mx = std::max(mx, v);
    }
    for (size_t q = 0; q < nxy; q++)
      t[(size_t)a * nxy + q] = mn == mx ? 0.f : (float)(((double)noise_scale[(size_t)a * nxy + q] - mn) / (mx - mn));
  }
  return CRAVA_OK;
}

}  // namespace

extern "C" {

crava_status crava_facies_prob_local_noise(crava_ctx* ctx, const crava_facies_desc* corners, int nang,
                                           const float* const* d_density, int density_row, const float* noise_scale,
                                           const float* const* d_post, int nx, int ny, int nz, int nxp, int nyp,
                                           float* const* d_prob, float* d_seis_lh, void* stream) {
  if (!ctx || !corners || !d_density || !d_post || !d_prob || (nang > 0 && !noise_scale))
    return fail(CRAVA_EINVAL, "null argument");
  if (nx < 1 || ny < 1 || nz < 1 || nxp < nx || nyp < ny) return fail(CRAVA_EINVAL, "bad grid dimensions");
  const crava_facies_desc* fd = corners;
  FaciesCornersHost hc;
  std::vector<float> t;
  if (crava_status s = facies_setup(corners, nang, d_density, density_row, noise_scale, nx, ny, d_prob, hc, t)) return s;
  const int nc = 1 << nang;
  CUDA_TRY(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  float* dt = nullptr;
  if (nang > 0) {
    CUDA_TRY(cudaMallocAsync((void**)&dt, sizeof(float) * t.size(), st));
    CUDA_TRY(cudaMemcpyAsync(dt, t.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice, st));
  }
  hc.t = dt;
  // facies-interleaved copies of the volumes for the lookups
  size_t pbytes = 0;
  for (int c = 0; c < nc; c++) pbytes += align256(facies_packed_bytes(hc.box[c], fd->nfacies));
  char* pk = nullptr;
  CUDA_TRY(cudaMallocAsync((void**)&pk, pbytes, st));
  for (int c = 0, off = 0; c < nc; c++) {
    hc.packed[c] = (float4*)(pk + off);
    off += (int)align256(facies_packed_bytes(hc.box[c], fd->nfacies));
  }
  // undefSum = p_undefined / (bins of the first density volume), as the reference
  const float undef_sum = fd->p_undefined / (float)(fd->nbins[0] * fd->nbins[1] * fd->nbins[2]);
  const int rnxp_in = 2 * (nxp / 2 + 1), rnxp_out = 2 * (nx / 2 + 1);
  cudaError_t e;
  {
    ProfScope ps(ctx, KT_FACIES, st);
    e = launch_facies_prob_corners(d_post[0], d_post[1], d_post[2], nx, ny, nz, rnxp_in, nyp, rnxp_out, hc,
                                   fd->nfacies, fd->prior, undef_sum, d_prob, d_seis_lh, st);
  }
  cudaFreeAsync(pk, st);
  if (dt) cudaFreeAsync(dt, st);
  if (e != cudaSuccess) return cuda_fail(e, "launch_facies_prob_corners");
  if (nang > 0) CUDA_TRY(cudaStreamSynchronize(st));   // the host t table
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->launches += 1 + nc;   // the packing of every volume and the lookups
  return CRAVA_OK;
}

crava_status crava_facies_prob(crava_ctx* ctx, const crava_facies_desc* fd, const float* d_density, int density_row,
                               const float* const* d_post, int nx, int ny, int nz, int nxp, int nyp,
                               float* const* d_prob, float* d_seis_lh, void* stream) {
  // the single-volume case of the local-noise form (no noise angles, one corner)
  return crava_facies_prob_local_noise(ctx, fd, 0, &d_density, density_row, nullptr, d_post, nx, ny, nz, nxp, nyp,
                                       d_prob, d_seis_lh, stream);
}

crava_status crava_job_set_facies(crava_job* job, const crava_facies_desc* corners, int nang,
                                  const float* const* d_density, int density_row, const float* noise_scale,
                                  float* const* d_prob, float* d_seis_lh) {
  if (!job) return fail(CRAVA_EINVAL, "null job");
  CUDA_TRY(cudaSetDevice(job->ctx->device));
  if (job->fac_mem) {
    CUDA_TRY(cudaDeviceSynchronize());   // a run still reading the packed volumes
    cudaFree(job->fac_mem);
    job->fac_mem = nullptr;
  }
  job->fac_on = false;
  if (!corners) return CRAVA_OK;   // cleared
  if (!d_density || !d_prob || (nang > 0 && !noise_scale)) return fail(CRAVA_EINVAL, "null argument");
  const crava_job_desc& d = job->d;
  FaciesCornersHost hc;
  std::vector<float> t;
  if (crava_status s = facies_setup(corners, nang, d_density, density_row, noise_scale, d.nx, d.ny, d_prob, hc, t))
    return s;
  const int nc = 1 << nang, nf = corners->nfacies;
  size_t bytes = align256(sizeof(float) * t.size());
  for (int c = 0; c < nc; c++) bytes += align256(facies_packed_bytes(hc.box[c], nf));
  CUDA_TRY(cudaMalloc((void**)&job->fac_mem, bytes));
  char* p = job->fac_mem;
  float* dt = (float*)p;
  p += align256(sizeof(float) * t.size());
  for (int c = 0; c < nc; c++) {
    hc.packed[c] = (float4*)p;
    p += align256(facies_packed_bytes(hc.box[c], nf));
  }
  if (!t.empty()) CUDA_TRY(cudaMemcpy(dt, t.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice));
  hc.t = nang > 0 ? dt : nullptr;
  CUDA_TRY(launch_facies_pack(hc, nf, nullptr));
  CUDA_TRY(cudaStreamSynchronize(nullptr));
  job->fac_hc = hc;
  job->fac_nf = nf;
  for (int f = 0; f < nf; f++) job->fac_prior[f] = corners->prior[f];
  // undefSum = p_undefined / (bins of the first density volume), as the reference
  job->fac_undef = corners->p_undefined / (float)(corners->nbins[0] * corners->nbins[1] * corners->nbins[2]);
  for (int f = 0; f <= nf; f++) job->fac_prob[f] = d_prob[f];
  job->fac_lh = d_seis_lh;
  job->fac_on = true;
  {
    std::lock_guard<std::mutex> lk(job->ctx->mu);
    job->ctx->launches += nc;
  }
  return CRAVA_OK;
}

}  // extern "C"
