"""Python binding of the C ABI in include/crava_gpu.h (ctypes; no torch types cross it).

The classes mirror the reference's objects on the hot path:

* ``Context``   -- one device (the process-wide FFTGrid/FFTW state of the reference)
* ``Job``       -- one AVOInversion on one block (src/avoinversion.cpp:53-111): upload the
                   inputs, ``run()`` = constructor transforms + computePostMeanResidAndFFTCov +
                   simulate + invFFTCovGrids, then download the outputs
* ``fft_r2c`` / ``fft_c2r`` -- FFTGrid::fftInPlace / invFFTInPlace on a device grid

The library is required: importing works without it, but every call raises
``CravaError`` when ``libcrava_gpu.so`` is missing, so no path silently falls back to the CPU.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcrava_gpu.so")

OK, EINVAL, ENOMEM, ECUDA, ETIMEDOUT, ENUMERIC, ENOTSUP, ESTATE, EBUSY, ECANCELED = range(10)
ROLE_DATA, ROLE_MEAN, ROLE_PRIOR_COV, ROLE_ERR_CORR, ROLE_POST_COV, ROLE_SIM, ROLE_NOISE, \
    ROLE_RESIDUAL, ROLE_POST_MEAN = range(9)
PRIOR_SEPARABLE, PRIOR_GRIDS = 0, 1
FLAG_HOST_NOISE, FLAG_KEEP_RESIDUAL, FLAG_SPECTRAL_COV, FLAG_NONCONST_THICK = 1, 2, 4, 8

# exported symbols the header declares (checked by the CPU tests)
EXPORTS = ["crava_ctx_create", "crava_ctx_destroy", "crava_last_error", "crava_status_string",
           "crava_job_create", "crava_job_destroy", "crava_job_footprint", "crava_job_upload",
           "crava_job_download", "crava_job_device_ptr", "crava_job_run", "crava_job_counters",
           "crava_fft_r2c", "crava_fft_c2r", "crava_ctx_kernel_launches", "crava_ctx_set_profiling",
           "crava_ctx_kernel_times", "crava_job_divide_data", "crava_job_fill_prior"]
KERNEL_CLASSES = ["x_r2c", "line_fwd", "zpass", "line_inv", "x_c2r", "xy_fwd", "xy_inv", "thick_divide",
                  "thick_fill", "local_noise", "facies", "fill_prior"]
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = range(4)


class CravaError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"crava status {status}: {msg}")
        self.status = status


_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)


class JobDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("nxp", ctypes.c_int), ("nyp", ctypes.c_int), ("nzp", ctypes.c_int),
                ("ntheta", ctypes.c_int), ("lz", ctypes.c_double), ("min_rel_thick", ctypes.c_double),
                ("low_cut", ctypes.c_float), ("high_cut", ctypes.c_float), ("wnc", ctypes.c_float),
                ("A", _dp), ("err_theta_cov", _dp), ("wavelet", _fp), ("wavelet_norm", _fp),
                ("prior_var0", _dp), ("prior_mode", ctypes.c_int), ("corr_xy", _fp),
                ("circ_corr_t", _fp), ("nsim", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("flags", ctypes.c_int), ("fp64_threshold", ctypes.c_float),
                ("rel_thick", _dp), ("energy_threshold", ctypes.c_float)]


class Counters(ctypes.Structure):
    _fields_ = [("inverted_bins", ctypes.c_longlong), ("chol_fallbacks", ctypes.c_longlong),
                ("sim_chol_zero", ctypes.c_longlong), ("fp64_bins", ctypes.c_longlong),
                ("post_var0", ctypes.c_float * 9), ("nonfinite_tiles", ctypes.c_longlong)]


class SimboxGeom(ctypes.Structure):
    _fields_ = [("x0", ctypes.c_double), ("y0", ctypes.c_double), ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("il0", ctypes.c_double), ("xl0", ctypes.c_double),
                ("il_step_x", ctypes.c_double), ("il_step_y", ctypes.c_double), ("xl_step_x", ctypes.c_double),
                ("xl_step_y", ctypes.c_double), ("angle", ctypes.c_double)]


class StormGeom(ctypes.Structure):
    _fields_ = [("xmin", ctypes.c_double), ("lx", ctypes.c_double), ("ymin", ctypes.c_double), ("ly", ctypes.c_double),
                ("lz", ctypes.c_double), ("angle", ctypes.c_double), ("cubetype", ctypes.c_int), ("flat", ctypes.c_int),
                ("top_name", ctypes.c_char_p), ("bot_name", ctypes.c_char_p)]


class SegyDesc(ctypes.Structure):
    _fields_ = [("x0", ctypes.c_double), ("y0", ctypes.c_double), ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("angle", ctypes.c_double), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dz", ctypes.c_double), ("top", _dp), ("top_z", ctypes.c_double), ("rel_thick", _dp),
                ("zmin", ctypes.c_double), ("zmax", ctypes.c_double), ("il0", ctypes.c_double),
                ("xl0", ctypes.c_double), ("il_step_x", ctypes.c_double), ("il_step_y", ctypes.c_double),
                ("xl_step_x", ctypes.c_double), ("xl_step_y", ctypes.c_double), ("z0", ctypes.c_float),
                ("header_format", ctypes.c_int), ("text", ctypes.POINTER(ctypes.c_char_p)), ("ntext", ctypes.c_int)]


class Wavelet3DDesc(ctypes.Structure):
    _fields_ = [("grad_x", _fp), ("grad_y", _fp), ("theta", _fp), ("filter_ni", ctypes.c_int),
                ("filter_nj", ctypes.c_int), ("filter_x0", ctypes.c_double), ("filter_y0", ctypes.c_double),
                ("filter_dx", ctypes.c_double), ("filter_dy", ctypes.c_double), ("alpha1", _fp),
                ("halpha", _fp), ("global_wavelet", _fp), ("global_wavelet_norm", _fp)]


def wavelet3d_desc(theta, alpha1, global_wavelet, global_wavelet_norm, filter_geom, grad_x=None, grad_y=None,
                   halpha=None):
    """A crava_wavelet3d_desc: theta (ntheta radians), alpha1 / halpha (ntheta, nj, ni) filter
    surfaces with filter_geom = (x0, y0, dx, dy) in degrees, the global wavelets (ntheta, nzp)
    and their norms, optional (ny, nx) depth gradient maps; returns (desc, keep-alive arrays)."""
    keep = []

    def arr(a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float32)
        keep.append(a)
        return a.ctypes.data_as(_fp)

    al = np.asarray(alpha1)
    d = Wavelet3DDesc()
    d.grad_x, d.grad_y = arr(grad_x), arr(grad_y)
    d.theta = arr(np.asarray(theta, dtype=np.float32).reshape(-1))
    d.filter_nj, d.filter_ni = int(al.shape[-2]), int(al.shape[-1])
    d.filter_x0, d.filter_y0, d.filter_dx, d.filter_dy = (float(v) for v in filter_geom)
    d.alpha1, d.halpha = arr(alpha1), arr(halpha)
    d.global_wavelet, d.global_wavelet_norm = arr(global_wavelet), arr(np.asarray(global_wavelet_norm).reshape(-1))
    return d, keep


def segy_desc(geom: dict, top=None, rel_thick=None, text=None):
    """A crava_segy_desc from geom (the scalar fields) and optional per-trace top / relative
    thickness arrays (ny, nx) and textual-header lines; returns (desc, keep-alive objects)."""
    d = SegyDesc(**{k: v for k, v in geom.items()})
    keep = []
    if top is not None:
        t = np.ascontiguousarray(top, dtype=np.float64)
        keep.append(t)
        d.top = t.ctypes.data_as(_dp)
    if rel_thick is not None:
        r = np.ascontiguousarray(rel_thick, dtype=np.float64)
        keep.append(r)
        d.rel_thick = r.ctypes.data_as(_dp)
    if text is not None:
        arr = (ctypes.c_char_p * len(text))(*[str(x).encode() for x in text])
        keep.append(arr)
        d.text = ctypes.cast(arr, ctypes.POINTER(ctypes.c_char_p))
        d.ntext = len(text)
    return d, keep


class FaciesDesc(ctypes.Structure):
    _fields_ = [("nfacies", ctypes.c_int), ("nbins", ctypes.c_int * 3), ("vmin", ctypes.c_double * 3),
                ("dv", ctypes.c_double * 3), ("prior", _fp), ("p_undefined", ctypes.c_float)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("status", ctypes.c_int), ("queue_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double)]


_lib = None


def lib() -> ctypes.CDLL:
    """Load the CUDA library; raises CravaError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CravaError(ENOTSUP, f"{LIB_PATH} is missing: build it with `python -m crava_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    L.crava_ctx_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_size_t]
    L.crava_ctx_destroy.argtypes = [vp]
    L.crava_last_error.restype = ctypes.c_char_p
    L.crava_status_string.restype = ctypes.c_char_p
    L.crava_status_string.argtypes = [ctypes.c_int]
    L.crava_job_create.argtypes = [vp, ctypes.POINTER(JobDesc), ctypes.POINTER(vp)]
    L.crava_job_destroy.argtypes = [vp]
    L.crava_job_footprint.argtypes = [ctypes.POINTER(JobDesc), ctypes.POINTER(ctypes.c_size_t)]
    L.crava_job_upload.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp]
    L.crava_job_download.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp]
    L.crava_job_device_ptr.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.crava_job_run.argtypes = [vp, vp]
    L.crava_job_divide_data.argtypes = [vp, vp]
    L.crava_job_fill_prior.argtypes = [vp, ctypes.c_float, ctypes.c_float, vp]
    L.crava_job_counters.argtypes = [vp, ctypes.POINTER(Counters)]
    L.crava_fft_r2c.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]
    L.crava_fft_c2r.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]
    L.crava_ctx_kernel_launches.argtypes = [vp]
    L.crava_ctx_kernel_launches.restype = ctypes.c_longlong
    L.crava_ctx_set_profiling.argtypes = [vp, ctypes.c_int]
    L.crava_ctx_kernel_times.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.c_int, ctypes.c_int]
    L.crava_batch_create.argtypes = [vp, ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.crava_batch_run.argtypes = [vp, vp]
    L.crava_batch_destroy.argtypes = [vp]
    L.crava_serve_start.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp)]
    L.crava_serve_submit.argtypes = [vp, ctypes.POINTER(JobDesc), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                     ctypes.POINTER(ctypes.c_uint64)]
    L.crava_serve_poll.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(RequestInfo)]
    L.crava_serve_wait.argtypes = [vp, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(RequestInfo)]
    L.crava_serve_stop.argtypes = [vp]
    L.crava_serve_set_queue_limit.argtypes = [vp, ctypes.c_int]
    L.crava_serve_cancel.argtypes = [vp, ctypes.c_uint64]
    L.crava_ctx_fail_next_allocs.argtypes = [vp, ctypes.c_int]
    L.crava_invert_noalloc.argtypes = [ctypes.POINTER(JobDesc), ctypes.POINTER(vp), ctypes.POINTER(vp), vp]
    L.crava_facies_smooth.argtypes = [vp, ctypes.POINTER(FaciesDesc), ctypes.POINTER(ctypes.c_double), vp, vp]
    L.crava_facies_prob.argtypes = [vp, ctypes.POINTER(FaciesDesc), vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp), vp, vp]
    L.crava_job_local_noise.argtypes = [vp, vp, vp]
    L.crava_job_set_wavelet_grids.argtypes = [vp, ctypes.c_int, vp, vp]
    L.crava_job_set_wavelet_3d.argtypes = [vp, ctypes.POINTER(Wavelet3DDesc)]
    L.crava_grid_write_storm.argtypes = [vp, ctypes.c_char_p, vp] + [ctypes.c_int] * 7 + [ctypes.POINTER(StormGeom), vp]
    L.crava_grid_read_storm.argtypes = [vp, ctypes.c_char_p, vp] + [ctypes.c_int] * 6 + [ctypes.POINTER(StormGeom), vp]
    L.crava_job_residual_synthetics.argtypes = [vp, vp]
    L.crava_grid_write_crava.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(SimboxGeom), vp]
    L.crava_grid_read_crava.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(SimboxGeom), vp]
    L.crava_facies_prob_local_noise.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.c_int, vp,
                                                ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp), vp, vp]
    L.crava_job_fill_prior_auto_cov.argtypes = [vp, vp, ctypes.c_float, ctypes.c_float, vp]
    L.crava_grid_write_segy.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(SegyDesc), vp]
    L.crava_job_set_facies.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.c_int, vp,
                                       ctypes.POINTER(vp), vp]
    L.crava_circ_corr_t.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]
    L.crava_circ_auto_cov.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, vp]
    L.crava_ctx_set_table_cache.argtypes = [vp, ctypes.c_size_t]
    L.crava_ctx_table_cache_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                             ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int)]
    L.crava_tuning_set.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
    L.crava_tuning_get.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.crava_tuning_load.argtypes = [ctypes.c_char_p]
    L.crava_tuning_path.restype = ctypes.c_char_p
    _lib = L
    return L


def _check(status: int):
    if status != OK:
        L = lib()
        raise CravaError(status, (L.crava_last_error() or b"").decode())


def tuning_set(key: str, n: int, value: int):
    """Override one schedule entry for this process (value < 0 removes it)."""
    _check(lib().crava_tuning_set(key.encode(), int(n), int(value)))


def tuning_get(key: str, n: int) -> int:
    """The schedule value a launch would use (-1: the built-in default)."""
    v = ctypes.c_int()
    _check(lib().crava_tuning_get(key.encode(), int(n), ctypes.byref(v)))
    return v.value


def tuning_load(path: str):
    _check(lib().crava_tuning_load(str(path).encode()))


def tuning_path() -> str:
    return (lib().crava_tuning_path() or b"").decode()


def circ_corr_t(prior_corr_t, min_int_fq: int, nzp: int) -> np.ndarray:
    """computeCircCorrT + makeCircCorrTPosDef on the host (crava_circ_corr_t)."""
    a = np.ascontiguousarray(prior_corr_t, dtype=np.float64)
    out = np.empty(nzp, dtype=np.float32)
    _check(lib().crava_circ_corr_t(a.ctypes.data, len(a), int(min_int_fq), int(nzp), out.ctypes.data))
    return out


def circ_auto_cov(auto_cov, nzp: int, dz: float) -> np.ndarray:
    """Estimated circular auto-covariances made positive definite and tapered
    (crava_circ_auto_cov); auto_cov (nlag, 3, 3); returns (6, nzp)."""
    a = np.ascontiguousarray(auto_cov, dtype=np.float64)
    out = np.empty((6, nzp), dtype=np.float32)
    _check(lib().crava_circ_auto_cov(a.ctypes.data, a.shape[0], int(nzp), float(dz), out.ctypes.data))
    return out


def pencil_key(nzp: int, ntheta: int) -> int:
    """Size key of the pencil-pass schedule entries."""
    return nzp * 16 + ntheta


class Context:
    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self._h = ctypes.c_void_p()
        _check(lib().crava_ctx_create(ctypes.byref(self._h), device, hbm_budget))

    @property
    def handle(self):
        return self._h

    def kernel_launches(self) -> int:
        return int(lib().crava_ctx_kernel_launches(self._h))

    def fail_next_allocs(self, n: int):
        """Fault injection: the next n job allocations fail with ENOMEM (crava_ctx_fail_next_allocs)."""
        _check(lib().crava_ctx_fail_next_allocs(self._h, int(n)))

    def set_profiling(self, on: bool):
        _check(lib().crava_ctx_set_profiling(self._h, int(on)))

    def kernel_times(self, reset: bool = True) -> dict:
        """{class: (total ms, launches)} for launches since the last reset."""
        n = len(KERNEL_CLASSES)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_longlong * n)()
        _check(lib().crava_ctx_kernel_times(self._h, ms, cnt, n, int(reset)))
        return {k: (ms[i], cnt[i]) for i, k in enumerate(KERNEL_CLASSES)}

    def set_table_cache(self, max_bytes: int):
        """Resident per-kz and lateral tables shared by jobs of the same model (0: off)."""
        _check(lib().crava_ctx_set_table_cache(self._h, int(max_bytes)))

    def table_cache_stats(self) -> dict:
        h, m, n = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_int()
        b = ctypes.c_size_t()
        _check(lib().crava_ctx_table_cache_stats(self._h, ctypes.byref(h), ctypes.byref(m), ctypes.byref(b),
                                                 ctypes.byref(n)))
        return {"hits": h.value, "misses": m.value, "bytes": b.value, "entries": n.value}

    def close(self):
        if self._h:
            lib().crava_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_desc(blk, prior_mode: int = PRIOR_SEPARABLE, flags: int = 0, seed: Optional[int] = None,
              nsim: Optional[int] = None, fp64_threshold: float = 0.0):
    """Job description of a synth.Block; returns (desc, keepalive arrays)."""
    keep = {
        "A": np.ascontiguousarray(blk.A, dtype=np.float64),
        "etc": np.ascontiguousarray(blk.err_theta_cov, dtype=np.float64),
        "wav": np.ascontiguousarray(blk.wavelet, dtype=np.float32),
        "wn": np.ascontiguousarray(blk.wavelet_norm, dtype=np.float32),
        "pv": np.ascontiguousarray(blk.prior_var0, dtype=np.float64),
        "cxy": np.ascontiguousarray(blk.corr_xy, dtype=np.float32),
        "cct": np.ascontiguousarray(blk.circ_corr_t, dtype=np.float32),
    }
    d = JobDesc()
    d.nx, d.ny, d.nz = blk.nx, blk.ny, blk.nz
    d.nxp, d.nyp, d.nzp = blk.nxp, blk.nyp, blk.nzp
    d.ntheta = blk.ntheta
    d.lz = float(blk.lz)
    d.min_rel_thick = float(blk.min_rel_thick)
    d.low_cut, d.high_cut, d.wnc = float(blk.low_cut), float(blk.high_cut), float(blk.wnc)
    d.A = keep["A"].ctypes.data_as(_dp)
    d.err_theta_cov = keep["etc"].ctypes.data_as(_dp)
    d.wavelet = keep["wav"].ctypes.data_as(_fp)
    d.wavelet_norm = keep["wn"].ctypes.data_as(_fp)
    d.prior_var0 = keep["pv"].ctypes.data_as(_dp)
    d.prior_mode = prior_mode
    d.corr_xy = keep["cxy"].ctypes.data_as(_fp)
    d.circ_corr_t = keep["cct"].ctypes.data_as(_fp)
    d.nsim = blk.nsim if nsim is None else nsim
    d.seed = int(blk.seed if seed is None else seed) & ((1 << 64) - 1)
    d.flags = flags
    d.fp64_threshold = float(fp64_threshold)
    if getattr(blk, "rel_thick", None) is not None:
        keep["relt"] = np.ascontiguousarray(blk.rel_thick, dtype=np.float64)
        d.rel_thick = keep["relt"].ctypes.data_as(_dp)
        d.energy_threshold = float(blk.energy_threshold)
        d.flags |= FLAG_NONCONST_THICK
    return d, keep


def footprint(blk, prior_mode=PRIOR_SEPARABLE, flags=0, nsim=None) -> int:
    d, _keep = make_desc(blk, prior_mode, flags, nsim=nsim)
    out = ctypes.c_size_t()
    _check(lib().crava_job_footprint(ctypes.byref(d), ctypes.byref(out)))
    return int(out.value)


class Job:
    """One inversion block on the device."""

    def __init__(self, ctx: Context, blk, prior_mode: int = PRIOR_SEPARABLE, flags: int = 0,
                 seed: Optional[int] = None, nsim: Optional[int] = None, fp64_threshold: float = 0.0):
        self.ctx = ctx
        self.blk = blk
        if getattr(blk, "rel_thick", None) is not None:
            flags |= FLAG_NONCONST_THICK
        self.flags = flags
        self.prior_mode = prior_mode
        self.nsim = blk.nsim if nsim is None else nsim
        desc, self._keep = make_desc(blk, prior_mode, flags, seed, nsim, fp64_threshold)
        self._h = ctypes.c_void_p()
        _check(lib().crava_job_create(ctx.handle, ctypes.byref(desc), ctypes.byref(self._h)))
        self.shape = (blk.nzp, blk.nyp, 2 * (blk.nxp // 2 + 1))

    def set_facies(self, corner_descs, d_densities, density_row: int, noise_scale, d_prob, d_seis_lh=None):
        """Facies probabilities written by every later run (crava_job_set_facies): 2^nang corner
        descriptions and device volumes, noise_scale (nang, ny, nx) host maps or None, nfacies+1
        device probability grids; corner_descs=None clears."""
        if corner_descs is None:
            _check(lib().crava_job_set_facies(self._h, None, 0, None, 0, None, None, None))
            return
        nang = int(np.asarray(noise_scale).shape[0]) if noise_scale is not None else 0
        assert len(corner_descs) == 1 << nang and len(d_densities) == 1 << nang
        arr = (FaciesDesc * len(corner_descs))(*corner_descs)
        dens = (ctypes.c_void_p * len(d_densities))(*d_densities)
        sc = np.ascontiguousarray(noise_scale, dtype=np.float32) if nang else None
        prob = (ctypes.c_void_p * len(d_prob))(*d_prob)
        _check(lib().crava_job_set_facies(self._h, arr, nang, dens, int(density_row),
                                          sc.ctypes.data if nang else None, prob, d_seis_lh))

    def upload(self, role: int, index: int, host: np.ndarray, stream=None):
        a = np.ascontiguousarray(host)
        if a.dtype == np.complex64:
            a = a.view(np.float32)
        assert a.dtype == np.float32 and a.size == int(np.prod(self.shape)), (a.dtype, a.shape)
        _check(lib().crava_job_upload(self._h, role, index, a.ctypes.data, stream))
        return a  # caller keeps it alive until the copy is done

    def download(self, role: int, index: int, out: Optional[np.ndarray] = None, stream=None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape, dtype=np.float32)
        _check(lib().crava_job_download(self._h, role, index, out.ctypes.data, stream))
        return out

    def device_ptr(self, role: int, index: int) -> int:
        p = ctypes.c_void_p()
        _check(lib().crava_job_device_ptr(self._h, role, index, ctypes.byref(p)))
        return int(p.value)

    def run(self, stream=None):
        _check(lib().crava_job_run(self._h, stream))

    def fill_prior(self, corr_grad_i: float = 0.0, corr_grad_j: float = 0.0, stream=None):
        """GRIDS-mode job: generate the six prior covariance grids and the error-correlation
        grid on the device from corr_xy and circ_corr_t (InitializeCorrelations)."""
        _check(lib().crava_job_fill_prior(self._h, float(corr_grad_i), float(corr_grad_j), stream))

    def fill_prior_auto_cov(self, circ_auto_cov, corr_grad_i: float = 0.0, corr_grad_j: float = 0.0, stream=None):
        """GRIDS-mode job with estimated covariance: the six covariance grids
        FillInLateralCorr(corrXY, circAutoCov_q) and the error-correlation grid on the device."""
        a = np.ascontiguousarray(circ_auto_cov, dtype=np.float32)
        assert a.shape == (6, self.blk.nzp), a.shape
        _check(lib().crava_job_fill_prior_auto_cov(self._h, a.ctypes.data, float(corr_grad_i), float(corr_grad_j),
                                                   stream))

    def divide_data(self, stream=None):
        """divideDataByScaleWavelet + interpolateSeismic on the uploaded data (non-constant
        thickness jobs); returns after the work is done."""
        _check(lib().crava_job_divide_data(self._h, stream))

    def set_wavelet_grids(self, angle: int, shift_ms=None, gain=None):
        """Local wavelet time shift (ms) and gain grids of one angle stack, (ny, nx) each or
        None; -999 entries mean no shift / unit gain."""
        arrs = []
        for a in (shift_ms, gain):
            if a is None:
                arrs.append(None)
                continue
            a = np.ascontiguousarray(a, dtype=np.float32)
            assert a.shape == (self.blk.ny, self.blk.nx), a.shape
            arrs.append(a)
        _check(lib().crava_job_set_wavelet_grids(self._h, int(angle), *[None if a is None else a.ctypes.data
                                                                         for a in arrs]))

    def set_wavelet_3d(self, theta, alpha1, global_wavelet, global_wavelet_norm, filter_geom, grad_x=None,
                       grad_y=None, halpha=None):
        """3D wavelets for every angle (crava_job_set_wavelet_3d); arguments as wavelet3d_desc."""
        nth, ny, nx = self.blk.ntheta, self.blk.ny, self.blk.nx
        for g in (grad_x, grad_y):
            assert g is None or np.shape(g) == (ny, nx), np.shape(g)
        assert np.shape(alpha1)[0] == nth and np.shape(global_wavelet) == (nth, self.blk.nzp)
        d, _keep = wavelet3d_desc(theta, alpha1, global_wavelet, global_wavelet_norm, filter_geom, grad_x, grad_y,
                                  halpha)
        _check(lib().crava_job_set_wavelet_3d(self._h, ctypes.byref(d)))

    def residual_synthetics(self, stream=None):
        """multiplyDataByScaleWaveletAndWriteToFile: after a run with KEEP_RESIDUAL the residual
        grids become the real residuals convolved with each trace's local wavelet."""
        _check(lib().crava_job_residual_synthetics(self._h, stream))

    def local_noise(self, scales: np.ndarray, stream=None):
        """correctVpVsRho and the local-noise mixing of the realisations, in place on the
        posterior mean and realisation grids; scales (ntheta, ny, nx) local noise scales."""
        a = np.ascontiguousarray(scales, dtype=np.float32)
        assert a.shape == (self.blk.ntheta, self.blk.ny, self.blk.nx), a.shape
        _check(lib().crava_job_local_noise(self._h, a.ctypes.data, stream))

    def counters(self) -> dict:
        """Per-job counters after a run; raises CravaError (status ENUMERIC) when the data
        or prior-mean grids held a NaN or Inf."""
        c = Counters()
        _check(lib().crava_job_counters(self._h, ctypes.byref(c)))
        return {"inverted_bins": c.inverted_bins, "chol_fallbacks": c.chol_fallbacks,
                "sim_chol_zero": c.sim_chol_zero, "fp64_bins": c.fp64_bins,
                "nonfinite_tiles": c.nonfinite_tiles,
                "post_var0": np.array(list(c.post_var0), dtype=np.float32).reshape(3, 3)}

    def upload_block(self, cov_grids=None, err_corr=None, noise=None):
        """Upload data and prior mean (and the GRIDS-mode prior, host noise)."""
        keep = []
        blk = self.blk
        for l in range(blk.ntheta):
            keep.append(self.upload(ROLE_DATA, l, blk.data[l]))
        for a in range(3):
            keep.append(self.upload(ROLE_MEAN, a, blk.mean[a]))
        if self.prior_mode == PRIOR_GRIDS:
            rnxp = self.shape[2]
            for q in range(6):
                g = np.zeros(self.shape, dtype=np.float32)
                g[..., :blk.nxp] = cov_grids[q]
                keep.append(self.upload(ROLE_PRIOR_COV, q, g))
            g = np.zeros(self.shape, dtype=np.float32)
            g[..., :blk.nxp] = err_corr
            keep.append(self.upload(ROLE_ERR_CORR, 0, g))
        if self.flags & FLAG_HOST_NOISE:
            for s in range(self.nsim):
                for a in range(3):
                    keep.append(self.upload(ROLE_NOISE, 3 * s + a, noise[s, a]))
        return keep

    def download_outputs(self) -> dict:
        blk = self.blk
        out = {"mean": np.stack([self.download(ROLE_POST_MEAN, a) for a in range(3)])}
        cov = np.stack([self.download(ROLE_POST_COV, q) for q in range(6)])
        if self.flags & FLAG_SPECTRAL_COV:
            out["cov_spec"] = cov.view(np.complex64)
        else:
            out["cov"] = cov
        if self.nsim:
            out["sims"] = np.stack([self.download(ROLE_SIM, q) for q in range(3 * self.nsim)]).reshape(
                (self.nsim, 3) + self.shape)
        if self.flags & FLAG_KEEP_RESIDUAL:
            out["resid_spec"] = np.stack([self.download(ROLE_RESIDUAL, l).view(np.complex64)
                                          for l in range(blk.ntheta)])
        return out

    def close(self):
        if self._h:
            lib().crava_job_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def invert_block(ctx: Context, blk, prior_mode=PRIOR_SEPARABLE, noise=None, keep_residual=False,
                 cov_grids=None, err_corr=None, seed=None, fp64_threshold=0.0, spectral_cov=False) -> dict:
    """Host-to-host inversion of one block (the e2e path): upload, run, download."""
    flags = (FLAG_HOST_NOISE if noise is not None else 0) | (FLAG_KEEP_RESIDUAL if keep_residual else 0) | \
        (FLAG_SPECTRAL_COV if spectral_cov else 0)
    job = Job(ctx, blk, prior_mode, flags, seed=seed, fp64_threshold=fp64_threshold)
    try:
        _keep = job.upload_block(cov_grids, err_corr, noise)
        if job.flags & FLAG_NONCONST_THICK:
            job.divide_data()
        job.run()
        out = job.download_outputs()
        out["counters"] = job.counters()
        return out
    finally:
        job.close()


def fft_r2c(ctx: Context, dptr: int, nxp: int, nyp: int, nzp: int, covariance: bool, stream=None):
    _check(lib().crava_fft_r2c(ctx.handle, ctypes.c_void_p(dptr), nxp, nyp, nzp, int(covariance), stream))


def fft_c2r(ctx: Context, dptr: int, nxp: int, nyp: int, nzp: int, covariance: bool, stream=None):
    _check(lib().crava_fft_c2r(ctx.handle, ctypes.c_void_p(dptr), nxp, nyp, nzp, int(covariance), stream))


class Batch:
    """Many created jobs replayed as one CUDA graph with concurrent branches."""

    def __init__(self, ctx: Context, jobs, branches: int = 16):
        self.ctx = ctx
        self.jobs = list(jobs)
        arr = (ctypes.c_void_p * len(self.jobs))(*[j._h.value for j in self.jobs])
        self._h = ctypes.c_void_p()
        _check(lib().crava_batch_create(ctx.handle, arr, len(self.jobs), branches, ctypes.byref(self._h)))

    def run(self, stream=None):
        _check(lib().crava_batch_run(self._h, stream))

    def close(self):
        if self._h:
            lib().crava_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The native serving loop: submit blocks (host buffers), poll/wait for completion."""

    def __init__(self, ctx: Context, max_inflight: int = 8):
        self.ctx = ctx
        self._h = ctypes.c_void_p()
        self._keep = {}
        _check(lib().crava_serve_start(ctx.handle, max_inflight, ctypes.byref(self._h)))

    def submit(self, blk, host_in, host_out, seed=None) -> int:
        """host_in / host_out: lists of host buffers (numpy float32 or pinned torch tensors)
        kept alive until the request finishes."""
        desc, keep = make_desc(blk, PRIOR_SEPARABLE, 0, seed=seed)
        ptr = lambda a: a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data
        ins = (ctypes.c_void_p * len(host_in))(*[ptr(a) for a in host_in])
        outs = (ctypes.c_void_p * len(host_out))(*[ptr(a) if a is not None else None for a in host_out])
        t = ctypes.c_uint64()
        _check(lib().crava_serve_submit(self._h, ctypes.byref(desc), ins, outs, ctypes.byref(t)))
        self._keep[t.value] = (desc, keep, host_in, host_out, ins, outs)
        return t.value

    def poll(self, ticket: int) -> dict:
        """A request's state; after its final state has been reported the ticket is released."""
        info = RequestInfo()
        _check(lib().crava_serve_poll(self._h, ticket, ctypes.byref(info)))
        if info.state in (REQ_DONE, REQ_FAILED):
            self._keep.pop(ticket, None)
        return {"state": info.state, "status": info.status, "queue_ms": info.queue_ms, "latency_ms": info.latency_ms}

    def wait(self, ticket: int, timeout_ms: float = 600000.0) -> dict:
        """Waits for a request; raises CravaError with the request's status when it failed."""
        info = RequestInfo()
        st = lib().crava_serve_wait(self._h, ticket, timeout_ms, ctypes.byref(info))
        if st != ETIMEDOUT:
            self._keep.pop(ticket, None)
        _check(st)
        return {"state": info.state, "status": info.status, "queue_ms": info.queue_ms, "latency_ms": info.latency_ms}

    def set_queue_limit(self, max_queued: int):
        """At most max_queued waiting requests; further submits raise CravaError(EBUSY)."""
        _check(lib().crava_serve_set_queue_limit(self._h, int(max_queued)))

    def cancel(self, ticket: int):
        """Cancels a request that is still queued (CravaError(ESTATE) once admitted)."""
        _check(lib().crava_serve_cancel(self._h, ticket))

    def stop(self):
        if self._h:
            lib().crava_serve_stop(self._h)
            self._h = ctypes.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


def facies_desc(prior, nbins, vmin, dv, p_undefined):
    pr = np.ascontiguousarray(prior, dtype=np.float32)
    fd = FaciesDesc()
    fd.nfacies = len(pr)
    for d in range(3):
        fd.nbins[d], fd.vmin[d], fd.dv[d] = int(nbins[d]), float(vmin[d]), float(dv[d])
    fd.prior = pr.ctypes.data_as(_fp)
    fd.p_undefined = float(p_undefined)
    return fd, pr


def facies_smooth(ctx: Context, fd, sigma_inv, d_hist: int, stream=None):
    """Gaussian smoothing of nfacies device histograms (FFTGrid layout) in place."""
    S = np.ascontiguousarray(sigma_inv, dtype=np.float64)
    _check(lib().crava_facies_smooth(ctx.handle, ctypes.byref(fd), S.ctypes.data_as(_dp), d_hist, stream))


def facies_prob(ctx: Context, fd, d_density: int, density_row: int, d_post, nx, ny, nz, nxp, nyp, d_prob,
                d_seis_lh=None, stream=None):
    post = (ctypes.c_void_p * 3)(*d_post)
    prob = (ctypes.c_void_p * len(d_prob))(*d_prob)
    _check(lib().crava_facies_prob(ctx.handle, ctypes.byref(fd), d_density, density_row, post, nx, ny, nz, nxp, nyp,
                                   prob, d_seis_lh, stream))


def facies_prob_local_noise(ctx: Context, corner_descs, d_densities, density_row: int, noise_scale, d_post, nx, ny,
                            nz, nxp, nyp, d_prob, d_seis_lh=None, stream=None):
    """Facies probabilities with local noise: 2^nang corner density volumes (corner_descs,
    d_densities), noise_scale (nang, ny, nx) host maps."""
    nang = int(np.asarray(noise_scale).shape[0]) if np.asarray(noise_scale).ndim == 3 else 0
    assert len(corner_descs) == 1 << nang and len(d_densities) == 1 << nang
    arr = (FaciesDesc * len(corner_descs))(*corner_descs)
    dens = (ctypes.c_void_p * len(d_densities))(*d_densities)
    sc = np.ascontiguousarray(noise_scale, dtype=np.float32)
    post = (ctypes.c_void_p * 3)(*d_post)
    prob = (ctypes.c_void_p * len(d_prob))(*d_prob)
    _check(lib().crava_facies_prob_local_noise(ctx.handle, arr, nang, dens, int(density_row),
                                               sc.ctypes.data if nang else None, post, nx, ny, nz, nxp, nyp, prob,
                                               d_seis_lh, stream))


def grid_write_crava(ctx: Context, path: str, d_grid: int, rnxp: int, nyp: int, nzp: int, geom: dict, stream=None):
    """FFTGrid::writeCravaFile of a device grid (rnxp x nyp x nzp floats)."""
    g = SimboxGeom(**geom)
    _check(lib().crava_grid_write_crava(ctx.handle, str(path).encode(), d_grid, rnxp, nyp, nzp, ctypes.byref(g), stream))


def grid_read_crava(ctx: Context, path: str, d_grid: int, rnxp: int, nyp: int, nzp: int, stream=None) -> dict:
    """FFTGrid::readCravaFile into a device grid; returns the file's simbox geometry."""
    g = SimboxGeom()
    _check(lib().crava_grid_read_crava(ctx.handle, str(path).encode(), d_grid, rnxp, nyp, nzp, ctypes.byref(g), stream))
    return {k: getattr(g, k) for k, _t in SimboxGeom._fields_}


def grid_write_segy(ctx: Context, path: str, d_grid: int, rnxp: int, nyp: int, nzp: int, desc, stream=None):
    """FFTGrid::writeSegyFile of a real device grid (rnxp x nyp x nzp floats); desc from segy_desc."""
    _check(lib().crava_grid_write_segy(ctx.handle, str(path).encode(), d_grid, rnxp, nyp, nzp, ctypes.byref(desc),
                                       stream))


def grid_write_storm(ctx: Context, path: str, d_grid: int, dims, padded_dims, geom: dict, padding: bool = False,
                     stream=None):
    """FFTGrid::writeStormFile (binary) of a padded real device grid; dims = (nx, ny, nz),
    padded_dims = (nxp, nyp, nzp); geom: xmin, lx, ymin, ly, lz, angle (radians), cubetype and
    either flat=1 or top_name/bot_name."""
    g = dict(geom)
    for k in ("top_name", "bot_name"):
        if g.get(k) is not None:
            g[k] = str(g[k]).encode()
    gs = StormGeom(**g)
    _check(lib().crava_grid_write_storm(ctx.handle, str(path).encode(), d_grid, *dims, *padded_dims, int(padding),
                                        ctypes.byref(gs), stream))


def grid_read_storm(ctx: Context, path: str, d_grid: int, dims, padded_dims, stream=None) -> dict:
    """A STORM binary grid into a padded real device grid with FFTGrid's padding fill; returns
    the header's geometry."""
    gs = StormGeom()
    _check(lib().crava_grid_read_storm(ctx.handle, str(path).encode(), d_grid, *dims, *padded_dims,
                                       ctypes.byref(gs), stream))
    return {k: getattr(gs, k) for k, _t in StormGeom._fields_ if k not in ("top_name", "bot_name")}
