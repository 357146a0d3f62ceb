"""ctypes bindings of the compiled checkers (test infrastructure only).

* ``_build/liboracle.so``  -- plain-C restatement of the reference's noise source.
* ``_ref/libref32.so``     -- the reference's FP32 numerics with the restated loops
                              (absent where the reference tree was not available at build).
* ``_ref/libsegyref.so``   -- FFTGrid::writeSegyFile over NRLib's own SegY header, geometry
                              and IBM-float code.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF32_LIB = os.path.join(HERE, "_ref", "libref32.so")
SEGYREF_LIB = os.path.join(HERE, "_ref", "libsegyref.so")

_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)


def _f(a):
    return a.ctypes.data_as(_fp)


def _d(a):
    return a.ctypes.data_as(_dp)


_oracle = None
_ref32 = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        _oracle = ctypes.CDLL(ORACLE_LIB)
        _oracle.oracle_sim_noise.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, _fp]
        _oracle.oracle_rnorm01.argtypes = [ctypes.POINTER(ctypes.c_uint32)]
        _oracle.oracle_rnorm01.restype = ctypes.c_double
    return _oracle


def ref32_available() -> bool:
    return os.path.exists(REF32_LIB)


class Ref32Block(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("nxp", ctypes.c_int), ("nyp", ctypes.c_int), ("nzp", ctypes.c_int),
                ("ntheta", ctypes.c_int),
                ("lz", ctypes.c_double), ("min_rel_thick", ctypes.c_double),
                ("low_cut", ctypes.c_float), ("high_cut", ctypes.c_float), ("wnc", ctypes.c_float),
                ("A", _dp), ("err_theta_cov", _dp), ("wavelet", _fp), ("wavelet_norm", _fp),
                ("prior_var0", _dp), ("nonconst", ctypes.c_int)]


def ref32_lib():
    global _ref32
    if _ref32 is None:
        _ref32 = ctypes.CDLL(REF32_LIB)
        P = ctypes.POINTER
        _ref32.ref32_invert.argtypes = [P(Ref32Block), P(_fp), P(_fp), _fp, P(_fp), ctypes.c_int,
                                        ctypes.c_uint, P(_fp), _fp, P(ctypes.c_longlong)]
        _ref32.ref32_fft.argtypes = [_fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _ref32.ref32_ifft.argtypes = [_fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _ref32.ref32_sim_noise.argtypes = [ctypes.c_uint, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, _fp]
        _ref32.ref32_divide_traces.argtypes = [_fp, ctypes.c_int, ctypes.c_int, _fp, _fp,
                                               ctypes.POINTER(ctypes.c_ubyte)]
        _ref32.ref32_facies_prob.argtypes = [P(_fp), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             P(_fp), P(ctypes.c_double), ctypes.c_int, _fp, ctypes.c_float, _fp, _fp]
    return _ref32


def ref32_divide(blk) -> np.ndarray:
    """AVOInversion::divideDataByScaleWavelet on every data grid with the reference's FFTW
    2.1.2 float transforms (ref32_divide_traces), the adjustment factor and band from the
    float32 restatement in ref64.  Returns (ntheta, nzp, nyp, rnxp) float32, the padding
    columns untouched."""
    from oracle import ref64
    f32 = np.float32
    nxp, nyp, nzp, nz = blk.nxp, blk.nyp, blk.nzp, blk.nz
    cn = nzp // 2 + 1
    tab = ref64.thick_tables(blk)
    tab["wnc"] = blk.wnc
    taper = np.ones(nzp, dtype=f32)
    for k in range(nzp):
        if k > nz:
            dk = f32(ref64.dist_to_boundary(k, nz, nzp))
            taper[k] = max(f32(1) - dk * dk, f32(0))
    rt = np.asarray(blk.rel_thick, dtype=np.float64)
    sf = rt.astype(f32).reshape(-1)
    deltaF = (float(nz) * 1000.0 / (rt * float(blk.lz) * float(nzp))).reshape(-1)
    k = np.arange(cn)
    fk = deltaF[:, None] * k[None, :]
    band = np.ascontiguousarray((fk < float(f32(blk.high_cut))) & (fk > float(f32(blk.low_cut))), dtype=np.uint8)
    out = np.array(blk.data, dtype=np.float32)
    for l in range(blk.ntheta):
        fac = ref64.adjustment_factor(tab, l, sf[:, None], k[None, :])
        fac = np.where(band.astype(bool), fac, 0.0)
        f = np.ascontiguousarray(fac.astype(np.complex64)).view(np.float32)
        traces = np.ascontiguousarray(np.moveaxis(out[l][..., :nxp], 0, -1).reshape(-1, nzp))
        ref32_lib().ref32_divide_traces(_f(traces), traces.shape[0], nzp, _f(taper), _f(f),
                                        band.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)))
        out[l][..., :nxp] = np.moveaxis(traces.reshape(nyp, nxp, nzp), -1, 0)
    return out


def sim_noise(seed: int, nsim: int, nxp: int, nyp: int, nzp: int, use_ref: bool = False) -> np.ndarray:
    """Complex noise grids (nsim, 3, nzp, nyp, cnxp) complex64 in simulate's draw order."""
    cnxp = nxp // 2 + 1
    out = np.empty((nsim, 3, nzp, nyp, cnxp), dtype=np.complex64)
    if use_ref:
        ref32_lib().ref32_sim_noise(seed, nsim, nxp, nyp, nzp, _f(out.view(np.float32)))
    else:
        oracle_lib().oracle_sim_noise(seed, nsim, nxp, nyp, nzp, _f(out.view(np.float32)))
    return out


def ref32_fft(grid: np.ndarray, nxp: int, covariance: bool) -> np.ndarray:
    """FFTGrid::fftInPlace with the reference FFTW on a padded (nzp,nyp,rnxp) float grid;
    returns the (nzp,nyp,cnxp) complex64 spectrum."""
    g = np.ascontiguousarray(grid, dtype=np.float32).copy()
    nzp, nyp, _ = g.shape
    ref32_lib().ref32_fft(_f(g), nxp, nyp, nzp, int(covariance))
    return g.view(np.complex64)


def ref32_ifft(spec: np.ndarray, nxp: int, covariance: bool) -> np.ndarray:
    g = np.ascontiguousarray(spec, dtype=np.complex64).copy()
    nzp, nyp, _ = g.shape
    r = g.view(np.float32)
    ref32_lib().ref32_ifft(_f(r), nxp, nyp, nzp, int(covariance))
    return r


class Ref32Result:
    def __init__(self):
        self.mean = None
        self.cov = None
        self.resid_spec = None
        self.sims = None
        self.n_inverted = 0
        self.n_chol_fail = 0


def ref32_invert(blk, cov_grids, err_corr, nsim=0, seed=0, noise=None, nonconst=False) -> Ref32Result:
    """Run the reference's FP32 path on one block.  cov_grids: six (nzp,nyp,nxp) float32
    prior covariance grids; err_corr: (nzp,nyp,nxp) float32; noise: optional
    (nsim,3,nzp,nyp,cnxp) complex64 replacing the RandomGen draws; nonconst: the
    non-constant-thickness branch of the per-bin step on blk.data taken as already divided."""
    lib = ref32_lib()
    nxp, nyp, nzp, nth = blk.nxp, blk.nyp, blk.nzp, blk.ntheta
    rnxp = 2 * (nxp // 2 + 1)

    def padded(x):
        g = np.zeros((nzp, nyp, rnxp), dtype=np.float32)
        g[..., :nxp] = x[..., :nxp]
        return g

    mean = [padded(blk.mean[a]) for a in range(3)]
    cov = [padded(c) for c in cov_grids]
    err = padded(err_corr)
    data = [padded(blk.data[l]) for l in range(nth)]
    sims = [np.zeros((nzp, nyp, rnxp), dtype=np.float32) for _ in range(3 * nsim)]
    A = np.ascontiguousarray(blk.A, dtype=np.float64)
    etc = np.ascontiguousarray(blk.err_theta_cov, dtype=np.float64)
    wav = np.ascontiguousarray(blk.wavelet, dtype=np.float32)
    wn = np.ascontiguousarray(blk.wavelet_norm, dtype=np.float32)
    pv = np.ascontiguousarray(blk.prior_var0, dtype=np.float64)
    b = Ref32Block(blk.nx, blk.ny, blk.nz, nxp, nyp, nzp, nth, float(blk.lz), float(blk.min_rel_thick),
                   float(blk.low_cut), float(blk.high_cut), float(blk.wnc), _d(A), _d(etc), _f(wav), _f(wn), _d(pv),
                   int(bool(nonconst)))
    arr = lambda L: (_fp * len(L))(*[_f(x) for x in L]) if L else None
    cnt = (ctypes.c_longlong * 2)()
    nz_in = None
    if noise is not None:
        noise = np.ascontiguousarray(noise, dtype=np.complex64)
        nz_in = _f(noise.view(np.float32))
    lib.ref32_invert(ctypes.byref(b), arr(mean), arr(cov), _f(err), arr(data), nsim, seed,
                     arr(sims) if nsim else None, nz_in, cnt)
    r = Ref32Result()
    r.mean = np.stack(mean)
    r.cov = np.stack(cov)
    r.resid_spec = np.stack([d.view(np.complex64) for d in data])
    r.sims = np.stack(sims).reshape(nsim, 3, nzp, nyp, rnxp) if nsim else None
    r.n_inverted, r.n_chol_fail = cnt[0], cnt[1]
    return r


def ref32_facies_prob(post, corners, prior, p_undefined, t):
    """calculateFaciesProb + findDensity in the reference's float arithmetic (ref32).
    post: 3 arrays (nz, ny, nx); corners: list of (dens (nf, nr, nb, na), nbins, vmin, dv);
    t: (nang, ny, nx) relative noise scales.  Returns (nf + 1, nz, ny, nx) float32."""
    lib = ref32_lib()
    nz, ny, nx = post[0].shape
    P = [np.ascontiguousarray(p, dtype=np.float32) for p in post]
    D = [np.ascontiguousarray(c[0], dtype=np.float32) for c in corners]
    box = np.array([list(c[2]) + list(c[3]) + list(c[1]) for c in corners], dtype=np.float64)
    nf = D[0].shape[0]
    pr = np.ascontiguousarray(prior, dtype=np.float32)
    tt = np.ascontiguousarray(t, dtype=np.float32)
    out = np.empty((nf + 1, nz, ny, nx), dtype=np.float32)
    lib.ref32_facies_prob((_fp * 3)(*[_f(p) for p in P]), nx, ny, nz, tt.shape[0], (_fp * len(D))(*[_f(d) for d in D]),
                          box.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nf, _f(pr), float(p_undefined),
                          _f(tt) if tt.size else None, _f(out))
    return out


def segy_ref_write(path: str, grid: np.ndarray, desc) -> None:
    """The reference's SegY file of a host grid (nzp, nyp, rnxp float32) for a crava_segy_desc
    (crava_b200.api.SegyDesc)."""
    L = ctypes.CDLL(SEGYREF_LIB)
    L.segy_ref_write.argtypes = [ctypes.c_char_p, _fp, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    g = np.ascontiguousarray(grid, dtype=np.float32)
    rc = L.segy_ref_write(str(path).encode(), _f(g), g.shape[2], g.shape[1], ctypes.addressof(desc))
    if rc != 0:
        raise RuntimeError(f"segy_ref_write failed ({rc})")
