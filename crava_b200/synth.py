"""Seeded synthetic inversion blocks with the shapes and value distributions of the
reference's model setup.

The reference builds these inputs from XML, wells and SegY files (model setup, out of
scope here).  This module builds the same objects directly, following the reference's
formulas, so that the hot path sees inputs of the right structure:

* reflection matrix A           -- CommonData::SetupDefaultReflectionMatrix
                                   (src/commondata.cpp:2915-2952), PP rows
* prior variance priorVar0      -- std_a * std_b * corr_ab
* lateral correlation surface   -- CommonData::FindCorrXYGrid (src/commondata.cpp:9180-9218)
                                   with SphericalVario::corr (src/vario.cpp:66-73)
* temporal correlation          -- Gaussian (GenExp power 2, src/vario.cpp:88-93) sampled at
                                   lag dz*j, j <= n_corr_T (src/commondata.cpp:8586-8604), then
                                   SeismicParametersHolder::computeCircCorrT + makeCircCorrTPosDef
                                   (src/seismicparametersholder.cpp:624-660, 805-840)
* low_int_cut                   -- main.cpp:258
* wavelets                      -- Ricker (src/wavelet.cpp:1484-1488), 239 samples at 1 ms
                                   (src/wavelet.cpp:161-176); a Ricker whose samples fall on
                                   the resampled grid is reproduced exactly by
                                   Wavelet::resample (src/wavelet.cpp:425-476), so it is sampled
                                   at dt in FFT order here; norm as in resample.
* angular error correlation     -- default GenExp power 1, range 10 deg
                                   (src/modelsettings.h:475; src/commondata.cpp:9864-9880)
* error theta covariance        -- ModelAVODynamic::ComputeDataVariance + SetupErrorCorrelation
                                   (src/modelavodynamic.cpp:574-650)
* seismic                       -- CravaResult::ComputeSyntSeismic / ComputeSeismicImpedance
                                   (src/cravaresult.cpp:2312-2405) applied to one seeded prior
                                   realisation, plus white noise with variance Var(signal)/SN.

All grids are FFTGrid-padded real arrays of shape (nzp, nyp, rnxp), x fastest, with
rnxp = 2*(nxp//2+1) (src/fftgrid.cpp:34-47).  The padding columns i >= nxp hold
RMISSING like the reference's fill routines; they never reach a transform result.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional, Sequence

import numpy as np

RMISSING = -99999.000  # definitions.h RMISSING


def _smooth(n: int) -> bool:
    for p in (2, 3, 5, 7):
        while n % p == 0:
            n //= p
    return n == 1


def smooth_sizes(lo: int, hi: int) -> list[int]:
    """2*3*5*7-smooth integers in [lo, hi] (FFTGrid::findClosestFactorableNumber's set)."""
    return [n for n in range(lo, hi + 1) if _smooth(n)]


def find_padding_size(n: int) -> int:
    """Smallest 2*3*5*7-smooth integer >= n (src/fftgrid.cpp:2630-2658)."""
    m = n
    while not _smooth(m):
        m += 1
    return m


@dataclasses.dataclass
class BlockSpec:
    """One inversion block (one interval of one vintage in the reference)."""
    nx: int = 64
    ny: int = 64
    nz: int = 128
    dx: float = 25.0
    dy: float = 25.0
    dt: float = 4.0                       # ms
    theta_deg: Sequence[float] = (10.0, 20.0, 30.0)
    peak_hz: Sequence[float] = (30.0, 30.0, 30.0)
    sn: Sequence[float] = (5.0, 5.0, 5.0)
    std: Sequence[float] = (0.08, 0.15, 0.05)
    corr: Sequence[float] = (0.7, 0.5, 0.4)       # vp-vs, vp-rho, vs-rho
    mean: Sequence[float] = (math.log(3000.0), math.log(1500.0), math.log(2300.0))
    lateral_range: float = 1000.0                  # m, spherical
    temporal_range: float = 40.0                   # ms, Gaussian
    angular: tuple = ("genexp1", 10.0)             # (kind, range in deg)
    vsvp: float = 0.5
    low_cut: float = 5.0
    high_cut: float = 55.0
    wnc: float = 0.1
    nsim: int = 1
    seed: int = 1
    nxp: Optional[int] = None
    nyp: Optional[int] = None
    nzp: Optional[int] = None
    corr_grad_i: float = 0.0
    corr_grad_j: float = 0.0

    def padded(self):
        return (self.nxp or self.nx, self.nyp or self.ny, self.nzp or self.nz)

    @property
    def ntheta(self) -> int:
        return len(self.theta_deg)


@dataclasses.dataclass
class Block:
    """Host-side inputs of one inversion block, in the reference's own representation."""
    spec: BlockSpec
    nx: int
    ny: int
    nz: int
    nxp: int
    nyp: int
    nzp: int
    lz: float
    A: np.ndarray              # (ntheta, 3) float64
    err_theta_cov: np.ndarray  # (ntheta, ntheta) float64
    wavelet: np.ndarray        # (ntheta, nzp) float32, FFT order
    wavelet_norm: np.ndarray   # (ntheta,) float32
    prior_var0: np.ndarray     # (3, 3) float64
    corr_xy: np.ndarray        # (nyp, nxp) float32, index i + nxp*j
    prior_corr_t: np.ndarray   # float64 lags
    circ_corr_t: np.ndarray    # (nzp,) float32 after makeCircCorrTPosDef
    low_int_cut: int
    mean: np.ndarray           # (3, nzp, nyp, rnxp) float32 padded
    data: np.ndarray           # (ntheta, nzp, nyp, rnxp) float32 padded
    low_cut: float
    high_cut: float
    wnc: float
    min_rel_thick: float = 1.0
    corr_grad_i: float = 0.0
    corr_grad_j: float = 0.0
    nsim: int = 1
    seed: int = 1
    rel_thick: Optional[np.ndarray] = None   # (nyp, nxp) float64: non-constant thickness
    energy_threshold: float = 0.0

    @property
    def ntheta(self) -> int:
        return self.A.shape[0]

    @property
    def cnxp(self) -> int:
        return self.nxp // 2 + 1

    @property
    def rnxp(self) -> int:
        return 2 * (self.nxp // 2 + 1)

    @property
    def n_voxels(self) -> int:
        return self.nxp * self.nyp * self.nzp


def reflection_matrix(theta_deg, vsvp: float) -> np.ndarray:
    """PP rows of CommonData::SetupDefaultReflectionMatrix (src/commondata.cpp:2925-2941);
    entries are stored through float like the reference."""
    th = np.deg2rad(np.asarray(theta_deg, dtype=np.float64))
    # the reference's angles are float (ModelSettings::getAngle)
    th = th.astype(np.float32).astype(np.float64)
    s2 = np.sin(th) ** 2
    t2 = np.tan(th) ** 2
    v2 = vsvp * vsvp
    A = np.stack([(1.0 + t2) / 2.0, -4.0 * v2 * s2, (1.0 - 4.0 * v2 * s2) / 2.0], axis=1)
    return A.astype(np.float32).astype(np.float64)


def spherical_corr(dist):
    d = np.asarray(dist, dtype=np.float64)
    return np.where(d >= 1.0, 0.0, 1.0 + d ** 3 / 2.0 - 1.5 * d)


def corr_xy_surface(nxp: int, nyp: int, dx: float, dy: float, rng_m: float) -> np.ndarray:
    """CommonData::FindCorrXYGrid with an isotropic spherical variogram."""
    i = np.arange(nxp)
    j = np.arange(nyp)
    ri = np.where(i < nxp // 2 + 1, i, i - nxp).astype(np.float32)
    rj = np.where(j < nyp // 2 + 1, j, j - nyp).astype(np.float32)
    DX = (ri[None, :] * np.float32(dx)).astype(np.float32)
    DY = (rj[:, None] * np.float32(dy)).astype(np.float32)
    inv = np.float32(1.0 / (rng_m * rng_m))
    dist = np.sqrt((inv * DX * DX + inv * DY * DY).astype(np.float32)).astype(np.float32)
    return spherical_corr(dist).astype(np.float32)


def prior_corr_t(nzp: int, dz: float, rng_ms: float) -> np.ndarray:
    """Temporal correlation lags 0..n_corr_T (src/commondata.cpp:8586-8604), Gaussian form."""
    n = nzp // 2 + 1 if nzp % 2 == 0 else nzp // 2
    j = np.arange(n + 1, dtype=np.float64)
    return np.exp(-3.0 * (dz * j / rng_ms) ** 2)


def circ_corr_t(prior_t: np.ndarray, min_int_fq: int, nzp: int) -> np.ndarray:
    """computeCircCorrT + makeCircCorrTPosDef (src/seismicparametersholder.cpp:624-660,
    805-840): circular extension, zero the spectrum at k <= minIntFq, take |.|, back
    transform and normalise by the lag-0 value.  Done in float64 here (the reference
    runs it through FFTW float; the difference is at float rounding level)."""
    n = len(prior_t)
    c = np.zeros(nzp, dtype=np.float64)
    for k in range(nzp):
        refk = k if k < nzp // 2 + 1 else nzp - k
        c[k] = prior_t[refk] if refk < n else 0.0
    c = c.astype(np.float32).astype(np.float64)
    F = np.fft.rfft(c)
    mag = np.abs(F)
    mag[: min_int_fq + 1] = 0.0
    back = np.fft.irfft(mag, n=nzp) * nzp  # FFTW c2r is unnormalised
    if not back[0] > 1e-5:
        raise ValueError("circular temporal correlation undefined (too few layers)")
    return (back / back[0]).astype(np.float32)


def angular_corr(theta_deg, kind: str, rng_deg: float) -> np.ndarray:
    th = np.asarray(theta_deg, dtype=np.float64)
    d = np.abs(th[:, None] - th[None, :]) / rng_deg
    if kind == "genexp1":
        return np.exp(-3.0 * d)
    if kind == "spherical":
        return spherical_corr(d)
    raise ValueError(kind)


def ricker(t_ms, peak_hz):
    c = math.pi * math.pi * peak_hz * peak_hz * np.asarray(t_ms, dtype=np.float64) ** 2 * 1e-6
    return (1 - 2 * c) * np.exp(-c)


def wavelet_fft_order(nzp: int, dt: float, peak_hz: float) -> np.ndarray:
    """Ricker of half-length 119 ms sampled at dt in FFT order (Wavelet::resample)."""
    k = np.arange(nzp)
    z = np.where(k < nzp // 2 + 1, dt * k, dt * (k - nzp)).astype(np.float32).astype(np.float64)
    w = np.where(np.abs(z) <= 119.0, ricker(z, peak_hz), 0.0)
    return w.astype(np.float32)


def wavelet_norm(w: np.ndarray) -> np.float32:
    w = w.astype(np.float32)
    return np.float32(math.sqrt(float(np.sum((w * w).astype(np.float64)))))


def pad_grid(values: np.ndarray, nxp: int, nyp: int, nzp: int) -> np.ndarray:
    """Real (nz, ny, nx) -> FFTGrid padded (nzp, nyp, rnxp), padding filled by the
    reference's linear taper (FFTGrid::fillInFromArray pads by smooth extension); here
    the padding is filled with the edge values blended cyclically, which keeps the
    padded grid smooth.  With padded dims equal to dims nothing is filled."""
    nz, ny, nx = values.shape
    rnxp = 2 * (nxp // 2 + 1)
    out = np.full((nzp, nyp, rnxp), RMISSING, dtype=np.float32)
    g = np.empty((nzp, nyp, nxp), dtype=np.float64)
    g[:nz, :ny, :nx] = values

    def taper(arr, n, axis):
        m = arr.shape[axis]
        if m == n:
            return
        idx0 = [slice(None)] * 3
        first = np.take(arr, [0], axis=axis)
        last = np.take(arr, [n - 1], axis=axis)
        for q in range(n, m):
            w = (q - n + 1) / (m - n + 1)
            idx0[axis] = slice(q, q + 1)
            arr[tuple(idx0)] = (1 - w) * last + w * first

    taper(g[:, :ny, :], nx, 2)
    taper(g[:, :, :], ny, 1)
    taper(g, nz, 0)
    out[:, :, :nxp] = g.astype(np.float32)
    return out


def _prior_realisation(rng, nx, ny, nz, nxp, nyp, nzp, corr_xy, circ_t, P0, mean):
    """One seeded prior realisation of (ln Vp, ln Vs, ln rho) on the padded grid.
    S(bin) = rho(bin) * P0 with rho = |F[corrXY] F[circCorrT]| (the reference's separable
    prior, |Re| as in getNextParameterCovariance), so the field is
    chol(P0) . F^-1[sqrt(rho) F[white]] with orthonormal transforms."""
    import scipy.fft as sfft

    Fxy = np.fft.rfft2(corr_xy.astype(np.float64))               # (nyp, cnxp)
    Ft = np.fft.fft(circ_t.astype(np.float64))                    # (nzp,)
    rho = np.abs((Ft[:, None, None] * Fxy[None, :, :]).real)
    amp = np.sqrt(rho).astype(np.float32)
    L = np.linalg.cholesky(P0)
    fields = []
    for a in range(3):
        w = rng.standard_normal((nzp, nyp, nxp), dtype=np.float32)
        W = sfft.rfftn(w, norm="ortho", workers=-1)
        W *= amp
        fields.append(sfft.irfftn(W, s=(nzp, nyp, nxp), norm="ortho", workers=-1).astype(np.float32))
    out = []
    for a in range(3):
        f = np.zeros((nzp, nyp, nxp), dtype=np.float32)
        for b in range(a + 1):
            f += np.float32(L[a, b]) * fields[b]
        out.append(f + np.float32(mean[a]))
    return out


def synt_seismic(m, A, wavelets, nz, nzp):
    """CravaResult::ComputeSyntSeismic (src/cravaresult.cpp:2312-2378): impedance
    A_l . m, cyclic backward difference along z, times the complex conjugate of the
    wavelet spectrum, inverse transform (scaled 1/nzp), first nz samples."""
    import scipy.fft as sfft

    out = []
    for l in range(A.shape[0]):
        imp = (np.float32(A[l, 0]) * m[0][:nz] + np.float32(A[l, 1]) * m[1][:nz]
               + np.float32(A[l, 2]) * m[2][:nz]).astype(np.float32)
        vec = np.empty((nzp,) + imp.shape[1:], dtype=np.float32)
        vec[:nz] = imp
        if nzp > nz:
            fac = 1.0 / (nzp - nz - 1) if nzp - nz - 1 > 0 else 0.0
            for k in range(nz, nzp):
                vec[k] = fac * ((k - nz) * imp[0] + (nzp - k - 1) * imp[nz - 1])
        diff = vec - np.roll(vec, 1, axis=0)
        R = sfft.rfft(diff, axis=0, workers=-1)
        Wc = np.fft.rfft(wavelets[l].astype(np.float64))
        R *= np.conj(Wc).astype(np.complex64)[:, None, None]
        s = sfft.irfft(R, n=nzp, axis=0, workers=-1)[:nz].astype(np.float32)
        out.append(s)
    return out


def make_block(spec: BlockSpec) -> Block:
    nxp, nyp, nzp = spec.padded()
    nx, ny, nz = spec.nx, spec.ny, spec.nz
    rng = np.random.default_rng(spec.seed)
    nth = spec.ntheta
    A = reflection_matrix(spec.theta_deg, spec.vsvp)
    sd = np.asarray(spec.std, dtype=np.float64)
    C = np.eye(3)
    C[0, 1] = C[1, 0] = spec.corr[0]
    C[0, 2] = C[2, 0] = spec.corr[1]
    C[1, 2] = C[2, 1] = spec.corr[2]
    P0 = (sd[:, None] * sd[None, :] * C).astype(np.float32).astype(np.float64)
    cxy = corr_xy_surface(nxp, nyp, spec.dx, spec.dy, spec.lateral_range)
    pct = prior_corr_t(nzp, spec.dt, spec.temporal_range)
    low_int_cut = int(math.floor(spec.low_cut * (nzp * 0.001 * spec.dt)))
    cct = circ_corr_t(pct, low_int_cut, nzp)
    wav = np.stack([wavelet_fft_order(nzp, spec.dt, f) for f in spec.peak_hz])
    wnorm = np.array([wavelet_norm(w) for w in wav], dtype=np.float32)

    m = _prior_realisation(rng, nx, ny, nz, nxp, nyp, nzp, cxy, cct, P0, spec.mean)
    sig = synt_seismic([f[:, :ny, :nx] for f in m], A, wav, nz, nzp)
    data = np.empty((nth, nzp, nyp, 2 * (nxp // 2 + 1)), dtype=np.float32)
    data_var = np.zeros(nth)
    for l in range(nth):
        s = sig[l]
        var_sig = float(np.mean(s.astype(np.float64) ** 2))
        noisy = s + rng.standard_normal(s.shape, dtype=np.float32) * np.float32(math.sqrt(var_sig / spec.sn[l]))
        data[l] = pad_grid(noisy, nxp, nyp, nzp)
        nzv = noisy[noisy != 0.0].astype(np.float32)
        data_var[l] = float(np.sum((nzv * nzv).astype(np.float64)) / max(nzv.size, 1))
    err_var = (data_var / np.asarray(spec.sn, dtype=np.float64)).astype(np.float32).astype(np.float64)
    ang = angular_corr(spec.theta_deg, spec.angular[0], spec.angular[1]).astype(np.float32)
    etc = (np.sqrt(err_var)[:, None] * np.sqrt(err_var)[None, :] * ang).astype(np.float32).astype(np.float64)

    mean = np.stack([pad_grid(np.full((nz, ny, nx), spec.mean[a], dtype=np.float32), nxp, nyp, nzp)
                     for a in range(3)])
    return Block(spec=spec, nx=nx, ny=ny, nz=nz, nxp=nxp, nyp=nyp, nzp=nzp, lz=nz * spec.dt,
                 A=A, err_theta_cov=etc, wavelet=wav, wavelet_norm=wnorm, prior_var0=P0,
                 corr_xy=cxy, prior_corr_t=pct, circ_corr_t=cct, low_int_cut=low_int_cut,
                 mean=mean, data=data, low_cut=spec.low_cut, high_cut=spec.high_cut,
                 wnc=spec.wnc, corr_grad_i=spec.corr_grad_i, corr_grad_j=spec.corr_grad_j,
                 nsim=spec.nsim, seed=spec.seed)


def make_block_fast(spec: BlockSpec, data: bool = True) -> Block:
    """Same shapes, operators and priors as make_block, with the seismic replaced by seeded
    white noise of seismic amplitude (no prior realisation, no forward model); data=False
    leaves the data and prior-mean grids out (None) for callers that supply their own
    buffers.  The inversion's cost does not depend on the data values, so throughput runs over many
    blocks use this to keep input synthesis short."""
    nxp, nyp, nzp = spec.padded()
    nx, ny, nz = spec.nx, spec.ny, spec.nz
    rng = np.random.default_rng(spec.seed)
    nth = spec.ntheta
    A = reflection_matrix(spec.theta_deg, spec.vsvp)
    sd = np.asarray(spec.std, dtype=np.float64)
    C = np.eye(3)
    C[0, 1] = C[1, 0] = spec.corr[0]
    C[0, 2] = C[2, 0] = spec.corr[1]
    C[1, 2] = C[2, 1] = spec.corr[2]
    P0 = (sd[:, None] * sd[None, :] * C).astype(np.float32).astype(np.float64)
    cxy = corr_xy_surface(nxp, nyp, spec.dx, spec.dy, spec.lateral_range)
    pct = prior_corr_t(nzp, spec.dt, spec.temporal_range)
    low_int_cut = int(math.floor(spec.low_cut * (nzp * 0.001 * spec.dt)))
    cct = circ_corr_t(pct, low_int_cut, nzp)
    wav = np.stack([wavelet_fft_order(nzp, spec.dt, f) for f in spec.peak_hz])
    wnorm = np.array([wavelet_norm(w) for w in wav], dtype=np.float32)
    rnxp = 2 * (nxp // 2 + 1)
    amp = np.float32(0.02)
    grids = data
    data = mean = None
    if grids:
        data = np.zeros((nth, nzp, nyp, rnxp), dtype=np.float32)
        for l in range(nth):
            data[l, :, :, :nxp] = rng.standard_normal((nzp, nyp, nxp), dtype=np.float32) * amp
        mean = np.zeros((3, nzp, nyp, rnxp), dtype=np.float32)
        for a in range(3):
            mean[a, :, :, :nxp] = np.float32(spec.mean[a])
    err_var = np.full(nth, float(amp) ** 2) / np.asarray(spec.sn, dtype=np.float64)
    ang = angular_corr(spec.theta_deg, spec.angular[0], spec.angular[1]).astype(np.float32)
    etc = (np.sqrt(err_var)[:, None] * np.sqrt(err_var)[None, :] * ang).astype(np.float32).astype(np.float64)
    return Block(spec=spec, nx=nx, ny=ny, nz=nz, nxp=nxp, nyp=nyp, nzp=nzp, lz=nz * spec.dt,
                 A=A, err_theta_cov=etc, wavelet=wav, wavelet_norm=wnorm, prior_var0=P0,
                 corr_xy=cxy, prior_corr_t=pct, circ_corr_t=cct, low_int_cut=low_int_cut,
                 mean=mean, data=data, low_cut=spec.low_cut, high_cut=spec.high_cut,
                 wnc=spec.wnc, nsim=spec.nsim, seed=spec.seed)


def rel_thick_surface(nxp: int, nyp: int, lo: float = 0.75, hi: float = 1.3, seed: int = 3) -> np.ndarray:
    """A smooth Simbox::getRelThick surface over the padded lateral grid, (nyp, nxp) float64
    in [lo, hi]: a non-constant-thickness block (top and base not parallel)."""
    rng = np.random.default_rng(seed)
    x = np.arange(nxp)[None, :] / nxp
    y = np.arange(nyp)[:, None] / nyp
    a, b = rng.uniform(0, 2 * np.pi, 2)
    s = 0.5 + 0.25 * np.sin(2 * np.pi * x + a) + 0.25 * np.cos(2 * np.pi * 1.5 * y + b)
    return (lo + (hi - lo) * s).astype(np.float64)


def with_rel_thick(blk: Block, seed: int = 3, threshold: float = 0.0) -> Block:
    """The block with a non-constant thickness surface (rel_thick, min_rel_thick over the
    simbox) and the interpolateSeismic energy threshold."""
    rt = rel_thick_surface(blk.nxp, blk.nyp, seed=seed)
    return dataclasses.replace(blk, rel_thick=rt, min_rel_thick=float(rt[:blk.ny, :blk.nx].min()),
                               energy_threshold=threshold)


def wavelet3d_model(blk: Block, theta_deg, seed: int = 5, halpha: bool = True, missing: bool = True,
                    flat: bool = False) -> dict:
    """Synthetic 3D-wavelet inputs for a block (the crava_wavelet3d_desc fields, keyed as
    api.Job.set_wavelet_3d takes them): smooth structure depth gradients of either sign up
    to about 0.4 with a strip of near-zero x gradients (findPhi's small-|a| branches), filter
    surfaces alpha1 = 1 + 0.2 sin(phi) cos(psi) and Halpha in 0.5..3 ms over phi 0..360 and
    psi 0..90 degrees on 30 x 10 degree nodes (with a few missing nodes), and global wavelets
    0.93 times the block's own, each with its norm.  flat: no gradients, theta 0, alpha1 1,
    no Halpha and the block's own wavelets (the neutral model)."""
    rng = np.random.default_rng(seed)
    nth, nx, ny = blk.ntheta, blk.nx, blk.ny
    ni, nj = 13, 10
    phi = np.arange(ni) * 30.0
    psi = np.arange(nj) * 10.0
    if flat:
        return dict(theta=np.zeros(nth, np.float32), alpha1=np.ones((nth, nj, ni), np.float32), halpha=None,
                    filter_geom=(0.0, 0.0, 30.0, 10.0), grad_x=None, grad_y=None,
                    global_wavelet=np.asarray(blk.wavelet, np.float32),
                    global_wavelet_norm=np.asarray(blk.wavelet_norm, np.float32))
    x = np.arange(nx)[None, :] / max(nx - 1, 1)
    y = np.arange(ny)[:, None] / max(ny - 1, 1)
    ph = rng.uniform(0, 2 * np.pi, 4)
    gx = 0.4 * np.sin(2 * np.pi * x + ph[0]) * np.cos(np.pi * y + ph[1])
    gy = 0.4 * np.cos(3 * np.pi * x + ph[2]) * np.sin(2 * np.pi * y + ph[3])
    gx[:, : max(1, nx // 8)] *= 1e-3
    a1 = np.empty((nth, nj, ni), np.float32)
    ha = np.empty((nth, nj, ni), np.float32)
    for l in range(nth):
        a1[l] = 1.0 + 0.2 * np.sin(np.deg2rad(phi)[None, :] + 0.3 * l) * np.cos(np.deg2rad(psi)[:, None])
        ha[l] = rng.uniform(0.0005, 0.003, (nj, ni))
        if missing:
            a1[l, 0, 3] = -999.0
            ha[l, 1, 5] = -999.0
    gw = (0.93 * np.asarray(blk.wavelet, np.float64)).astype(np.float32)
    gnorm = np.sqrt((gw.astype(np.float64) ** 2).sum(axis=1)).astype(np.float32)
    return dict(theta=np.deg2rad(np.asarray(theta_deg, np.float64)).astype(np.float32), alpha1=a1,
                halpha=ha if halpha else None, filter_geom=(0.0, 0.0, 30.0, 10.0),
                grad_x=gx.astype(np.float32), grad_y=gy.astype(np.float32), global_wavelet=gw,
                global_wavelet_norm=gnorm)


# --- the configurations of the benchmark suite -------------------------------------

def config0(seed: int = 11) -> BlockSpec:
    """64x64x128, dt 4 ms, 3 angles 10/20/30 deg, 30 Hz Ricker, S/N 5, 1 realisation."""
    return BlockSpec(seed=seed)


def config1(seed: int = 21) -> BlockSpec:
    """540x540x256, 5 angles 5..45 deg, Ricker 25-35 Hz, lateral range 2000 m, angular
    error correlation 0.3 between neighbouring angles (spherical), 4 realisations."""
    th = (5.0, 15.0, 25.0, 35.0, 45.0)
    # spherical range R with corr(10 deg / R) = 0.3: 1 - 1.5 d + 0.5 d^3 = 0.3
    d = 0.5
    for _ in range(60):
        f = 1 - 1.5 * d + 0.5 * d ** 3 - 0.3
        d -= f / (-1.5 + 1.5 * d * d)
    return BlockSpec(nx=540, ny=540, nz=256, theta_deg=th, peak_hz=(25.0, 27.5, 30.0, 32.5, 35.0),
                     sn=(5.0,) * 5, lateral_range=2000.0, angular=("spherical", 10.0 / d),
                     nsim=4, seed=seed)


def config3(seed: int = 31) -> BlockSpec:
    """768x768x320, 6 angles 5..50 deg, band 2-120 Hz so edge bins are inverted,
    S/N 2..10 across angles, 1 realisation."""
    th = tuple(np.linspace(5.0, 50.0, 6))
    return BlockSpec(nx=768, ny=768, nz=320, theta_deg=th, peak_hz=(30.0,) * 6,
                     sn=tuple(np.linspace(2.0, 10.0, 6)), low_cut=2.0, high_cut=120.0,
                     nsim=1, seed=seed)


def served_specs(n_jobs: int = 48, seed: int = 51, nsim: int = 16) -> list[BlockSpec]:
    """Served stream: grids log-uniform between 64x64x64 and 512x512x256 voxels (2,3,5,7-
    smooth), 3..6 angles, priors as the mixed-size batch."""
    rng = np.random.default_rng(seed)
    xy = np.array(smooth_sizes(64, 512))
    zz = np.array(smooth_sizes(64, 256))
    lo, hi = math.log(64 * 64 * 64), math.log(512 * 512 * 256)
    base = config0()
    out = []
    for b in range(n_jobs):
        target = math.exp(rng.uniform(lo, hi))
        f = (target / (64 * 64 * 64)) ** (1.0 / 3.0)
        nz = int(zz[np.argmin(np.abs(zz - min(256, 64 * f)))])
        nxy = math.sqrt(target / nz)
        nx = int(xy[np.argmin(np.abs(xy - nxy * rng.uniform(0.85, 1.15)))])
        ny = int(xy[np.argmin(np.abs(xy - nxy * rng.uniform(0.85, 1.15)))])
        nth = int(rng.integers(3, 7))
        out.append(BlockSpec(nx=nx, ny=ny, nz=nz, theta_deg=tuple(np.linspace(5.0, 45.0, nth)),
                             peak_hz=(30.0,) * nth, sn=(5.0,) * nth, std=base.std, corr=base.corr,
                             nsim=nsim, seed=seed * 1000 + b))
    return out


def served_stream_specs(n_jobs: int = 48, n_models: int = 6, seed: int = 61, nsim: int = 16) -> list[BlockSpec]:
    """A served stream of fresh requests: n_models interval models (nz smooth in [64, 256],
    3..6 angles 5..45 deg, priors within +-30% of the 64x64x128 block, Ricker 30 Hz) and, per
    request, one model and a lateral shape such that the voxel counts are log-uniform between
    64x64x64 and 512x512x256 (x, y smooth in [64, 512])."""
    rng = np.random.default_rng(seed)
    xy = np.array(smooth_sizes(64, 512))
    zz = np.array(smooth_sizes(64, 256))
    base = config0()
    models = []
    for m in range(n_models):
        nth = int(rng.integers(3, 7))
        jit = lambda v: tuple(float(x) * float(rng.uniform(0.7, 1.3)) for x in v)
        models.append(dict(nz=int(rng.choice(zz)), theta_deg=tuple(np.linspace(5.0, 45.0, nth)),
                           peak_hz=(30.0,) * nth, sn=(5.0,) * nth, std=jit(base.std),
                           corr=tuple(float(np.clip(c * rng.uniform(0.7, 1.3), -0.9, 0.9)) for c in base.corr),
                           lateral_range=base.lateral_range * float(rng.uniform(0.7, 1.3)),
                           temporal_range=base.temporal_range * float(rng.uniform(0.7, 1.3))))
    lo, hi = math.log(64 * 64 * 64), math.log(512 * 512 * 256)
    out = []
    for b in range(n_jobs):
        m = models[int(rng.integers(0, n_models))]
        target = math.exp(rng.uniform(lo, hi))
        nxy = math.sqrt(target / m["nz"])
        nx = int(xy[np.argmin(np.abs(xy - nxy * rng.uniform(0.85, 1.15)))])
        ny = int(xy[np.argmin(np.abs(xy - nxy * rng.uniform(0.85, 1.15)))])
        out.append(BlockSpec(nx=nx, ny=ny, nsim=nsim, seed=seed * 1000 + b, **m))
    return out


def batch_specs(n_blocks: int = 64, seed: int = 41, nsim: int = 16,
                xy_range=(64, 256), z_range=(64, 200)) -> list[BlockSpec]:
    """Mixed-size blocks: nx, ny uniform over smooth sizes in xy_range, nz over z_range,
    2..6 angles, priors within +-30% of the 64x64x128 block."""
    rng = np.random.default_rng(seed)
    xy = smooth_sizes(*xy_range)
    zz = smooth_sizes(*z_range)
    base = config0()
    out = []
    for b in range(n_blocks):
        nth = int(rng.integers(2, 7))
        th = tuple(np.linspace(5.0, 45.0, nth)) if nth > 1 else (20.0,)
        jit = lambda v: tuple(float(x) * float(rng.uniform(0.7, 1.3)) for x in v)
        cr = tuple(float(np.clip(c * rng.uniform(0.7, 1.3), -0.9, 0.9)) for c in base.corr)
        out.append(BlockSpec(nx=int(rng.choice(xy)), ny=int(rng.choice(xy)), nz=int(rng.choice(zz)),
                             theta_deg=th, peak_hz=(30.0,) * nth, sn=(5.0,) * nth,
                             std=jit(base.std), corr=cr,
                             lateral_range=base.lateral_range * float(rng.uniform(0.7, 1.3)),
                             temporal_range=base.temporal_range * float(rng.uniform(0.7, 1.3)),
                             nsim=nsim, seed=seed * 1000 + b))
    return out
