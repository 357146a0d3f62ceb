"""FP64 oracle: a numpy restatement of the reference's FFT-domain AVO inversion.

TEST INFRASTRUCTURE ONLY.  Nothing in the product path imports this module; it is the
checker the CUDA path is compared against (tests, the smoke check and the CPU leg of the
benchmark).

Restated from the reference, in float64 with numpy's pocketfft transforms:

* FFTGrid::fftInPlace / invFFTInPlace            src/fftgrid.cpp:1587-1643
    forward = rfftw3d r2c (unnormalised, e^{-2 pi i}), grid pre-scaled by 1/sqrt(N) unless
    the grid is a COVARIANCE grid; inverse = c2r then x 1/N (COVARIANCE) or 1/sqrt(N).
* FFTGrid::fillInParamCorr / fillInErrCorr       src/fftgrid.cpp:777-828, 878-928
* SeismicParametersHolder::InitializeCorrelations src/seismicparametersholder.cpp:325-351
* SeismicParametersHolder::getNextParameterCovariance  :485-557  (|Re|, Im dropped)
* Wavelet1D diff operators                        src/wavelet1D.cpp:389-500
* Wavelet::getCAmp / findNorm                     src/wavelet.cpp:318-334, 882-900
* AVOInversion::computePostMeanResidAndFFTCov     src/avoinversion.cpp:794-1091
    K = diag(conj(W) kD) A (:948-975), getNextErrorVariance (:1236-1272), per-bin posterior
    (:1016-1082) with lib_matrCholCpx (libs/lib/lib_matr.c:78-168) and
    lib_matrAXeqBMatCpx (:330-378)
* AVOInversion::simulate                          src/avoinversion.cpp:1354-1526
    lib_matrCholCpx(3) + lib_matrProdCholVec (libs/lib/lib_matr.c:453-471)
* SeismicParametersHolder::updatePriorVar / createPostCov00   :1031-1067

Layout: real grids are (nzp, nyp, rnxp) float arrays (FFTGrid index i + rnxp*j +
rnxp*nyp*k); spectra are (nzp, nyp, cnxp) complex arrays (index i + cnxp*j + cnxp*nyp*k).
"""
from __future__ import annotations

import math

import numpy as np

TOL = 1e-20  # libs/lib/lib_matr.c:20


# ---------------------------------------------------------------- transforms

def fft_in_place(real_padded: np.ndarray, nxp: int, covariance: bool) -> np.ndarray:
    """FFTGrid::fftInPlace (src/fftgrid.cpp:1587-1612) in float64."""
    x = real_padded[..., :nxp].astype(np.float64)
    N = x.size
    if not covariance:
        x = x / math.sqrt(N)
    return np.fft.rfftn(x, axes=(0, 1, 2))


def inv_fft_in_place(spec: np.ndarray, nxp: int, covariance: bool) -> np.ndarray:
    """FFTGrid::invFFTInPlace (src/fftgrid.cpp:1615-1643): c2r (unnormalised), then the
    1/N (COVARIANCE) or 1/sqrt(N) scale.  Returns the padded real layout."""
    nzp, nyp, cnxp = spec.shape
    out = np.fft.irfftn(spec, s=(nzp, nyp, nxp), axes=(0, 1, 2))  # = c2r / N
    N = nzp * nyp * nxp
    if not covariance:
        out = out * math.sqrt(N)
    res = np.zeros((nzp, nyp, 2 * cnxp))
    res[..., :nxp] = out
    return res


# ---------------------------------------------------------------- prior grids

def fill_param_corr(corr_xy, circ_corr_t, nxp, nyp, nzp, grad_i=0.0, grad_j=0.0):
    """FFTGrid::fillInParamCorr (src/fftgrid.cpp:878-928), float arithmetic as the
    reference; returns (nzp, nyp, nxp) float32."""
    f32 = np.float32
    i = np.arange(nxp)
    j = np.arange(nyp)
    ci = np.where(i < -(i - nxp), i, i - nxp)
    cj = np.where(j < -(j - nyp), j, j - nyp)
    out = np.empty((nzp, nyp, nxp), dtype=np.float32)
    cxy = corr_xy.astype(np.float32)
    ct = circ_corr_t.astype(np.float32)
    for k in range(nzp):
        subk = (f32(k) + (ci[None, :] * f32(grad_i)).astype(np.float32)
                + (cj[:, None] * f32(grad_j)).astype(np.float32)).astype(np.float32)
        basek = np.floor(subk).astype(np.int64)
        subk = (subk - basek).astype(np.float32)
        basek = np.mod(basek, nzp)
        nxt = np.where(basek != nzp - 1, basek + 1, 0)
        v = ((f32(1) - subk) * ct[basek] + subk * ct[nxt]).astype(np.float32)
        out[k] = (v * cxy).astype(np.float32)
    return out


def fill_err_corr(corr_xy, nxp, nyp, nzp, grad_i=0.0, grad_j=0.0):
    """FFTGrid::fillInErrCorr (src/fftgrid.cpp:777-828): corrXY at the (rotated) k=0 lag,
    subK = k + cycleI*gradI + cycleJ*gradJ in float left to right as the reference."""
    f32 = np.float32
    cxy = corr_xy.astype(f32)
    i = np.arange(nxp)
    j = np.arange(nyp)
    ci = np.where(i < -(i - nxp), i, i - nxp).astype(f32)
    cj = np.where(j < -(j - nyp), j, j - nyp).astype(f32)
    ti = (ci * f32(grad_i)).astype(f32)[None, :]
    tj = (cj * f32(grad_j)).astype(f32)[:, None]
    out = np.zeros((nzp, nyp, nxp), dtype=f32)
    for k in range(nzp):
        sub = ((f32(k) + ti).astype(f32) + tj).astype(f32)                 # (nyp, nxp)
        hit = (np.abs(sub) < f32(1.0)) | (np.abs((sub - f32(nzp)).astype(f32)) < f32(1.0))
        base = np.trunc(sub).astype(np.int64)
        s = (sub - base.astype(f32)).astype(f32)
        base = np.where(base < -1, base + nzp, base)
        base = np.where(base >= 1, base - nzp, base)
        s = np.where(base < 0, (f32(1) - s).astype(f32), s)
        out[k] = np.where(hit, ((f32(1) - s).astype(f32) * cxy).astype(f32), f32(0))
    return out


def fill_err_corr_zero_grad(corr_xy, nxp, nyp, nzp):
    """fillInErrCorr with zero correlation gradients: corrXY on the k = 0 plane only."""
    out = np.zeros((nzp, nyp, nxp), dtype=np.float32)
    out[0] = corr_xy.astype(np.float32)
    return out


def prior_cov_grids(blk, full_grid=True):
    """The six prior covariance grids (COVARIANCE type) of InitializeCorrelations
    (src/seismicparametersholder.cpp:334-348): fillInParamCorr x priorVar0(a,b), in the
    order Vp, Vs, Rho, VpVs, VpRho, VsRho."""
    base = fill_param_corr(blk.corr_xy, blk.circ_corr_t, blk.nxp, blk.nyp, blk.nzp,
                           blk.corr_grad_i, blk.corr_grad_j)
    pv = blk.prior_var0
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    return [(base * np.float32(pv[a, b])).astype(np.float32) for a, b in pairs], pairs


# ---------------------------------------------------------------- wavelets / per-kz

def wavelet_spectrum_full(w: np.ndarray) -> np.ndarray:
    """Wavelet::fft1DInPlace + getCAmp(k) with the Hermitian mirror for k >= cnzp
    (src/wavelet.cpp:255-270, 318-334): the full DFT (e^{-2 pi i}) at every k."""
    return np.fft.fft(w.astype(np.float64))


def diff_forward(w):
    """Wavelet1D(w, FIRSTORDERFORWARDDIFF) (src/wavelet1D.cpp:447-452)."""
    return np.roll(w, -1) - w


def diff_backward(w):
    return w - np.roll(w, 1)


def diff_central(w):
    return 0.5 * (np.roll(w, -1) - np.roll(w, 1))


def real_norm(w):
    """Wavelet::findNorm for a real vector (src/wavelet.cpp:882-889)."""
    return math.sqrt(float(np.sum(np.asarray(w, dtype=np.float64) ** 2)))


def per_kz_operators(blk):
    """Per-kz quantities of computePostMeanResidAndFFTCov's constant-thickness branch
    (src/avoinversion.cpp:845-975):
      K[k]   = diag(conj(W_l(k)) * kD(k)) A          (fillkW, ProdScalVec, ProdDiagCpxR)
      e1[k]  = conj(W_l(k)) / |w_l|                   (fillkWNorm on seisWaveletForNorm)
      e2[k]  = conj(E3_l(k)) / |e3_l|                 (fillkWNorm on errorSmooth3)
      e3[k]  = 1                                      (lib_matrFillOnesVecCpx)
      inv[k] = lowCut*minRelThick < f(k) < highCut    (:946, :1029)
    """
    nzp, nth = blk.nzp, blk.ntheta
    d1 = np.zeros(nzp)
    d1[0] = -1.0
    d1[nzp - 1] = 1.0
    kD = np.fft.fft(d1)
    K = np.zeros((nzp, nth, 3), dtype=np.complex128)
    e1 = np.zeros((nzp, nth), dtype=np.complex128)
    e2 = np.zeros((nzp, nth), dtype=np.complex128)
    e3 = np.ones((nzp, nth))
    nonconst = getattr(blk, "rel_thick", None) is not None
    kD3 = np.fft.fft(diff_central(diff_backward(d1)))
    for l in range(nth):
        w = blk.wavelet[l].astype(np.float64)
        W = wavelet_spectrum_full(w)
        es3 = diff_central(diff_backward(diff_forward(w)))
        if nonconst:
            # non-constant thickness (src/avoinversion.cpp:976-1014): K = kD A, errMult1 =
            # 1/|w|, errMult2 = kD3/|errorSmooth3|, errMult3 = fillInverseAbskWRobust
            K[:, l, :] = kD[:, None] * blk.A[l][None, :]
            e1[:, l] = 1.0 / float(blk.wavelet_norm[l])
            e2[:, l] = kD3 / real_norm(es3)
            e3[:, l] = inverse_abs_kw_robust(W, float(blk.wavelet_norm[l]))
            continue
        kW = np.conj(W) * kD
        K[:, l, :] = kW[:, None] * blk.A[l][None, :]
        e1[:, l] = np.conj(W) / float(blk.wavelet_norm[l])
        e2[:, l] = np.conj(np.fft.fft(es3)) / real_norm(es3)
    inv = invert_mask(blk)
    return K, e1, e2, e3, inv


def camp_scaled32(c: np.ndarray, k, scale):
    """Wavelet::getCAmp(k, scale) (src/wavelet.cpp:337-382) for 0 <= k < cnzp: linear
    interpolation of the half spectrum c (complex64, cnzp entries) at k / scale, divided
    by scale, in float32 with the reference's operation order.  k and scale broadcast."""
    cn = c.shape[0]
    f32 = np.float32
    k = np.asarray(k)
    scale = np.asarray(scale, dtype=f32)
    om = k.astype(f32) / scale
    valid = om < f32(cn)
    lo = np.where(valid, np.floor(om), 0).astype(np.int64)
    hi = lo + 1
    hi = np.where(hi >= cn, hi - 1, hi)
    d = (om - lo.astype(f32)).astype(f32)
    e = (f32(1.0) - d).astype(f32)
    cr, ci = c.real.astype(f32), c.imag.astype(f32)
    re = (cr[lo] * e + cr[hi] * d) / scale
    im = (ci[lo] * e + ci[hi] * d) / scale
    re = np.where(valid, re, f32(0))
    im = np.where(valid, im, f32(0))
    return re.astype(f32), im.astype(f32)


def interp_scaled32(at, cn: int, k, scale):
    """Wavelet::getCAmp(k, scale) as camp_scaled32 for a spectrum given by at(m) -> (re, im)
    float32 arrays (m an index array broadcasting with k and scale)."""
    f32 = np.float32
    k = np.asarray(k)
    scale = np.asarray(scale, dtype=f32)
    om = k.astype(f32) / scale
    valid = om < f32(cn)
    lo = np.where(valid, np.floor(om), 0).astype(np.int64)
    hi = lo + 1
    hi = np.where(hi >= cn, hi - 1, hi)
    d = (om - lo.astype(f32)).astype(f32)
    e = (f32(1.0) - d).astype(f32)
    ar, ai = at(lo)
    br, bi = at(hi)
    re = ((ar * e).astype(f32) + (br * d).astype(f32)).astype(f32) / scale
    im = ((ai * e).astype(f32) + (bi * d).astype(f32)).astype(f32) / scale
    re = np.where(valid, re, f32(0))
    im = np.where(valid, im, f32(0))
    return re.astype(f32), im.astype(f32)


def shift_scale32(c: np.ndarray, ish, gain, m, nzp: int):
    """Wavelet1D::shiftAndScale (src/wavelet1D.cpp:580-602) at bins m of the half spectrum c
    (complex64): multiplier float(gain cos(a)) + i float(gain sin(-a)) with
    a = 2 (pi iShift m) / float(nzp) in double, product in float32.  Returns (re, im)."""
    m = np.asarray(m)
    return shift_scale_vals32(c.real.astype(np.float32)[m], c.imag.astype(np.float32)[m], ish, gain, m, nzp)


def shift_scale_vals32(cr, ci, ish, gain, m, nzp: int):
    """shift_scale32 on the values (cr, ci) of bins m (float32 arrays)."""
    f32 = np.float32
    m = np.asarray(m)
    a = 2.0 * (math.pi * np.asarray(ish, dtype=f32).astype(np.float64) * m.astype(np.float64)) / float(f32(nzp))
    g = np.asarray(gain, dtype=f32).astype(np.float64)
    mr = (g * np.cos(a)).astype(f32)
    mi = (g * np.sin(-a)).astype(f32)
    return ((mr * cr).astype(f32) - (mi * ci).astype(f32)).astype(f32), \
        ((mi * cr).astype(f32) + (mr * ci).astype(f32)).astype(f32)


def inverse_abs_kw_robust(W: np.ndarray, wnorm: float) -> np.ndarray:
    """AVOInversion::fillInverseAbskWRobust (src/avoinversion.cpp:1296-1322): per kz,
    1/sqrt(max(|W(k)|^2, |W(k; 0.999)|^2)) in float32 (W the full spectrum; a large
    number where both vanish)."""
    n = W.shape[0]
    cn = n // 2 + 1
    f32 = np.float32
    c = W[:cn].astype(np.complex64)
    k = np.arange(n)
    refk = np.where(k < cn, k, n - k)
    v = W.astype(np.complex64)
    m = (v.real * v.real + v.imag * v.imag).astype(f32)
    fr, fi = camp_scaled32(c, refk, f32(0.999))
    mf = (fr * fr + fi * fi).astype(f32)
    mx = np.maximum(m, mf)
    big = f32(wnorm) * f32(n) * f32(n) * f32(100.0)
    with np.errstate(divide="ignore"):
        r = np.where(mx > 0, (1.0 / np.sqrt(mx)).astype(f32), big)
    return r.astype(np.float64)


# ---------------------------------------------------------------- non-constant thickness

def dist_to_boundary(i: int, n: int, np_: int) -> float:
    """FFTGrid::getDistToBoundary (src/fftgrid.cpp:1158-1197), float32."""
    if i < n:
        return 0.0
    taper = np.float32(min(n, np_ - n) / 2.1)
    below, above = np_ - i, i - (n - 1)
    return float(np.float32(above) / taper if above < below else np.float32(below) / taper)


def fill_number(i: int, n: int, np_: int) -> int:
    """FFTGrid::getFillNumber (src/fftgrid.cpp:1103-1141)."""
    if i < n:
        return i
    below, above = np_ - i - 1, i - n + 1
    return max(n - above, n // 2) if above < below else min(below, n // 2)


def thick_tables(blk):
    """Per-angle tables of AVOInversion::computeAdjustmentFactor (src/avoinversion.cpp:630-719)
    over kz < cnzp, float32 where the reference computes in float: the wavelet half
    spectrum, the band-normalised spectrum of errorSmooth3 (with the RMISSING that
    multiplyRAmpByConstant writes into the floats at index >= nzp, src/wavelet.cpp:507-515),
    |Re| of the reflection-coefficient covariance spectrum (:369-401) and the scalars."""
    f32 = np.float32
    n, nth = blk.nzp, blk.ntheta
    cn = n // 2 + 1
    dz = f32(blk.lz / blk.nz)
    dOmega = f32(1.0 / float(f32(n * dz) * 0.001))
    loI = max(0, int(np.floor(f32(blk.low_cut) / dOmega)))
    hiI = min(cn, int(np.ceil(f32(blk.high_cut) / dOmega)))
    maxfreq = f32((n // 2) * 1000.0 * blk.nz) / f32(blk.lz * n)
    circ = blk.circ_corr_t.astype(f32)
    corrT = np.zeros(n, dtype=f32)
    for i in range(n):
        refk = i if i < n // 2 + 1 else n - i
        corrT[i] = circ[refk] / circ[0] if refk < blk.nz else f32(0)
    out = {"wamp": [], "es3": [], "tau2": [], "wn2": [], "modW": [], "err_var": []}
    for l in range(nth):
        wf = blk.wavelet[l].astype(f32)
        W = np.fft.fft(wf.astype(np.float64))
        f1 = (np.roll(wf, -1) - wf).astype(f32)
        f2 = (f1 - np.roll(f1, 1)).astype(f32)
        f3 = (0.5 * (np.roll(f2, -1) - np.roll(f2, 1)).astype(np.float64)).astype(f32)
        E3 = np.fft.fft(f3.astype(np.float64))[:cn].astype(np.complex64)
        fac = 1.0 / n
        sq = (E3.real * E3.real + E3.imag * E3.imag).astype(f32)
        norm2 = 0.0
        for i in range(loI, hiI):
            norm2 += 2.0 * fac * float(sq[i])
        if loI == 0:
            norm2 -= fac * float(sq[0])
        c3 = f32(1.0) / f32(np.sqrt(norm2))
        es3 = (E3.real * c3).astype(f32) + 1j * (E3.imag * c3).astype(f32)
        es3 = es3.astype(np.complex64)
        out.setdefault("es3_last", []).append(es3[cn - 1])
        es3.imag[cn - 1] = -99999.0
        if n % 2 == 0:
            es3.real[cn - 1] = -99999.0
        Al = blk.A[l].astype(f32)
        pv = blk.prior_var0
        eiVar = 0.0
        for a in range(3):
            for b in range(3):
                eiVar += float(Al[a] * f32(pv[a, b]) * Al[b])
        rc = (eiVar * corrT.astype(np.float64)).astype(f32)
        first, prev = rc[0], rc[n - 1]
        for i in range(n - 1):
            curr, nxt = rc[i], rc[i + 1]
            rc[i] = f32(2) * curr - nxt - prev
            prev = curr
        rc[n - 1] = f32(2) * rc[n - 1] - first - prev
        RC = np.fft.fft(rc.astype(np.float64))[:cn]
        norm = f32(blk.wavelet_norm[l])
        modW = norm * norm
        modW = f32(modW * (maxfreq / f32(blk.high_cut)))
        out["wamp"].append(W[:cn].astype(np.complex64))
        out["es3"].append(es3)
        out["tau2"].append(np.abs(RC.real.astype(f32)))
        out["wn2"].append(f32(norm * norm))
        out["modW"].append(modW)
        out["err_var"].append(f32(blk.err_theta_cov[l, l]))
    return out


def adjustment_factor(tab, l: int, sf, k) -> np.ndarray:
    """computeAdjustmentFactor (src/avoinversion.cpp:674-712) of angle l at kz k (< cnzp)
    for traces stretched by sf (float32), local wavelet = global wavelet; float32 with the
    reference's operation order.  sf and k broadcast; returns complex128."""
    f32 = np.float32
    wa, es = tab["wamp"][l], tab["es3"][l]
    wn2, modW, ev = tab["wn2"][l], tab["modW"][l], tab["err_var"][l]
    wnc = f32(tab["wnc"])
    k = np.asarray(k)
    lr, li = camp_scaled32(wa, k, sf)
    wLoc2 = (lr * lr + li * li).astype(f32)
    gr, gi = wa.real.astype(f32)[k], wa.imag.astype(f32)[k]
    wGlob2 = (gr * gr + gi * gi).astype(f32)
    er, ei = camp_scaled32(es, k, sf)
    sL = (wLoc2 / wn2 + (er * er + ei * ei)).astype(f32)
    sgr, sgi = es.real.astype(f32)[k], es.imag.astype(f32)[k]
    sG = (wGlob2 / wn2 + (sgr * sgr + sgi * sgi)).astype(f32)
    c = (f32(1.0) - wnc) * f32(0.5)
    s2L = (ev * (wnc + c * sL)).astype(f32)
    s2G = (ev * (wnc + c * sG)).astype(f32)
    tau2 = tab["tau2"][l][k]
    tm = f32(0.05) * modW
    wG2A = np.where(wGlob2 < tm, f32(0.5) * (wGlob2 + tm), wGlob2).astype(f32)
    wL2A = np.where(wLoc2 < tm, f32(0.5) * (wLoc2 + tm), wLoc2).astype(f32)
    tg = (f32(0.05) * wG2A).astype(f32)
    adj = wL2A < tg
    wL2A = np.where(adj, f32(0.5) * (wLoc2 + tg), wL2A).astype(f32)
    with np.errstate(divide="ignore", invalid="ignore"):
        s2L = np.where(adj, s2L * (wL2A / wLoc2), s2L).astype(f32)
        dL = (tau2 * wL2A + s2L).astype(f32)
        q = (wG2A / (tau2 * wGlob2 + s2G)).astype(f32)
        fr = ((lr / dL) / q).astype(f32)
        fi = ((li / dL) / q).astype(f32)
    return fr.astype(np.float64) + 1j * fi.astype(np.float64)


def adjustment_factor_local(tab, l: int, sf, k, ish, gn, nzp: int, w3=None) -> np.ndarray:
    """computeAdjustmentFactor (src/avoinversion.cpp:630-719) for traces whose local wavelet
    carries a shift ish (samples) and a gain gn (createLocalWavelet1D + shiftAndScale,
    src/wavelet1D.cpp:518-602): wLoc and eSkLoc from the shifted and scaled spectra stretched
    by sf, eSkGlob from the same spectra unstretched, wGlob from the global wavelet.  The
    local errorSmooth3 is the global one turned by the unit-modulus multiplier (its band
    normalisation removes the gain) with the RMISSING entry at cnzp - 1 kept; the
    reference's round trip of the local wavelet through the time domain is not restated.
    float32 in the reference's operation order; sf, k, ish, gn broadcast.  w3: 3D wavelets
    (wavelet3d_params of the angle: per-trace mult, H, wn2, gam broadcasting with ish, and the
    global wavelet's half spectrum wglob, its modW and the bin spacing den); the local spectra
    then carry the dip factor (dip_factor32), errorSmooth3 also gamma, the norm is the adjusted
    wavelet's and wGlob the global wavelet's."""
    f32 = np.float32
    wa, es = tab["wamp"][l], tab["es3"][l]
    es_last = tab["es3_last"][l]
    cn = wa.shape[0]
    wn2, modW, ev = tab["wn2"][l], tab["modW"][l], tab["err_var"][l]
    if w3 is not None:
        wn2, modW = w3["wn2"], f32(w3["modW"])
    wnc = f32(tab["wnc"])
    k = np.asarray(k)
    es_true = es.copy()
    es_true[cn - 1] = es_last

    def wl(m):
        m = np.asarray(m)
        cr, ci = wa.real.astype(f32)[m], wa.imag.astype(f32)[m]
        if w3 is not None:
            f = dip_factor32(w3["den"], m, w3["mult"], w3["H"])
            cr, ci = (cr * f).astype(f32), (ci * f).astype(f32)
        return shift_scale_vals32(cr, ci, ish, gn, m, nzp)

    def el(m):
        m = np.asarray(m)
        cr, ci = es_true.real.astype(f32)[m], es_true.imag.astype(f32)[m]
        if w3 is not None:
            f = dip_factor32(w3["den"], m, w3["mult"], w3["H"])
            cr = ((cr * f).astype(f32) * w3["gam"]).astype(f32)
            ci = ((ci * f).astype(f32) * w3["gam"]).astype(f32)
        r, i = shift_scale_vals32(cr, ci, ish, f32(1.0), m, nzp)
        last = np.asarray(m) == cn - 1
        i = np.where(last, f32(-99999.0), i).astype(f32)
        if nzp % 2 == 0:
            r = np.where(last, f32(-99999.0), r).astype(f32)
        return r, i

    lr, li = interp_scaled32(wl, cn, k, sf)
    wLoc2 = (lr * lr + li * li).astype(f32)
    er, ei = interp_scaled32(el, cn, k, sf)
    sL = (wLoc2 / wn2 + (er * er + ei * ei)).astype(f32)
    gr, gi = wl(np.broadcast_to(k, np.broadcast(k, ish).shape))
    sgr, sgi = el(np.broadcast_to(k, np.broadcast(k, ish).shape))
    sG = ((gr * gr + gi * gi).astype(f32) / wn2 + (sgr * sgr + sgi * sgi)).astype(f32)
    c = (f32(1.0) - wnc) * f32(0.5)
    s2L = (ev * (wnc + c * sL)).astype(f32)
    s2G = (ev * (wnc + c * sG)).astype(f32)
    wgs = w3["wglob"] if w3 is not None else wa
    wgr, wgi = wgs.real.astype(f32)[k], wgs.imag.astype(f32)[k]
    wGlob2 = (wgr * wgr + wgi * wgi).astype(f32)
    tau2 = tab["tau2"][l][k]
    tm = f32(0.05) * modW
    wG2A = np.where(wGlob2 < tm, f32(0.5) * (wGlob2 + tm), wGlob2).astype(f32)
    wL2A = np.where(wLoc2 < tm, f32(0.5) * (wLoc2 + tm), wLoc2).astype(f32)
    tg = (f32(0.05) * wG2A).astype(f32)
    adj = wL2A < tg
    wL2A = np.where(adj, f32(0.5) * (wLoc2 + tg), wL2A).astype(f32)
    with np.errstate(divide="ignore", invalid="ignore"):
        s2L = np.where(adj, s2L * (wL2A / wLoc2), s2L).astype(f32)
        dL = (tau2 * wL2A + s2L).astype(f32)
        q = (wG2A / (tau2 * wGlob2 + s2G)).astype(f32)
        fr = ((lr / dL) / q).astype(f32)
        fi = ((li / dL) / q).astype(f32)
    return fr.astype(np.float64) + 1j * fi.astype(np.float64)


def dip_factor32(den: float, m, mult, H):
    """Wavelet1D::adjustForAmplitudeEffect (src/wavelet1D.cpp:605-636) at bins m: the factor
    float(multiplyer * float(exp(-pi omega Halpha))) with omega = m / den (den =
    double(nzp dz 1e-3)), or float(multiplyer) where Halpha <= 0.  float32 array."""
    f32 = np.float32
    m = np.asarray(m).astype(np.float64)
    mult = np.asarray(mult, dtype=np.float64)
    H = np.asarray(H, dtype=f32)
    om = m / float(den)
    am = np.exp((-math.pi * om) * H.astype(np.float64)).astype(f32)
    return np.where(H > f32(0), (mult * am.astype(np.float64)).astype(f32), mult.astype(f32)).astype(f32)


def surface_z(z: np.ndarray, geom, x: float, y: float) -> float:
    """NRLib::RegularSurface<float>::GetZ (libs/nrlib/surface/regularsurface.hpp:367-394 with
    GetCorners :670-703, FindGeneralIndex :640-644, CellRelX/Y :851-863, GetBilinearZ :328-337,
    GetBilinearZMissingCorners :340-363) on z (nj, ni) with geom = (x0, y0, dx, dy); -999 is
    missing.  Returns a float32 value."""
    f32 = np.float32
    miss = f32(-999.0)
    nj, ni = z.shape
    x0, y0, dx, dy = (float(v) for v in geom)
    fx, fy = (x - x0) / dx, (y - y0) / dy
    i, j = int(math.floor(fx)), int(math.floor(fy))
    c = [miss] * 4
    if i + 1 >= 0 and i < ni and j + 1 >= 0 and j < nj:
        if i >= 0 and j >= 0:
            c[0] = f32(z[j, i])
        if i + 1 < ni and j >= 0:
            c[1] = f32(z[j, i + 1])
        if i >= 0 and j + 1 < nj:
            c[2] = f32(z[j + 1, i])
        if i + 1 < ni and j + 1 < nj:
            c[3] = f32(z[j + 1, i + 1])
    nmiss = sum(1 for v in c if v == miss)
    if nmiss == 4:
        return miss
    u, v = math.modf(fx)[0], math.modf(fy)[0]
    if nmiss == 0:
        a = c[0]
        b, cc = f32(c[1] - a), f32(c[2] - a)
        d = f32(f32(f32(c[3] - a) - b) - cc)
        return f32(float(a) + float(b) * u + float(cc) * v + float(d) * u * v)
    w = [(1.0 - u) * (1.0 - v), u * (1.0 - v), (1.0 - u) * v, u * v]
    sm = sw = 0.0
    for q in range(4):
        if c[q] != miss:
            sm += w[q] * float(c[q])
            sw += w[q]
    return miss if sw == 0.0 else f32(sm / sw)


def find_phi(a, b) -> float:
    """Wavelet3D::findPhi (src/wavelet3D.cpp:819-838) of float32 gradients a, b; its float atan
    taken as the double atan rounded to float32."""
    f32 = np.float32
    a, b = f32(a), f32(b)
    eps = 0.001

    def at():
        return float(f32(math.atan(float(f32(b / a)))))
    if a > eps and b >= 0:
        return at()
    if a > eps and b < 0:
        return 2 * math.pi + at()
    if a < -eps:
        return math.pi + at()
    return 0.5 * math.pi if b >= 0 else 1.5 * math.pi


def find_psi(r) -> float:
    """Wavelet3D::findPsi (src/wavelet3D.cpp:841-851)."""
    return math.acos(1.0 / float(r)) if r > 1 else 0.0


def wavelet3d_params(blk, w3):
    """Per angle and unpadded trace the dip adjustment of 3D wavelets (Wavelet3D::
    getLocalStretch / createLocalWavelet1D / dipAdjustWavelet, src/wavelet3D.cpp:328-459):
    phi and psi from the depth gradients, alpha1 and Halpha from the filter surfaces at
    (phi, psi) in degrees, multiplyer = alpha1 cos(psi) cos(theta) (cos of the float angle
    rounded to float32), the stretch float32(cos(psi) cos(theta)), the norm^2 of the adjusted
    wavelet (Wavelet::findNorm by Parseval over its half spectrum in float64, then
    float32(norm)^2) and gamma = 1 / findNormWithinFrequencyBand of the job's normalised
    errorSmooth3 times the dip factor.  w3: dict with theta, alpha1 / halpha (ntheta, nj, ni),
    filter_geom (x0, y0, dx, dy), grad_x / grad_y (ny, nx) or None, global_wavelet (ntheta, nzp),
    global_wavelet_norm.  Returns per angle a dict of (ny, nx) arrays mult, H, stretch, wn2,
    gam and the scalars of adjustment_factor_local (wglob, modW, den)."""
    f32 = np.float32
    nx, ny, n = blk.nx, blk.ny, blk.nzp
    cn = n // 2 + 1
    tab = thick_tables(blk)
    dz = f32(blk.lz / blk.nz)
    den = float(f32(f32(n) * dz)) * 1e-3
    dOmega = f32(1.0 / float(f32(n * dz) * 0.001))
    loI = max(0, int(np.floor(f32(blk.low_cut) / dOmega)))
    hiI = min(cn, int(np.ceil(f32(blk.high_cut) / dOmega)))
    maxfreq = f32((n // 2) * 1000.0 * blk.nz) / f32(blk.lz * n)
    gx = np.zeros((ny, nx), f32) if w3.get("grad_x") is None else np.asarray(w3["grad_x"], f32)
    gy = np.zeros((ny, nx), f32) if w3.get("grad_y") is None else np.asarray(w3["grad_y"], f32)
    k = np.arange(cn)
    wk = np.where((k == 0) | ((k == cn - 1) & (n % 2 == 0)), 1.0, 2.0)
    out = []
    for l in range(blk.ntheta):
        cth = float(f32(math.cos(float(f32(w3["theta"][l])))))
        wa = tab["wamp"][l]
        es = tab["es3"][l].copy()
        es[cn - 1] = tab["es3_last"][l]
        P = {k2: np.zeros((ny, nx), dt) for k2, dt in
             (("mult", np.float64), ("H", f32), ("stretch", f32), ("wn2", f32), ("gam", f32))}
        for j in range(ny):
            for i in range(nx):
                a, b = gx[j, i], gy[j, i]
                phi = find_phi(a, b)
                r = f32(np.sqrt(f32(f32(a * a) + f32(b * b)) + f32(1)))
                psi = find_psi(r)
                cpsi = math.cos(psi) * cth
                xd, yd = phi * 180.0 / math.pi, psi * 180.0 / math.pi
                a1 = surface_z(np.asarray(w3["alpha1"][l]), w3["filter_geom"], xd, yd)
                H = f32(0) if w3.get("halpha") is None else surface_z(np.asarray(w3["halpha"][l]), w3["filter_geom"], xd, yd)
                mult = float(a1) * cpsi
                f = dip_factor32(den, k, mult, H)
                cr, ci = (wa.real.astype(f32) * f).astype(f32), (wa.imag.astype(f32) * f).astype(f32)
                n2 = float(np.sum(wk * (cr.astype(np.float64) ** 2 + ci.astype(np.float64) ** 2)))
                norm = f32(math.sqrt(n2 / n))
                er, ei = (es.real.astype(f32) * f).astype(f32), (es.imag.astype(f32) * f).astype(f32)
                p = (er * er + ei * ei).astype(f32)
                e2 = sum(2.0 * (1.0 / n) * float(p[q]) for q in range(loI, hiI))
                if loI == 0:
                    e2 -= (1.0 / n) * float(p[0])
                P["mult"][j, i] = mult
                P["H"][j, i] = H
                P["stretch"][j, i] = f32(cpsi)
                P["wn2"][j, i] = f32(norm * norm)
                P["gam"][j, i] = f32(1) / f32(math.sqrt(e2))
        gw = np.asarray(w3["global_wavelet"][l], f32)
        P["wglob"] = np.fft.fft(gw.astype(np.float64))[:cn].astype(np.complex64)
        gn_ = f32(w3["global_wavelet_norm"][l])
        P["modW"] = f32(f32(gn_ * gn_) * (maxfreq / f32(blk.high_cut)))
        P["den"] = den
        out.append(P)
    return out


def wavelet_index(i: int, n: int, np_: int) -> int:
    """The unpadded trace whose local wavelet padded trace i uses (src/avoinversion.cpp:525-543)."""
    if i > 3 * n - 1:
        i = 0
    if i > (np_ + n) // 2:
        i = np_ - i
    if i >= n:
        i = 2 * n - i - 1
    return i


def local_wavelet_maps(blk, shift_ms, gain):
    """Per angle and padded trace (ntheta, nyp, nxp) the shift in samples (float(shift) /
    float(dz), dz = lz / nz) and the gain of the local wavelet; -999 entries are no shift and
    unit gain; None grids are none."""
    f32 = np.float32
    nth, nx, ny, nxp, nyp = blk.ntheta, blk.nx, blk.ny, blk.nxp, blk.nyp
    dz = f32(blk.lz / blk.nz)
    ish = np.zeros((nth, ny, nx), dtype=f32)
    gn = np.ones((nth, ny, nx), dtype=f32)
    for l in range(nth):
        if shift_ms is not None and shift_ms[l] is not None:
            sh = np.asarray(shift_ms[l], dtype=f32)
            ish[l] = np.where(sh != f32(-999.0), (sh / dz).astype(f32), f32(0))
        if gain is not None and gain[l] is not None:
            g = np.asarray(gain[l], dtype=f32)
            gn[l] = np.where(g != f32(-999.0), g, f32(1))
    ii = np.array([wavelet_index(i, nx, nxp) for i in range(nxp)])
    jj = np.array([wavelet_index(j, ny, nyp) for j in range(nyp)])
    return ish[:, jj][:, :, ii], gn[:, jj][:, :, ii]


def _w3_padded(blk, P):
    """wavelet3d_params of one angle mapped onto the padded traces (nyp, nxp) by
    wavelet_index; the scalars as they are."""
    ii = np.array([wavelet_index(i, blk.nx, blk.nxp) for i in range(blk.nxp)])
    jj = np.array([wavelet_index(j, blk.ny, blk.nyp) for j in range(blk.nyp)])
    return {k: (v[jj][:, ii] if isinstance(v, np.ndarray) and v.shape == (blk.ny, blk.nx) else v)
            for k, v in P.items()}


def divide_data_by_scale_wavelet(blk, shift_ms=None, gain=None, w3=None) -> np.ndarray:
    """AVOInversion::divideDataByScaleWavelet (src/avoinversion.cpp:484-612) on every data
    grid: per trace (i < nxp, j < nyp) the 1/sqrt(nzp) scale and z taper, r2c along z,
    the adjustment factor inside the band deltaF*k in (lowCut, highCut) with
    deltaF = nz*1000/(relThick*lz*nzp) and zero outside, c2r, 1/sqrt(nzp).  The transforms
    in float64.  shift_ms / gain: per angle (ny, nx) local wavelet grids or None
    (adjustment_factor_local).  w3: 3D wavelets (the wavelet3d_params input dict): the stretch
    becomes float32(relThick * double(local stretch)) (src/avoinversion.cpp:557) and the
    factor adjustment_factor_local's 3D form.  Returns (ntheta, nzp, nyp, rnxp) float64
    (padding columns zero)."""
    f32 = np.float32
    nxp, nyp, nzp, nz = blk.nxp, blk.nyp, blk.nzp, blk.nz
    cn = nzp // 2 + 1
    tab = thick_tables(blk)
    tab["wnc"] = blk.wnc
    rsq = f32(np.sqrt(f32(nzp)))
    taper = np.ones(nzp, dtype=f32)
    for k in range(nzp):
        if k > nz:
            dk = f32(dist_to_boundary(k, nz, nzp))
            taper[k] = max(f32(1) - dk * dk, f32(0))
    rt = np.asarray(blk.rel_thick, dtype=np.float64)            # (nyp, nxp)
    sf = rt.astype(f32)
    deltaF = float(nz) * 1000.0 / (rt * float(blk.lz) * float(nzp))
    k = np.arange(cn)
    fk = deltaF[None] * k[:, None, None]                         # (cn, nyp, nxp)
    band = (fk < float(f32(blk.high_cut))) & (fk > float(f32(blk.low_cut)))
    out = np.zeros((blk.ntheta, nzp, nyp, 2 * (nxp // 2 + 1)))
    local = shift_ms is not None or gain is not None or w3 is not None
    if local:
        ish, gn = local_wavelet_maps(blk, shift_ms, gain)
    w3p = wavelet3d_params(blk, w3) if w3 is not None else None
    for l in range(blk.ntheta):
        v = (blk.data[l][..., :nxp].astype(f32) / rsq).astype(f32) * taper[:, None, None]
        spec = np.fft.rfft(v.astype(np.float64), axis=0)
        if w3p is not None:
            P = _w3_padded(blk, w3p[l])
            sfl = (rt * P["stretch"].astype(np.float64)).astype(f32)
            W3 = {kk: (vv[None] if isinstance(vv, np.ndarray) and vv.ndim == 2 else vv) for kk, vv in P.items()}
            fac = adjustment_factor_local(tab, l, sfl[None], k[:, None, None], ish[l][None], gn[l][None], nzp, w3=W3)
        elif local:
            fac = adjustment_factor_local(tab, l, sf[None], k[:, None, None], ish[l][None], gn[l][None], nzp)
        else:
            fac = adjustment_factor(tab, l, sf[None], k[:, None, None])
        spec = np.where(band, spec * fac, 0.0)
        res = np.fft.irfft(spec, n=nzp, axis=0) * nzp / float(rsq)
        out[l, ..., :nxp] = res
    return out


def residual_synthetics(blk, resid: np.ndarray, shift_ms=None, gain=None, w3=None) -> np.ndarray:
    """AVOInversion::multiplyDataByScaleWaveletAndWriteToFile (src/avoinversion.cpp:721-790)
    on real residual grids resid (ntheta, nzp, nyp, rnxp) (after invFFTInPlace): every trace
    i < nx, j < ny divided by float(sqrt(float(nzp))), r2c along z, times the conjugate of
    its local wavelet's spectrum stretched by relThick (getCAmp(k, sf)), c2r, divided by
    float(sqrt(double(nzp))); the other traces as given.  w3: 3D wavelets (wavelet3d_params'
    input): the local wavelet carries the dip factor and the stretch is float32(relThick) *
    local stretch (:748).  Transforms in float64."""
    f32 = np.float32
    nx, ny, nzp = blk.nx, blk.ny, blk.nzp
    cn = nzp // 2 + 1
    rsq = f32(np.sqrt(f32(nzp)))
    rsq_out = f32(np.sqrt(float(nzp)))
    W = [np.fft.fft(blk.wavelet[l].astype(f32).astype(np.float64))[:cn].astype(np.complex64)
         for l in range(blk.ntheta)]
    rt = getattr(blk, "rel_thick", None)
    sf = (np.asarray(rt, dtype=np.float64)[:ny, :nx].astype(f32) if rt is not None
          else np.ones((ny, nx), dtype=f32))
    ish, gn = local_wavelet_maps(blk, shift_ms, gain)
    k = np.arange(cn)[:, None, None]
    out = np.array(resid, dtype=np.float64, copy=True)
    w3p = wavelet3d_params(blk, w3) if w3 is not None else None
    for l in range(blk.ntheta):
        v = (np.asarray(resid[l][:, :ny, :nx], dtype=f32) / rsq).astype(f32)
        spec = np.fft.rfft(v.astype(np.float64), axis=0)
        sfl = sf
        if w3p is not None:
            P = w3p[l]
            sfl = (sf * P["stretch"]).astype(f32)

        def at(m, l=l):
            m = np.asarray(m)
            cr, ci = W[l].real.astype(f32)[m], W[l].imag.astype(f32)[m]
            if w3p is not None:
                fct = dip_factor32(w3p[l]["den"], m, w3p[l]["mult"][None], w3p[l]["H"][None])
                cr, ci = (cr * fct).astype(f32), (ci * fct).astype(f32)
            return shift_scale_vals32(cr, ci, ish[l][None, :ny, :nx], gn[l][None, :ny, :nx], m, nzp)
        wr, wi = interp_scaled32(at, cn, k, sfl[None])
        spec = spec * (wr.astype(np.float64) - 1j * wi.astype(np.float64))
        out[l][:, :ny, :nx] = np.fft.irfft(spec, n=nzp, axis=0) * nzp / float(rsq_out)
    return out


def plan_trace_interpolation(energy: np.ndarray, nx: int, ny: int, threshold: float):
    """The control flow of FFTGrid::interpolateSeismic / interpolateTrace
    (src/fftgrid.cpp:2349-2480) on one angle's energy map (ny, nx) float32: returns the
    interpolations in the reference's order as (target, [neighbour indices]) with index
    i + nx*j, and the box (imin, imax, jmin, jmax) of good traces."""
    e = np.asarray(energy, dtype=np.float32).reshape(-1)
    n = nx * ny
    total = np.float32(0)
    for q in range(n):
        total = np.float32(total + e[q])
    limit = np.float32(np.float32(threshold) * total / np.float32(n))
    flags = [0] * n
    imin, imax, jmin, jmax, flag = nx, 0, ny, 0, 0
    for q in range(n):
        i, j = q % nx, q // nx
        cur = 1 if e[q] <= limit else 0
        flags[q] = flag + cur
        if cur:
            flag = 2
        else:
            imin, imax, jmin, jmax = min(imin, i), max(imax, i), min(jmin, j), max(jmax, j)
    ops = []

    def interp(index, i, j):
        nb = []
        if i > 0 and flags[index - 1] % 2 == 0:
            nb.append(index - 1)
        if i < nx - 1 and flags[index + 1] % 2 == 0:
            nb.append(index + 1)
        if j > 0 and flags[index - nx] % 2 == 0:
            nb.append(index - nx)
        if j < ny - 1 and flags[index + nx] % 2 == 0:
            nb.append(index + nx)
        if len(nb) > 1:
            ops.append((index, nb))
            flags[index] -= 1
        return flags[index]

    for cur in range(n):
        i, j = cur % nx, cur // nx
        if flags[cur] % 2 == 1 and interp(cur, i, j) % 2 == 0:
            index = cur - 1
            while index >= 0 and flags[index] > 1:
                if flags[index] % 2 == 1:
                    interp(index, index % nx, index // nx)
                index -= 1
            index = max(index, 0) + 1
            while index <= cur and flags[index - 1] == 0:
                if flags[index] > 1:
                    flags[index] -= 2
                index += 1
    return ops, (imin, imax, jmin, jmax)


def interpolate_seismic(grid: np.ndarray, blk, threshold: float) -> np.ndarray:
    """FFTGrid::interpolateSeismic (src/fftgrid.cpp:2349-2437) on one real grid (nzp, nyp,
    rnxp): energies over k < nz in float32 order, the interpolation plan, then
    extrapolateSeismic (:2484-2516) outside the box of good traces.  Returns a new grid."""
    nx, ny, nz, nxp, nyp, nzp = blk.nx, blk.ny, blk.nz, blk.nxp, blk.nyp, blk.nzp
    g = np.array(grid, dtype=np.float64)
    v32 = g[:nz, :ny, :nx].astype(np.float32)
    energy = np.zeros((ny, nx), dtype=np.float32)
    for k in range(nz):
        energy = (energy + v32[k] * v32[k]).astype(np.float32)
    ops, (imin, imax, jmin, jmax) = plan_trace_interpolation(energy, nx, ny, threshold)
    for t, nb in ops:
        s = sum(g[:, q // nx, q % nx] for q in nb)
        g[:, t // nx, t % nx] = s / len(nb)
    if imin > imax or jmin > jmax:
        return g
    dx = np.array([dist_to_boundary(i, nx, nxp) for i in range(nxp)], dtype=np.float32)
    dy = np.array([dist_to_boundary(j, ny, nyp) for j in range(nyp)], dtype=np.float32)
    dzv = np.array([dist_to_boundary(k, nz, nzp) for k in range(nzp)], dtype=np.float32)
    ri = np.clip([fill_number(i, nx, nxp) for i in range(nxp)], imin, imax)
    rj = np.clip([fill_number(j, ny, nyp) for j in range(nyp)], jmin, jmax)
    I = np.arange(nxp)[None, :]
    J = np.arange(nyp)[:, None]
    outside = (I < imin) | (I > imax) | (J < jmin) | (J > jmax)        # (nyp, nxp)
    src = g[:, rj[:, None], ri[None, :]]                               # (nzp, nyp, nxp)
    t = 1.0 - (dx * dx)[None, None, :].astype(np.float64) - (dy * dy)[None, :, None].astype(np.float64) \
        - (dzv * dzv)[:, None, None].astype(np.float64)
    mult = np.maximum(t, 0.0) ** 3
    g[..., :nxp] = np.where(outside[None], mult * src, g[..., :nxp])
    return g


def real_frequency(blk) -> np.ndarray:
    """realFrequency (src/avoinversion.cpp:946), evaluated exactly as the reference:
    (float(nz)*1000.0f) / (lz * nzp) * min(k, nzp-k) in double, stored as float."""
    k = np.arange(blk.nzp)
    kk = np.minimum(k, blk.nzp - k).astype(np.float64)
    nz1000 = float(np.float32(blk.nz) * np.float32(1000.0))
    return (nz1000 / (float(blk.lz) * blk.nzp) * kk).astype(np.float32)


def invert_mask(blk) -> np.ndarray:
    f = real_frequency(blk).astype(np.float64)
    lo = float(np.float32(blk.low_cut)) * float(blk.min_rel_thick)
    hi = float(np.float32(blk.high_cut))
    return (f > lo) & (f < hi)


# ---------------------------------------------------------------- per-bin algebra

def chol_cpx(M: np.ndarray):
    """lib_matrCholCpx (libs/lib/lib_matr.c:78-168) vectorised over leading axes.
    Scales by M[0,0].re, rejects a non-positive scale, a scaled diagonal <= TOL before the
    update and an updated pivot <= TOL.  Returns (L, ok)."""
    n = M.shape[-1]
    fac = M[..., 0, 0].real
    ok = fac > 0
    safe = np.where(ok, fac, 1.0)
    X = M / safe[..., None, None]
    L = np.zeros_like(X)
    for i in range(n):
        ok &= X[..., i, i].real > TOL
        for j in range(i):
            s = np.zeros(X.shape[:-2], dtype=X.dtype)
            for k in range(j):
                s = s + L[..., i, k] * np.conj(L[..., j, k])
            L[..., i, j] = (X[..., i, j] - s) / L[..., j, j]
        r = X[..., i, i].real - sum(np.abs(L[..., i, k]) ** 2 for k in range(i)) if i else X[..., i, i].real
        ok &= r > TOL
        L[..., i, i] = np.sqrt(np.where(r > TOL, r, 1.0))
    L = L * np.sqrt(safe)[..., None, None]
    return L, ok


def chol_solve(L, B):
    """lib_matrAXeqBMatCpx (libs/lib/lib_matr.c:330-378): X = (L L^H)^{-1} B."""
    n = L.shape[-1]
    Y = np.array(B, copy=True)
    for i in range(n):
        acc = Y[..., i, :]
        for j in range(i):
            acc = acc - L[..., i, j, None] * Y[..., j, :]
        Y[..., i, :] = acc / L[..., i, i, None]
    for i in range(n - 1, -1, -1):
        acc = Y[..., i, :]
        for j in range(i + 1, n):
            acc = acc - np.conj(L[..., j, i, None]) * Y[..., j, :]
        Y[..., i, :] = acc / np.conj(L[..., i, i, None])
    return Y


def param_cov_from_spectra(spec6, pv):
    """getNextParameterCovariance (src/seismicparametersholder.cpp:485-557):
    S_ab = |Re(spec_ab) / pv_ab| * pv_ab (division skipped when pv_ab == 0), Im = 0."""
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    shp = spec6[0].shape
    S = np.zeros(shp + (3, 3), dtype=np.complex128)
    for s, (a, b) in zip(spec6, pairs):
        p = float(pv[a, b])
        v = np.abs(s.real / p) * p if p != 0 else np.abs(s.real)
        S[..., a, b] = v
        S[..., b, a] = v
    return S


# ---------------------------------------------------------------- the inversion

def _data_system(K, e1, e2, e3, Sth, wnc, S, lam, k0, k1):
    """K S and Sd = K S K^H + Sigma_e for kz in [k0, k1) (src/avoinversion.cpp:1036-1044
    with getNextErrorVariance :1236-1272).  S (z,y,x,3,3), lam (z,y,x)."""
    nth = K.shape[-2]
    Kk = K[k0:k1][:, None, None]                      # (z,1,1,nth,3)
    e1k = e1[k0:k1][:, None, None]
    e2k = e2[k0:k1][:, None, None]
    e3k = e3[k0:k1][:, None, None]
    E = 0.5 * (1.0 - wnc) * Sth * lam[..., None, None] * (
        e1k[..., :, None] * np.conj(e1k[..., None, :]) + e2k[..., :, None] * np.conj(e2k[..., None, :]))
    E = E + np.eye(nth) * (wnc * np.diag(Sth) * np.abs(e3k) ** 2)[..., None, :]
    KS = Kk @ S
    Sd = KS @ np.conj(np.swapaxes(Kk, -1, -2)) + E
    return Kk, KS, Sd


def post_cov_given_inputs(blk, S6, lam, slab: int = 16):
    """Posterior covariance spectra per bin, S_post = S - (KS)^H Sd^-1 KS, in FP64 from a
    given prior covariance spectrum S6 (6, nzp, nyp, cnxp) real, order Vp, Vs, Rho, VpVs,
    VpRho, VsRho, and error-correlation spectrum lam (nzp, nyp, cnxp), real >= 0: the
    per-bin algebra of computePostMeanResidAndFFTCov (src/avoinversion.cpp:1036-1061)
    without the transforms that make its inputs.  Returns (cov_spec (6, ...), ok) with ok
    the bins that were inverted and factorised; the others keep S."""
    K, e1, e2, e3, inv = per_kz_operators(blk)
    Sth = blk.err_theta_cov
    wnc = float(np.float32(blk.wnc))
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    nzp = S6.shape[1]
    cs = np.zeros(S6.shape, dtype=np.complex128)
    okall = np.zeros(S6.shape[1:], dtype=bool)
    for k0 in range(0, nzp, slab):
        k1 = min(nzp, k0 + slab)
        S = np.zeros(S6[:, k0:k1].shape[1:] + (3, 3), dtype=np.complex128)
        for g, (a, b) in enumerate(pairs):
            S[..., a, b] = S6[g, k0:k1]
            S[..., b, a] = S6[g, k0:k1]
        _, KS, Sd = _data_system(K, e1, e2, e3, Sth, wnc, S, lam[k0:k1], k0, k1)
        L, ok = chol_cpx(Sd)
        ok &= np.broadcast_to(inv[k0:k1][:, None, None], ok.shape)
        red = np.conj(np.swapaxes(KS, -1, -2)) @ chol_solve(L, KS)
        Spost = np.where(ok[..., None, None], S - red, S)
        for g, (a, b) in enumerate(pairs):
            cs[g, k0:k1] = Spost[..., a, b]
        okall[k0:k1] = ok
    return cs, okall


class Posterior:
    """Outputs of computePostMeanResidAndFFTCov + invFFTCovGrids, float64."""

    def __init__(self):
        self.mean_spec = None     # (3, nzp, nyp, cnxp)
        self.cov_spec = None      # (6, ...) Vp, Vs, Rho, VpVs, VpRho, VsRho
        self.resid_spec = None    # (ntheta, ...)
        self.mean = None          # (3, nzp, nyp, rnxp) real, 1/sqrt(N)
        self.cov = None           # (6, nzp, nyp, rnxp) real, 1/N
        self.n_inverted = 0
        self.n_chol_fail = 0


def posterior(blk, slab: int = 16, cov_grids=None, separable: bool = False) -> Posterior:
    """AVOInversion constructor FFTs + computePostMeanResidAndFFTCov + invFFTCovGrids;
    cov_grids: the six prior covariance grids when not those of prior_cov_grids(blk).
    separable (zero correlation gradients only): the prior and error-correlation spectra
    formed slab by slab as FFT2(corrXY) x FFT1(circCorrT) (and FFT2(corrXY) for the error
    correlation, a delta in time) instead of transforming the seven full grids; equal to the
    grid path up to the float32 rounding of the grids' products corrXY * circCorrT, and without
    their memory, for full-size blocks."""
    nxp, nyp, nzp, nth = blk.nxp, blk.nyp, blk.nzp, blk.ntheta
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    if separable:
        assert cov_grids is None and blk.corr_grad_i == 0 and blk.corr_grad_j == 0
        c2 = np.fft.rfft2(np.asarray(blk.corr_xy, dtype=np.float64))        # (nyp, cnxp)
        c1 = np.fft.fft(np.asarray(blk.circ_corr_t, dtype=np.float64))      # (nzp,)
        pvs = [float(np.float32(blk.prior_var0[a, b])) for a, b in pairs]
        cov_spec = None
        err_spec = None
    else:
        covs, pairs = prior_cov_grids(blk)
        if cov_grids is not None:
            covs = [np.asarray(c, dtype=np.float32) for c in cov_grids]
        cov_spec = [fft_in_place(c, nxp, True) for c in covs]
        if abs(blk.corr_grad_i) > 0 or abs(blk.corr_grad_j) > 0:
            ec = fill_err_corr(blk.corr_xy, nxp, nyp, nzp, blk.corr_grad_i, blk.corr_grad_j)
        else:
            ec = fill_err_corr_zero_grad(blk.corr_xy, nxp, nyp, nzp)
        err_spec = fft_in_place(ec, nxp, True)
    data_spec = np.stack([fft_in_place(blk.data[l], nxp, False) for l in range(nth)])
    mean_spec = np.stack([fft_in_place(blk.mean[a], nxp, False) for a in range(3)])
    K, e1, e2, e3, inv = per_kz_operators(blk)
    Sth = blk.err_theta_cov
    wnc = float(np.float32(blk.wnc))
    out = Posterior()
    out.mean_spec = mean_spec.copy()
    out.resid_spec = data_spec.copy()
    cs = np.zeros((6,) + mean_spec.shape[1:], dtype=np.complex128)
    for k0 in range(0, nzp, slab):
        k1 = min(nzp, k0 + slab)
        if separable:
            base = c1[k0:k1, None, None] * c2[None]
            S = param_cov_from_spectra([pv * base for pv in pvs], blk.prior_var0)
            lam = np.broadcast_to(np.abs(c2.real)[None], base.shape)
            del base
        else:
            S = param_cov_from_spectra([c[k0:k1] for c in cov_spec], blk.prior_var0)  # (z,y,x,3,3)
            lam = np.abs(err_spec[k0:k1].real)
        Kk, KS, Sd = _data_system(K, e1, e2, e3, Sth, wnc, S, lam, k0, k1)
        L, ok = chol_cpx(Sd)
        invk = np.broadcast_to(inv[k0:k1][:, None, None], ok.shape)
        ok_eff = ok & invk
        M = chol_solve(L, KS)                               # Sd^{-1} K S
        red = np.conj(np.swapaxes(KS, -1, -2)) @ M
        Spost = np.where(ok_eff[..., None, None], S - red, S)
        mu = np.moveaxis(mean_spec[:, k0:k1], 0, -1)       # (z,y,x,3)
        d = np.moveaxis(data_spec[:, k0:k1], 0, -1)        # (z,y,x,nth)
        dm = d - (Kk @ mu[..., None])[..., 0]
        mu_post = mu + (np.conj(np.swapaxes(M, -1, -2)) @ dm[..., None])[..., 0]
        res = d - (Kk @ mu_post[..., None])[..., 0]
        mu_post = np.where(ok_eff[..., None], mu_post, mu)
        res = np.where(ok_eff[..., None], res, d)
        out.mean_spec[:, k0:k1] = np.moveaxis(mu_post, -1, 0)
        out.resid_spec[:, k0:k1] = np.moveaxis(res, -1, 0)
        for g, (a, b) in enumerate(pairs):
            cs[g, k0:k1] = Spost[..., a, b]
        out.n_inverted += int(invk.sum())
        out.n_chol_fail += int((invk & ~ok).sum())
    out.cov_spec = cs
    out.mean = np.stack([inv_fft_in_place(out.mean_spec[a], nxp, False) for a in range(3)])
    out.cov = np.stack([inv_fft_in_place(cs[g], nxp, True) for g in range(6)])
    return out


def simulate(blk, post: Posterior, noise: np.ndarray) -> np.ndarray:
    """AVOInversion::simulate (src/avoinversion.cpp:1401-1511) for one realisation given
    its three complex noise grids noise (3, nzp, nyp, cnxp).  Returns (3, nzp, nyp, rnxp)."""
    cs = post.cov_spec
    C = np.zeros(cs.shape[1:] + (3, 3), dtype=np.complex128)
    C[..., 0, 0] = cs[0]
    C[..., 1, 1] = cs[1]
    C[..., 2, 2] = cs[2]
    C[..., 0, 1] = cs[3]
    C[..., 0, 2] = cs[4]
    C[..., 1, 2] = cs[5]
    C[..., 1, 0] = np.conj(cs[3])
    C[..., 2, 0] = np.conj(cs[4])
    C[..., 2, 1] = np.conj(cs[5])
    L, ok = chol_cpx(C)
    z = np.moveaxis(noise.astype(np.complex128), 0, -1)
    s = (np.tril(L) @ z[..., None])[..., 0]
    s = np.where(ok[..., None], s, 0.0)
    s = np.moveaxis(s, -1, 0)
    real = np.stack([inv_fft_in_place(s[a], blk.nxp, False) for a in range(3)])
    return real + post.mean


def post_var0(post: Posterior) -> np.ndarray:
    """updatePriorVar (src/seismicparametersholder.cpp:1031-1043): cov grids at (0,0,0)."""
    v = post.cov[:, 0, 0, 0]
    P = np.zeros((3, 3))
    P[0, 0], P[1, 1], P[2, 2] = v[0], v[1], v[2]
    P[0, 1] = P[1, 0] = v[3]
    P[0, 2] = P[2, 0] = v[4]
    P[1, 2] = P[2, 1] = v[5]
    return P


def post_cov00(post: Posterior, nz: int) -> np.ndarray:
    """createPostCov00 (src/seismicparametersholder.cpp:1056-1067) for Vp, Vs, Rho."""
    return post.cov[:3, :nz, 0, 0].copy()


def rel_err(x, ref) -> float:
    """Norm-wise relative error ||x - ref|| / ||ref||."""
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.linalg.norm(ref)
    return float(np.linalg.norm(x - ref) / (den if den > 0 else 1.0))


def max_rel_err(x, ref) -> float:
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.max(np.abs(ref))
    return float(np.max(np.abs(x - ref)) / (den if den > 0 else 1.0))


# ---------------------------------------------------------------- facies probabilities

def facies_smoother(nbins, dv, sigma_inv):
    """Normalised Gaussian smoother with cyclic bin offsets (FaciesProb::makeFaciesDens,
    src/faciesprob.cpp:447-496), (nr, nb, na) array."""
    na, nb, nr = nbins
    cyc = lambda n: np.where(np.arange(n) <= n // 2, np.arange(n), np.arange(n) - n).astype(np.float64)
    jj, kk, ll = cyc(na)[None, None, :] * dv[0], cyc(nb)[None, :, None] * dv[1], cyc(nr)[:, None, None] * dv[2]
    S = np.asarray(sigma_inv, dtype=np.float64)
    f = (jj * jj * S[0, 0] + kk * kk * S[1, 1] + ll * ll * S[2, 2] + 2 * jj * kk * S[1, 0] + 2 * jj * ll * S[2, 0]
         + 2 * kk * ll * S[2, 1])
    sm = np.exp(-0.5 * f)
    return sm / sm.sum()


def facies_smooth(hist, nbins, dv, sigma_inv):
    """Circular convolution of each (nr, nb, na) histogram with the smoother, the effect
    of fftInPlace / multiply / invFFTInPlace / x sqrt(N) in makeFaciesDens (:505-515)."""
    sm = facies_smoother(nbins, dv, sigma_inv)
    Fs = np.fft.rfftn(sm)
    return np.stack([np.fft.irfftn(np.fft.rfftn(h) * Fs, s=h.shape, axes=(0, 1, 2)) for h in np.asarray(hist, dtype=np.float64)])


def facies_prob(post, dens, nbins, vmin, dv, prior, p_undefined, nx, ny, nz):
    """FaciesProb::calculateFaciesProb with findDensity (src/faciesprob.cpp:1909-2075,
    1307-1423), one density volume per facies (no local-noise corners).
    post: three real (nz, ny, >=nx) arrays of ln Vp, ln Vs, ln rho; dens: (nf, nr, nb, na).
    Returns (nf+1, nz, ny, nx): facies probabilities and the undefined class."""
    nf = len(prior)
    v = [np.asarray(post[d][:nz, :ny, :nx], dtype=np.float64) for d in range(3)]
    idx, w = [], []
    for d in range(3):
        f = (v[d] - vmin[d]) / dv[d] - 0.5
        i1 = np.floor(f).astype(np.int64)
        lo = i1 < 0
        hi = i1 >= nbins[d] - 1
        ww = np.where(lo | hi, 0.0, f - i1)
        i1 = np.where(lo, 0, np.where(hi, nbins[d] - 1, i1))
        i2 = np.where(lo | hi, i1, i1 + 1)
        idx.append((i1, i2))
        w.append(ww)
    undef = p_undefined / float(nbins[0] * nbins[1] * nbins[2])
    vals = []
    for f in range(nf):
        D = np.maximum(np.asarray(dens[f], dtype=np.float64), 0.0)
        d = 0.0
        for a in (0, 1):
            wa = w[0] if a else 1 - w[0]
            for b in (0, 1):
                wb = w[1] if b else 1 - w[1]
                for c in (0, 1):
                    wc = w[2] if c else 1 - w[2]
                    d = d + wa * wb * wc * D[idx[2][c], idx[1][b], idx[0][a]]
        vals.append(prior[f] * np.maximum(d, 0.0))
    s = undef + sum(vals)
    return np.stack([x / s for x in vals] + [undef / s])


# ---------------------------------------------------------------- local noise (row f3)

def _sym_eig_sorted(a):
    """Eigen-decomposition of a real symmetric matrix, eigenvalues descending (NRLib::Sort3x3
    order), each eigenvector's largest-magnitude component positive (the reference takes
    LAPACK's signs, which this environment cannot reproduce)."""
    w, v = np.linalg.eigh(0.5 * (a + a.T))
    idx = np.argsort(-w, kind="stable")
    w, v = w[idx], v[:, idx]
    big = np.argmax(np.abs(v), axis=0)
    sg = np.sign(v[big, np.arange(v.shape[1])])
    sg[sg == 0] = 1.0
    return w, v * sg


def _sym_fun(a, f):
    """V diag(f(w)) V^T of symmetric a (batched over leading axes)."""
    w, v = np.linalg.eigh(0.5 * (a + np.swapaxes(a, -1, -2)))
    return (v * f(w)[..., None, :]) @ np.swapaxes(v, -1, -2)


def compute_g(Sm, Smd, Sth):
    """AVOInversion::computeG (src/avoinversion.cpp:1943-2026): G = Sth^1/2 Lg Evec^T Sm^-1/2
    with (Eval, Evec) the sorted eigen-decomposition of Sm^-1/2 (Sm - Smd)_+ Sm^-1/2 and
    Lg(i, i) = sqrt(Eval_i / (1 - Eval_i)) for i < min(ntheta, 3)."""
    n = Sth.shape[0]
    Sdel = _sym_fun(Sm - Smd, lambda w: np.where(w > 0, w, 0.0))
    Sinv = _sym_fun(Sm, lambda w: np.where(w > 1e-7, 1.0 / np.sqrt(np.maximum(w, 1e-300)), 0.0))
    A = Sinv @ Sdel @ Sinv
    ew, ev = _sym_eig_sorted(A)
    Lg = np.zeros((n, 3))
    for i in range(min(n, 3)):
        if ew[i] > 0:
            Lg[i, i] = np.sqrt(ew[i] / (1.0 - ew[i]))
    S12 = _sym_fun(Sth, lambda w: np.sqrt(np.maximum(w, 0.0)))
    return S12 @ Lg @ ev.T @ Sinv


def local_noise_maps(Sm, Smd, Sth, scales):
    """newPosteriorCovPointwise (src/avoinversion.cpp:2028-2118) per trace: the map S of the
    posterior deviation from the prior mean and the map Msim of a realisation's deviation
    (sigmamdnew_ times postVar0^-1/2, :2226-2239).  scales: (ntheta, ny, nx) already divided
    by each angle's minimum.  Returns S, Msim of shape (ny, nx, 3, 3)."""
    G = compute_g(Sm, Smd, Sth)
    d = np.sqrt(np.moveaxis(scales, 0, -1))                       # (ny, nx, n)
    M = G @ Sm @ G.T + d[..., :, None] * Sth * d[..., None, :]
    Minv = _sym_fun(M, lambda w: np.where(w > 1e-8, 1.0 / np.where(w > 1e-8, w, 1.0), 0.0))
    delta = Sm @ G.T @ Minv @ G @ Sm
    smd = Sm - delta
    rs = _sym_fun(smd, lambda w: np.sqrt(np.maximum(w, 0.0)))
    rd = _sym_fun(delta, lambda w: np.sqrt(np.maximum(w, 0.0)))
    sdel = _sym_fun(Sm - Smd, lambda w: np.where(w > 1e-7, 1.0 / np.sqrt(np.maximum(w, 1e-300)), 0.0))
    smdi = _sym_fun(Smd, lambda w: np.where(w > 0, 1.0 / np.sqrt(np.maximum(w, 1e-300)), 0.0))
    return rd @ sdel, rs @ smdi


def local_noise_correct(blk, post_mean, sims, scales, post_var0_mat):
    """correctVpVsRho (src/avoinversion.cpp:2146-2270) on the posterior mean (3, nzp, nyp,
    rnxp) and the local-noise mixing of simulate (:1485-1504) on realisations (nsim, 3, ...)
    holding posterior + noise; scales (ntheta, ny, nx) raw local noise scales.  Returns the
    corrected copies."""
    nx, ny, nz = blk.nx, blk.ny, blk.nz
    sc = scales / scales.reshape(scales.shape[0], -1).min(axis=1)[:, None, None]
    S, Ms = local_noise_maps(np.asarray(blk.prior_var0, dtype=np.float64), np.asarray(post_var0_mat, np.float64),
                             np.asarray(blk.err_theta_cov, dtype=np.float64), sc)
    pm = np.asarray(blk.mean, dtype=np.float64)[:, :nz, :ny, :nx]
    pr = np.asarray(post_mean, dtype=np.float64)[:, :nz, :ny, :nx]
    dev = pr - pm
    new = pm + np.einsum("yxab,bzyx->azyx", S, dev)
    out_mean = np.array(post_mean, dtype=np.float64, copy=True)
    out_mean[:, :nz, :ny, :nx] = new
    out_sims = None
    if sims is not None:
        out_sims = np.array(sims, dtype=np.float64, copy=True)
        for s in range(sims.shape[0]):
            noise = np.asarray(sims[s], dtype=np.float64)[:, :nz, :ny, :nx] - pr
            out_sims[s, :, :nz, :ny, :nx] = new + np.einsum("yxab,bzyx->azyx", Ms, noise)
    return out_mean, out_sims


# ---------------------------------------------------------------- temporal prior functions (row f2)

def circ_corr_t(prior_t, min_int_fq: int, nzp: int) -> np.ndarray:
    """SeismicParametersHolder::computeCircCorrT + makeCircCorrTPosDef
    (src/seismicparametersholder.cpp:624-660, 805-840) in float64: circular extension of the
    lags (as float), spectrum zeroed at k <= minIntFq and |.| elsewhere, unnormalised back
    transform divided by its lag-0 value."""
    n = len(prior_t)
    c = np.zeros(nzp)
    for k in range(nzp):
        refk = k if k < nzp // 2 + 1 else nzp - k
        c[k] = float(np.float32(prior_t[refk])) if refk < n else 0.0
    mag = np.abs(np.fft.rfft(c))
    mag[: min_int_fq + 1] = 0.0
    back = np.fft.irfft(mag, n=nzp) * nzp
    if not back[0] > 1e-5:
        raise ValueError("circular temporal correlation undefined")
    return (back / back[0]).astype(np.float32)


def circ_auto_cov(auto_cov, nzp: int, dz: float) -> np.ndarray:
    """ComputeCircAutoCov + MakeCircAutoCovPosDef + TaperCircAutoCovFunction
    (src/seismicparametersholder.cpp:559-757) with the lag-0 test of InitializeCorrelations
    (:247-274), in float64.  auto_cov: (nlag, 3, 3); returns (6, nzp) float32 in the order
    Vp, Vs, Rho, VpVs, VpRho, VsRho."""
    ac = np.asarray(auto_cov, dtype=np.float64)
    nlag = ac.shape[0]
    circ = np.zeros((3, 3, nzp))
    for i in range(3):
        for j in range(3):
            zero = not abs(ac[0, i, j]) > 1e-10
            for k in range(nlag):
                if k < nzp:
                    circ[i, j, k] = 0.0 if zero else float(np.float32(ac[k, i, j]))
                if k < nlag - 1 and 0 <= nzp - k - 1 < nzp:
                    circ[i, j, nzp - k - 1] = 0.0 if zero else float(np.float32(ac[k + 1, j, i]))
    F = np.fft.rfft(circ, axis=-1)                      # (3, 3, nh)
    d = np.sqrt(np.array([circ[i, i, 0] for i in range(3)]))
    A = np.moveaxis(F, -1, 0) / (d[:, None] * d[None, :])   # (nh, 3, 3)
    A = 0.5 * (A + np.conj(np.swapaxes(A, -1, -2)))
    w, v = np.linalg.eigh(A)
    Aa = (v * np.abs(w)[:, None, :]) @ np.conj(np.swapaxes(v, -1, -2))
    F2 = np.moveaxis(Aa * (d[:, None] * d[None, :]), 0, -1)
    back = np.fft.irfft(F2, n=nzp, axis=-1)             # irfft divides by nzp already
    sd = min(50.0 / dz, nzp / 2.0)
    t = np.arange(nzp)
    m = np.where(t < nzp // 2 + 1, t, nzp - t).astype(np.float32).astype(np.float64)
    e = np.exp(-0.5 * (m / sd) ** 2)
    taper = np.where(e > 1e-10, e.astype(np.float32).astype(np.float64), 0.0)
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    return np.stack([back[a, b] * taper for a, b in pairs]).astype(np.float32)


def facies_density_corners(post, corners, scales, nx, ny, nz, t=None):
    """findDensity with local noise (src/faciesprob.cpp:1307-1423) and the relative noise
    scales of calculateFaciesProb (:1961-1977), float64.  corners: list of 2^nang tuples
    (dens (nf, nr, nb, na), nbins, vmin, dv); scales: (nang, ny, nx), or t: the relative
    scales themselves.  Returns (nf, nz, ny, nx) densities (before the prior weighting)."""
    if t is None:
        nang = scales.shape[0]
        t = np.zeros_like(np.asarray(scales, dtype=np.float64))
        for a in range(nang):
            mn, mx = float(scales[a].min()), float(scales[a].max())
            t[a] = 0.0 if mn == mx else ((scales[a].astype(np.float64) - mn) / (mx - mn)).astype(np.float32)
    t = np.asarray(t, dtype=np.float64)
    nang = t.shape[0]
    v = [np.asarray(post[d][:nz, :ny, :nx], dtype=np.float64) for d in range(3)]
    nf = corners[0][0].shape[0]
    out = np.zeros((nf, nz, ny, nx))
    for c, (dens, nbins, vmin, dv) in enumerate(corners):
        idx, w = [], []
        for d in range(3):
            f = (v[d] - vmin[d]) / dv[d] - 0.5
            i1 = np.floor(f).astype(np.int64)
            lo = i1 < 0
            hi = i1 >= nbins[d] - 1
            idx.append((np.where(lo, 0, np.where(hi, nbins[d] - 1, i1)),
                        np.where(lo | hi, np.where(lo, 0, nbins[d] - 1), i1 + 1)))
            w.append(np.where(lo | hi, 0.0, f - i1))
        wc = np.ones((ny, nx))
        for a in range(nang):
            wc = wc * (t[a] if (c >> a) & 1 else 1.0 - t[a])
        for f in range(nf):
            D = np.maximum(np.asarray(dens[f], dtype=np.float64), 0.0)
            d = 0.0
            for a in (0, 1):
                wa = w[0] if a else 1 - w[0]
                for b in (0, 1):
                    wb = w[1] if b else 1 - w[1]
                    for e in (0, 1):
                        we = w[2] if e else 1 - w[2]
                        d = d + wa * wb * we * D[idx[2][e], idx[1][b], idx[0][a]]
            out[f] += d * wc[None]
    return np.maximum(out, 0.0)


# ---------------------------------------------------------------- STORM grids

def storm_padding(vals: np.ndarray, nxp: int, nyp: int, nzp: int) -> np.ndarray:
    """FFTGrid(const StormContGrid*, nxp, nyp, nzp) (src/fftgrid.cpp:215-302): the interior
    values vals (nz, ny, nx) float32 in a padded real grid (nzp, nyp, rnxp) whose padding is
    the float32 blend c1 w1 + c2 w2 of two edge values, in the reference's loop and branch
    order (k, then j, then i; z padding, else y padding, else x padding; zero beyond nxp)."""
    f32 = np.float32
    nz, ny, nx = vals.shape
    rnxp = 2 * (nxp // 2 + 1)
    g = np.zeros((nzp, nyp, rnxp), dtype=f32)
    sc = f32(1.0) / f32(nzp - nz + 1)
    sb = f32(1.0) / f32(nyp - ny + 1)
    sa = f32(1.0) / f32(nxp - nx + 1)
    ii = np.arange(nx, nxp)
    wa1 = (sa * (ii - nx + 1).astype(f32)).astype(f32)
    wa2 = (sa * (nxp - ii).astype(f32)).astype(f32)
    for k in range(nzp):
        for j in range(nyp):
            row = g[k, j]
            if k >= nz:
                w1 = f32(sc * f32(k - nz + 1))
                w2 = f32(sc * f32(nzp - k))
                row[:nxp] = (g[0, j, :nxp] * w1).astype(f32) + (g[nz - 1, j, :nxp] * w2).astype(f32)
            elif j >= ny:
                w1 = f32(sb * f32(j - ny + 1))
                w2 = f32(sb * f32(nyp - j))
                row[:nxp] = (g[k, 0, :nxp] * w1).astype(f32) + (g[k, ny - 1, :nxp] * w2).astype(f32)
            else:
                row[:nx] = vals[k, j]
                row[nx:nxp] = (row[0] * wa1).astype(f32) + (row[nx - 1] * wa2).astype(f32)
    return g
