"""The C++ host layer (crava_b200/host: FFTGrid / AVOInversion over the C ABI) against the
FP64 oracle, through its demo driver: DATA and PARAMETER grids go in as FFTGrid objects,
computePostMeanResidAndFFTCov and simulate run, and the posterior is read back from the
same grids, as the reference's AVOInversion leaves it.

Tolerances (norm-wise relative): posterior mean 1e-4, covariance 1e-3, realisations 1e-4,
residual spectra 2e-3 (a residual is a small difference of FP32 spectra, so its relative
error is larger than the mean's); Cholesky fallbacks and inverted bins exactly.
"""
import os
import subprocess

import numpy as np
import pytest

from crava_b200 import synth
from oracle import bindings as ob
from oracle import ref64

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEMO = os.path.join(ROOT, "crava_b200", "host", "avo_host_demo")


def crel(x, ref):
    x = np.asarray(x, dtype=np.complex128)
    ref = np.asarray(ref, dtype=np.complex128)
    return float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))


def write_block(path, blk, grids, noise, w3=None):
    rnxp = 2 * (blk.nxp // 2 + 1)
    shape = (blk.nzp, blk.nyp, rnxp)

    def padded(a):
        g = np.zeros(shape, dtype=np.float32)
        g[..., :a.shape[-1]] = a
        return g

    with open(path, "wb") as f:
        np.array([blk.nx, blk.ny, blk.nz, blk.nxp, blk.nyp, blk.nzp, blk.ntheta, blk.nsim,
                  1 if grids else 0, 1 if noise is not None else 0], dtype=np.int32).tofile(f)
        np.array([blk.seed], dtype=np.uint64).tofile(f)
        np.array([blk.lz, blk.min_rel_thick, blk.low_cut, blk.high_cut, blk.wnc], dtype=np.float64).tofile(f)
        np.asarray(blk.A, dtype=np.float64).tofile(f)
        np.asarray(blk.err_theta_cov, dtype=np.float64).tofile(f)
        np.asarray(blk.prior_var0, dtype=np.float64).tofile(f)
        np.asarray(blk.wavelet, dtype=np.float32).tofile(f)
        np.asarray(blk.wavelet_norm, dtype=np.float32).tofile(f)
        if grids:
            covs, _ = ref64.prior_cov_grids(blk)
            for c in covs:
                padded(c).tofile(f)
            padded(ref64.fill_err_corr_zero_grad(blk.corr_xy, blk.nxp, blk.nyp, blk.nzp)).tofile(f)
        else:
            np.asarray(blk.corr_xy, dtype=np.float32).tofile(f)
            np.asarray(blk.circ_corr_t, dtype=np.float32).tofile(f)
        for l in range(blk.ntheta):
            np.asarray(blk.data[l], dtype=np.float32).tofile(f)
        for a in range(3):
            np.asarray(blk.mean[a], dtype=np.float32).tofile(f)
        if noise is not None:
            np.ascontiguousarray(noise, dtype=np.complex64).tofile(f)
        nonconst = getattr(blk, "rel_thick", None) is not None
        grads = not grids and (blk.corr_grad_i != 0.0 or blk.corr_grad_j != 0.0)
        if nonconst or grads or w3 is not None:
            np.array([1 if nonconst else 0], dtype=np.int32).tofile(f)
        if nonconst:
            np.ascontiguousarray(blk.rel_thick, dtype=np.float64).tofile(f)
            np.array([blk.energy_threshold], dtype=np.float32).tofile(f)
        if grads or w3 is not None:
            np.array([1 if grads else 0], dtype=np.int32).tofile(f)
        if grads:
            np.array([blk.corr_grad_i, blk.corr_grad_j], dtype=np.float32).tofile(f)
        if w3 is not None:
            a1 = np.asarray(w3["alpha1"], dtype=np.float32)
            has_grad, has_h = w3["grad_x"] is not None, w3["halpha"] is not None
            np.array([1, a1.shape[2], a1.shape[1], int(has_grad), int(has_h)], dtype=np.int32).tofile(f)
            np.array(w3["filter_geom"], dtype=np.float64).tofile(f)
            np.asarray(w3["theta"], dtype=np.float32).tofile(f)
            if has_grad:
                np.asarray(w3["grad_x"], dtype=np.float32).tofile(f)
                np.asarray(w3["grad_y"], dtype=np.float32).tofile(f)
            a1.tofile(f)
            if has_h:
                np.asarray(w3["halpha"], dtype=np.float32).tofile(f)
            np.asarray(w3["global_wavelet"], dtype=np.float32).tofile(f)
            np.asarray(w3["global_wavelet_norm"], dtype=np.float32).tofile(f)


def read_out(path, blk):
    rnxp = 2 * (blk.nxp // 2 + 1)
    rs = blk.nzp * blk.nyp * rnxp
    shape = (blk.nzp, blk.nyp, rnxp)
    with open(path, "rb") as f:
        grids = np.fromfile(f, dtype=np.float32, count=rs * (9 + 3 * blk.nsim + blk.ntheta))
        cnt = np.fromfile(f, dtype=np.int64, count=4)
        pv = np.fromfile(f, dtype=np.float32, count=9)
        rt = np.fromfile(f, dtype=np.float32, count=1)
    grids = grids.reshape((-1,) + shape)
    return {"mean": grids[:3], "cov": grids[3:9], "sims": grids[9:9 + 3 * blk.nsim].reshape((blk.nsim, 3) + shape),
            "resid": grids[9 + 3 * blk.nsim:].view(np.complex64), "counters": cnt, "post_var0": pv,
            "fft_roundtrip": float(rt[0])}


@pytest.mark.parametrize("grids", [False, True])
def test_host_layer_matches_oracle(tmp_path, grids):
    assert os.path.exists(DEMO), "crava_b200/host/avo_host_demo is not built (python -m crava_b200.build)"
    blk = synth.make_block(synth.BlockSpec(nx=30, ny=28, nz=40, theta_deg=(8.0, 20.0, 32.0), peak_hz=(30.0,) * 3,
                                           sn=(5.0,) * 3, nsim=2, seed=17))
    noise = ob.sim_noise(23, blk.nsim, blk.nxp, blk.nyp, blk.nzp)
    fin, fout = tmp_path / "block.bin", tmp_path / "out.bin"
    write_block(fin, blk, grids, noise)
    r = subprocess.run([DEMO, str(fin), str(fout)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = read_out(fout, blk)
    post = ref64.posterior(blk)
    nx = blk.nxp
    assert out["counters"][0] == post.n_inverted
    assert out["counters"][1] == post.n_chol_fail
    for a in range(3):
        assert crel(out["mean"][a][..., :nx], post.mean[a][..., :nx]) < 1e-4, ("mean", a)
    for q in range(6):
        assert crel(out["cov"][q][..., :nx], post.cov[q][..., :nx]) < 1e-3, ("cov", q)
    for l in range(blk.ntheta):
        assert crel(out["resid"][l], post.resid_spec[l]) < 2e-3, ("resid", l)
    for s in range(blk.nsim):
        sim = ref64.simulate(blk, post, noise[s])
        for a in range(3):
            assert crel(out["sims"][s, a][..., :nx], sim[a][..., :nx]) < 1e-4, ("sim", s, a)
    assert np.allclose(out["post_var0"].reshape(3, 3), ref64.post_var0(post), rtol=1e-3)
    scale = float(np.abs(blk.data[0]).max())
    assert out["fft_roundtrip"] < 1e-5 * scale


@pytest.mark.parametrize("grids,wavelet3d", [(False, False), (True, False), (False, True)])
def test_host_layer_nonconst_thickness(tmp_path, grids, wavelet3d):
    """AVOInversionSettings::relThick: the layer divides the data by the scale wavelet
    (crava_job_divide_data) before the inversion, and in GRIDS mode reads the temporal
    correlation from the covVp grid's (0, 0) column; with waveletDim 3 the division uses the
    dip-adjusted local wavelets of 3D wavelets (crava_job_set_wavelet_3d)."""
    import dataclasses
    assert os.path.exists(DEMO)
    blk = synth.make_block(synth.BlockSpec(nx=30, ny=28, nz=40, nxp=36, nyp=32, nzp=48, theta_deg=(8.0, 20.0, 32.0),
                                           peak_hz=(30.0,) * 3, sn=(5.0,) * 3, nsim=0, seed=19))
    blk = synth.with_rel_thick(blk, seed=7)
    w3 = synth.wavelet3d_model(blk, blk.spec.theta_deg, seed=11) if wavelet3d else None
    fin, fout = tmp_path / "block.bin", tmp_path / "out.bin"
    write_block(fin, blk, grids, None, w3=w3)
    r = subprocess.run([DEMO, str(fin), str(fout)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = read_out(fout, blk)
    div = ref64.divide_data_by_scale_wavelet(blk, w3=w3)
    divided = np.stack([ref64.interpolate_seismic(div[l], blk, blk.energy_threshold) for l in range(blk.ntheta)])
    post = ref64.posterior(dataclasses.replace(blk, data=divided))
    nx = blk.nxp
    assert out["counters"][0] == post.n_inverted
    for a in range(3):
        assert crel(out["mean"][a][..., :nx], post.mean[a][..., :nx]) < 1e-4, ("mean", a)
    for q in range(6):
        assert crel(out["cov"][q][..., :nx], post.cov[q][..., :nx]) < 1e-3, ("cov", q)


def test_host_layer_correlation_gradients(tmp_path):
    """AVOInversionSettings::corrGradI/J with the separable factors: the layer generates
    InitializeCorrelations' grids on the device (crava_job_fill_prior) and inverts in GRIDS
    mode; the result matches the oracle's posterior on the gradient prior."""
    assert os.path.exists(DEMO)
    blk = synth.make_block(synth.BlockSpec(nx=30, ny=28, nz=40, theta_deg=(8.0, 20.0, 32.0), peak_hz=(30.0,) * 3,
                                           sn=(5.0,) * 3, nsim=0, seed=29, corr_grad_i=0.37, corr_grad_j=-0.21))
    fin, fout = tmp_path / "block.bin", tmp_path / "out.bin"
    write_block(fin, blk, False, None)
    r = subprocess.run([DEMO, str(fin), str(fout)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = read_out(fout, blk)
    post = ref64.posterior(blk)
    nx = blk.nxp
    assert out["counters"][0] == post.n_inverted
    for a in range(3):
        assert crel(out["mean"][a][..., :nx], post.mean[a][..., :nx]) < 1e-4, ("mean", a)
    for q in range(6):
        assert crel(out["cov"][q][..., :nx], post.cov[q][..., :nx]) < 1e-3, ("cov", q)
