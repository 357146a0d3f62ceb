"""Parity of the CUDA path (through the C ABI) with the oracle.

Tolerances (norm-wise relative error ||x - ref|| / ||ref|| per grid):
  posterior mean 1e-4, posterior covariance 1e-3, realisations 1e-4 against the FP64
  oracle; transforms 2e-6 against numpy's float64 FFT.
"""
import math

import numpy as np
import pytest

from crava_b200 import api, synth
from oracle import bindings as ob
from oracle import ref64

pytestmark = pytest.mark.gpu

TOL_MEAN = 1e-4
TOL_COV = 1e-3
TOL_SIM = 1e-4
TOL_FFT = 2e-6


def crel(x, ref):
    x = np.asarray(x, dtype=np.complex128)
    ref = np.asarray(ref, dtype=np.complex128)
    return float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("dims", [(64, 64, 128), (15, 12, 20), (27, 25, 14), (7, 5, 9), (540, 8, 6), (6, 768, 10),
                                  (8, 6, 320), (245, 3, 2), (2, 2, 2), (540, 540, 3), (768, 768, 2)])
@pytest.mark.parametrize("covariance", [False, True])
def test_fft_matches_numpy(ctx, dims, covariance):
    import torch
    nxp, nyp, nzp = dims
    rnxp = 2 * (nxp // 2 + 1)
    rng = np.random.default_rng(nxp * 7 + nyp * 3 + nzp)
    x = rng.standard_normal((nzp, nyp, nxp)).astype(np.float32)
    g = torch.zeros((nzp, nyp, rnxp), dtype=torch.float32, device="cuda")
    g[..., :nxp] = torch.from_numpy(x).cuda()
    api.fft_r2c(ctx, g.data_ptr(), nxp, nyp, nzp, covariance)
    torch.cuda.synchronize()
    spec = g.cpu().numpy().view(np.complex64)
    N = nxp * nyp * nzp
    ref = np.fft.rfftn(x.astype(np.float64)) * (1.0 if covariance else 1.0 / math.sqrt(N))
    assert crel(spec, ref) < TOL_FFT
    api.fft_c2r(ctx, g.data_ptr(), nxp, nyp, nzp, covariance)
    torch.cuda.synchronize()
    back = g.cpu().numpy()[..., :nxp]
    assert crel(back, x) < TOL_FFT
    if ob.ref32_available():  # the reference's own FFTW on the same grid
        pad = np.zeros((nzp, nyp, rnxp), dtype=np.float32)
        pad[..., :nxp] = x
        r32 = ob.ref32_fft(pad, nxp, covariance)
        assert crel(spec, r32) < 4 * TOL_FFT


@pytest.fixture(scope="module")
def block0():
    return synth.make_block(synth.config0())


@pytest.fixture(scope="module")
def post0(block0):
    return ref64.posterior(block0)


def _check_posterior(blk, out, post, n_inv=None):
    nx = blk.nxp
    for a in range(3):
        assert crel(out["mean"][a][..., :nx], post.mean[a][..., :nx]) < TOL_MEAN, ("mean", a)
    for q in range(6):
        assert crel(out["cov"][q][..., :nx], post.cov[q][..., :nx]) < TOL_COV, ("cov", q)
    if n_inv is not None:
        assert out["counters"]["inverted_bins"] == n_inv
        assert out["counters"]["chol_fallbacks"] == post.n_chol_fail


def test_posterior_separable_config0(ctx, block0, post0):
    noise = ob.sim_noise(block0.seed, block0.nsim, block0.nxp, block0.nyp, block0.nzp)
    out = api.invert_block(ctx, block0, api.PRIOR_SEPARABLE, noise=noise, keep_residual=True)
    _check_posterior(block0, out, post0, post0.n_inverted)
    for l in range(block0.ntheta):
        assert crel(out["resid_spec"][l], post0.resid_spec[l]) < 1e-3, ("resid", l)
    for s in range(block0.nsim):
        sim = ref64.simulate(block0, post0, noise[s])
        for a in range(3):
            assert crel(out["sims"][s, a][..., :block0.nxp], sim[a][..., :block0.nxp]) < TOL_SIM
    pv = out["counters"]["post_var0"]
    assert np.allclose(pv, ref64.post_var0(post0), rtol=1e-3)


def test_posterior_grids_mode_config0(ctx, block0, post0):
    covs, _ = ref64.prior_cov_grids(block0)
    ec = ref64.fill_err_corr_zero_grad(block0.corr_xy, block0.nxp, block0.nyp, block0.nzp)
    out = api.invert_block(ctx, block0, api.PRIOR_GRIDS, cov_grids=covs, err_corr=ec,
                           noise=ob.sim_noise(3, block0.nsim, block0.nxp, block0.nyp, block0.nzp))
    _check_posterior(block0, out, post0, post0.n_inverted)


@pytest.mark.parametrize("spec", [
    dict(nx=15, ny=12, nz=21, theta_deg=(8.0, 24.0), peak_hz=(28.0, 32.0), sn=(4.0, 6.0), nsim=2, seed=5),
    dict(nx=13, ny=11, nz=19, nxp=14, nyp=12, nzp=20, theta_deg=(5.0, 15.0, 25.0, 35.0, 45.0, 55.0),
         peak_hz=(30.0,) * 6, sn=(3.0,) * 6, nsim=1, seed=6),
    dict(nx=25, ny=27, nz=35, theta_deg=(10.0,), peak_hz=(25.0,), sn=(10.0,), nsim=1, seed=7),
    dict(nx=16, ny=16, nz=32, theta_deg=tuple(np.linspace(5, 50, 8)), peak_hz=(35.0,) * 8, sn=(5.0,) * 8,
         nsim=3, seed=8, low_cut=2.0, high_cut=120.0),
])
def test_posterior_small_blocks(ctx, spec):
    blk = synth.make_block(synth.BlockSpec(**spec))
    post = ref64.posterior(blk)
    noise = ob.sim_noise(11, blk.nsim, blk.nxp, blk.nyp, blk.nzp)
    out = api.invert_block(ctx, blk, api.PRIOR_SEPARABLE, noise=noise)
    _check_posterior(blk, out, post, post.n_inverted)
    for s in range(blk.nsim):
        sim = ref64.simulate(blk, post, noise[s])
        for a in range(3):
            assert crel(out["sims"][s, a][..., :blk.nxp], sim[a][..., :blk.nxp]) < TOL_SIM


def test_posterior_grids_with_gradients(ctx):
    blk = synth.make_block(synth.BlockSpec(nx=12, ny=10, nz=16, theta_deg=(10.0, 30.0), peak_hz=(30.0, 30.0),
                                           sn=(5.0, 5.0), nsim=1, seed=9, corr_grad_i=0.3, corr_grad_j=-0.2))
    post = ref64.posterior(blk)
    covs, _ = ref64.prior_cov_grids(blk)
    ec = ref64.fill_err_corr(blk.corr_xy, blk.nxp, blk.nyp, blk.nzp, blk.corr_grad_i, blk.corr_grad_j)
    out = api.invert_block(ctx, blk, api.PRIOR_GRIDS, cov_grids=covs, err_corr=ec,
                           noise=ob.sim_noise(1, 1, blk.nxp, blk.nyp, blk.nzp))
    _check_posterior(blk, out, post, post.n_inverted)


def test_fp64_refine_every_bin_config0(ctx, block0, post0):
    """fp64_threshold 1 flags (nearly) every inverted bin: the FP64 re-factorisation with
    its refinement step reproduces the oracle like the FP32 path does."""
    noise = ob.sim_noise(block0.seed, block0.nsim, block0.nxp, block0.nyp, block0.nzp)
    out = api.invert_block(ctx, block0, api.PRIOR_SEPARABLE, noise=noise, keep_residual=True, fp64_threshold=1.0)
    _check_posterior(block0, out, post0, post0.n_inverted)
    assert out["counters"]["fp64_bins"] > 0.9 * post0.n_inverted
    for l in range(block0.ntheta):
        assert crel(out["resid_spec"][l], post0.resid_spec[l]) < 1e-3, ("resid", l)
    sim = ref64.simulate(block0, post0, noise[0])
    for a in range(3):
        assert crel(out["sims"][0, a][..., :block0.nxp], sim[a][..., :block0.nxp]) < TOL_SIM


def test_spectral_cov_matches_oracle_spectrum(ctx, block0, post0):
    """CRAVA_FLAG_SPECTRAL_COV leaves S_post per bin, the oracle's cov_spec."""
    job = api.Job(ctx, block0, api.PRIOR_SEPARABLE, api.FLAG_SPECTRAL_COV, nsim=0)
    _keep = job.upload_block()
    job.run()
    out = job.download_outputs()
    job.close()
    for q in range(6):
        assert crel(out["cov_spec"][q], post0.cov_spec[q]) < TOL_COV, q


def test_descriptor_rejects_unknown_flag_and_bad_threshold(ctx, block0):
    for kw in (dict(flags=64), dict(fp64_threshold=-1.0), dict(fp64_threshold=float("inf"))):
        with pytest.raises(api.CravaError):
            api.Job(ctx, block0, api.PRIOR_SEPARABLE, **kw)


def test_device_noise_statistics(ctx, block0, post0):
    """Product-mode noise: each realisation's deviation from the posterior mean has, per
    voxel, the posterior variance (the covariance grids at lag 0)."""
    job = api.Job(ctx, block0, api.PRIOR_SEPARABLE, 0, seed=1234, nsim=8)
    _keep = job.upload_block()
    job.run()
    out = job.download_outputs()
    nx = block0.nxp
    dev = out["sims"][..., :nx] - out["mean"][None, ..., :nx]
    for a in range(3):
        emp = float(np.mean(dev[:, a].astype(np.float64) ** 2))
        assert 0.85 < emp / post0.cov[a, 0, 0, 0] < 1.15, (a, emp, post0.cov[a, 0, 0, 0])
    # realisations differ from one another and from another seed's
    assert np.abs(dev[0, 0] - dev[1, 0]).max() > 0
    job.close()


def test_inputs_preserved_and_rerun_bitwise(ctx, block0):
    job = api.Job(ctx, block0, api.PRIOR_SEPARABLE, 0, seed=77)
    _keep = job.upload_block()
    job.run()
    a = job.download_outputs()
    d0 = job.download(api.ROLE_DATA, 0)
    assert np.array_equal(d0, block0.data[0])
    job.run()
    b = job.download_outputs()
    for k in ("mean", "cov", "sims"):
        assert np.array_equal(a[k], b[k]), k
    job.close()


from tests.golden import golden_io  # noqa: E402


@pytest.mark.parametrize("name", golden_io.names())
def test_against_reference_fixtures(ctx, name):
    """GPU (grids mode, reference RandomGen noise) against the reference's own FP32 path."""
    blk, z = golden_io.load(name)
    out = api.invert_block(ctx, blk, api.PRIOR_GRIDS, cov_grids=list(z["cov_grids"]), err_corr=z["err_corr"],
                           noise=z["noise"], keep_residual=True)
    nx = blk.nxp
    assert out["counters"]["inverted_bins"] == int(z["ref_n_inverted"])
    assert out["counters"]["chol_fallbacks"] == int(z["ref_n_chol_fail"])
    for a in range(3):
        assert crel(out["mean"][a][..., :nx], z["ref_mean"][a][..., :nx]) < TOL_MEAN
    for q in range(6):
        assert crel(out["cov"][q][..., :nx], z["ref_cov"][q][..., :nx]) < TOL_COV
    for l in range(blk.ntheta):
        assert crel(out["resid_spec"][l], z["ref_resid_spec"][l]) < 1e-3
    for s in range(blk.nsim):
        for a in range(3):
            assert crel(out["sims"][s, a][..., :nx], z["ref_sims"][s, a][..., :nx]) < TOL_SIM
    if not (blk.corr_grad_i or blk.corr_grad_j):
        sep = api.invert_block(ctx, blk, api.PRIOR_SEPARABLE, noise=z["noise"])
        for a in range(3):
            assert crel(sep["mean"][a][..., :nx], z["ref_mean"][a][..., :nx]) < TOL_MEAN
        for q in range(6):
            assert crel(sep["cov"][q][..., :nx], z["ref_cov"][q][..., :nx]) < TOL_COV


# ------------------------------------------------------------------ the production workload's instantiation

def _production_block(nx, ny):
    """The 540x540x256 workload (5 angles 5..45 deg, Ricker 25..35 Hz, nzp 256, 4 realisations,
    separable prior) on a lateral window whose long side keeps the 540-point transform."""
    spec = synth.config1(seed=21)
    spec.nx, spec.ny = nx, ny
    return synth.make_block(spec)


@pytest.mark.parametrize("lateral,sb", [((540, 12), None), ((12, 540), None), ((540, 12), 0)])
def test_production_instantiation_against_fp64_oracle(ctx, lateral, sb):
    """Same pencil-pass instantiation as the full 540x540x256 block (5 angle stacks, nzp 256
    through the 16x16 four-step z split, 4 realisations) and the 540-point row (x) or column
    (y) transforms, with the reference RandomGen noise (parity mode): posterior mean 1e-4,
    covariance 1e-3, realisations 1e-4 against the FP64 oracle.

    Residual spectra: every bin of the prior-mean spectrum carries the FP32 rounding of the
    large constant background (ln 3000 over 1.66 M voxels) through K mu, so FP32 residuals
    differ from FP64 ones by up to a few 1e-3 here; the reference's own FP32 path (FFTW 2.1.2
    float, oracle/_ref) reaches 3.5e-3 on this block.  The bound is therefore "no worse than
    the reference's FP32 path" (1.5 x its error, at least 1e-3) when oracle/_ref is present,
    else 5e-3."""
    blk = _production_block(*lateral)
    post = ref64.posterior(blk)
    noise = ob.sim_noise(17, blk.nsim, blk.nxp, blk.nyp, blk.nzp)
    # sb = 0: the pencil pass without realisation slots (the mean stored first and added back
    # to every realisation)
    pk = api.pencil_key(blk.nzp, blk.ntheta)
    saved = api.tuning_get("pencil_sb", pk)
    if sb is not None:
        api.tuning_set("pencil_sb", pk, sb)
    try:
        out = api.invert_block(ctx, blk, api.PRIOR_SEPARABLE, noise=noise, keep_residual=True)
    finally:
        api.tuning_set("pencil_sb", pk, saved)
    _check_posterior(blk, out, post, post.n_inverted)
    if ob.ref32_available():
        covs, _ = ref64.prior_cov_grids(blk)
        ec = ref64.fill_err_corr_zero_grad(blk.corr_xy, blk.nxp, blk.nyp, blk.nzp)
        r32 = ob.ref32_invert(blk, covs, ec, nsim=0, seed=1)
        bound = [max(1e-3, 1.5 * crel(r32.resid_spec[l], post.resid_spec[l])) for l in range(blk.ntheta)]
    else:
        bound = [5e-3] * blk.ntheta
    for l in range(blk.ntheta):
        assert crel(out["resid_spec"][l], post.resid_spec[l]) < bound[l], ("resid", l, bound[l])
    for s in range(blk.nsim):
        sim = ref64.simulate(blk, post, noise[s])
        for a in range(3):
            assert crel(out["sims"][s, a][..., :blk.nxp], sim[a][..., :blk.nxp]) < TOL_SIM, (s, a)


def test_production_instantiation_device_noise_statistics(ctx):
    """Product-mode noise on the production instantiation: per voxel, each realisation's
    deviation from the posterior mean has the posterior variance (covariance at lag 0), and
    the mean and covariance match the FP64 oracle as in parity mode."""
    blk = _production_block(540, 12)
    post = ref64.posterior(blk)
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=99)
    _keep = job.upload_block()
    job.run()
    out = job.download_outputs()
    c = job.counters()
    job.close()
    nx = blk.nxp
    assert c["inverted_bins"] == post.n_inverted
    for a in range(3):
        assert crel(out["mean"][a][..., :nx], post.mean[a][..., :nx]) < TOL_MEAN
    for q in range(6):
        assert crel(out["cov"][q][..., :nx], post.cov[q][..., :nx]) < TOL_COV
    dev = out["sims"][..., :nx] - out["mean"][None, ..., :nx]
    for a in range(3):
        emp = float(np.mean(dev[:, a].astype(np.float64) ** 2))
        assert 0.85 < emp / post.cov[a, 0, 0, 0] < 1.15, (a, emp, post.cov[a, 0, 0, 0])


@pytest.mark.parametrize("grid", ["data", "mean"])
def test_non_finite_grid_reported_as_numeric(ctx, grid):
    """A single NaN voxel in a data or prior-mean grid: the run completes, and the counters
    call reports CRAVA_ENUMERIC (the NaN reaches every bin through the transforms)."""
    blk = synth.make_block(synth.BlockSpec(nx=16, ny=12, nz=20, nsim=1, seed=3))
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=5)
    _keep = job.upload_block()
    g = np.array((blk.data[1] if grid == "data" else blk.mean[2]), copy=True)
    g[7, 5, 3] = np.nan
    _keep.append(job.upload(api.ROLE_DATA if grid == "data" else api.ROLE_MEAN, 1 if grid == "data" else 2, g))
    job.run()
    with pytest.raises(api.CravaError) as ei:
        job.counters()
    assert ei.value.status == api.ENUMERIC
    # the same job with finite inputs runs clean again
    _keep.append(job.upload(api.ROLE_DATA if grid == "data" else api.ROLE_MEAN, 1 if grid == "data" else 2,
                            blk.data[1] if grid == "data" else blk.mean[2]))
    job.run()
    assert job.counters()["nonfinite_tiles"] == 0
    job.close()
