"""Non-constant thickness on the GPU through the C ABI, against the oracle.

divideDataByScaleWavelet + interpolateSeismic (crava_job_divide_data) and the posterior of
the non-constant branch (K = kD A, src/avoinversion.cpp:976-1014).

Tolerances (norm-wise relative per grid): divided data 2e-5 against the oracle (FP32
trace transforms against float64 ones; the adjustment factor is the same float32
arithmetic on both sides); posterior mean 1e-4 and covariance 1e-3 as the constant-
thickness parity tests.  The trace interpolation is checked exactly: an interpolated trace
is the float32 mean of its neighbours in the kernel's own output.
"""
import dataclasses

import numpy as np
import pytest

from crava_b200 import api, synth
from oracle import ref64

pytestmark = pytest.mark.gpu

TOL_DIV = 2e-5
TOL_MEAN = 1e-4
TOL_COV = 1e-3


def rel(x, ref):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))


def thick_block(nx=40, ny=30, nz=50, nxp=48, nyp=40, nzp=64, nsim=1, seed=5, threshold=0.0, theta=(8.0, 20.0, 32.0)):
    spec = synth.BlockSpec(nx=nx, ny=ny, nz=nz, nxp=nxp, nyp=nyp, nzp=nzp, nsim=nsim, seed=seed, theta_deg=theta,
                           peak_hz=(30.0,) * len(theta), sn=(6.0,) * len(theta))
    return synth.with_rel_thick(synth.make_block(spec), seed=seed, threshold=threshold)


def oracle_divided(blk):
    div = ref64.divide_data_by_scale_wavelet(blk)
    return np.stack([ref64.interpolate_seismic(div[l], blk, blk.energy_threshold) for l in range(blk.ntheta)])


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def gpu_divided(ctx, blk):
    job = api.Job(ctx, blk)
    try:
        _keep = job.upload_block()
        job.divide_data()
        return np.stack([job.download(api.ROLE_DATA, l) for l in range(blk.ntheta)])
    finally:
        job.close()


@pytest.mark.parametrize("dims", [(40, 30, 50, 48, 40, 64), (40, 30, 50, 45, 36, 60), (33, 21, 90, 35, 27, 100)])
def test_divide_data_matches_oracle(ctx, dims):
    nx, ny, nz, nxp, nyp, nzp = dims
    blk = thick_block(nx, ny, nz, nxp, nyp, nzp)
    got = gpu_divided(ctx, blk)
    ref = oracle_divided(blk)
    for l in range(blk.ntheta):
        assert rel(got[l][..., :nxp], ref[l][..., :nxp]) < TOL_DIV, l
    # the division changed the data (it is not an identity)
    assert rel(got[0][..., :nxp], blk.data[0][..., :nxp]) > 1e-2


def test_unit_thickness_interior_is_a_deconvolution(ctx):
    """rel_thick = 1: the factor is 1/conj(W) wherever the stabilisation is inactive, so
    re-applying the wavelet (K's conj(W) of the constant branch) gives back the band-passed
    data; checked through the oracle factor and the GPU result agreeing."""
    blk = thick_block()
    blk = dataclasses.replace(blk, rel_thick=np.ones((blk.nyp, blk.nxp)), min_rel_thick=1.0)
    got = gpu_divided(ctx, blk)
    ref = oracle_divided(blk)
    assert rel(got[..., :blk.nxp], ref[..., :blk.nxp]) < TOL_DIV


def plant_dead_traces(blk, weak=None):
    data = blk.data.copy()
    dead = [(5, 5), (0, 0), (1, 0)] + [(i, 8) for i in range(10, 15)] + [(20, 12), (21, 12), (20, 13), (21, 13)]
    for (i, j) in dead:
        data[:, :, j, i] = 0.0
    for (i, j) in (weak or []):
        data[:, :, j, i] *= 1e-3
    return dataclasses.replace(blk, data=data), dead


@pytest.mark.parametrize("threshold", [0.0, 0.05])
def test_dead_traces_interpolated(ctx, threshold):
    blk = thick_block(threshold=threshold)
    weak = [(30, 20), (31, 25)] if threshold > 0 else None
    blk, dead = plant_dead_traces(blk, weak)
    got = gpu_divided(ctx, blk)
    ref = oracle_divided(blk)
    nxp = blk.nxp
    for l in range(blk.ntheta):
        assert rel(got[l][..., :nxp], ref[l][..., :nxp]) < TOL_DIV, l
    # the isolated dead trace is exactly the float32 mean of its four neighbours
    g = got[0]
    i, j = 5, 5
    s = np.float32(0)
    for (a, b) in [(i - 1, j), (i + 1, j), (i, j - 1), (i, j + 1)]:
        s = (s + g[:, b, a]).astype(np.float32)
    assert np.array_equal(g[:, j, i], (s / np.float32(4)).astype(np.float32))
    # the reference leaves the first dead trace of the scan without a second good
    # neighbour at its turn ((0,0): only (0,1) is good) and never revisits it: it keeps
    # its divided value, zero
    assert np.all(g[:, 0, 0] == 0.0)
    assert np.any(g[:, 0, 1] != 0.0)   # (1,0) was interpolated from (2,0) and (1,1)
    if weak:
        for (i, j) in weak:
            assert np.any(got[0][:, j, i] != 0.0)


@pytest.mark.parametrize("prior_mode,fp64,dims", [
    (api.PRIOR_SEPARABLE, 0.0, None), (api.PRIOR_GRIDS, 0.0, None),
    (api.PRIOR_SEPARABLE, 1.0, None),                      # every bin refactorised in FP64
    (api.PRIOR_SEPARABLE, 0.0, (33, 21, 90, 35, 27, 105)),  # odd nxp and nzp
])
def test_nonconst_inversion_matches_oracle(ctx, prior_mode, fp64, dims):
    blk = thick_block(*dims, nsim=0) if dims else thick_block(nsim=0)
    kw = {"fp64_threshold": fp64}
    if prior_mode == api.PRIOR_GRIDS:
        covs, _pairs = ref64.prior_cov_grids(blk)
        kw.update(cov_grids=[c[..., :blk.nxp] for c in covs],
                  err_corr=ref64.fill_err_corr_zero_grad(blk.corr_xy, blk.nxp, blk.nyp, blk.nzp)[..., :blk.nxp])
    out = api.invert_block(ctx, blk, prior_mode=prior_mode, **kw)
    ref_blk = dataclasses.replace(blk, data=oracle_divided(blk))
    post = ref64.posterior(ref_blk)
    nxp = blk.nxp
    for a in range(3):
        assert rel(out["mean"][a][..., :nxp], post.mean[a][..., :nxp]) < TOL_MEAN, a
    for q in range(6):
        assert rel(out["cov"][q][..., :nxp], post.cov[q][..., :nxp]) < TOL_COV, q
    assert out["counters"]["inverted_bins"] == post.n_inverted
    # the non-constant branch differs from the constant one on the same data
    const = ref64.posterior(dataclasses.replace(ref_blk, rel_thick=None))
    assert rel(const.mean[0][..., :nxp], post.mean[0][..., :nxp]) > 1e-3


def test_divide_data_needs_the_flag(ctx):
    blk = synth.make_block(synth.BlockSpec(nx=16, ny=12, nz=20, nsim=0))
    job = api.Job(ctx, blk)
    try:
        with pytest.raises(api.CravaError) as ei:
            job.divide_data()
        assert ei.value.status == api.ESTATE
    finally:
        job.close()


def test_noalloc_and_serving_reject_nonconst(ctx):
    blk = thick_block(nsim=0)
    d, _keep = api.make_desc(blk)
    assert d.flags & api.FLAG_NONCONST_THICK
    vp = __import__("ctypes").c_void_p
    arr_in = (vp * (blk.ntheta + 3))(*([1] * (blk.ntheta + 3)))
    arr_out = (vp * 9)(*([1] * 9))
    st = api.lib().crava_invert_noalloc(__import__("ctypes").byref(d), arr_in, arr_out, None)
    assert st == api.ENOTSUP


def test_divide_data_matches_the_golden_fixture(ctx):
    """The GPU division against the reference-FFTW division frozen in
    tests/golden/t1_nonconst.npz (followed by the oracle's interpolateSeismic, which for
    this block only rebuilds the padding)."""
    from tests.golden import golden_io
    blk, z = golden_io.load("t1_nonconst")
    got = gpu_divided(ctx, blk)
    ref = np.stack([ref64.interpolate_seismic(z["ref_divided"][l].astype(np.float64), blk, blk.energy_threshold)
                    for l in range(blk.ntheta)])
    for l in range(blk.ntheta):
        assert rel(got[l][..., :blk.nxp], ref[l][..., :blk.nxp]) < TOL_DIV, l


def test_nonconst_posterior_against_reference_arithmetic(ctx):
    """The non-constant branch of the per-bin step (K = kD A with the wavelet-normalised error
    multipliers and fillInverseAbskWRobust, src/avoinversion.cpp:976-1014, 1296-1322) against the
    reference's FP32 numerics (oracle/_ref: FFTW 2.1.2, lib_matr.c and that branch restated
    around them), both on the same divided data: mean 1e-4, covariance 1e-3, inverted bins and
    Cholesky fallbacks equal."""
    from oracle import bindings as ob
    if not ob.ref32_available():
        pytest.skip("oracle/_ref not built")
    blk = thick_block(nsim=0)
    job = api.Job(ctx, blk)
    try:
        _keep = job.upload_block()
        job.divide_data()
        div = np.stack([job.download(api.ROLE_DATA, l) for l in range(blk.ntheta)])
        job.run()
        out = job.download_outputs()
        cnt = job.counters()
    finally:
        job.close()
    nxp = blk.nxp
    ref_blk = dataclasses.replace(blk, data=div[..., :nxp])
    covs, _ = ref64.prior_cov_grids(ref_blk)
    ec = ref64.fill_err_corr_zero_grad(blk.corr_xy, blk.nxp, blk.nyp, blk.nzp)
    r32 = ob.ref32_invert(ref_blk, covs, ec, nsim=0, seed=1, nonconst=True)
    assert cnt["inverted_bins"] == r32.n_inverted and cnt["chol_fallbacks"] == r32.n_chol_fail
    for a in range(3):
        assert rel(out["mean"][a][..., :nxp], r32.mean[a][..., :nxp]) < TOL_MEAN, a
    for q in range(6):
        assert rel(out["cov"][q][..., :nxp], r32.cov[q][..., :nxp]) < TOL_COV, q
