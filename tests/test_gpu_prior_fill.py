"""Prior grids generated on the device (crava_job_fill_prior) against the oracle.

InitializeCorrelations' six covariance grids (fillInParamCorr x priorVar0) and fillInErrCorr
with lateral correlation gradients: the device grids equal the oracle's float32 restatement of
the reference's float arithmetic bit for bit; the inversion on them matches the FP64 oracle
with the constant-thickness parity tolerances (mean 1e-4, covariance 1e-3).
"""
import dataclasses

import numpy as np
import pytest

from crava_b200 import api, synth
from oracle import ref64

pytestmark = pytest.mark.gpu


def rel(x, ref):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def grad_block(gi, gj, dims=(30, 24, 40, 32, 27, 48), nsim=0):
    nx, ny, nz, nxp, nyp, nzp = dims
    spec = synth.BlockSpec(nx=nx, ny=ny, nz=nz, nxp=nxp, nyp=nyp, nzp=nzp, theta_deg=(8.0, 20.0, 32.0),
                           peak_hz=(30.0,) * 3, sn=(5.0,) * 3, nsim=nsim, seed=23, corr_grad_i=gi, corr_grad_j=gj)
    return synth.make_block(spec)


@pytest.mark.parametrize("gi,gj", [(0.0, 0.0), (0.37, -0.21), (-1.3, 0.8)])
def test_filled_grids_equal_the_reference_float_grids(ctx, gi, gj):
    blk = grad_block(gi, gj)
    job = api.Job(ctx, blk, api.PRIOR_GRIDS)
    try:
        job.fill_prior(blk.corr_grad_i, blk.corr_grad_j)
        covs, _pairs = ref64.prior_cov_grids(blk)
        for q in range(6):
            got = job.download(api.ROLE_PRIOR_COV, q)[..., :blk.nxp]
            assert np.array_equal(got, covs[q]), q
        err = ref64.fill_err_corr(blk.corr_xy, blk.nxp, blk.nyp, blk.nzp, blk.corr_grad_i, blk.corr_grad_j)
        assert np.array_equal(job.download(api.ROLE_ERR_CORR, 0)[..., :blk.nxp], err)
    finally:
        job.close()


def test_inversion_on_filled_grids_matches_oracle(ctx):
    blk = grad_block(0.37, -0.21)
    job = api.Job(ctx, blk, api.PRIOR_GRIDS)
    try:
        for l in range(blk.ntheta):
            job.upload(api.ROLE_DATA, l, blk.data[l])
        for a in range(3):
            job.upload(api.ROLE_MEAN, a, blk.mean[a])
        job.fill_prior(blk.corr_grad_i, blk.corr_grad_j)
        job.run()
        out = job.download_outputs()
        cnt = job.counters()
    finally:
        job.close()
    post = ref64.posterior(blk)
    nxp = blk.nxp
    for a in range(3):
        assert rel(out["mean"][a][..., :nxp], post.mean[a][..., :nxp]) < 1e-4, a
    for q in range(6):
        assert rel(out["cov"][q][..., :nxp], post.cov[q][..., :nxp]) < 1e-3, q
    assert cnt["inverted_bins"] == post.n_inverted
    # the gradients matter: the zero-gradient prior gives a different posterior
    flat = ref64.posterior(dataclasses.replace(blk, corr_grad_i=0.0, corr_grad_j=0.0))
    assert rel(flat.cov[0][..., :nxp], post.cov[0][..., :nxp]) > 1e-3


def test_fill_prior_needs_a_grids_job(ctx):
    blk = grad_block(0.0, 0.0)
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE)
    try:
        with pytest.raises(api.CravaError) as ei:
            job.fill_prior(0.1, 0.1)
        assert ei.value.status == api.ESTATE
    finally:
        job.close()


def test_estimated_auto_cov_grids_and_inversion(ctx):
    """Estimated covariance (InitializeCorrelations with cov_estimated): the six grids
    FillInLateralCorr(corrXY, circAutoCov_q) equal the oracle's float restatement bit for bit,
    and the inversion on them matches the FP64 oracle (mean 1e-4, covariance 1e-3)."""
    blk = grad_block(0.37, -0.21)
    nlag = 12
    lag = np.arange(nlag)
    rho = np.exp(-3.0 * (4.0 * lag / 40.0) ** 2)
    ac = blk.prior_var0[None] * rho[:, None, None]
    ac[:, 0, 1] *= np.exp(-0.02 * lag)          # a cross-covariance that differs forward / backward
    act = api.circ_auto_cov(ac, blk.nzp, 4.0)
    job = api.Job(ctx, blk, api.PRIOR_GRIDS)
    try:
        job.fill_prior_auto_cov(act, blk.corr_grad_i, blk.corr_grad_j)
        covs = [ref64.fill_param_corr(blk.corr_xy, act[q], blk.nxp, blk.nyp, blk.nzp, blk.corr_grad_i,
                                      blk.corr_grad_j) for q in range(6)]
        for q in range(6):
            got = job.download(api.ROLE_PRIOR_COV, q)[..., :blk.nxp]
            assert np.array_equal(got, covs[q]), q
        for l in range(blk.ntheta):
            job.upload(api.ROLE_DATA, l, blk.data[l])
        for a in range(3):
            job.upload(api.ROLE_MEAN, a, blk.mean[a])
        job.run()
        out = job.download_outputs()
        post = ref64.posterior(blk, cov_grids=covs)
        for a in range(3):
            assert rel(out["mean"][a][..., :blk.nxp], post.mean[a][..., :blk.nxp]) < 1e-4, a
        for q in range(6):
            assert rel(out["cov"][q][..., :blk.nxp], post.cov[q][..., :blk.nxp]) < 1e-3, q
    finally:
        job.close()


def test_base_prior_path_equals_the_six_spectra_path(ctx):
    """After crava_job_fill_prior the run transforms one prior grid and scales it per pair;
    re-uploading the same six grids takes the six-spectra path.  Both agree to the float
    rounding of the grids' products."""
    blk = grad_block(0.37, -0.21, nsim=1)
    outs = []
    for reupload in (False, True):
        job = api.Job(ctx, blk, api.PRIOR_GRIDS, seed=4)
        try:
            for l in range(blk.ntheta):
                job.upload(api.ROLE_DATA, l, blk.data[l])
            for a in range(3):
                job.upload(api.ROLE_MEAN, a, blk.mean[a])
            job.fill_prior(blk.corr_grad_i, blk.corr_grad_j)
            if reupload:
                for q in range(6):
                    job.upload(api.ROLE_PRIOR_COV, q, job.download(api.ROLE_PRIOR_COV, q))
            job.run()
            o = job.download_outputs()
            o["counters"] = job.counters()
            outs.append(o)
        finally:
            job.close()
    a, b = outs
    nxp = blk.nxp
    for q in range(3):
        assert rel(a["mean"][q][..., :nxp], b["mean"][q][..., :nxp]) < 1e-5, q
    for q in range(6):
        assert rel(a["cov"][q][..., :nxp], b["cov"][q][..., :nxp]) < 1e-5, q
    assert rel(a["sims"][..., :nxp], b["sims"][..., :nxp]) < 1e-4
    assert a["counters"]["inverted_bins"] == b["counters"]["inverted_bins"]
