"""The oracle against the reference's own numerics (golden fixtures) and its self-checks.

Fixtures: tests/golden/*.npz, written by tests/golden/make_golden.py from oracle/_ref
(FFTW 2.1.2 float + lib_matr.c + RandomGen of the reference).  Tolerances: the FP64
restatement against the FP32 reference path, posterior mean 1e-4, covariance 1e-3,
realisations 1e-4 (norm-wise relative); the noise source bit for bit.
"""
import math

import numpy as np
import pytest

from oracle import bindings as ob
from oracle import ref64
from tests.golden import golden_io

CASES = golden_io.names()


def crel(x, ref):
    x = np.asarray(x, dtype=np.complex128)
    ref = np.asarray(ref, dtype=np.complex128)
    return float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))


def test_fixtures_present():
    assert len(CASES) >= 5


@pytest.mark.parametrize("name", CASES)
def test_noise_restatement_bit_exact(name):
    blk, z = golden_io.load(name)
    n = ob.sim_noise(int(z["noise_seed"]), blk.nsim, blk.nxp, blk.nyp, blk.nzp, use_ref=False)
    assert np.array_equal(n, z["noise"])


@pytest.mark.parametrize("name", CASES)
def test_fp64_oracle_matches_reference_path(name):
    blk, z = golden_io.load(name)
    post = ref64.posterior(blk)
    nx = blk.nxp
    assert post.n_inverted == int(z["ref_n_inverted"])
    assert post.n_chol_fail == int(z["ref_n_chol_fail"])
    for a in range(3):
        assert crel(post.mean[a][..., :nx], z["ref_mean"][a][..., :nx]) < 1e-4
    for q in range(6):
        assert crel(post.cov[q][..., :nx], z["ref_cov"][q][..., :nx]) < 1e-3
    for l in range(blk.ntheta):
        assert crel(post.resid_spec[l], z["ref_resid_spec"][l]) < 1e-3
    for s in range(blk.nsim):
        sim = ref64.simulate(blk, post, z["noise"][s])
        for a in range(3):
            assert crel(sim[a][..., :nx], z["ref_sims"][s, a][..., :nx]) < 1e-4


@pytest.mark.skipif(not ob.ref32_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", CASES[:2])
def test_reference_path_reproduces_fixture(name):
    blk, z = golden_io.load(name)
    r = ob.ref32_invert(blk, list(z["cov_grids"]), z["err_corr"], nsim=blk.nsim, seed=int(z["noise_seed"]))
    assert np.array_equal(r.mean, z["ref_mean"])
    assert np.array_equal(r.cov, z["ref_cov"])
    assert np.array_equal(r.sims, z["ref_sims"])


def test_fft_scalings_round_trip_and_parseval():
    rng = np.random.default_rng(0)
    nzp, nyp, nxp = 10, 12, 15
    x = np.zeros((nzp, nyp, 2 * (nxp // 2 + 1)))
    x[..., :nxp] = rng.standard_normal((nzp, nyp, nxp))
    for cov in (False, True):
        spec = ref64.fft_in_place(x, nxp, cov)
        back = ref64.inv_fft_in_place(spec, nxp, cov)
        assert np.allclose(back[..., :nxp], x[..., :nxp], atol=1e-12)
    # PARAMETER scaling is unitary: Parseval over the full (Hermitian-extended) spectrum
    spec = np.fft.fftn(x[..., :nxp]) / math.sqrt(x[..., :nxp].size)
    assert np.isclose(np.sum(np.abs(spec) ** 2), np.sum(x[..., :nxp] ** 2))


@pytest.fixture(scope="module")
def g1():
    return golden_io.load("g1_even")


def test_not_inverted_bins_keep_prior(g1):
    blk, z = g1
    post = ref64.posterior(blk)
    inv = ref64.invert_mask(blk)
    mean_spec = np.stack([ref64.fft_in_place(blk.mean[a], blk.nxp, False) for a in range(3)])
    assert np.allclose(post.mean_spec[:, ~inv], mean_spec[:, ~inv])
    data_spec = np.stack([ref64.fft_in_place(blk.data[l], blk.nxp, False) for l in range(blk.ntheta)])
    assert np.allclose(post.resid_spec[:, ~inv], data_spec[:, ~inv])


def test_posterior_variance_not_above_prior(g1):
    blk, z = g1
    post = ref64.posterior(blk)
    covs, _ = ref64.prior_cov_grids(blk)
    S = ref64.param_cov_from_spectra([ref64.fft_in_place(c, blk.nxp, True) for c in covs], blk.prior_var0)
    for q in range(3):
        assert np.all(post.cov_spec[q].real <= S[..., q, q].real * (1 + 1e-9) + 1e-15)


def test_data_free_limit_gives_prior(g1):
    blk, z = g1
    import copy
    b2 = copy.copy(blk)
    b2.err_theta_cov = blk.err_theta_cov * 1e14
    post = ref64.posterior(b2)
    mean_spec = np.stack([ref64.fft_in_place(blk.mean[a], blk.nxp, False) for a in range(3)])
    assert crel(post.mean_spec, mean_spec) < 1e-6
    covs, _ = ref64.prior_cov_grids(blk)
    S = ref64.param_cov_from_spectra([ref64.fft_in_place(c, blk.nxp, True) for c in covs], blk.prior_var0)
    for q, (a, b) in enumerate([(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]):
        assert crel(post.cov_spec[q], S[..., a, b]) < 1e-6


def test_noise_free_limit_rank3():
    """Three angle stacks, negligible error: inverted bins reproduce the data exactly."""
    from crava_b200 import synth
    blk = synth.make_block(synth.BlockSpec(nx=8, ny=8, nz=32, theta_deg=(10.0, 25.0, 40.0), peak_hz=(30.0,) * 3,
                                           sn=(5.0,) * 3, nsim=1, seed=3, wnc=1e-6))
    blk.err_theta_cov = blk.err_theta_cov * 1e-10
    post = ref64.posterior(blk)
    inv = ref64.invert_mask(blk)
    data_spec = np.stack([ref64.fft_in_place(blk.data[l], blk.nxp, False) for l in range(blk.ntheta)])
    assert np.linalg.norm(post.resid_spec[:, inv]) < 1e-4 * np.linalg.norm(data_spec[:, inv])


def test_cholesky_rejections_follow_reference():
    # non-positive scale
    M = np.array([[[0.0, 0.0], [0.0, 1.0]]], dtype=np.complex128)
    _, ok = ref64.chol_cpx(M)
    assert not ok[0]
    # pivot below 1e-20 after scaling
    M = np.array([[[1.0, 1.0], [1.0, 1.0 + 1e-22]]], dtype=np.complex128)
    _, ok = ref64.chol_cpx(M)
    assert not ok[0]
    # a Hermitian positive definite matrix factors to L L^H
    rng = np.random.default_rng(1)
    B = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
    M = (B @ B.conj().T + 4 * np.eye(4))[None]
    L, ok = ref64.chol_cpx(M)
    assert ok[0]
    assert np.allclose(np.tril(L[0]) @ np.tril(L[0]).conj().T, M[0])


def test_separable_posterior_equals_the_grid_path():
    """The slab-wise separable spectra give the grid path's posterior up to the float32
    rounding of the prior grids' products."""
    from crava_b200 import synth
    blk = synth.make_block(synth.BlockSpec(nx=24, ny=20, nz=40, nsim=0, seed=4))
    a = ref64.posterior(blk)
    b = ref64.posterior(blk, slab=7, separable=True)
    for x, y in ((b.mean, a.mean), (b.cov, a.cov)):
        assert np.linalg.norm(x - y) / np.linalg.norm(y) < 1e-6
    assert a.n_inverted == b.n_inverted and a.n_chol_fail == b.n_chol_fail


def test_nonconst_branch_restatement_matches_reference_arithmetic():
    """The FP64 restatement of the non-constant-thickness per-bin step (K = kD A, error
    multipliers 1/norm, kD3/norm(errorSmooth3), fillInverseAbskWRobust) against the same branch
    restated around the reference's FFTW 2.1.2 and lib_matr.c (oracle/_ref), on the same
    divided data: mean and covariance within 1e-5; the constant-thickness branch differs."""
    import dataclasses
    from oracle import bindings as ob
    if not ob.ref32_available():
        pytest.skip("oracle/_ref not built")
    from crava_b200 import synth
    spec = synth.BlockSpec(nx=40, ny=30, nz=50, nxp=48, nyp=40, nzp=64, nsim=0, seed=5, theta_deg=(8.0, 20.0, 32.0),
                           peak_hz=(30.0,) * 3, sn=(6.0,) * 3)
    blk = synth.with_rel_thick(synth.make_block(spec), seed=5, threshold=0.0)
    div = ref64.divide_data_by_scale_wavelet(blk)
    div = np.stack([ref64.interpolate_seismic(div[l], blk, blk.energy_threshold) for l in range(blk.ntheta)])
    rb = dataclasses.replace(blk, data=div)
    post = ref64.posterior(rb)
    covs, _ = ref64.prior_cov_grids(rb)
    ec = ref64.fill_err_corr_zero_grad(blk.corr_xy, blk.nxp, blk.nyp, blk.nzp)
    r32 = ob.ref32_invert(rb, covs, ec, nsim=0, seed=1, nonconst=True)
    nx = blk.nxp
    rel = lambda a, b: float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))
    assert r32.n_inverted == post.n_inverted and r32.n_chol_fail == 0
    assert max(rel(r32.mean[a][..., :nx], post.mean[a][..., :nx]) for a in range(3)) < 1e-5
    assert max(rel(r32.cov[q][..., :nx], post.cov[q][..., :nx]) for q in range(6)) < 1e-5
    r32c = ob.ref32_invert(rb, covs, ec, nsim=0, seed=1, nonconst=False)
    assert rel(r32c.mean[0][..., :nx], post.mean[0][..., :nx]) > 1e-3
