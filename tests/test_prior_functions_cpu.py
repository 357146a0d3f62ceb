"""Host-side temporal prior functions of the C ABI against the oracle (no device):
crava_circ_corr_t (computeCircCorrT + makeCircCorrTPosDef) and crava_circ_auto_cov
(ComputeCircAutoCov + MakeCircAutoCovPosDef + TaperCircAutoCovFunction), 1e-6 norm-wise."""
import numpy as np
import pytest

from crava_b200 import api, synth
from oracle import ref64


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("nzp,dz,rng_ms,cut", [(128, 4.0, 40.0, 2), (90, 4.0, 60.0, 1), (256, 2.0, 30.0, 3)])
def test_circ_corr_t_matches_oracle_and_generator(nzp, dz, rng_ms, cut):
    pt = synth.prior_corr_t(nzp, dz, rng_ms)
    got = api.circ_corr_t(pt, cut, nzp)
    assert rel(got, ref64.circ_corr_t(pt, cut, nzp)) < 1e-6
    assert rel(got, synth.circ_corr_t(pt, cut, nzp)) < 1e-6
    assert got[0] == 1.0
    # its spectrum is non-negative and zero at k <= cut (makeCircCorrTPosDef)
    spec = np.fft.rfft(got.astype(np.float64))
    assert np.all(spec.real > -1e-5 * np.abs(spec).max()) and np.all(np.abs(spec[:cut + 1]) < 1e-4 * np.abs(spec).max())


def test_circ_corr_t_rejects_too_few_layers():
    with pytest.raises(api.CravaError) as e:
        api.circ_corr_t(np.array([1.0]), 40, 64)   # every frequency cut: lag 0 vanishes
    assert e.value.status == api.EINVAL


def _auto_cov(nlag, seed, separable):
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((3, 3))
    P0 = B @ B.T * 1e-3 + np.eye(3) * 1e-3
    lag = np.arange(nlag)
    rho = np.exp(-3.0 * (4.0 * lag / 40.0) ** 2)
    ac = P0[None] * rho[:, None, None]
    if not separable:   # a cross term that is not symmetric in lag
        ac[:, 0, 1] *= np.exp(-0.01 * lag)
        ac[:, 1, 0] *= np.exp(0.005 * lag) / np.exp(0.005 * lag[-1])
        ac[0, 1, 0] = ac[0, 0, 1]
    return ac, P0, rho


@pytest.mark.parametrize("separable", [True, False])
def test_circ_auto_cov_matches_oracle(separable):
    ac, _, _ = _auto_cov(20, 3, separable)
    got = api.circ_auto_cov(ac, 96, 4.0)
    ref = ref64.circ_auto_cov(ac, 96, 4.0)
    for q in range(6):
        assert rel(got[q], ref[q]) < 1e-6, q


def test_circ_auto_cov_keeps_a_positive_definite_separable_covariance():
    """A separable auto-covariance whose temporal spectrum is positive is already positive
    definite: the result is P0_ab times the circular correlation times the taper."""
    nzp, dz = 128, 4.0
    ac, P0, rho = _auto_cov(30, 5, True)
    got = api.circ_auto_cov(ac, nzp, dz)
    circ = np.zeros(nzp)
    for k in range(30):
        circ[k] = np.float32(rho[k])
        if k < 29:
            circ[nzp - k - 1] = np.float32(rho[k + 1])
    sd = min(50.0 / dz, nzp / 2)
    t = np.arange(nzp)
    m = np.where(t < nzp // 2 + 1, t, nzp - t)
    taper = np.exp(-0.5 * (m / sd) ** 2)
    for q, (a, b) in enumerate([(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]):
        want = np.float32(P0[a, b]) * circ * taper
        assert rel(got[q], want) < 1e-5, q
