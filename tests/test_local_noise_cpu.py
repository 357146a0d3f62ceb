"""The local-noise oracle (correctVpVsRho / newPosteriorCovPointwise / computeG restated in
oracle/ref64.py) on its own: with every scale equal and Sm - Smd positive definite, the local
posterior is the global one, so both per-trace maps are the identity; larger local noise
moves the posterior back toward the prior (the map shrinks the update)."""
import numpy as np

from oracle import ref64


def _mats(n, seed):
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((3, 3))
    Sm = B @ B.T + np.eye(3)
    C = rng.standard_normal((3, 3))
    Smd = Sm - 0.05 * (C @ C.T) - 0.05 * np.eye(3)   # Smd < Sm
    E = rng.standard_normal((n, n))
    Sth = E @ E.T + np.eye(n)
    return Sm, Smd, Sth


def test_g_reproduces_the_global_posterior():
    for n in (3, 4, 6):
        Sm, Smd, Sth = _mats(n, n)
        G = ref64.compute_g(Sm, Smd, Sth)
        delta = Sm @ G.T @ np.linalg.inv(G @ Sm @ G.T + Sth) @ G @ Sm
        assert np.abs(delta - (Sm - Smd)).max() < 1e-12


def test_unit_scales_leave_posterior_and_realisations_unchanged():
    n = 4
    Sm, Smd, Sth = _mats(n, 7)
    S, Ms = ref64.local_noise_maps(Sm, Smd, Sth, np.ones((n, 3, 5)))
    assert np.abs(S - np.eye(3)).max() < 1e-10
    assert np.abs(Ms - np.eye(3)).max() < 1e-10


def test_larger_noise_shrinks_the_update():
    n = 4
    Sm, Smd, Sth = _mats(n, 9)
    sc = np.ones((n, 1, 2))
    sc[:, 0, 1] = 4.0                       # the second trace is four times noisier
    S, _ = ref64.local_noise_maps(Sm, Smd, Sth, sc)
    dev = np.array([0.3, -0.2, 0.1])
    assert np.linalg.norm(S[0, 1] @ dev) < np.linalg.norm(S[0, 0] @ dev)
