"""Synthetic inputs follow the reference's set-up formulas."""
import math

import numpy as np

from crava_b200 import synth


def test_smooth_sizes_and_padding():
    s = synth.smooth_sizes(64, 256)
    assert 64 in s and 256 in s and 243 in s and 245 in s and 67 not in s
    assert synth.find_padding_size(131) == 135
    assert synth.find_padding_size(540) == 540


def test_reflection_matrix_pp_rows():
    A = synth.reflection_matrix([0.0, 30.0], 0.5)
    assert np.allclose(A[0], [0.5, 0.0, 0.5])
    th = math.radians(30.0)
    assert np.isclose(A[1, 0], (1 + math.tan(th) ** 2) / 2, rtol=1e-6)
    assert np.isclose(A[1, 1], -4 * 0.25 * math.sin(th) ** 2, rtol=1e-6)


def test_lateral_correlation_is_symmetric_and_one_at_origin():
    c = synth.corr_xy_surface(20, 16, 25.0, 25.0, 200.0)
    assert c[0, 0] == 1.0
    assert np.allclose(c[:, 1:], c[:, 1:][:, ::-1])
    assert np.allclose(c[1:, :], c[1:, :][::-1, :])


def test_circular_temporal_correlation_is_psd_and_band_cut():
    nzp, dt = 64, 4.0
    low = int(math.floor(5.0 * nzp * 0.001 * dt))
    c = synth.circ_corr_t(synth.prior_corr_t(nzp, dt, 40.0), low, nzp)
    assert np.isclose(c[0], 1.0)
    F = np.fft.rfft(c.astype(np.float64))
    assert np.all(F.real > -1e-5)
    assert np.all(np.abs(F[: low + 1]) < 1e-5)


def test_block_shapes_and_padding():
    b = synth.make_block(synth.BlockSpec(nx=13, ny=11, nz=19, nxp=14, nyp=12, nzp=20, nsim=1))
    assert b.data.shape == (3, 20, 12, 16)
    assert b.mean.shape == (3, 20, 12, 16)
    assert np.all(b.data[..., 14:] == synth.RMISSING)
    assert np.all(np.isfinite(b.data[..., :14]))
    assert np.allclose(b.err_theta_cov, b.err_theta_cov.T)
    assert np.all(np.linalg.eigvalsh(b.prior_var0) > 0)


def test_batch_specs_are_valid():
    specs = synth.batch_specs(n_blocks=8, nsim=2)
    for s in specs:
        assert 64 <= s.nx <= 256 and 64 <= s.ny <= 256 and 64 <= s.nz <= 200
        assert 2 <= len(s.theta_deg) <= 6
