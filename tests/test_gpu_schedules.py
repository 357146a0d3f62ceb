"""Schedule entries change speed, not results: the transform and pencil kernels give the same
bits under every schedule form they accept (one block at the production lengths of x and y,
540 points, with a short z axis)."""
import numpy as np
import pytest

from crava_b200 import api, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def outputs(ctx, blk, sched):
    saved = {}
    for (k, n), v in sched.items():
        saved[(k, n)] = api.tuning_get(k, n)
        api.tuning_set(k, n, v)
    try:
        o = api.invert_block(ctx, blk, api.PRIOR_SEPARABLE, seed=3)
    finally:
        for (k, n), v in saved.items():
            api.tuning_set(k, n, v)
    return o


@pytest.mark.parametrize("sched", [
    {("x4_stage_fwd", 270): 0, ("x4_stage_inv", 270): 0},
    {("x4_threads_fwd", 270): 256, ("x4_threads_inv", 270): 192},
    {("line4_threads_fwd", 540): 320, ("line4_threads_inv", 540): 448},
    {("line4_w_fwd", 540): 16, ("line4_w_inv", 540): 8, ("line4_threads_inv", 540): 512},
])
def test_schedule_forms_give_identical_results(ctx, sched):
    spec = synth.BlockSpec(nx=540, ny=540, nz=20, nzp=24, nsim=1, seed=9, theta_deg=(10.0, 25.0),
                           peak_hz=(30.0, 30.0), sn=(5.0, 5.0))
    blk = synth.make_block_fast(spec)
    base = outputs(ctx, blk, {})
    other = outputs(ctx, blk, sched)
    for key in ("mean", "cov", "sims"):
        assert np.array_equal(base[key], other[key]), key


@pytest.mark.parametrize("dims", [(96, 40, 256), (64, 30, 320)])
def test_pencil_without_realisation_slots(ctx, dims):
    """pencil_sb = 0 (the eigen-form pencil pass storing the mean first and adding it back to each
    realisation) against the default: the same mean and covariance bits, realisations equal to
    FP32 rounding (IFFT(mu) + IFFT(L z) against IFFT(mu + L z)); at nzp 320 with 6 angles it is the
    form that fits 8-bin tiles."""
    nx, ny, nz = dims
    nth = 5 if nz == 256 else 6
    spec = synth.BlockSpec(nx=nx, ny=ny, nz=nz, nsim=3, seed=11, theta_deg=tuple(np.linspace(5.0, 45.0, nth)),
                           peak_hz=(30.0,) * nth, sn=(5.0,) * nth)
    blk = synth.make_block_fast(spec)
    pk = api.pencil_key(blk.nzp, blk.ntheta)
    base = outputs(ctx, blk, {("pencil_kernel", pk): 2, ("pencil_sb", pk): 1, ("pencil_w", pk): 4})
    other = outputs(ctx, blk, {("pencil_kernel", pk): 2, ("pencil_sb", pk): 0, ("pencil_w", pk): 4})
    wide = outputs(ctx, blk, {("pencil_kernel", pk): 2, ("pencil_sb", pk): 0, ("pencil_w", pk): 8})
    for o in (other, wide):
        assert np.array_equal(base["mean"], o["mean"]) and np.array_equal(base["cov"], o["cov"])
        d = np.linalg.norm((o["sims"] - base["sims"]).astype(np.float64)) / np.linalg.norm(base["sims"])
        assert d < 1e-6, d
