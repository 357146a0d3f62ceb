"""Local-noise shrinkage on the GPU (crava_job_local_noise: correctVpVsRho and the
local-noise mixing of simulate) against the FP64 oracle restatement, applied to the job's
own posterior and realisations: posterior mean and realisations within 1e-5 (norm-wise
relative), the padding untouched."""
import numpy as np
import pytest

from crava_b200 import api, synth
from oracle import ref64

pytestmark = pytest.mark.gpu


def crel(x, ref):
    return float(np.linalg.norm(np.asarray(x, np.float64) - ref) / np.linalg.norm(ref))


@pytest.mark.parametrize("spec", [
    dict(nx=30, ny=20, nz=32, nxp=32, nyp=24, nzp=40, theta_deg=(5.0, 15.0, 25.0, 35.0), peak_hz=(30.0,) * 4,
         sn=(5.0,) * 4, nsim=2, seed=4),
    dict(nx=24, ny=18, nz=30, theta_deg=(10.0, 30.0), peak_hz=(30.0,) * 2, sn=(6.0,) * 2, nsim=1, seed=5),
])
def test_local_noise_matches_oracle(spec):
    blk = synth.make_block(synth.BlockSpec(**spec))
    ctx = api.Context(0)
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=31)
    _k = job.upload_block()
    job.run()
    before = job.download_outputs()
    pv0 = job.counters()["post_var0"].astype(np.float64)
    rng = np.random.default_rng(spec["seed"])
    scales = (1.0 + 3.0 * rng.random((blk.ntheta, blk.ny, blk.nx))).astype(np.float32)
    job.local_noise(scales)
    after = job.download_outputs()
    job.close()
    ctx.close()
    ref_mean, ref_sims = ref64.local_noise_correct(blk, before["mean"], before["sims"], scales.astype(np.float64), pv0)
    nx, ny, nz = blk.nx, blk.ny, blk.nz
    for a in range(3):
        assert crel(after["mean"][a, :nz, :ny, :nx], ref_mean[a, :nz, :ny, :nx]) < 1e-5, a
        # the padding keeps the uncorrected values
        assert np.array_equal(after["mean"][a, nz:], before["mean"][a, nz:])
    for s in range(blk.nsim):
        for a in range(3):
            assert crel(after["sims"][s, a, :nz, :ny, :nx], ref_sims[s, a, :nz, :ny, :nx]) < 1e-5, (s, a)
    # the correction changed something where the noise is not uniform
    assert not np.array_equal(after["mean"], before["mean"])
