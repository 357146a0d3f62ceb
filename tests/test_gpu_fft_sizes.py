"""The four-step transforms over the whole size table: 3D r2c / c2r through the C ABI against
numpy float64 for lengths of every split shape (x through the half-length rows, y and z
through the column kernels), both FFTGrid scalings."""
import math

import numpy as np
import pytest

from crava_b200 import api

pytestmark = pytest.mark.gpu

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


# (nxp, nyp, nzp): nxp / 2, nyp and nzp cover splits with both factors odd, both even,
# prime-power factors (25, 27, 49), sevens, and the 32 x 32 end of the table
SHAPES = [(144, 72, 16), (90, 100, 18), (250, 125, 21), (126, 243, 20), (196, 49, 28), (350, 81, 30),
          (450, 98, 25), (648, 36, 27), (1008, 45, 32), (2048, 16, 40), (168, 1024, 6), (882, 441, 4)]


@pytest.mark.parametrize("dims", SHAPES)
@pytest.mark.parametrize("covariance", [False, True])
def test_four_step_sizes_match_numpy(ctx, dims, covariance):
    import torch
    nxp, nyp, nzp = dims
    rnxp = 2 * (nxp // 2 + 1)
    rng = np.random.default_rng(nxp + 3 * nyp + 7 * nzp)
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
    assert crel(g.cpu().numpy()[..., :nxp], x) < TOL_FFT
