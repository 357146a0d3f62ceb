"""CRAVA binary grid files (crava_grid_write_crava / crava_grid_read_crava) against the format
of FFTGrid::writeCravaFile (src/fftgrid.cpp:2183-2270) read independently with numpy: the tag
line, the simbox geometry and padded dimensions big-endian, the grid as big-endian floats;
a round trip through the file is exact; a file of other dimensions is rejected."""
import numpy as np
import pytest

from crava_b200 import api, synth

pytestmark = pytest.mark.gpu

GEOM = dict(x0=456000.0, y0=6780000.5, dx=25.0, dy=12.5, nx=61, ny=37, il0=1001.0, xl0=2001.0, il_step_x=0.5,
            il_step_y=-0.25, xl_step_x=0.125, xl_step_y=2.0, angle=0.3)


@pytest.mark.parametrize("dims", [(61, 37, 45), (300, 200, 250)])   # the second spans several staging chunks
def test_crava_file_round_trip_and_format(tmp_path, dims):
    import torch
    nxp, nyp, nzp = dims
    rnxp = 2 * (nxp // 2 + 1)
    rng = np.random.default_rng(nzp)
    grid = rng.standard_normal((nzp, nyp, rnxp)).astype(np.float32)
    ctx = api.Context(0)
    d = torch.from_numpy(grid).cuda()
    path = tmp_path / "g.crava"
    api.grid_write_crava(ctx, str(path), d.data_ptr(), rnxp, nyp, nzp, GEOM)
    raw = path.read_bytes()
    tag = b"crava_fftgrid_binary\n"
    assert raw.startswith(tag)
    h = raw[len(tag):]
    dbl = np.frombuffer(h[:32], dtype=">f8")
    assert list(dbl) == [GEOM["x0"], GEOM["y0"], GEOM["dx"], GEOM["dy"]]
    assert list(np.frombuffer(h[32:40], dtype=">i4")) == [GEOM["nx"], GEOM["ny"]]
    assert list(np.frombuffer(h[40:96], dtype=">f8")) == [GEOM[k] for k in ("il0", "xl0", "il_step_x", "il_step_y",
                                                                         "xl_step_x", "xl_step_y", "angle")]
    assert list(np.frombuffer(h[96:108], dtype=">i4")) == [rnxp, nyp, nzp]
    vals = np.frombuffer(h[108:], dtype=">f4")
    assert vals.size == grid.size and np.array_equal(vals.reshape(grid.shape), grid)
    back = torch.zeros_like(d)
    g2 = api.grid_read_crava(ctx, str(path), back.data_ptr(), rnxp, nyp, nzp)
    assert np.array_equal(back.cpu().numpy(), grid)
    assert g2 == pytest.approx(GEOM)
    with pytest.raises(api.CravaError) as e:
        api.grid_read_crava(ctx, str(path), back.data_ptr(), rnxp, nyp, nzp + 1)
    assert e.value.status == api.EINVAL
    ctx.close()


def test_posterior_mean_written_as_crava_file(tmp_path):
    """A job's posterior mean written straight from the device reads back as its download."""
    import torch
    blk = synth.make_block(synth.BlockSpec(nx=20, ny=16, nz=24, nsim=0, seed=2))
    ctx = api.Context(0)
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=1, nsim=0)
    _k = job.upload_block()
    job.run()
    rnxp, nyp, nzp = job.shape[2], job.shape[1], job.shape[0]
    path = tmp_path / "postvp.crava"
    api.grid_write_crava(ctx, str(path), job.device_ptr(api.ROLE_POST_MEAN, 0), rnxp, nyp, nzp, GEOM)
    vals = np.frombuffer(path.read_bytes()[len(b"crava_fftgrid_binary\n") + 108:], dtype=">f4")
    assert np.array_equal(vals.reshape(job.shape), job.download(api.ROLE_POST_MEAN, 0))
    job.close()
    ctx.close()
