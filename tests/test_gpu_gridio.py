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


STORM = dict(xmin=456000.0, lx=1525.0, ymin=6780000.5, ly=462.5, lz=120.0, angle=0.3, cubetype=3)


def storm_header(g, nx, ny, nz, flat, top="", bot=""):
    """Simbox::getStormHeader (src/simbox.cpp:1012-1034) restated with Python formatting."""
    f = lambda x: "%.6f" % x
    h = "storm_petro_binary\n0 %d %s\nFFTGrid\n" % (g["cubetype"], f(-99999.0))
    h += " ".join(f(g[k]) for k in ("xmin", "lx", "ymin", "ly")) + " "
    h += ("0.0 %s 0.0 0.0\n" % f(g["lz"])) if flat else ("%s %s 0.0 0.0\n" % (top, bot))
    h += "%s %s\n\n%d %d %d\n" % (f(g["lz"]), f(g["angle"] * 180.0 / np.pi), nx, ny, nz)
    return h.encode()


@pytest.mark.parametrize("dims,flat,padding", [((61, 37, 45, 64, 40, 50), True, False),
                                               ((61, 37, 45, 64, 40, 50), False, True),
                                               ((300, 200, 250, 320, 210, 256), True, False)])
def test_storm_file_format_round_trip_and_padding(tmp_path, dims, flat, padding):
    import torch
    from oracle import ref64
    nx, ny, nz, nxp, nyp, nzp = dims
    rnxp = 2 * (nxp // 2 + 1)
    rng = np.random.default_rng(nx + nz)
    grid = rng.standard_normal((nzp, nyp, rnxp)).astype(np.float32)
    ctx = api.Context(0)
    d = torch.from_numpy(grid).cuda()
    path = tmp_path / "g.storm"
    geom = dict(STORM, flat=1) if flat else dict(STORM, flat=0, top_name="top.irap", bot_name="base.irap")
    api.grid_write_storm(ctx, str(path), d.data_ptr(), (nx, ny, nz), (nxp, nyp, nzp), geom, padding=padding)
    raw = path.read_bytes()
    wx, wy, wz = (nxp, nyp, nzp) if padding else (nx, ny, nz)
    head = storm_header(STORM, wx, wy, wz, flat, "top.irap", "base.irap")
    assert raw[:len(head)] == head
    assert raw.endswith(b"0\n")
    vals = np.frombuffer(raw[len(head):-2], dtype=">f4").reshape(wz, wy, wx)
    assert np.array_equal(vals, grid[:wz, :wy, :wx])
    if padding:
        return
    # read back: the interior as written, the padding as the StormContGrid constructor fills it
    back = torch.full_like(d, 7.0)
    g2 = api.grid_read_storm(ctx, str(path), back.data_ptr(), (nx, ny, nz), (nxp, nyp, nzp))
    got = back.cpu().numpy()
    ref = ref64.storm_padding(grid[:nz, :ny, :nx], nxp, nyp, nzp)
    assert np.array_equal(got, ref)
    assert g2["cubetype"] == STORM["cubetype"] and g2["flat"] == 1
    assert g2["lz"] == pytest.approx(STORM["lz"]) and g2["angle"] == pytest.approx(STORM["angle"], abs=1e-7)
    assert g2["xmin"] == pytest.approx(STORM["xmin"]) and g2["ly"] == pytest.approx(STORM["ly"])
    with pytest.raises(api.CravaError) as e:
        api.grid_read_storm(ctx, str(path), back.data_ptr(), (nx, ny, nz + 1), (nxp, nyp, nzp))
    assert e.value.status == api.EINVAL
    bad = tmp_path / "bad.storm"
    bad.write_bytes(b"crava_fftgrid_binary\n" + raw[:200])
    with pytest.raises(api.CravaError) as e:
        api.grid_read_storm(ctx, str(bad), back.data_ptr(), (nx, ny, nz), (nxp, nyp, nzp))
    assert e.value.status == api.EINVAL
    ctx.close()


def _segy_case(case, rng):
    """A small padded grid and a SegY description: 7 x 5 traces of 12 cells (padded 8 x 6 x 16),
    rotated simbox; inline along y ('il_y') or along x ('il_x', records transposed by the
    inline/crossline sort); per-trace tops with one missing trace and relative thickness, or a
    constant top; the regular axis starting above the tops and ending inside or below them."""
    import math
    nx, ny, nz, rnxp, nyp, nzp = 7, 5, 12, 10, 6, 16
    grid = rng.standard_normal((nzp, nyp, rnxp)).astype(np.float32)
    ang, dx, dy = 0.3, 25.0, 12.5
    c, s = math.cos(ang), math.sin(ang)
    if case["axes"] == "il_y":
        steps = dict(il_step_x=-s / dy, il_step_y=c / dy, xl_step_x=c / dx, xl_step_y=s / dx)
    else:
        steps = dict(il_step_x=c / dx, il_step_y=s / dx, xl_step_x=-s / dy, xl_step_y=c / dy)
    geom = dict(x0=456000.3, y0=6780000.7, dx=dx, dy=dy, angle=ang, nx=nx, ny=ny, nz=nz, dz=case["dz"], top_z=1001.5,
                zmin=1000.0, zmax=case["zmax"], z0=case["z0"], header_format=case["fmt"], il0=99.5, xl0=9.5,
                **steps)
    top = rel = None
    if case["tops"]:
        top = 1000.0 + 3.0 * rng.random((ny, nx))
        top[1, 2] = -99999.0
        rel = 0.9 + 0.2 * rng.random((ny, nx))
    text = ["CRAVA B200 SEGY TEST", "line three [bracketed] ^caret", "x" * 90] if case["text"] else None
    return grid, geom, top, rel, text


SEGY_CASES = [
    dict(axes="il_y", fmt=0, dz=4.0, zmax=1100.0, z0=990.0, tops=True, text=False),
    dict(axes="il_x", fmt=2, dz=4.0, zmax=1100.0, z0=990.0, tops=True, text=True),
    dict(axes="il_x", fmt=1, dz=3.6, zmax=1030.0, z0=1002.0, tops=False, text=False),   # ends inside the grid
    dict(axes="il_y", fmt=5, dz=0.3, zmax=1010.0, z0=995.5, tops=True, text=False),     # dz rounds to 0 -> 1
    dict(axes="il_y", fmt=3, dz=4.0, zmax=1100.0, z0=1040.0, tops=False, text=True),    # starts below the data
    dict(axes="il_x", fmt=4, dz=4.0, zmax=1100.0, z0=990.0, tops=True, text=False),
]


@pytest.mark.parametrize("case", SEGY_CASES, ids=lambda c: f"{c['axes']}-fmt{c['fmt']}-dz{c['dz']}-z0{c['z0']}")
def test_segy_file_equals_the_reference_writer(tmp_path, case):
    """crava_grid_write_segy byte for byte against FFTGrid::writeSegyFile restated over NRLib's
    own SegY header, geometry and IBM-float code (oracle/_ref/libsegyref.so): textual, binary
    and trace headers, inline/crossline order, missing traces, the regular-z interpolation with
    its edge rules, every trace-header format."""
    import os
    import torch
    from oracle import bindings as ob
    if not os.path.exists(ob.SEGYREF_LIB):
        pytest.skip("oracle/_ref/libsegyref.so not built")
    rng = np.random.default_rng(len(str(case)))
    grid, geom, top, rel, text = _segy_case(case, rng)
    d, keep = api.segy_desc(geom, top=top, rel_thick=rel, text=text)
    ref = tmp_path / "ref.sgy"
    ob.segy_ref_write(str(ref), grid, d)
    ctx = api.Context(0)
    dg = torch.from_numpy(grid).cuda()
    got = tmp_path / "got.sgy"
    api.grid_write_segy(ctx, str(got), dg.data_ptr(), grid.shape[2], grid.shape[1], grid.shape[0], d)
    rb, gb = ref.read_bytes(), got.read_bytes()
    ctx.close()
    assert len(gb) == len(rb)
    if gb != rb:
        first = next(i for i in range(len(rb)) if rb[i] != gb[i])
        raise AssertionError(f"first differing byte {first} of {len(rb)}")
