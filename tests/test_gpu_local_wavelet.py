"""Local wavelets (shift and gain grids) and the wavelet-convolved residuals on the GPU through
the C ABI, against the oracle.

crava_job_set_wavelet_grids feeds divideDataByScaleWavelet's local wavelets
(createLocalWavelet1D + shiftAndScale, src/wavelet1D.cpp:518-602, inside
computeAdjustmentFactor, src/avoinversion.cpp:630-719); crava_job_set_wavelet_3d makes them 3D
wavelets adjusted for the local dip (Wavelet3D, src/wavelet3D.cpp:328-459);
crava_job_residual_synthetics is multiplyDataByScaleWaveletAndWriteToFile
(src/avoinversion.cpp:721-790).

Tolerances (norm-wise relative per grid): 2e-5, FP32 trace transforms against float64 ones
with the same float32 factor arithmetic on both sides (the divided-data tolerance of the
non-constant-thickness tests).
"""
import numpy as np
import pytest

from crava_b200 import api, synth
from oracle import ref64

pytestmark = pytest.mark.gpu

TOL = 2e-5


def rel(x, ref):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def thick_block(nx=40, ny=30, nz=50, nxp=48, nyp=40, nzp=64, seed=5, nsim=1):
    theta = (8.0, 20.0, 32.0)
    spec = synth.BlockSpec(nx=nx, ny=ny, nz=nz, nxp=nxp, nyp=nyp, nzp=nzp, nsim=nsim, seed=seed, theta_deg=theta,
                           peak_hz=(30.0,) * 3, sn=(6.0,) * 3)
    return synth.with_rel_thick(synth.make_block(spec), seed=seed, threshold=0.0)


def const_block(nx=40, ny=30, nz=50, nxp=48, nyp=40, nzp=64, seed=7):
    theta = (8.0, 20.0, 32.0)
    spec = synth.BlockSpec(nx=nx, ny=ny, nz=nz, nxp=nxp, nyp=nyp, nzp=nzp, nsim=0, seed=seed, theta_deg=theta,
                           peak_hz=(30.0,) * 3, sn=(6.0,) * 3)
    return synth.make_block(spec)


def wavelet_grids(blk, seed, missing=True):
    """Per angle a shift grid (ms, within +-2 samples) and a gain grid (0.5..2), with some
    WELLMISSING (-999) entries."""
    rng = np.random.default_rng(seed)
    dz = blk.lz / blk.nz
    shifts, gains = [], []
    for _ in range(blk.ntheta):
        s = rng.uniform(-2.0, 2.0, (blk.ny, blk.nx)) * dz
        g = rng.uniform(0.5, 2.0, (blk.ny, blk.nx))
        if missing:
            s[rng.random(s.shape) < 0.1] = -999.0
            g[rng.random(g.shape) < 0.1] = -999.0
        shifts.append(s.astype(np.float32))
        gains.append(g.astype(np.float32))
    return shifts, gains


def gpu_divided(ctx, blk, shifts=None, gains=None, w3=None):
    job = api.Job(ctx, blk)
    try:
        _keep = job.upload_block()
        if shifts is not None:
            for l in range(blk.ntheta):
                job.set_wavelet_grids(l, shifts[l], gains[l])
        if w3 is not None:
            job.set_wavelet_3d(**w3)
        job.divide_data()
        return np.stack([job.download(api.ROLE_DATA, l) for l in range(blk.ntheta)])
    finally:
        job.close()


@pytest.mark.parametrize("dims", [(40, 30, 50, 48, 40, 64), (33, 21, 90, 35, 27, 100), (30, 20, 40, 36, 24, 45)])
def test_divide_with_wavelet_grids_matches_oracle(ctx, dims):
    blk = thick_block(*dims)
    shifts, gains = wavelet_grids(blk, seed=sum(dims))
    got = gpu_divided(ctx, blk, shifts, gains)
    div = ref64.divide_data_by_scale_wavelet(blk, shifts, gains)
    ref = np.stack([ref64.interpolate_seismic(div[l], blk, blk.energy_threshold) for l in range(blk.ntheta)])
    nxp = blk.nxp
    for l in range(blk.ntheta):
        assert rel(got[l][..., :nxp], ref[l][..., :nxp]) < TOL, l
    # the grids change the division
    plain = gpu_divided(ctx, blk)
    assert rel(got[0][..., :nxp], plain[0][..., :nxp]) > 1e-3


def test_neutral_grids_equal_the_global_wavelet(ctx):
    """Zero shift and unit gain everywhere: the per-trace factor is the tabulated one."""
    blk = thick_block(seed=11)
    z = [np.zeros((blk.ny, blk.nx), np.float32)] * blk.ntheta
    o = [np.ones((blk.ny, blk.nx), np.float32)] * blk.ntheta
    got = gpu_divided(ctx, blk, z, o)
    plain = gpu_divided(ctx, blk)
    assert rel(got, plain) < 1e-7


def gpu_residual_synthetics(ctx, blk, shifts=None, gains=None, w3=None):
    job = api.Job(ctx, blk, flags=api.FLAG_KEEP_RESIDUAL, nsim=0)
    try:
        _keep = job.upload_block()
        if blk_is_nonconst(blk):
            job.divide_data()
        if shifts is not None:
            for l in range(blk.ntheta):
                job.set_wavelet_grids(l, shifts[l], gains[l])
        if w3 is not None:
            job.set_wavelet_3d(**w3)
        job.run()
        spec = np.stack([job.download(api.ROLE_RESIDUAL, l).view(np.complex64) for l in range(blk.ntheta)])
        job.residual_synthetics()
        got = np.stack([job.download(api.ROLE_RESIDUAL, l) for l in range(blk.ntheta)])
        with pytest.raises(api.CravaError) as ei:
            job.residual_synthetics()
        assert ei.value.status == api.ESTATE
        return spec, got
    finally:
        job.close()


def blk_is_nonconst(blk):
    return getattr(blk, "rel_thick", None) is not None


@pytest.mark.parametrize("kind", ["const", "const_grids", "nonconst_grids", "const_3d", "nonconst_grids_3d"])
def test_residual_synthetics_match_oracle(ctx, kind):
    blk = thick_block(seed=13) if kind.startswith("nonconst") else const_block()
    shifts = gains = w3 = None
    if "grids" in kind:
        shifts, gains = wavelet_grids(blk, seed=17)
    if kind.endswith("3d"):
        w3 = synth.wavelet3d_model(blk, blk.spec.theta_deg, seed=19)
    spec, got = gpu_residual_synthetics(ctx, blk, shifts, gains, w3)
    resid = np.stack([ref64.inv_fft_in_place(spec[l].astype(np.complex128), blk.nxp, False)
                      for l in range(blk.ntheta)])
    ref = ref64.residual_synthetics(blk, resid, shifts, gains, w3=w3)
    nxp = blk.nxp
    for l in range(blk.ntheta):
        assert rel(got[l][..., :nxp], ref[l][..., :nxp]) < TOL, l
        # the interior traces were convolved, the padding traces only transformed back
        assert rel(got[l][:, :blk.ny, :blk.nx], resid[l][:, :blk.ny, :blk.nx]) > 1e-2
        assert rel(got[l][:, blk.ny:, :nxp], resid[l][:, blk.ny:, :nxp]) < TOL


def test_residual_synthetics_state(ctx):
    blk = const_block(seed=3)
    job = api.Job(ctx, blk, nsim=0)
    try:
        with pytest.raises(api.CravaError) as ei:
            job.residual_synthetics()
        assert ei.value.status == api.ESTATE          # no KEEP_RESIDUAL
    finally:
        job.close()
    job = api.Job(ctx, blk, flags=api.FLAG_KEEP_RESIDUAL, nsim=0)
    try:
        with pytest.raises(api.CravaError) as ei:
            job.residual_synthetics()
        assert ei.value.status == api.ESTATE          # before the run
        with pytest.raises(api.CravaError) as ei:
            job.set_wavelet_grids(blk.ntheta, None, None)
        assert ei.value.status == api.EINVAL
        bad = np.zeros((blk.ny, blk.nx), np.float32)
        bad[0, 0] = np.nan
        with pytest.raises(api.CravaError) as ei:
            job.set_wavelet_grids(0, bad, None)
        assert ei.value.status == api.EINVAL
    finally:
        job.close()


# ---------------------------------------------------------------- 3D wavelets

@pytest.mark.parametrize("dims,halpha,grids", [((40, 30, 50, 48, 40, 64), True, False),
                                               ((33, 21, 90, 35, 27, 100), True, True),
                                               ((30, 20, 40, 36, 24, 45), False, False)])
def test_divide_with_3d_wavelets_matches_oracle(ctx, dims, halpha, grids):
    """Dip-adjusted local wavelets (gradients of either sign, filter surfaces with missing
    nodes, with and without Halpha, with and without shift/gain grids) against the oracle."""
    blk = thick_block(*dims)
    w3 = synth.wavelet3d_model(blk, blk.spec.theta_deg, seed=sum(dims), halpha=halpha)
    shifts = gains = None
    if grids:
        shifts, gains = wavelet_grids(blk, seed=sum(dims) + 1)
    got = gpu_divided(ctx, blk, shifts, gains, w3=w3)
    div = ref64.divide_data_by_scale_wavelet(blk, shifts, gains, w3=w3)
    ref = np.stack([ref64.interpolate_seismic(div[l], blk, blk.energy_threshold) for l in range(blk.ntheta)])
    nxp = blk.nxp
    for l in range(blk.ntheta):
        assert rel(got[l][..., :nxp], ref[l][..., :nxp]) < TOL, l
    plain = gpu_divided(ctx, blk, shifts, gains)
    assert rel(got[0][..., :nxp], plain[0][..., :nxp]) > 1e-3


def test_neutral_3d_model_equals_the_1d_wavelets(ctx):
    """Flat gradients, theta 0, alpha1 1, no Halpha and the block's own wavelets as the global
    ones: the dip factor, the stretch and gamma are exactly 1 and the norm is the wavelet's."""
    blk = thick_block(seed=23)
    w3 = synth.wavelet3d_model(blk, blk.spec.theta_deg, flat=True)
    got = gpu_divided(ctx, blk, w3=w3)
    plain = gpu_divided(ctx, blk)
    assert rel(got, plain) < 1e-7


def test_wavelet_3d_arguments(ctx):
    blk = thick_block(seed=29)
    job = api.Job(ctx, blk)
    try:
        w3 = synth.wavelet3d_model(blk, blk.spec.theta_deg, seed=2)
        for key, val in [("filter_geom", (0.0, 0.0, 0.0, 10.0)), ("filter_geom", (0.0, np.nan, 30.0, 10.0))]:
            with pytest.raises(api.CravaError) as ei:
                job.set_wavelet_3d(**dict(w3, **{key: val}))
            assert ei.value.status == api.EINVAL
        bad = np.array(w3["grad_x"])
        bad[1, 2] = np.inf
        with pytest.raises(api.CravaError) as ei:
            job.set_wavelet_3d(**dict(w3, grad_x=bad))
        assert ei.value.status == api.EINVAL
        with pytest.raises(api.CravaError) as ei:
            job.set_wavelet_3d(**dict(w3, global_wavelet_norm=np.zeros(blk.ntheta, np.float32)))
        assert ei.value.status == api.EINVAL
        job.set_wavelet_3d(**w3)
    finally:
        job.close()
