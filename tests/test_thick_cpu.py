"""The oracle's restatement of the non-constant-thickness pre-processing, on the CPU.

Pins: FFTGrid::getFillNumber / getDistToBoundary against the sequences the reference
documents beside them (src/fftgrid.cpp:1105-1108, 1160-1163); the interpolation plan of
interpolateSeismic against hand-traced cases; the adjustment factor's limit (unit
stretch, no stabilisation: 1/conj(W)); the division against the reference's FFTW trace
loop (oracle/_ref); the ABI's validation of the new fields.
"""
import ctypes
import dataclasses

import numpy as np
import pytest

from crava_b200 import api, synth
from oracle import ref64


def test_fill_number_matches_the_documented_sequences():
    # "GetFillNumber(i, 5 , 8) returns 0,1,2,3,4,4,1,0", "(i, 4, 8) 0,1,2,3,3,2,1,0",
    # "(i, 3, 8) 0,1,2,2,1,1,1,0"
    assert [ref64.fill_number(i, 5, 8) for i in range(8)] == [0, 1, 2, 3, 4, 4, 1, 0]
    assert [ref64.fill_number(i, 4, 8) for i in range(8)] == [0, 1, 2, 3, 3, 2, 1, 0]
    assert [ref64.fill_number(i, 3, 8) for i in range(8)] == [0, 1, 2, 2, 1, 1, 1, 0]


def test_dist_to_boundary_matches_the_documented_pattern():
    # "(i, 5, 8) returns 0,0,0,0,0,p,r,p  p between 0 and 1, r larger than 1", and the
    # same shape for (4, 8) and (3, 8)
    for n, pattern in [(5, "00000prp"), (4, "0000prrp"), (3, "000prrrp")]:
        d = [ref64.dist_to_boundary(i, n, 8) for i in range(8)]
        for v, c in zip(d, pattern):
            if c == "0":
                assert v == 0.0
            elif c == "p":
                assert 0.0 < v < 1.0
            else:
                assert v > 1.0


def _plan(mask, threshold=0.0):
    e = np.asarray(mask, dtype=np.float32)
    return ref64.plan_trace_interpolation(e, e.shape[1], e.shape[0], threshold)


def test_plan_isolated_dead_trace():
    ops, box = _plan([[1, 1, 1], [1, 0, 1], [1, 1, 1]])
    assert ops == [(4, [3, 5, 1, 7])]
    assert box == (0, 2, 0, 2)


def test_plan_first_dead_trace_without_two_good_neighbours_is_left():
    # (0,0) has one good neighbour at its turn; the backtrack after (1,0) stops at flags <= 1
    ops, box = _plan([[0, 0, 1], [1, 1, 1], [1, 1, 1]])
    assert ops == [(1, [2, 4])]
    assert box == (0, 2, 0, 2)


def test_plan_backtracks_to_an_earlier_trace():
    # (1,0) is dead with one good neighbour (1,1) at its turn; after (2,1) -- dead, with
    # (3,1), (2,0)... -- is filled, the backtrack revisits it
    m = [[1, 0, 1, 1],
         [1, 0, 0, 1],
         [1, 1, 1, 1]]
    ops, _ = _plan(m)
    targets = [t for t, _ in ops]
    assert sorted(targets) == [1, 5, 6]
    for t, nb in ops:
        assert len(nb) >= 2


def test_plan_threshold_uses_the_mean_energy():
    e = np.ones((4, 4), dtype=np.float32)
    e[1, 2] = 0.01
    ops, _ = ref64.plan_trace_interpolation(e, 4, 4, 0.05)
    assert [t for t, _ in ops] == [1 * 4 + 2]
    ops, _ = ref64.plan_trace_interpolation(e, 4, 4, 0.0)
    assert ops == []


@pytest.fixture(scope="module")
def blk():
    b = synth.make_block(synth.BlockSpec(nx=24, ny=20, nz=50, nxp=30, nyp=24, nzp=64, nsim=0))
    return dataclasses.replace(b, rel_thick=np.full((b.nyp, b.nxp), 1.0))


def test_unit_stretch_factor_is_the_inverse_wavelet(blk):
    tab = ref64.thick_tables(blk)
    tab["wnc"] = blk.wnc
    cn = blk.nzp // 2 + 1
    k = np.arange(cn)
    for l in range(blk.ntheta):
        f = ref64.adjustment_factor(tab, l, np.float32(1.0), k)
        W = tab["wamp"][l].astype(np.complex128)
        strong = np.abs(W) ** 2 > 0.2 * tab["modW"][l]
        assert strong.sum() > 5
        assert np.abs(f[strong] * np.conj(W[strong]) - 1).max() < 1e-6


def test_error_smooth_table_is_band_normalised_with_the_rmissing_tail(blk):
    tab = ref64.thick_tables(blk)
    n = blk.nzp
    cn = n // 2 + 1
    es = tab["es3"][0]
    assert es.real[cn - 1] == -99999.0 and es.imag[cn - 1] == -99999.0   # even nzp
    dz = np.float32(blk.lz / blk.nz)
    dO = np.float32(1.0 / float(np.float32(n * dz) * 0.001))
    lo = max(0, int(np.floor(np.float32(blk.low_cut) / dO)))
    hi = min(cn, int(np.ceil(np.float32(blk.high_cut) / dO)))
    s = sum(2.0 / n * abs(complex(es[i])) ** 2 for i in range(lo, hi))
    if lo == 0:
        s -= abs(complex(es[0])) ** 2 / n
    assert abs(s - 1.0) < 1e-5


def test_nonconst_branch_operators(blk):
    K, e1, e2, e3, _inv = ref64.per_kz_operators(blk)
    d1 = np.zeros(blk.nzp)
    d1[0], d1[-1] = -1.0, 1.0
    kD = np.fft.fft(d1)
    assert np.allclose(K[:, 0, :], kD[:, None] * blk.A[0][None, :])
    assert np.allclose(e1[:, 1], 1.0 / float(blk.wavelet_norm[1]))
    assert np.all(e3 > 0)


def test_abi_validates_the_thickness_fields(blk):
    d, keep = api.make_desc(blk)
    assert d.flags & api.FLAG_NONCONST_THICK
    out = ctypes.c_size_t()
    assert api.lib().crava_job_footprint(ctypes.byref(d), ctypes.byref(out)) == api.OK
    with_thick = out.value
    d2, keep2 = api.make_desc(dataclasses.replace(blk, rel_thick=None))
    assert api.lib().crava_job_footprint(ctypes.byref(d2), ctypes.byref(out)) == api.OK
    assert with_thick > out.value
    bad = keep["relt"].copy()
    bad[3, 4] = 0.0
    d.rel_thick = bad.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert api.lib().crava_job_footprint(ctypes.byref(d), ctypes.byref(out)) == api.EINVAL
    d.rel_thick = None
    assert api.lib().crava_job_footprint(ctypes.byref(d), ctypes.byref(out)) == api.EINVAL
    d.rel_thick = keep["relt"].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    d.energy_threshold = -1.0
    assert api.lib().crava_job_footprint(ctypes.byref(d), ctypes.byref(out)) == api.EINVAL


def test_division_restatement_matches_the_reference_fftw():
    """divideDataByScaleWavelet in float64 (ref64) against the same trace loop over the
    reference's own FFTW 2.1.2 float transforms (oracle/_ref): the two agree to FP32
    rounding, so the float64 restatement carries the reference's transform conventions
    (scalings, half spectrum, band cut)."""
    from oracle import bindings as ob
    if not ob.ref32_available():
        pytest.skip("oracle/_ref not built")
    b = synth.make_block(synth.BlockSpec(nx=20, ny=16, nz=50, nxp=24, nyp=18, nzp=64, nsim=0, seed=9))
    b = synth.with_rel_thick(b, seed=4)
    ref = ob.ref32_divide(b)
    mine = ref64.divide_data_by_scale_wavelet(b)
    for l in range(b.ntheta):
        x, r = mine[l][..., :b.nxp], ref[l][..., :b.nxp].astype(np.float64)
        assert np.linalg.norm(x - r) / np.linalg.norm(r) < 2e-6
        assert np.linalg.norm(r - b.data[l][..., :b.nxp]) > 1e-2 * np.linalg.norm(r)


def test_division_restatement_matches_the_golden_fixture():
    """The committed fixture tests/golden/t1_nonconst.npz holds the division computed over
    the reference's FFTW 2.1.2 float plans (make_golden.py); the float64 restatement agrees."""
    from tests.golden import golden_io
    b, z = golden_io.load("t1_nonconst")
    mine = ref64.divide_data_by_scale_wavelet(b)
    ref = z["ref_divided"]
    for l in range(b.ntheta):
        x, r = mine[l][..., :b.nxp], ref[l][..., :b.nxp].astype(np.float64)
        assert np.linalg.norm(x - r) / np.linalg.norm(r) < 2e-6, l


def test_local_factor_with_neutral_grids_is_the_global_factor(blk):
    """Zero shift and unit gain: the local-wavelet restatement of computeAdjustmentFactor
    gives the global one bit for bit."""
    tab = ref64.thick_tables(blk)
    tab["wnc"] = blk.wnc
    cn = blk.nzp // 2 + 1
    k = np.arange(cn)[:, None]
    sf = np.array([[0.8, 1.0, 1.3]], dtype=np.float32)
    for l in range(blk.ntheta):
        g = ref64.adjustment_factor(tab, l, sf, k)
        loc = ref64.adjustment_factor_local(tab, l, sf, k, np.float32(0.0), np.float32(1.0), blk.nzp)
        assert np.array_equal(g, loc)


def test_wavelet_index_maps_padding_onto_the_interior():
    n, np_ = 10, 16
    idx = [ref64.wavelet_index(i, n, np_) for i in range(np_)]
    assert idx[:n] == list(range(n))
    assert all(0 <= i < n for i in idx)
    assert idx[n] == n - 1 and idx[np_ - 1] == 1


def test_residual_convolution_with_an_integer_shift_and_gain(blk):
    """shiftAndScale by a whole number of samples s and a gain g: the convolved residual is
    the unshifted one advanced by s samples and scaled by g (constant thickness, sf = 1)."""
    b = dataclasses.replace(blk, rel_thick=None)
    rng = np.random.default_rng(2)
    resid = rng.standard_normal((b.ntheta, b.nzp, b.nyp, 2 * (b.nxp // 2 + 1)))
    dz = b.lz / b.nz
    s, g = 3, 1.5
    shifts = [np.full((b.ny, b.nx), s * dz, np.float32)] * b.ntheta
    gains = [np.full((b.ny, b.nx), g, np.float32)] * b.ntheta
    base = ref64.residual_synthetics(b, resid)
    got = ref64.residual_synthetics(b, resid, shifts, gains)
    want = g * np.roll(base[:, :, :b.ny, :b.nx], -s, axis=1)
    err = np.linalg.norm(got[:, :, :b.ny, :b.nx] - want) / np.linalg.norm(want)
    assert err < 1e-5
    # the traces outside the interior are untouched
    assert np.array_equal(got[:, :, b.ny:], resid[:, :, b.ny:])


def test_storm_padding_restatement_blends_the_edges():
    """The StormContGrid padding: z padding blends slices 0 and nz-1 with weights that step
    from the last slice's value towards the first slice's across the padding."""
    rng = np.random.default_rng(1)
    vals = rng.standard_normal((5, 4, 3)).astype(np.float32)
    g = ref64.storm_padding(vals, 6, 7, 9)
    assert np.array_equal(g[:5, :4, :3], vals)
    assert np.all(g[..., 6:] == 0)
    sc = np.float32(1.0) / np.float32(9 - 5 + 1)
    k = 5
    want = (g[0, 2, 1] * np.float32(sc * np.float32(k - 5 + 1))).astype(np.float32) + \
        (g[4, 2, 1] * np.float32(sc * np.float32(9 - k))).astype(np.float32)
    assert g[k, 2, 1] == want
    # x padding of an interior row is the blend of its first and last values
    sa = np.float32(1.0) / np.float32(6 - 3 + 1)
    assert g[1, 1, 3] == (g[1, 1, 0] * np.float32(sa * 1)).astype(np.float32) + \
        (g[1, 1, 2] * np.float32(sa * 3)).astype(np.float32)
