"""The C ABI without a GPU: the library loads, exports every entry point the header
declares, sizes jobs and rejects invalid descriptions; the Python binding fails loudly when
the library is missing."""
import ctypes
import os
import re

import numpy as np
import pytest

from crava_b200 import api, synth

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "crava_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(crava_[a-z0-9_]+)\s*\(", src)))


def test_library_built():
    assert os.path.exists(api.LIB_PATH), "run python -m crava_b200.build"


def test_every_declared_entry_point_is_exported():
    L = ctypes.CDLL(api.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings():
    L = api.lib()
    for s in range(8):
        assert L.crava_status_string(s)


def _desc(blk, **over):
    d, keep = api.make_desc(blk)
    for k, v in over.items():
        setattr(d, k, v)
    return d, keep


@pytest.fixture(scope="module")
def small():
    return synth.make_block(synth.BlockSpec(nx=16, ny=12, nz=20, nsim=2))


def test_footprint_counts_grids_and_tables(small):
    blk = small
    nb = api.footprint(blk)
    cnxp = blk.nxp // 2 + 1
    grid = -(-(8 * cnxp * blk.nyp * blk.nzp) // 256) * 256
    ngrids = 2 * (blk.ntheta + 3) + 6 + 3 * blk.nsim
    assert nb >= ngrids * grid
    assert nb < ngrids * grid + 64 * 1024
    nb_grids = api.footprint(blk, prior_mode=api.PRIOR_GRIDS)
    # eight more grids (six covariance, the error correlation and its spectrum) and the
    # small fill buffers of crava_job_fill_prior, less the separable lateral factor
    assert 8 * grid - 64 * 1024 < nb_grids - nb < 8 * grid + 64 * 1024
    nb_noise = api.footprint(blk, flags=api.FLAG_HOST_NOISE)
    assert nb_noise - nb == 3 * blk.nsim * grid


@pytest.mark.parametrize("field,value,status", [
    ("nxp", 11 * 13, api.ENOTSUP),     # not 2,3,5,7-smooth
    ("ntheta", 9, api.ENOTSUP),
    ("nsim", 17, api.ENOTSUP),
    ("nxp", 8, api.EINVAL),            # padded below simbox size
    ("lz", 0.0, api.EINVAL),
    ("prior_mode", 7, api.EINVAL),
])
def test_invalid_descriptions_rejected(small, field, value, status):
    d, _k = _desc(small, **{field: value})
    out = ctypes.c_size_t()
    st = api.lib().crava_job_footprint(ctypes.byref(d), ctypes.byref(out))
    assert st == status
    assert api.lib().crava_last_error()


def test_null_description_rejected():
    out = ctypes.c_size_t()
    assert api.lib().crava_job_footprint(None, ctypes.byref(out)) == api.EINVAL


def test_context_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(api.CravaError):
        api.Context(0)


def test_missing_library_raises(monkeypatch):
    monkeypatch.setattr(api, "_lib", None)
    monkeypatch.setattr(api, "LIB_PATH", "/nonexistent/libcrava_gpu.so")
    with pytest.raises(api.CravaError):
        api.lib()


def test_host_layer_built_and_exports_the_reference_entry_points():
    """The C++ host layer keeps the reference's class and method names."""
    import subprocess
    lib = os.path.join(os.path.dirname(api.LIB_PATH), "libcrava_host.so")
    assert os.path.exists(lib), "run python -m crava_b200.build"
    syms = subprocess.run(["nm", "-DC", lib], capture_output=True, text=True, check=True).stdout
    for name in ("crava_b200::FFTGrid::fftInPlace()", "crava_b200::FFTGrid::invFFTInPlace()",
                 "crava_b200::AVOInversion::computePostMeanResidAndFFTCov()",
                 "crava_b200::AVOInversion::simulate(", "crava_b200::FFTGrid::getNextComplex()",
                 "crava_b200::FFTGrid::setRealValue("):
        assert name in syms, name


@pytest.mark.parametrize("array", ["A", "err_theta_cov", "prior_var0", "wavelet", "corr_xy", "circ_corr_t"])
def test_non_finite_description_rejected_as_numeric(small, array):
    """A NaN in any of the description's host arrays is reported as CRAVA_ENUMERIC before
    anything reaches a device (a job whose prior or wavelets are not finite would spread NaN
    through every bin of the block)."""
    blk = small
    src = {"A": blk.A, "err_theta_cov": blk.err_theta_cov, "prior_var0": blk.prior_var0,
           "wavelet": blk.wavelet, "corr_xy": blk.corr_xy, "circ_corr_t": blk.circ_corr_t}[array]
    bad = np.array(src, copy=True)
    bad.flat[bad.size // 2] = np.nan
    d, keep = api.make_desc(blk)
    ptype = ctypes.POINTER(ctypes.c_double if bad.dtype == np.float64 else ctypes.c_float)
    bad = np.ascontiguousarray(bad)
    setattr(d, array, bad.ctypes.data_as(ptype))
    out = ctypes.c_size_t()
    assert api.lib().crava_job_footprint(ctypes.byref(d), ctypes.byref(out)) == api.ENUMERIC
    assert b"non-finite" in api.lib().crava_last_error()


def test_schedule_table_set_get_load(tmp_path):
    """The schedule table: per-size entries, the any-size entry (n = -1), removal, and a file
    of "key n value" lines with comments replacing the table."""
    key = "test_only_key"
    assert api.tuning_get(key, 7) == -1
    api.tuning_set(key, -1, 3)
    assert api.tuning_get(key, 7) == 3
    api.tuning_set(key, 7, 5)
    assert api.tuning_get(key, 7) == 5 and api.tuning_get(key, 8) == 3
    api.tuning_set(key, 7, -1)
    api.tuning_set(key, -1, -1)
    assert api.tuning_get(key, 7) == -1
    f = tmp_path / "sched.txt"
    f.write_text("# comment line\n" + key + " 256 4   # trailing comment\n" + key + " -1 2\n")
    before = api.tuning_path()
    api.tuning_load(str(f))
    try:
        assert api.tuning_path() == str(f)
        assert api.tuning_get(key, 256) == 4 and api.tuning_get(key, 320) == 2
    finally:
        if before:
            api.tuning_load(before)
    with pytest.raises(api.CravaError):
        api.tuning_load(str(tmp_path / "missing.txt"))
