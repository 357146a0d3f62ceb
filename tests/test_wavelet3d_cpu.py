"""3D wavelets on the CPU: the oracle's restatement of the filter-surface lookup against
NRLib's own RegularSurface<float>::GetZ (libs/nrlib/surface/regularsurface.hpp, a header-only
template compiled from the reference tree), findPhi's quadrants, and the neutral 3D model
(flat gradients, theta 0, alpha1 1, no Halpha, the block's own wavelets as the global ones)
giving the 1D division and residual convolution exactly."""
import math
import os
import struct
import subprocess

import numpy as np
import pytest

from crava_b200 import synth
from oracle import ref64

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("CRAVA_REFERENCE") or os.path.join(os.sep, "root", "reference")


def test_surface_lookup_matches_nrlib(tmp_path):
    hdr = os.path.join(REF, "libs", "nrlib", "surface", "regularsurface.hpp")
    if not os.path.exists(hdr):
        pytest.skip("reference tree not present")
    exe = str(tmp_path / "surface_check")
    subprocess.run(["g++", "-O2", "-std=c++11", os.path.join(ROOT, "tests", "native", "surface_check.cpp"),
                    "-I" + os.path.join(REF, "libs", "nrlib"), "-I" + os.path.join(REF, "libs"), "-o", exe],
                   check=True)
    rng = np.random.default_rng(8)
    ni, nj = 13, 10
    geom = (0.0, 0.0, 30.0, 10.0)
    z = rng.uniform(0.5, 1.5, (nj, ni)).astype(np.float32)
    z[0, 3] = z[4, 7] = z[9, 12] = -999.0
    pts = [(rng.uniform(-40.0, 400.0), rng.uniform(-15.0, 100.0)) for _ in range(3000)]
    # nodes, cell edges, the last row and column, and points beside missing nodes
    pts += [(30.0 * i, 10.0 * j) for i in range(ni) for j in range(nj)]
    pts += [(90.0 + 7.5, 0.0), (360.0, 45.0), (359.9, 89.9), (210.0 + 1e-9, 40.0), (-30.0, -10.0), (-1e-12, 5.0)]
    path = tmp_path / "surf.bin"
    with open(path, "wb") as f:
        f.write(struct.pack("<ii4d", ni, nj, *geom))
        f.write(z.astype("<f4").tobytes())
        f.write(struct.pack("<i", len(pts)))
        f.write(np.asarray(pts, "<f8").tobytes())
    out = subprocess.run([exe, str(path)], capture_output=True, text=True, check=True)
    ref = np.array([float(v) for v in out.stdout.split()], dtype=np.float32)
    got = np.array([ref64.surface_z(z, geom, x, y) for x, y in pts], dtype=np.float32)
    assert len(ref) == len(pts)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert (ref == -999.0).any() and (ref != -999.0).sum() > 2000


def test_find_phi_quadrants():
    for a, b, lo, hi in [(1.0, 0.5, 0, math.pi / 2), (-1.0, 0.5, math.pi / 2, math.pi),
                         (-1.0, -0.5, math.pi, 1.5 * math.pi), (1.0, -0.5, 1.5 * math.pi, 2 * math.pi)]:
        assert lo <= ref64.find_phi(a, b) < hi
    assert ref64.find_phi(0.0005, 1.0) == 0.5 * math.pi
    assert ref64.find_phi(-0.0005, -1.0) == 1.5 * math.pi
    assert ref64.find_psi(np.float32(1.0)) == 0.0
    assert abs(ref64.find_psi(np.float32(2.0)) - math.pi / 3) < 1e-7


def small_block(seed=5):
    theta = (8.0, 20.0, 32.0)
    spec = synth.BlockSpec(nx=12, ny=10, nz=50, nxp=16, nyp=12, nzp=64, nsim=1, seed=seed, theta_deg=theta,
                           peak_hz=(30.0,) * 3, sn=(6.0,) * 3)
    return synth.with_rel_thick(synth.make_block(spec), seed=seed, threshold=0.0)


def test_neutral_3d_model_is_the_1d_path():
    blk = small_block()
    w3 = synth.wavelet3d_model(blk, blk.spec.theta_deg, flat=True)
    P = ref64.wavelet3d_params(blk, w3)
    tab = ref64.thick_tables(blk)
    for l in range(blk.ntheta):
        assert np.all(P[l]["mult"] == 1.0) and np.all(P[l]["stretch"] == 1.0) and np.all(P[l]["gam"] == 1.0)
        assert np.all(P[l]["wn2"] == tab["wn2"][l])
    a = ref64.divide_data_by_scale_wavelet(blk)
    b = ref64.divide_data_by_scale_wavelet(blk, w3=w3)
    assert np.array_equal(a, b)
    rng = np.random.default_rng(2)
    resid = rng.standard_normal((blk.ntheta, blk.nzp, blk.nyp, 2 * (blk.nxp // 2 + 1)))
    assert np.array_equal(ref64.residual_synthetics(blk, resid), ref64.residual_synthetics(blk, resid, w3=w3))


def test_3d_model_changes_the_division():
    blk = small_block(seed=6)
    w3 = synth.wavelet3d_model(blk, blk.spec.theta_deg, seed=4)
    a = ref64.divide_data_by_scale_wavelet(blk)
    b = ref64.divide_data_by_scale_wavelet(blk, w3=w3)
    assert np.isfinite(b).all()
    assert np.linalg.norm(a - b) / np.linalg.norm(a) > 1e-2
