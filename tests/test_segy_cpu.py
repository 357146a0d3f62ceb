"""SegY pieces on the CPU: the IEEE -> IBM float conversion of the library (ibm_float.h)
against the reference's own bit arithmetic (NRLib fileio.hpp, compiled from the reference
tree), and the SegY oracle (oracle/_ref/libsegyref.so: FFTGrid::writeSegyFile over NRLib's
header and geometry code) against an independent numpy reading of its file: EBCDIC card
images, binary header, sorted inline/crossline records, trace samples within the IBM
truncation (2^-20 relative) of a float64 interpolation."""
import codecs
import math
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("CRAVA_REFERENCE") or os.path.join(os.sep, "root", "reference")


def test_ibm_conversion_matches_reference_bit_arithmetic(tmp_path):
    hdr = os.path.join(REF, "libs", "nrlib", "iotools", "fileio.hpp")
    if not os.path.exists(hdr):
        pytest.skip("reference tree not present")
    exe = str(tmp_path / "ibm_check")
    subprocess.run(["g++", "-O2", "-std=c++11", os.path.join(ROOT, "tests", "native", "ibm_check.cpp"),
                    "-I" + os.path.join(REF, "libs", "nrlib"), "-I" + os.path.join(REF, "libs"),
                    "-I" + os.path.join(ROOT, "crava_b200", "csrc"), "-o", exe], check=True)
    out = subprocess.run([exe, "97"], capture_output=True, text=True)
    n, bad = (int(v) for v in out.stdout.split())
    assert n > 44_000_000 and bad == 0


def ibm_to_float(words):
    w = words.astype(np.uint64)
    sign = np.where(w >> 31, -1.0, 1.0)
    ex = ((w >> 24) & 0x7F).astype(np.int64) - 64
    fr = (w & 0xFFFFFF).astype(np.float64) / 2.0 ** 24
    return sign * fr * 16.0 ** ex


def test_segy_oracle_file_reads_back():
    from crava_b200 import api
    from oracle import bindings as ob
    if not os.path.exists(ob.SEGYREF_LIB):
        pytest.skip("oracle/_ref/libsegyref.so not built")
    nx, ny, nz, rnxp, nyp, nzp = 7, 5, 12, 10, 6, 16
    rng = np.random.default_rng(4)
    grid = rng.standard_normal((nzp, nyp, rnxp)).astype(np.float32)
    ang, dx, dy = 0.3, 25.0, 12.5
    c, s = math.cos(ang), math.sin(ang)
    geom = dict(x0=456000.3, y0=6780000.7, dx=dx, dy=dy, angle=ang, nx=nx, ny=ny, nz=nz, dz=4.0, top_z=0.0,
                zmin=1000.0, zmax=1100.0, z0=990.0, header_format=0, il0=99.5, xl0=9.5, il_step_x=c / dx,
                il_step_y=s / dx, xl_step_x=-s / dy, xl_step_y=c / dy)
    top = 1000.0 + 3.0 * rng.random((ny, nx))
    top[1, 2] = -99999.0
    rel = 0.9 + 0.2 * rng.random((ny, nx))
    d, keep = api.segy_desc(geom, top=top, rel_thick=rel)
    path = os.path.join(ROOT, "oracle", "_build", "segy_check.sgy")
    os.makedirs(os.path.dirname(path), exist_ok=True)
    ob.segy_ref_write(path, grid, d)
    b = open(path, "rb").read()
    os.remove(path)
    text = codecs.decode(b[:3200], "cp037")
    assert text[:3] == "C 1" and text[39 * 80:39 * 80 + 14] == "C40 END EBCDIC"
    assert "THE CRAVA PROGRAM" in text[13 * 80:14 * 80]
    ns = int.from_bytes(b[3220:3222], "big")
    assert ns == 28 and int.from_bytes(b[3216:3218], "big") == 4000 and int.from_bytes(b[3224:3226], "big") == 1
    rec = 240 + 4 * ns
    nrec = (len(b) - 3600) // rec
    assert nrec == nx * ny - 1 and len(b) == 3600 + nrec * rec
    keys = []
    for r in range(nrec):
        h = b[3600 + r * rec:3600 + r * rec + 240]
        il = int.from_bytes(h[8:12], "big", signed=True)
        xl = int.from_bytes(h[20:24], "big", signed=True)
        keys.append((il, xl))
        i, j = il - 100, xl - 10          # inline along x, crossline along y here
        assert int.from_bytes(h[114:116], "big") == ns and int.from_bytes(h[108:110], "big") == 990
        rx, ry = (i + 0.5) * dx, (j + 0.5) * dy
        assert int.from_bytes(h[72:76], "big", signed=True) == int(np.float32(rx * c - ry * s + geom["x0"]))
        w = np.frombuffer(b[3600 + r * rec + 240:3600 + (r + 1) * rec], dtype=">u4")
        got = ibm_to_float(w)
        gdz = 4.0 * rel[j, i]
        z = top[j, i]
        first = math.floor(0.5 + (z - 990.0) / 4.0)
        end = min(math.floor(0.5 + ((z - 990.0) + nz * gdz) / 4.0), ns)
        want = np.zeros(ns)
        for k in range(max(first, 0), end):
            t = (990.0 + 4.0 * k - z) / gdz
            kg = int(t)
            t -= kg
            if kg < 0:
                kg, t = 0, 0.0
            elif kg > nz - 2:
                kg, t = nz - 2, 1.0
            want[k] = (1 - t) * grid[kg, j, i] + t * grid[kg + 1, j, i]
        assert np.allclose(got, want, rtol=2e-6, atol=2e-6)
    assert keys == sorted(keys)
