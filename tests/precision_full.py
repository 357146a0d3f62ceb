"""Precision at the full 768x768x320 block of the precision study (6 angles 5..50 deg, band
2..120 Hz, S/N 2..10): the GPU posterior mean and covariance, FP32 alone and with the FP64
re-factorisation of flagged bins (fp64_threshold 100), against the FP64 oracle end to end in
real space.  A script, not a pytest test: the oracle needs about 75 GB of host memory and ten
minutes of one core at this size.

    python tests/precision_full.py --out report.json            # full size
    python tests/precision_full.py --dims 96,96,320             # the reduced study's size

The oracle forms the separable prior and error-correlation spectra slab by slab
(ref64.posterior(separable=True)); the data are the synthetic seismic of the reduced study at
full lateral size.  Reported per output grid: norm-wise relative error and max|x-x_ref| /
max|x_ref|.
"""
import argparse
import dataclasses
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

from crava_b200 import api, synth  # noqa: E402
from oracle import ref64  # noqa: E402


def errors(x, ref):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return {"rel": float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300)),
            "max_rel": float(np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", default=None, help="nx,ny,nz instead of 768,768,320")
    ap.add_argument("--out", default=None, help="write the report as JSON here")
    args = ap.parse_args()
    spec = dataclasses.replace(synth.config3(), nsim=0)
    if args.dims:
        nx, ny, nz = (int(v) for v in args.dims.split(","))
        spec = dataclasses.replace(spec, nx=nx, ny=ny, nz=nz)
    t0 = time.time()
    blk = synth.make_block(spec)
    rep = {"dims": [blk.nx, blk.ny, blk.nz], "padded": [blk.nxp, blk.nyp, blk.nzp], "ntheta": blk.ntheta,
           "synth_s": time.time() - t0}
    ctx = api.Context(0)
    gpu = {}
    for t in (0.0, 100.0):
        t1 = time.time()
        o = api.invert_block(ctx, blk, api.PRIOR_SEPARABLE, fp64_threshold=t)
        gpu[t] = (o["mean"], o["cov"])
        rep[f"t={t:g}"] = {"counters": {k: v for k, v in o["counters"].items() if k != "post_var0"},
                           "gpu_s": time.time() - t1}
        del o
    ctx.close()
    t2 = time.time()
    post = ref64.posterior(blk, slab=8, separable=True)
    rep["oracle_s"] = time.time() - t2
    rep["oracle_inverted"] = post.n_inverted
    rep["oracle_chol_fallbacks"] = post.n_chol_fail
    nxp = blk.nxp
    names = ["Vp", "Vs", "Rho", "VpVs", "VpRho", "VsRho"]
    for t in (0.0, 100.0):
        mean, cov = gpu[t]
        r = rep[f"t={t:g}"]
        r["mean"] = {names[a]: errors(mean[a][..., :nxp], post.mean[a][..., :nxp]) for a in range(3)}
        r["cov"] = {names[q]: errors(cov[q][..., :nxp], post.cov[q][..., :nxp]) for q in range(6)}
        r["worst"] = {"mean": max(v["rel"] for v in r["mean"].values()),
                      "cov": max(v["rel"] for v in r["cov"].values())}
    line = json.dumps(rep)
    print(line)
    if args.out:
        Path(args.out).write_text(line + "\n")


if __name__ == "__main__":
    main()
