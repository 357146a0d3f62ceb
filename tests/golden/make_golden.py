"""Generate the golden fixtures of tests/golden/ from the reference's own FP32 numerics.

    python tests/golden/make_golden.py [name ...]   (needs oracle/_ref/libref32.so, built by
                                                     `make -C oracle` from the reference tree)

Each fixture holds one small block's inputs (the synth.Block arrays), the reference-path
outputs computed by oracle/_ref (FFTW 2.1.2 float + lib_matr.c with the restated loops):
posterior mean, posterior covariance, residual spectra, realisations drawn with the
reference RandomGen, the inverted-bin and Cholesky-fallback counts, and the noise grids
themselves.  The cases cover even, odd and padded sizes, 1..6 angle stacks, and a prior
with correlation gradients (covariance grids that are not separable).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from crava_b200 import synth  # noqa: E402
from oracle import bindings as ob  # noqa: E402
from oracle import ref64  # noqa: E402

CASES = {
    "g1_even": dict(nx=16, ny=12, nz=20, theta_deg=(8.0, 24.0), peak_hz=(28.0, 32.0), sn=(4.0, 6.0), nsim=1, seed=5),
    "g2_odd": dict(nx=15, ny=9, nz=21, theta_deg=(10.0, 20.0, 30.0), peak_hz=(30.0,) * 3, sn=(5.0,) * 3, nsim=2,
                   seed=6),
    "g3_padded": dict(nx=13, ny=11, nz=19, nxp=14, nyp=12, nzp=20, theta_deg=(5.0, 15.0, 25.0, 35.0, 45.0, 55.0),
                      peak_hz=(30.0,) * 6, sn=(3.0,) * 6, nsim=1, seed=7),
    "g4_gradients": dict(nx=12, ny=10, nz=16, theta_deg=(10.0, 30.0), peak_hz=(30.0, 30.0), sn=(5.0, 5.0), nsim=1,
                         seed=9, corr_grad_i=0.3, corr_grad_j=-0.2),
    "g5_one_angle_wideband": dict(nx=10, ny=8, nz=24, theta_deg=(20.0,), peak_hz=(40.0,), sn=(8.0,), nsim=1, seed=10,
                                  low_cut=1.0, high_cut=200.0),
    # the production block's z length, angle stacks and realisations (540x540x256 workload:
    # 5 angles 5..45 deg, Ricker 25..35 Hz, nzp 256, 4 realisations) on a 6x4 lateral window,
    # so the pencil pass runs the same instantiation as on the full block
    "g6_production_pencil": dict(nx=6, ny=4, nz=256, theta_deg=(5.0, 15.0, 25.0, 35.0, 45.0),
                                 peak_hz=(25.0, 27.5, 30.0, 32.5, 35.0), sn=(5.0,) * 5, lateral_range=2000.0,
                                 angular=("spherical", 20.0), nsim=4, seed=21),
}

SCALARS = ["nx", "ny", "nz", "nxp", "nyp", "nzp", "lz", "low_int_cut", "low_cut", "high_cut", "wnc",
           "min_rel_thick", "corr_grad_i", "corr_grad_j", "nsim", "seed"]
ARRAYS = ["A", "err_theta_cov", "wavelet", "wavelet_norm", "prior_var0", "corr_xy", "prior_corr_t",
          "circ_corr_t", "mean", "data"]


def make(name, kw, noise_seed=1234):
    blk = synth.make_block(synth.BlockSpec(**kw))
    covs, _ = ref64.prior_cov_grids(blk)
    if blk.corr_grad_i or blk.corr_grad_j:
        ec = ref64.fill_err_corr(blk.corr_xy, blk.nxp, blk.nyp, blk.nzp, blk.corr_grad_i, blk.corr_grad_j)
    else:
        ec = ref64.fill_err_corr_zero_grad(blk.corr_xy, blk.nxp, blk.nyp, blk.nzp)
    noise = ob.sim_noise(noise_seed, blk.nsim, blk.nxp, blk.nyp, blk.nzp, use_ref=True)
    r = ob.ref32_invert(blk, covs, ec, nsim=blk.nsim, seed=noise_seed)
    out = {k: np.asarray(getattr(blk, k)) for k in SCALARS}
    out.update({k: getattr(blk, k) for k in ARRAYS})
    out.update({"cov_grids": np.stack(covs), "err_corr": ec, "noise": noise, "noise_seed": np.int64(noise_seed),
                "ref_mean": r.mean, "ref_cov": r.cov, "ref_resid_spec": r.resid_spec, "ref_sims": r.sims,
                "ref_n_inverted": np.int64(r.n_inverted), "ref_n_chol_fail": np.int64(r.n_chol_fail)})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return out


# Non-constant thickness: divideDataByScaleWavelet's trace loop over the reference's FFTW
# 2.1.2 float plans (oracle/_ref ref32_divide_traces), padded block, rel_thick surface.
THICK_CASES = {
    "t1_nonconst": (dict(nx=14, ny=10, nz=24, nxp=16, nyp=12, nzp=32, theta_deg=(8.0, 20.0, 32.0),
                         peak_hz=(30.0,) * 3, sn=(5.0,) * 3, nsim=0, seed=12), 11),
}


def make_thick(name, kw, surface_seed):
    blk = synth.with_rel_thick(synth.make_block(synth.BlockSpec(**kw)), seed=surface_seed)
    out = {k: np.asarray(getattr(blk, k)) for k in SCALARS}
    out.update({k: getattr(blk, k) for k in ARRAYS})
    out.update({"rel_thick": blk.rel_thick, "energy_threshold": np.float32(blk.energy_threshold),
                "ref_divided": ob.ref32_divide(blk)})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return out


# Facies probabilities with local-noise corners: calculateFaciesProb + findDensity in the
# reference's float arithmetic (oracle/_ref ref32_facies_prob) on seeded posterior values,
# 2^2 corner density volumes with their own boxes, and relative noise scales.
FACIES_CASES = {"f1_facies_corners": dict(nx=9, ny=7, nz=11, nang=2, nf=3, nbins=(12, 10, 8), seed=13)}


def make_facies(name, kw):
    rng = np.random.default_rng(kw["seed"])
    nx, ny, nz, nang, nf, nbins = kw["nx"], kw["ny"], kw["nz"], kw["nang"], kw["nf"], kw["nbins"]
    centre = np.array([np.log(3000.0), np.log(1500.0), np.log(2300.0)])
    post = [(centre[a] + 0.15 * rng.standard_normal((nz, ny, nx))).astype(np.float32) for a in range(3)]
    dens, boxes = [], []
    for c in range(1 << nang):
        widen = 0.1 * (1 + c)
        vmin = [float(p.min()) - widen for p in post]
        dv = [(float(p.max()) + widen - vmin[d]) / nbins[d] for d, p in enumerate(post)]
        d = rng.random((nf, nbins[2], nbins[1], nbins[0])).astype(np.float32)
        d[:, :2] -= 0.3        # some negative entries: findDensity clamps them to zero
        dens.append(d)
        boxes.append(np.array(vmin + dv + list(nbins), dtype=np.float64))
    prior = np.array([0.2, 0.5, 0.3], dtype=np.float32)[:nf]
    scales = (1.0 + 2.0 * rng.random((nang, ny, nx))).astype(np.float32)
    # calculateFaciesProb's relative scales (src/faciesprob.cpp:1961-1977): double, stored as float
    t = np.stack([((scales[a].astype(np.float64) - scales[a].min()) / (float(scales[a].max()) - scales[a].min()))
                  for a in range(nang)]).astype(np.float32)
    corners = [(dens[c], nbins, list(boxes[c][:3]), list(boxes[c][3:6])) for c in range(1 << nang)]
    out = ob.ref32_facies_prob(post, corners, prior, 0.05, t)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), post=np.stack(post), dens=np.stack(dens),
                        boxes=np.stack(boxes), prior=prior, p_undefined=np.float32(0.05), scales=scales, t=t,
                        ref_prob=out)


if __name__ == "__main__":
    if not ob.ref32_available():
        sys.exit("oracle/_ref/libref32.so missing: run `make -C oracle` with the reference tree present")
    only = set(sys.argv[1:])   # optional fixture names; all of them by default
    for name, kw in CASES.items():
        if not only or name in only:
            make(name, kw)
            print("wrote", name)
    for name, (kw, sseed) in THICK_CASES.items():
        if not only or name in only:
            make_thick(name, kw, sseed)
            print("wrote", name)
    for name, kw in FACIES_CASES.items():
        if not only or name in only:
            make_facies(name, kw)
            print("wrote", name)
