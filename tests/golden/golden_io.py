"""Loader of the golden fixtures written by make_golden.py."""
import glob
import os

import numpy as np

from crava_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))


def names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(HERE, "g*.npz")))


def load(name):
    """Returns (Block, dict of the fixture's arrays)."""
    z = dict(np.load(os.path.join(HERE, name + ".npz")))
    sc = lambda k: z[k].item()
    blk = synth.Block(spec=None, nx=int(sc("nx")), ny=int(sc("ny")), nz=int(sc("nz")), nxp=int(sc("nxp")),
                      nyp=int(sc("nyp")), nzp=int(sc("nzp")), lz=float(sc("lz")), A=z["A"],
                      err_theta_cov=z["err_theta_cov"], wavelet=z["wavelet"], wavelet_norm=z["wavelet_norm"],
                      prior_var0=z["prior_var0"], corr_xy=z["corr_xy"], prior_corr_t=z["prior_corr_t"],
                      circ_corr_t=z["circ_corr_t"], low_int_cut=int(sc("low_int_cut")), mean=z["mean"],
                      data=z["data"], low_cut=float(sc("low_cut")), high_cut=float(sc("high_cut")),
                      wnc=float(sc("wnc")), min_rel_thick=float(sc("min_rel_thick")),
                      corr_grad_i=float(sc("corr_grad_i")), corr_grad_j=float(sc("corr_grad_j")),
                      nsim=int(sc("nsim")), seed=int(sc("seed")))
    if "rel_thick" in z:
        blk.rel_thick = z["rel_thick"]
        blk.energy_threshold = float(z["energy_threshold"])
    return blk, z
