"""Facies oracle: the vectorised restatement against a literal per-voxel restatement of
findDensity / calculateFaciesProb (src/faciesprob.cpp:1307-1423, 1909-2075)."""
import numpy as np

from oracle import ref64


def find_density_loop(vp, vs, rho, D, nb, vmin, dv):
    def axis(v, d):
        full = (v - vmin[d]) / dv[d] - 0.5
        i1 = int(np.floor(full))
        if i1 < 0:
            return 0, 0, 0.0
        if i1 >= nb[d] - 1:
            return nb[d] - 1, nb[d] - 1, 0.0
        return i1, i1 + 1, full - i1
    j1, j2, wj = axis(vp, 0)
    k1, k2, wk = axis(vs, 1)
    l1, l2, wl = axis(rho, 2)
    g = lambda j, k, l: max(0.0, D[l, k, j])
    v = 0.0
    v += (1 - wj) * (1 - wk) * (1 - wl) * g(j1, k1, l1)
    v += (1 - wj) * (1 - wk) * wl * g(j1, k1, l2)
    v += (1 - wj) * wk * (1 - wl) * g(j1, k2, l1)
    v += (1 - wj) * wk * wl * g(j1, k2, l2)
    v += wj * (1 - wk) * (1 - wl) * g(j2, k1, l1)
    v += wj * (1 - wk) * wl * g(j2, k1, l2)
    v += wj * wk * (1 - wl) * g(j2, k2, l1)
    v += wj * wk * wl * g(j2, k2, l2)
    return v if v > 0 else 0.0


def test_facies_prob_matches_literal_loop():
    rng = np.random.default_rng(3)
    nb = (10, 8, 6)
    vmin = (7.9, 7.1, 7.6)
    dv = (0.04, 0.07, 0.03)
    nf = 3
    dens = rng.random((nf, nb[2], nb[1], nb[0]))
    dens[0, 0, 0, 0] = -1.0
    prior = [0.5, 0.3, 0.2]
    nz, ny, nx = 4, 3, 5
    post = [rng.uniform(vmin[d] - 0.1, vmin[d] + nb[d] * dv[d] + 0.1, (nz, ny, nx + 2)) for d in range(3)]
    got = ref64.facies_prob(post, dens, nb, vmin, dv, prior, 0.1, nx, ny, nz)
    undef = 0.1 / np.prod(nb)
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                vals = [prior[f] * find_density_loop(post[0][k, j, i], post[1][k, j, i], post[2][k, j, i], dens[f], nb,
                                                     vmin, dv) for f in range(nf)]
                s = undef + sum(vals)
                assert np.allclose(got[:nf, k, j, i], np.array(vals) / s)
                assert np.isclose(got[nf, k, j, i], undef / s)


def test_facies_smoother_is_normalised_and_symmetric():
    S = np.linalg.inv(np.array([[0.01, 0.002, 0.0], [0.002, 0.02, 0.001], [0.0, 0.001, 0.005]]))
    sm = ref64.facies_smoother((10, 8, 6), (0.05, 0.05, 0.05), S)
    assert np.isclose(sm.sum(), 1.0)
    assert sm[0, 0, 0] == sm.max()
    h = np.zeros((1, 6, 8, 10))
    h[0, 2, 3, 4] = 1.0
    out = ref64.facies_smooth(h, (10, 8, 6), (0.05, 0.05, 0.05), S)
    assert np.isclose(out.sum(), 1.0)


def test_corner_density_oracle_matches_reference_arithmetic_fixture():
    """The float64 restatement of findDensity with local-noise corners against the
    reference's float arithmetic (tests/golden/f1_facies_corners.npz, written by
    tests/golden/make_golden.py from oracle/_ref): 1e-6."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "f1_facies_corners.npz"))
    post = list(z["post"])
    nz, ny, nx = post[0].shape
    corners = [(z["dens"][c], tuple(int(v) for v in z["boxes"][c][6:9]), list(z["boxes"][c][:3]),
                list(z["boxes"][c][3:6])) for c in range(z["dens"].shape[0])]
    dens = ref64.facies_density_corners(post, corners, None, nx, ny, nz, t=z["t"])
    nb = corners[0][1]
    undef = float(z["p_undefined"]) / float(nb[0] * nb[1] * nb[2])
    val = z["prior"].astype(np.float64)[:, None, None, None] * dens
    tot = undef + val.sum(axis=0)
    ref = np.concatenate([val / tot, (undef / tot)[None]])
    got = z["ref_prob"].astype(np.float64)
    assert np.linalg.norm(ref - got) / np.linalg.norm(got) < 1e-6
