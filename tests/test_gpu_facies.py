"""Facies probabilities on the GPU against the oracle restatement (norm-wise relative
tolerance 5e-5 for the smoothed densities, an FP32 3D transform of up to 500k bins, and
1e-5 for the probabilities)."""
import numpy as np
import pytest

from crava_b200 import api, synth
from oracle import ref64

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("nbins", [(100, 100, 50), (20, 16, 10), (15, 12, 9)])
def test_smoothing_matches_oracle(ctx, nbins):
    import torch
    rng = np.random.default_rng(sum(nbins))
    nf = 3
    na, nb, nr = nbins
    rna = 2 * (na // 2 + 1)
    hist = np.zeros((nf, nr, nb, na))
    for f in range(nf):
        idx = rng.integers(0, [nr, nb, na], size=(200, 3))
        for l, k, j in idx:
            hist[f, l, k, j] += 1.0 / 200
    dv = (0.02, 0.03, 0.01)
    sig = np.array([[0.003, 0.001, 0.0005], [0.001, 0.004, 0.0002], [0.0005, 0.0002, 0.001]])
    S = np.linalg.inv(sig)
    g = np.zeros((nf, nr, nb, rna), dtype=np.float32)
    g[..., :na] = hist
    d = torch.from_numpy(g).cuda()
    fd, _k = api.facies_desc([0.4, 0.4, 0.2], nbins, (7.9, 7.0, 7.7), dv, 0.05)
    api.facies_smooth(ctx, fd, S, d.data_ptr())
    torch.cuda.synchronize()
    got = d.cpu().numpy()[..., :na]
    ref = ref64.facies_smooth(hist, nbins, dv, S)
    assert rel(got, ref) < 5e-5


def test_facies_prob_on_posterior_mean(ctx):
    import torch
    blk = synth.make_block(synth.config0())
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=3)
    _k = job.upload_block()
    job.run()
    mean = [job.download(api.ROLE_POST_MEAN, a) for a in range(3)]
    nbins = (100, 100, 50)
    m = [x[..., :blk.nx] for x in mean]
    vmin = [float(x.min()) - 0.05 for x in m]
    dv = [(float(x.max()) + 0.05 - vmin[i]) / nbins[i] for i, x in enumerate(m)]
    rng = np.random.default_rng(5)
    nf = 4
    dens = rng.random((nf, nbins[2], nbins[1], nbins[0])).astype(np.float32)
    prior = [0.1, 0.2, 0.3, 0.4]
    fd, _k2 = api.facies_desc(prior, nbins, vmin, dv, 0.02)
    d_dens = torch.from_numpy(dens).cuda()
    d_mean = [torch.from_numpy(x).cuda() for x in mean]
    rnx = 2 * (blk.nx // 2 + 1)
    outs = [torch.zeros((blk.nz, blk.ny, rnx), dtype=torch.float32, device="cuda") for _ in range(nf + 1)]
    lh = torch.zeros((blk.nz, blk.ny, rnx), dtype=torch.float32, device="cuda")
    api.facies_prob(ctx, fd, d_dens.data_ptr(), nbins[0], [t.data_ptr() for t in d_mean], blk.nx, blk.ny, blk.nz,
                    blk.nxp, blk.nyp, [t.data_ptr() for t in outs], lh.data_ptr())
    torch.cuda.synchronize()
    got = np.stack([t.cpu().numpy()[..., :blk.nx] for t in outs])
    ref = ref64.facies_prob(mean, dens, nbins, vmin, dv, prior, 0.02, blk.nx, blk.ny, blk.nz)
    assert rel(got, ref) < 1e-5
    assert np.allclose(got.sum(axis=0), 1.0, atol=1e-5)
    pad = outs[0].cpu().numpy()[..., blk.nx:]
    assert pad.size == 0 or np.all(pad == -99999.0)
    job.close()


@pytest.mark.parametrize("nang", [0, 2, 3])
def test_facies_prob_with_local_noise_corners(ctx, nang):
    """findDensity with local noise: 2^nang corner volumes (each its own box), weighted per
    trace by the relative noise scales, against the oracle (1e-5); nang = 0 equals the
    single-volume entry point."""
    import torch
    blk = synth.make_block(synth.config0())
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=3)
    _k = job.upload_block()
    job.run()
    mean = [job.download(api.ROLE_POST_MEAN, a) for a in range(3)]
    job.close()
    m = [x[..., :blk.nx] for x in mean]
    rng = np.random.default_rng(11 + nang)
    nf, nbins = 3, (24, 20, 12)
    prior = [0.3, 0.3, 0.4]
    corners, descs, keep, d_dens = [], [], [], []
    for c in range(1 << nang):
        widen = 0.05 * (1 + c)          # the corner boxes differ
        vmin = [float(x.min()) - widen for x in m]
        dv = [(float(x.max()) + widen - vmin[i]) / nbins[i] for i, x in enumerate(m)]
        dens = rng.random((nf, nbins[2], nbins[1], nbins[0])).astype(np.float32)
        corners.append((dens, nbins, vmin, dv))
        fd, k = api.facies_desc(prior, nbins, vmin, dv, 0.02)
        descs.append(fd)
        keep.append(k)
        d_dens.append(torch.from_numpy(dens).cuda())
    scales = (1.0 + 2.0 * rng.random((nang, blk.ny, blk.nx))).astype(np.float32)
    rnx = 2 * (blk.nx // 2 + 1)
    outs = [torch.zeros((blk.nz, blk.ny, rnx), dtype=torch.float32, device="cuda") for _ in range(nf + 1)]
    d_mean = [torch.from_numpy(x).cuda() for x in mean]
    api.facies_prob_local_noise(ctx, descs, [t.data_ptr() for t in d_dens], nbins[0], scales,
                                [t.data_ptr() for t in d_mean], blk.nx, blk.ny, blk.nz, blk.nxp, blk.nyp,
                                [t.data_ptr() for t in outs])
    torch.cuda.synchronize()
    got = np.stack([t.cpu().numpy()[..., :blk.nx] for t in outs])
    dens_ref = ref64.facies_density_corners(mean, corners, scales, blk.nx, blk.ny, blk.nz)
    undef = 0.02 / float(np.prod(nbins))
    val = np.asarray(prior)[:, None, None, None] * dens_ref
    tot = undef + val.sum(axis=0)
    ref = np.concatenate([val / tot, (undef / tot)[None]])
    assert rel(got, ref) < 1e-5
    if nang == 0:
        ref1 = ref64.facies_prob(mean, corners[0][0], nbins, corners[0][2], corners[0][3], prior, 0.02,
                                 blk.nx, blk.ny, blk.nz)
        assert rel(got, ref1) < 1e-5


def test_facies_corners_against_reference_arithmetic_fixture(ctx):
    """crava_facies_prob_local_noise against the reference's float arithmetic
    (tests/golden/f1_facies_corners.npz from oracle/_ref): 2 local-noise angles, 4 corner
    volumes with their own boxes, negative density entries clamped; 1e-6."""
    import os
    import torch
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "f1_facies_corners.npz"))
    nz, ny, nx = z["post"][0].shape
    rnx = 2 * (nx // 2 + 1)
    d_post = []
    for a in range(3):
        g = np.zeros((nz, ny, rnx), dtype=np.float32)
        g[..., :nx] = z["post"][a]
        d_post.append(torch.from_numpy(g).cuda())
    descs, keep, d_dens = [], [], []
    prior = [float(p) for p in z["prior"]]
    for c in range(z["dens"].shape[0]):
        b = z["boxes"][c]
        nb = tuple(int(v) for v in b[6:9])
        fd, k = api.facies_desc(prior, nb, list(b[:3]), list(b[3:6]), float(z["p_undefined"]))
        descs.append(fd)
        keep.append(k)
        d_dens.append(torch.from_numpy(np.ascontiguousarray(z["dens"][c])).cuda())
    nf = len(prior)
    outs = [torch.zeros((nz, ny, rnx), dtype=torch.float32, device="cuda") for _ in range(nf + 1)]
    api.facies_prob_local_noise(ctx, descs, [t.data_ptr() for t in d_dens], int(z["boxes"][0][6]), z["scales"],
                                [t.data_ptr() for t in d_post], nx, ny, nz, nx, ny, [t.data_ptr() for t in outs])
    torch.cuda.synchronize()
    got = np.stack([t.cpu().numpy()[..., :nx] for t in outs])
    assert rel(got, z["ref_prob"].astype(np.float64)) < 1e-6


@pytest.mark.parametrize("dims,nang", [((64, 64, 128), 0), ((64, 64, 128), 2), ((540, 12, 32), 1), ((28, 20, 24), 2)])
def test_job_facies_in_the_mean_transform(ctx, dims, nang):
    """crava_job_set_facies: the probabilities written by crava_job_run equal
    crava_facies_prob_local_noise on the job's posterior mean bit for bit, and the posterior
    mean itself is unchanged, with the evaluation inside the inverse x transform of the mean
    (schedule entry facies_fused = 1, where nxp/2 has a four-step split: 32 and 270 here) and
    as a separate pass (the default; the only form for nxp 28)."""
    import torch
    spec = synth.config0()
    spec.nx, spec.ny, spec.nz = dims
    blk = synth.make_block(spec)
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=3)
    _k = job.upload_block()
    job.run()
    torch.cuda.synchronize()
    mean = [job.download(api.ROLE_POST_MEAN, a) for a in range(3)]
    m = [x[..., :blk.nx] for x in mean]
    rng = np.random.default_rng(7 + nang)
    nf, nbins = 3, (24, 20, 12)
    prior = [0.25, 0.35, 0.4]
    descs, keep, d_dens = [], [], []
    for c in range(1 << nang):
        widen = 0.04 * (1 + c)
        vmin = [float(x.min()) - widen for x in m]
        dv = [(float(x.max()) + widen - vmin[i]) / nbins[i] for i, x in enumerate(m)]
        fd, k = api.facies_desc(prior, nbins, vmin, dv, 0.02)
        descs.append(fd)
        keep.append(k)
        d_dens.append(torch.from_numpy(rng.random((nf, nbins[2], nbins[1], nbins[0])).astype(np.float32)).cuda())
    scales = (1.0 + rng.random((nang, blk.ny, blk.nx))).astype(np.float32) if nang else None
    rnx = 2 * (blk.nx // 2 + 1)

    def grids():
        return [torch.full((blk.nz, blk.ny, rnx), 7.0, dtype=torch.float32, device="cuda") for _ in range(nf + 2)]

    ref = grids()
    d_mean = [torch.from_numpy(x).cuda() for x in mean]
    api.facies_prob_local_noise(ctx, descs, [t.data_ptr() for t in d_dens], nbins[0],
                                scales if nang else np.zeros((0,)), [t.data_ptr() for t in d_mean], blk.nx, blk.ny,
                                blk.nz, blk.nxp, blk.nyp, [t.data_ptr() for t in ref[:-1]], ref[-1].data_ptr())
    got = grids()
    job.set_facies(descs, [t.data_ptr() for t in d_dens], nbins[0], scales, [t.data_ptr() for t in got[:-1]],
                   got[-1].data_ptr())
    del d_dens   # the job holds packed copies
    for fused in (1, 0):
        api.tuning_set("facies_fused", blk.nxp // 2, fused)
        for rep in range(2):
            for t in got:
                t.fill_(7.0)
            job.run()
            torch.cuda.synchronize()
            for a in range(3):
                assert np.array_equal(job.download(api.ROLE_POST_MEAN, a), mean[a])
            for g, r in zip(got, ref):
                assert torch.equal(g, r)
    api.tuning_set("facies_fused", blk.nxp // 2, -1)
    assert np.all(got[0].cpu().numpy()[..., blk.nx:] == -99999.0)
    job.set_facies(None, None, 0, None, None)
    for t in got:
        t.fill_(7.0)
    job.run()
    torch.cuda.synchronize()
    assert bool((got[0] == 7.0).all())
    job.close()
