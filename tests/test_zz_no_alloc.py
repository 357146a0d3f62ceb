"""crava_invert_noalloc: the inversion entry point that allocates no device memory.

It exists for callers that cannot allocate device memory (a plugin inside an application
that owns the device memory pool and admits no other allocator).  Its
intermediates live in a fixed array inside the library; this test calls it through the
C ABI twice in a row on the same block and checks each call against the ordinary job
entry point (crava_job_create / crava_job_run), and the posterior mean and covariance
against the FP64 oracle, with the tolerances of the parity tests:
posterior mean 1e-4, covariance 1e-3, realisations 1e-4 (norm-wise relative).  The file
sorts last so that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from crava_b200 import api, synth

pytestmark = pytest.mark.gpu

TOL = {"mean": 1e-4, "cov": 1e-3, "sims": 1e-4}


def rel(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / max(np.linalg.norm(b.astype(np.float64)), 1e-300))


def _noalloc_fn():
    L = api.lib()
    f = L.crava_invert_noalloc
    f.argtypes = [ctypes.POINTER(api.JobDesc), ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                  ctypes.c_void_p]
    return f


def test_noalloc_matches_job_entry_point_twice():
    import torch
    blk = synth.make_block(synth.config0())
    seed = 4242
    ctx = api.Context(0)
    # the ordinary entry point
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=seed)
    _keep = job.upload_block()
    job.run()
    ref = job.download_outputs()
    job.close()

    shape = job.shape
    d_in = [torch.from_numpy(np.ascontiguousarray(blk.data[l])).cuda() for l in range(blk.ntheta)] + \
           [torch.from_numpy(np.ascontiguousarray(blk.mean[a])).cuda() for a in range(3)]
    nout = 9 + 3 * blk.nsim
    d_out = [torch.zeros(shape, dtype=torch.float32, device="cuda") for _ in range(nout)]
    desc, _k = api.make_desc(blk, api.PRIOR_SEPARABLE, 0, seed=seed)
    ins = (ctypes.c_void_p * len(d_in))(*[t.data_ptr() for t in d_in])
    outs = (ctypes.c_void_p * nout)(*[t.data_ptr() for t in d_out])
    f = _noalloc_fn()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        for t in d_out:
            t.fill_(float("nan"))
        st = f(ctypes.byref(desc), ins, outs, stream)
        assert st == api.OK, api.lib().crava_last_error()
        torch.cuda.synchronize()
        got = [t.cpu().numpy() for t in d_out]
        nx = blk.nxp
        for a in range(3):
            assert rel(got[a][..., :nx], ref["mean"][a][..., :nx]) < TOL["mean"], (call, "mean", a)
        for q in range(6):
            assert rel(got[3 + q][..., :nx], ref["cov"][q][..., :nx]) < TOL["cov"], (call, "cov", q)
        for s in range(blk.nsim):
            for a in range(3):
                assert rel(got[9 + 3 * s + a][..., :nx], ref["sims"][s, a][..., :nx]) < TOL["sims"], (call, "sim", s, a)
    # inputs are read only
    for l in range(blk.ntheta):
        assert np.array_equal(d_in[l].cpu().numpy(), blk.data[l])
    # and the posterior itself against the FP64 oracle (realisations use device noise, so
    # they are checked against the job entry point above only)
    from oracle import ref64
    post = ref64.posterior(blk)
    for a in range(3):
        assert rel(got[a][..., :nx], post.mean[a][..., :nx]) < TOL["mean"], ("oracle mean", a)
    for q in range(6):
        assert rel(got[3 + q][..., :nx], post.cov[q][..., :nx]) < TOL["cov"], ("oracle cov", q)
    ctx.close()


def test_noalloc_rejects_blocks_beyond_its_scratch():
    import torch
    blk = synth.make_block(synth.BlockSpec(nx=16, ny=16, nz=16, nsim=1))
    desc, _k = api.make_desc(blk, api.PRIOR_SEPARABLE, 0, seed=1)
    # a 512x512x256 block with 6 angle stacks needs ~1.6 GB of data intermediates
    desc.nx = desc.nxp = 512
    desc.ny = desc.nyp = 512
    desc.nz = desc.nzp = 256
    desc.lz = 256 * 4.0
    wav = np.zeros((blk.ntheta, 256), dtype=np.float32)
    wav[:, 0] = 1.0
    desc.wavelet = wav.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    cxy = np.ones(512 * 512, dtype=np.float32)
    cct = np.ones(256, dtype=np.float32)
    desc.corr_xy = cxy.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    desc.circ_corr_t = cct.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    dummy = torch.zeros(4, device="cuda")
    ins = (ctypes.c_void_p * (blk.ntheta + 3))(*([dummy.data_ptr()] * (blk.ntheta + 3)))
    outs = (ctypes.c_void_p * 12)(*([dummy.data_ptr()] * 12))
    st = _noalloc_fn()(ctypes.byref(desc), ins, outs, None)
    assert st == api.ENOTSUP
    assert b"scratch" in api.lib().crava_last_error()
