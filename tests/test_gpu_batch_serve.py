"""Batches and the serving loop: every block's result is the same alone, in a batch and in
a served mix (bitwise: the kernels are deterministic and the per-block work does not depend
on what else runs)."""
import numpy as np
import pytest

from crava_b200 import api, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


SPECS = [
    dict(nx=64, ny=48, nz=64, theta_deg=(10.0, 30.0), peak_hz=(30.0, 30.0), sn=(5.0, 5.0), nsim=2, seed=1),
    dict(nx=75, ny=90, nz=81, theta_deg=(5.0, 20.0, 35.0, 50.0), peak_hz=(28.0,) * 4, sn=(4.0,) * 4, nsim=1, seed=2),
    dict(nx=96, ny=80, nz=100, theta_deg=tuple(np.linspace(5, 45, 6)), peak_hz=(32.0,) * 6, sn=(6.0,) * 6, nsim=3,
         seed=3),
    dict(nx=45, ny=64, nz=128, theta_deg=(15.0, 25.0, 35.0), peak_hz=(30.0,) * 3, sn=(5.0,) * 3, nsim=1, seed=4),
]


@pytest.fixture(scope="module")
def blocks():
    return [synth.make_block(synth.BlockSpec(**s)) for s in SPECS]


@pytest.fixture(scope="module")
def alone(ctx, blocks):
    outs = []
    for i, b in enumerate(blocks):
        j = api.Job(ctx, b, api.PRIOR_SEPARABLE, 0, seed=100 + i)
        _k = j.upload_block()
        j.run()
        outs.append(j.download_outputs())
        j.close()
    return outs


def test_batch_matches_alone(ctx, blocks, alone):
    jobs = []
    for i, b in enumerate(blocks):
        j = api.Job(ctx, b, api.PRIOR_SEPARABLE, 0, seed=100 + i)
        j._k = j.upload_block()
        jobs.append(j)
    bt = api.Batch(ctx, jobs, branches=3)
    l0 = ctx.kernel_launches()
    for _ in range(2):
        bt.run()
    import torch
    torch.cuda.synchronize()
    assert ctx.kernel_launches() - l0 == 2 * 5 * len(jobs)
    for j, ref in zip(jobs, alone):
        got = j.download_outputs()
        for k in ("mean", "cov", "sims"):
            assert np.array_equal(got[k], ref[k]), k
    bt.close()
    for j in jobs:
        j.close()


def _host_buffers(b, nsim):
    import torch
    shape = (b.nzp, b.nyp, 2 * (b.nxp // 2 + 1))
    ins = [torch.from_numpy(np.ascontiguousarray(b.data[l])).pin_memory() for l in range(b.ntheta)] + \
          [torch.from_numpy(np.ascontiguousarray(b.mean[a])).pin_memory() for a in range(3)]
    outs = [torch.empty(shape, dtype=torch.float32).pin_memory() for _ in range(9 + 3 * nsim)]
    return ins, outs


def test_served_mix_matches_alone(ctx, blocks, alone):
    sv = api.Server(ctx, max_inflight=3)
    tickets, bufs = [], []
    for rep in range(2):
        for i, b in enumerate(blocks):
            ins, outs = _host_buffers(b, b.nsim)
            tickets.append((i, sv.submit(b, ins, outs, seed=100 + i)))
            bufs.append(outs)
    for (i, t), outs in zip(tickets, bufs):
        info = sv.wait(t, timeout_ms=120000)
        assert info["state"] == api.REQ_DONE
        assert info["latency_ms"] > 0
        ref = alone[i]
        got_mean = np.stack([o.numpy() for o in outs[:3]])
        got_cov = np.stack([o.numpy() for o in outs[3:9]])
        assert np.array_equal(got_mean, ref["mean"])
        assert np.array_equal(got_cov, ref["cov"])
        got_sims = np.stack([o.numpy() for o in outs[9:]]).reshape(ref["sims"].shape)
        assert np.array_equal(got_sims, ref["sims"])
    sv.stop()


def test_served_admission_by_budget(blocks):
    """A budget that holds one job at a time: requests queue and still all complete."""
    fp = max(api.footprint(b) for b in blocks)
    c = api.Context(0, hbm_budget=int(fp * 1.2))
    sv = api.Server(c, max_inflight=4)
    ts = []
    keep = []
    for i, b in enumerate(blocks):
        ins, outs = _host_buffers(b, b.nsim)
        keep.append((ins, outs))
        ts.append(sv.submit(b, ins, outs, seed=7))
    infos = [sv.wait(t, timeout_ms=120000) for t in ts]
    assert all(x["state"] == api.REQ_DONE for x in infos)
    # later requests waited in the queue for memory
    assert max(x["queue_ms"] for x in infos) > 0
    sv.stop()
    c.close()


def test_wait_times_out_and_stop_fails_queued(ctx, blocks):
    sv = api.Server(ctx, max_inflight=1)
    b = blocks[2]
    bufs = [_host_buffers(b, b.nsim) for _ in range(3)]
    ts = [sv.submit(b, ins, outs, seed=1) for ins, outs in bufs]
    with pytest.raises(api.CravaError) as e:
        sv.wait(ts[-1], timeout_ms=0.01)
    assert e.value.status == api.ETIMEDOUT
    sv.wait(ts[0], timeout_ms=120000)
    sv.stop()


def test_served_oversized_request_fails_and_the_next_one_runs(blocks):
    """A request larger than the context budget is refused at submit; one that cannot be
    allocated with nothing else in flight fails with ENOMEM instead of holding the queue, and
    the request behind it completes."""
    small = blocks[0]
    fp = api.footprint(small)
    c = api.Context(0, hbm_budget=int(fp * 1.5))
    sv = api.Server(c, max_inflight=2)
    big = synth.make_block_fast(synth.BlockSpec(nx=200, ny=200, nz=128, nsim=16, seed=3))
    bi, bo = _host_buffers(big, big.nsim)
    with pytest.raises(api.CravaError) as e:
        sv.submit(big, bi, bo, seed=1)
    assert e.value.status == api.ENOMEM
    si, so = _host_buffers(small, small.nsim)
    t = sv.submit(small, si, so, seed=2)
    assert sv.wait(t, timeout_ms=120000)["state"] == api.REQ_DONE
    sv.stop()
    c.close()


def test_served_non_finite_request_fails_with_numeric(ctx, blocks):
    b = blocks[1]
    sv = api.Server(ctx, max_inflight=2)
    ins, outs = _host_buffers(b, b.nsim)
    ins[0].numpy()[3, 2, 1] = np.nan
    t_bad = sv.submit(b, ins, outs, seed=1)
    ins2, outs2 = _host_buffers(b, b.nsim)
    t_ok = sv.submit(b, ins2, outs2, seed=1)
    with pytest.raises(api.CravaError) as e:
        sv.wait(t_bad, timeout_ms=120000)
    assert e.value.status == api.ENUMERIC
    assert sv.wait(t_ok, timeout_ms=120000)["state"] == api.REQ_DONE
    # the final state has been reported: the ticket is released
    with pytest.raises(api.CravaError):
        sv.poll(t_ok)
    sv.stop()


def test_table_cache_hits_and_results_unchanged(blocks, alone):
    """Jobs with the same model share resident tables: the second job of a model is a cache
    hit, and its results equal the uncached job's bit for bit."""
    c = api.Context(0)
    c.set_table_cache(64 << 20)
    for rep in range(2):
        for i, b in enumerate(blocks):
            j = api.Job(c, b, api.PRIOR_SEPARABLE, 0, seed=100 + i)
            _k = j.upload_block()
            j.run()
            got = j.download_outputs()
            for k in ("mean", "cov", "sims"):
                assert np.array_equal(got[k], alone[i][k]), (rep, i, k)
            j.close()
    st = c.table_cache_stats()
    assert st["hits"] >= 2 * len(blocks) and st["entries"] >= len(blocks)
    c.close()


def test_served_queue_limit_and_cancel(ctx, blocks):
    """With one request running, a queue limit of 2 refuses the third waiting request with
    EBUSY (nothing queued); a queued request can be cancelled (it fails with ECANCELED, reported
    once), a running one cannot (ESTATE); the others complete."""
    import time
    sv = api.Server(ctx, max_inflight=1)
    sv.set_queue_limit(2)
    big = synth.make_block_fast(synth.BlockSpec(nx=256, ny=256, nz=128, nsim=16, seed=5))
    bi, bo = _host_buffers(big, big.nsim)
    t0 = sv.submit(big, bi, bo, seed=1)
    deadline = time.time() + 60
    while sv.poll(t0)["state"] == api.REQ_QUEUED and time.time() < deadline:
        time.sleep(0.0005)
    b = blocks[0]
    bufs = [_host_buffers(b, b.nsim) for _ in range(3)]
    t1 = sv.submit(b, *bufs[0], seed=2)
    t2 = sv.submit(b, *bufs[1], seed=3)
    with pytest.raises(api.CravaError) as e:
        sv.submit(b, *bufs[2], seed=4)
    assert e.value.status == api.EBUSY
    sv.cancel(t2)
    info = sv.poll(t2)
    assert info["state"] == api.REQ_FAILED and info["status"] == api.ECANCELED
    with pytest.raises(api.CravaError) as e:
        sv.poll(t2)                      # the final state was reported once
    assert e.value.status == api.EINVAL
    with pytest.raises(api.CravaError) as e:
        sv.cancel(t0)
    assert e.value.status == api.ESTATE
    assert sv.wait(t0, timeout_ms=120000)["state"] == api.REQ_DONE
    assert sv.wait(t1, timeout_ms=120000)["state"] == api.REQ_DONE
    sv.stop()


def test_injected_allocation_failures(blocks):
    """crava_ctx_fail_next_allocs: the next job creation fails with ENOMEM and the one after it
    succeeds; a served request whose allocation fails with nothing in flight fails with ENOMEM
    and the request behind it completes with the same result as alone."""
    c = api.Context(0)
    b = blocks[0]
    c.fail_next_allocs(1)
    with pytest.raises(api.CravaError) as e:
        api.Job(c, b, api.PRIOR_SEPARABLE, 0, seed=1)
    assert e.value.status == api.ENOMEM
    j = api.Job(c, b, api.PRIOR_SEPARABLE, 0, seed=1)
    j.close()
    sv = api.Server(c, max_inflight=1)
    c.fail_next_allocs(1)
    bi, bo = _host_buffers(b, b.nsim)
    t_bad = sv.submit(b, bi, bo, seed=1)
    with pytest.raises(api.CravaError) as e:
        sv.wait(t_bad, timeout_ms=120000)
    assert e.value.status == api.ENOMEM
    gi, go = _host_buffers(b, b.nsim)
    t_ok = sv.submit(b, gi, go, seed=1)
    assert sv.wait(t_ok, timeout_ms=120000)["state"] == api.REQ_DONE
    sv.stop()
    c.close()
