"""bench.py host logic: algorithmic byte counts, clock-log parsing, and the max-over-ranks
reduction of the multi-GPU launch (world size 2 on gloo)."""
import os
import socket

import pytest

import bench
from crava_b200 import synth


def test_alg_bytes_model():
    blk = synth.make_block(synth.BlockSpec(nx=16, ny=12, nz=20, nsim=2))
    N = 16 * 12 * 20
    Nc = 9 * 12 * 20
    assert bench.alg_bytes(blk, 2, "zpass", 1) == 8 * Nc * ((3 + 3) + (9 + 6))
    assert bench.alg_bytes(blk, 2, "line_fwd", 6) == 6 * 16 * Nc
    assert bench.alg_bytes(blk, 2, "x_r2c", 6) == 6 * (4 * N + 8 * Nc)


def test_clock_summary(tmp_path):
    p = tmp_path / "c.csv"
    p.write_text(
        "index, clocks.sm [MHz], clocks.max.sm [MHz], power.draw [W], active, hw, hwt, swt, swpc\n"
        "0, 1965 MHz, 1965 MHz, 700 W, 0x0, Not Active, Not Active, Not Active, Not Active\n"
        "0, 1800 MHz, 1965 MHz, 990 W, 0x4, Not Active, Not Active, Not Active, Active\n"
        "1, 900 MHz, 1965 MHz, 100 W, 0x0, Active, Not Active, Not Active, Not Active\n")
    c = bench.summarize_clocks(str(p), 0)
    assert c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"]
    assert c["samples"] == 2


def test_clock_merge_prefers_the_timed_region_samples(tmp_path):
    p = tmp_path / "c.csv"
    p.write_text(
        "index, clocks.sm [MHz], clocks.max.sm [MHz], power.draw [W], active, hw, hwt, swt, swpc\n"
        "0, 345 MHz, 1965 MHz, 120 W, 0x1, Not Active, Not Active, Not Active, Not Active\n"
        "0, 1800 MHz, 1965 MHz, 990 W, 0x4, Not Active, Not Active, Not Active, Active\n")
    smi = bench.summarize_clocks(str(p), 0)

    class Nvml:
        sm = [1965.0, 1950.0, 1965.0]
        reasons = {"hw_slowdown"}
        max_mhz = 1965.0
    c = bench.merge_clocks(smi, Nvml())
    assert c["sm_mhz"] == 1965.0 and c["samples"] == 3 and c["nvidia_smi_samples"] == 2
    assert c["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert "_sm" not in c and "_sm" not in bench.merge_clocks(smi, None)
    assert bench.merge_clocks(None, None) is None


def test_fifo_replay():
    span, lat = bench.fifo_replay([0.0, 0.1, 0.15, 1.0], [0.2, 0.05, 0.1, 0.05])
    assert abs(span - 1.05) < 1e-12
    assert [round(v, 6) for v in lat] == [200.0, 150.0, 200.0, 50.0]


def test_physical_gpu_index(monkeypatch):
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "3,5")
    assert bench.physical_gpu_index(1) == 5
    monkeypatch.delenv("CUDA_VISIBLE_DEVICES")
    assert bench.physical_gpu_index(2) == 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    v = bench.max_over_ranks(10.0 + 5.0 * rank, dist, device="cpu")
    q.put((rank, v))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_world2_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 15.0), (1, 15.0)]


def test_max_over_ranks_single_process():
    assert bench.max_over_ranks(3.0, None) == 3.0
