#!/usr/bin/env python
"""Benchmark of the B200 FFT-domain AVO inversion (posterior mean + covariance + realisations).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one whole inversion block of the 540x540x256 production workload (5 angle
stacks 5..45 deg, 4 conditional realisations, separable prior): forward transforms of the
data and prior mean, the fused per-bin posterior and simulation pencil pass, inverse
transforms of mean, covariance and realisations.  Under torchrun every rank inverts its own
block (weak scaling, no collective on the data path).

`value` is voxels/s with inputs resident in HBM; `e2e` is the same metric through the
C-ABI job calls with pinned host buffers (uploads, run, downloads of every output inside
the timed region), for a stream of blocks on two jobs and two streams so that one block's
copies overlap the next one's.  `--impl reference` times the reference's own CPU numerics (FFTW 2.1.2
float + lib_matr, built into oracle/_ref) on bounded samples of the same workload on the
host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "posterior voxels/s batched+served vs plain GPU at ≤1e-4 rel err; p99 latency"
UNIT = "voxels/s"
HBM_FALLBACK_GBS = 6650.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def workload_spec(rank: int = 0, dims=None):
    from crava_b200 import synth
    spec = synth.config1(seed=21 + rank)
    if dims:
        spec.nx, spec.ny, spec.nz = dims
    return spec


def sample_spec(seed: int = 101):
    """Bounded CPU sample of the same workload: the 540x540x256 block's parameters on a
    135x135x256 lateral window (1/16 of the voxels, same z length and angle count)."""
    from crava_b200 import synth
    spec = synth.config1(seed=seed)
    spec.nx = spec.ny = 135
    return spec


# ------------------------------------------------------------------ clocks

CLOCK_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def start_clock_sampler(path):
    try:
        f = open(path, "w")
        p = subprocess.Popen(["nvidia-smi", f"--query-gpu={CLOCK_FIELDS}", "--format=csv", "-lms", "200"],
                             stdout=f, stderr=subprocess.DEVNULL)
        return p, f
    except Exception:
        return None, None


def stop_clock_sampler(p, f):
    if p is None:
        return
    p.terminate()
    try:
        p.wait(timeout=5)
    except Exception:
        p.kill()
    f.close()


class NvmlClockSampler:
    """SM clock and clock-event reasons of one GPU read through NVML every `interval` seconds
    by a thread (reads only), so that a timed region of a fraction of a second still gets a
    dozen samples beside nvidia-smi's 200 ms ones."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, gpu_index, interval=0.01):
        import threading
        self.sm, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._t = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(gpu_index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM))
            self._reason = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        except Exception:
            self._nv = None
            return
        self._interval = interval
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)))
                r = self._reason(self._h)
                for name, const in self.REASONS:
                    if r & getattr(nv, const, 0):
                        self.reasons.add(name)
            except Exception:
                return
            self._stop.wait(self._interval)

    def stop(self):
        if self._t is not None:
            self._stop.set()
            self._t.join(timeout=2)
        if self._nv is not None:
            try:
                self._nv.nvmlShutdown()
            except Exception:
                pass
        return self


def merge_clocks(smi, nv):
    """One clocks record: the median SM clock of the NVML samples, taken inside the timed region
    alone, and the throttle reasons seen by either sampler (nvidia-smi's run also covers a
    short idle lead-in, so its clocks only stand in when NVML gave nothing)."""
    if smi is not None:
        smi = {k: v for k, v in smi.items() if k != "_sm"}
    if nv is None or not nv.sm:
        return smi
    reasons = set(nv.reasons) | set((smi or {}).get("reasons", []))
    mx = nv.max_mhz if nv.max_mhz is not None else (smi or {}).get("sm_max_mhz")
    return {"sm_mhz": statistics.median(nv.sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(nv.sm),
            "sampler": "NVML every 10 ms over the timed steps", "nvidia_smi_samples": (smi or {}).get("samples", 0)}


def summarize_clocks(path, gpu_index):
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    sm, mx, reasons = [], None, set()
    try:
        with open(path) as f:
            lines = [l.strip() for l in f if l.strip()]
    except Exception:
        return None
    for l in lines[1:]:
        parts = [p.strip() for p in l.split(",")]
        if len(parts) < 9 or not parts[0].isdigit() or int(parts[0]) != gpu_index:
            continue
        try:
            sm.append(float(parts[1].split()[0]))
            mx = float(parts[2].split()[0])
        except ValueError:
            continue
        for nm, v in zip(names, parts[5:9]):
            if v.lower() == "active":
                reasons.add(nm)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
            "_sm": sm}


def physical_gpu_index(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return int(ids[local_rank])
    return local_rank


# ------------------------------------------------------------------ CPU reference (oracle/_ref)

_worker_block = None


def _ref_worker_init(seed):
    global _worker_block
    from crava_b200 import synth
    _worker_block = synth.make_block(sample_spec(seed))


def _ref_worker_run(_):
    """One sample inversion with the reference numerics; returns (voxels, seconds)."""
    from oracle import bindings as ob
    from oracle import ref64
    blk = _worker_block
    covs, _ = ref64.prior_cov_grids(blk)
    ec = ref64.fill_err_corr_zero_grad(blk.corr_xy, blk.nxp, blk.nyp, blk.nzp)
    t = time.perf_counter()
    ob.ref32_invert(blk, covs, ec, nsim=blk.nsim, seed=blk.seed)
    return blk.n_voxels, time.perf_counter() - t


def cpu_reference_available():
    from oracle import bindings as ob
    return ob.ref32_available()


def run_cpu_sample(nproc=1, steps=1, warmup=0):
    """Runs the sample on nproc spawned processes; returns per-step (voxels/s) list."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    vals = []
    with ctx.Pool(nproc, initializer=_ref_worker_init, initargs=(101,)) as pool:
        for s in range(warmup + steps):
            t0 = time.perf_counter()
            res = pool.map(_ref_worker_run, range(nproc), chunksize=1)
            dt = time.perf_counter() - t0
            if s >= warmup:
                vals.append(sum(r[0] for r in res) / dt)
    return vals


def reference_main(args, rank, world):
    spec = workload_spec(0)
    cfg = {"workload": f"{spec.nx}x{spec.ny}x{spec.nz}, {len(spec.theta_deg)} angles, {spec.nsim} realisations",
           "prior": "separable (reference: six covariance grids + errCorr grid, as InitializeCorrelations builds)"}
    if rank != 0:
        return
    if not cpu_reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref32.so was not built (reference tree absent at build time)"}))
        return
    ncores = os.cpu_count() or 1
    nproc = max(1, min(64, ncores))
    vals = run_cpu_sample(nproc=nproc, steps=args.steps, warmup=args.warmup)
    v = statistics.median(vals)
    smp = sample_spec()
    vox = smp.nx * smp.ny * smp.nz
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * nproc * vox / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nproc, "kind": "reference",
                             "sample": f"{nproc} processes, each one full inversion (5 angles, 4 realisations) of a "
                                       f"{smp.nx}x{smp.ny}x{smp.nz} window of the workload per step; FFTW 2.1.2 float "
                                       f"and lib_matr.c from the reference, single-threaded as in the reference; "
                                       f"host has {ncores} logical cores"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ------------------------------------------------------------------ GPU arm

def max_over_ranks(x: float, dist, device: str = "cuda") -> float:
    """Max of a per-rank timing over all ranks (a no-op without a process group)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def alg_bytes(blk, nsim, cls, ngrids):
    """Algorithmic HBM bytes of one launch of a kernel class over ngrids grids."""
    N = blk.nxp * blk.nyp * blk.nzp
    Nc = (blk.nxp // 2 + 1) * blk.nyp * blk.nzp
    if cls in ("x_r2c", "xy_fwd"):   # the fused xy pass keeps the x->y intermediate in L2
        return ngrids * (4 * N + 8 * Nc)
    if cls in ("x_c2r", "xy_inv"):
        return ngrids * (8 * Nc + 4 * N)
    if cls in ("line_fwd", "line_inv"):
        return ngrids * 16 * Nc
    if cls == "zpass":
        return 8 * Nc * ((blk.ntheta + 3) + (9 + 3 * nsim))
    raise ValueError(cls)


# ncu summary of the kernel each timer class measures at the production size
PROFILE_OF_CLASS = {"zpass": "pencil"}


def read_traffic(kernel_class):
    """dram bytes per launch from the committed ncu summary (line 'traffic_bytes_per_launch')."""
    path = os.path.join(ROOT, "profiles", f"{PROFILE_OF_CLASS.get(kernel_class, kernel_class)}_540x540x256.md")
    try:
        with open(path) as f:
            for l in f:
                if l.startswith("traffic_bytes_per_launch:"):
                    return float(l.split(":", 1)[1].strip())
    except Exception:
        pass
    return None


def batched_leg(ctx, torch, n_blocks=64, nsim=16, reps=3, branch_counts=(1, 2, 4, 16)):
    """64 blocks of uneven size and angle count (nx, ny smooth in [64,256], nz smooth in
    [64,200], 2..6 angles, 16 realisations): one-job-at-a-time (run, wait) against the whole
    batch replayed as one CUDA graph with concurrent branches (each branch count of
    branch_counts timed; the line reports the fastest and lists all); inputs resident."""
    from crava_b200 import api, synth
    blocks = [synth.make_block_fast(s) for s in synth.batch_specs(n_blocks, nsim=nsim)]
    jobs = []
    for i, b in enumerate(blocks):
        j = api.Job(ctx, b, api.PRIOR_SEPARABLE, 0, seed=500 + i)
        j._keep_in = j.upload_block()
        jobs.append(j)
    vox = sum(b.n_voxels for b in blocks)
    st = torch.cuda.current_stream()
    sh = st.cuda_stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for j in jobs:
        j.run(sh)
    torch.cuda.synchronize()
    e0.record(st)
    for j in jobs:
        j.run(sh)
        st.synchronize()
    e1.record(st)
    torch.cuda.synchronize()
    t_plain = e0.elapsed_time(e1) / 1000.0
    # the ceiling of any batching: the plain path's wall time against the device time of its
    # kernels (per-launch CUDA events); a plain path whose wall time is mostly kernel time
    # leaves batching little to gain
    ctx.set_profiling(True)
    ctx.kernel_times(reset=True)
    for j in jobs:
        j.run(sh)
        st.synchronize()
    torch.cuda.synchronize()
    kt = ctx.kernel_times(reset=True)
    ctx.set_profiling(False)
    t_kernels = sum(v[0] for v in kt.values()) / 1000.0
    per_branches = {}
    best = None
    for branches in branch_counts:
        bt = api.Batch(ctx, jobs, branches=branches)
        bt.run(sh)
        torch.cuda.synchronize()
        l0 = ctx.kernel_launches()
        e0.record(st)
        for _ in range(reps):
            bt.run(sh)
        e1.record(st)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1000.0 / reps
        per_branches[str(branches)] = 1000 * t
        if best is None or t < best[0]:
            best = (t, branches, (ctx.kernel_launches() - l0) // reps)
        bt.close()
    t_b, branches, launches = best
    for j in jobs:
        j.close()
    return {"workload": f"{n_blocks} blocks, nx,ny in smooth[64,256], nz in smooth[64,200], 2..6 angles, "
                        f"{nsim} realisations, separable prior, white-noise seismic of seismic amplitude",
            "voxels": vox, "voxels_per_s": vox / t_b, "jobs_per_s": n_blocks / t_b, "ms_per_batch": 1000 * t_b,
            "plain_voxels_per_s": vox / t_plain, "plain_jobs_per_s": n_blocks / t_plain,
            "speedup_vs_plain": t_plain / t_b, "branches": branches, "ms_per_batch_by_branches": per_branches,
            "gpu_launches_per_batch": launches,
            "plain_kernel_ms_sum": 1000 * t_kernels, "plain_wall_ms": 1000 * t_plain,
            "plain_gpu_busy": t_kernels / t_plain,
            "speedup_ceiling": t_plain / t_kernels,
            "ceiling_note": "plain wall time / sum of its kernel times: batching can remove host gaps and "
                            "overlap launch tails, not kernel work"}


def cfg3_leg(torch, steps, warmup):
    """The precision-study block 768x768x320 (6 angles 5..50 deg, band 2..120 Hz, S/N 2..10,
    1 realisation): ms per job on resident inputs and its job roofline
    B_alg = 12 N (G_in + G_out) = 12 * 188,743,680 * (9 + 12) bytes = 47.56 GB."""
    from crava_b200 import api, synth
    blk = synth.make_block_fast(synth.config3())
    ctx = api.Context(torch.cuda.current_device())
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=3000)
    keep = job.upload_block()
    st = torch.cuda.current_stream()
    sh = st.cuda_stream
    for _ in range(warmup):
        job.run(sh)
    torch.cuda.synchronize()
    ctx.set_profiling(True)
    ctx.kernel_times(reset=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        job.run(sh)
    e1.record(st)
    torch.cuda.synchronize()
    kt = ctx.kernel_times(reset=True)
    ctx.set_profiling(False)
    ms = e0.elapsed_time(e1) / steps
    peak, peak_kind = peaks()
    nin, nout = blk.ntheta + 3, 9 + 3 * job.nsim
    B_alg = 12 * blk.n_voxels * (nin + nout)
    del keep
    job.close()
    ctx.close()
    return {"workload": f"single block {blk.nx}x{blk.ny}x{blk.nz}, {blk.ntheta} angles 5..50 deg, band 2..120 Hz, "
                        f"S/N 2..10, {job.nsim} realisation, separable prior; inputs white noise of seismic amplitude",
            "steps": steps, "warmup": warmup, "ms_per_job": ms, "voxels_per_s": blk.n_voxels / (ms / 1000.0),
            "job_roofline": {"alg_bytes": B_alg, "achieved_gbs": B_alg / (ms / 1000.0) / 1e9,
                             "frac": B_alg / (ms / 1000.0) / 1e9 / peak, "peak_gbs": peak, "peak_kind": peak_kind,
                             "target_frac": 0.6, "target_ms": B_alg / (0.6 * peak * 1e9) * 1000.0},
            "kernel_ms_per_job": {c: kt[c][0] / steps for c in kt if kt[c][1]}}


def cufft_leg(torch, dims=(540, 540, 256), reps=10):
    """Comparator only (not on the product path): one 3D real transform of a 540x540x256 grid
    each way, the library's drop-in for FFTGrid::fftInPlace / invFFTInPlace (crava_fft_r2c /
    crava_fft_c2r, in place on the padded layout) against cuFFT through torch.fft.rfftn /
    irfftn (out of place), device time per transform with CUDA events."""
    from crava_b200 import api
    nx, ny, nz = dims
    rnx = 2 * (nx // 2 + 1)
    ctx = api.Context(torch.cuda.current_device())
    g = torch.randn((nz, ny, rnx), device="cuda", dtype=torch.float32)
    x = torch.randn((nz, ny, nx), device="cuda", dtype=torch.float32)
    st = torch.cuda.current_stream()
    sh = st.cuda_stream

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {}
    out["crava_r2c_ms"] = timed(lambda: api.fft_r2c(ctx, g.data_ptr(), nx, ny, nz, False, sh))
    out["crava_c2r_ms"] = timed(lambda: api.fft_c2r(ctx, g.data_ptr(), nx, ny, nz, False, sh))
    y = torch.fft.rfftn(x, dim=(0, 1, 2))
    out["cufft_r2c_ms"] = timed(lambda: torch.fft.rfftn(x, dim=(0, 1, 2)))
    out["cufft_c2r_ms"] = timed(lambda: torch.fft.irfftn(y, s=(nz, ny, nx), dim=(0, 1, 2)))
    del g, x, y
    ctx.close()
    return {"workload": f"one {nx}x{ny}x{nz} real grid, 3D r2c and c2r", "reps": reps, **out,
            "note": "cuFFT is a comparator only; the library's transforms are the product path"}


def fifo_replay(arrivals, service):
    """One server taking requests in arrival order: request k starts at max(its arrival, the
    previous one's end) and runs for its measured service time.  Returns (makespan in s,
    latencies in ms); times in s from the same origin as the arrivals."""
    done, lat = 0.0, []
    for a, sv in zip(arrivals, service):
        done = max(float(a), done) + float(sv)
        lat.append((done - float(a)) * 1000.0)
    return done, lat


def served_leg(torch, n_jobs=48, n_models=6, rate=20.0, nsim=16, max_inflight=8, budget_gb=120):
    """Served stream: Poisson arrivals at `rate` jobs/s; every request drawn fresh: one of
    n_models interval models (nz, 3..6 angles, priors within +-30% of the 64x64x128 block,
    wavelets) and its own lateral shape, so that voxel counts are log-uniform between 64^3 and
    512x512x256; 16 realisations; host->device inputs, inversion, device->host of the
    posterior mean, covariance and first realisation per request.  Against the plain
    one-job-at-a-time path (create, upload, run, download, release) on a context without the
    resident table cache: back to back for the saturated run, and for the Poisson run its
    measured per-request times replayed under the same arrivals.  Input values come from a shared random pinned pool and outputs
    land in a shared pinned scratch (the inversion's cost does not depend on the values; the
    test suite checks every result alone and in a served mix)."""
    import numpy as np
    from crava_b200 import api, synth
    specs = synth.served_stream_specs(n_jobs, n_models=n_models, nsim=nsim)
    blocks = [synth.make_block_fast(sp, data=False) for sp in specs]
    shapes = [(b.nzp, b.nyp, 2 * (b.nxp // 2 + 1)) for b in blocks]
    gmax = max(int(np.prod(sh)) for sh in shapes)
    rng = np.random.default_rng(5)
    pool_in = torch.empty(9 * gmax, dtype=torch.float32).pin_memory()
    pool_in.numpy()[:] = rng.standard_normal(9 * gmax, dtype=np.float32) * np.float32(0.02)
    pool_out = torch.empty(12 * gmax, dtype=torch.float32).pin_memory()

    def bufs(k):
        b, n = blocks[k], int(np.prod(shapes[k]))
        ins = [pool_in[q * gmax:q * gmax + n].view(shapes[k]) for q in range(b.ntheta + 3)]
        outs = [pool_out[q * gmax:q * gmax + n].view(shapes[k]) for q in range(12)] + [None] * (3 * nsim - 3)
        return ins, outs

    vox = sum(b.n_voxels for b in blocks)
    # plain path
    ctx = api.Context(torch.cuda.current_device(), hbm_budget=int(budget_gb * 1e9))
    t0 = time.perf_counter()
    service = []
    for k, b in enumerate(blocks):
        tk = time.perf_counter()
        j = api.Job(ctx, b, api.PRIOR_SEPARABLE, 0, seed=900 + k)
        ins, outs = bufs(k)
        for q, h in enumerate(ins):
            role, idx = (api.ROLE_DATA, q) if q < b.ntheta else (api.ROLE_MEAN, q - b.ntheta)
            api._check(api.lib().crava_job_upload(j._h, role, idx, h.data_ptr(), None))
        j.run()
        for q in range(12):
            role, idx = (api.ROLE_POST_MEAN, q) if q < 3 else ((api.ROLE_POST_COV, q - 3) if q < 9 else (api.ROLE_SIM, q - 9))
            api._check(api.lib().crava_job_download(j._h, role, idx, outs[q].data_ptr(), None))
        torch.cuda.synchronize()
        j.close()
        service.append(time.perf_counter() - tk)
    t_plain = time.perf_counter() - t0
    ctx.close()
    # served at `rate` (Poisson) and saturated (all at once), each on a fresh context
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_jobs))
    res = {}
    for mode in ("poisson", "saturated"):
        ctx = api.Context(torch.cuda.current_device(), hbm_budget=int(budget_gb * 1e9))
        sv = api.Server(ctx, max_inflight=max_inflight)
        tickets = []
        t0 = time.perf_counter()
        for k, b in enumerate(blocks):
            if mode == "poisson":
                dt = arrivals[k] - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
            ins, outs = bufs(k)
            tickets.append(sv.submit(b, ins, outs, seed=900 + k))
        infos = [sv.wait(t, timeout_ms=600000) for t in tickets]
        t_all = time.perf_counter() - t0
        sv.stop()
        cache = ctx.table_cache_stats()
        ctx.close()
        lat = np.array([x["latency_ms"] for x in infos])
        res[mode] = {"jobs_per_s": n_jobs / t_all, "voxels_per_s": vox / t_all,
                     "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                     "speedup_vs_plain": t_plain / t_all,
                     "table_cache": {"hits": cache["hits"], "misses": cache["misses"], "entries": cache["entries"]}}
        if mode == "poisson":
            # the plain path under the same arrivals: its measured per-request times replayed
            # through one first-come-first-served server (arrival-limited, like the served run)
            span, plat = fifo_replay(arrivals, service)
            res[mode]["speedup_vs_plain"] = span / t_all
            res[mode]["plain_same_arrivals"] = {"jobs_per_s": n_jobs / span, "p50_ms": float(np.percentile(plat, 50)),
                                                "p99_ms": float(np.percentile(plat, 99))}
    return {"workload": f"{n_jobs} requests, each drawn fresh: one of {n_models} interval models (nz, 3..6 angles, "
                        f"+-30% priors, wavelets) and its own lateral shape, voxels log-uniform 64^3..512x512x256, "
                        f"{nsim} realisations; outputs mean+cov+1 realisation to host; {rate:g} jobs/s Poisson",
            "voxels": vox, "plain_jobs_per_s": n_jobs / t_plain, "plain_voxels_per_s": vox / t_plain,
            "max_inflight": max_inflight, "budget_gb": budget_gb, **res}


def nonconst_main(args):
    """Non-constant thickness on the same workload (one GPU): a step is
    crava_job_divide_data (divideDataByScaleWavelet + interpolateSeismic) followed by the
    inversion, on resident inputs; the data grids are uploaded again before each step
    (outside the timed region) because the division works in place.  Prints one JSON
    line of its own; the headline line is the default mode's."""
    import numpy as np
    import torch
    from crava_b200 import api, synth

    dims = tuple(int(v) for v in args.dims.split(",")) if args.dims else None
    blk = synth.with_rel_thick(synth.make_block_fast(workload_spec(0, dims)))
    ctx = api.Context(0)
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=1000)
    keep = job.upload_block()
    if args.wavelet3d:
        job.set_wavelet_3d(**synth.wavelet3d_model(blk, blk.spec.theta_deg, seed=7))

    def restore():
        for l in range(blk.ntheta):
            keep.append(job.upload(api.ROLE_DATA, l, blk.data[l]))

    for _ in range(args.warmup):
        restore()
        job.divide_data()
        job.run()
    torch.cuda.synchronize()
    ctx.set_profiling(True)
    ctx.kernel_times(reset=True)
    stream = torch.cuda.current_stream()
    tot = 0.0
    launches0 = ctx.kernel_launches()
    for _ in range(args.steps):
        restore()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        job.divide_data()
        job.run()
        e1.record(stream)
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    launches = ctx.kernel_launches() - launches0
    kt = ctx.kernel_times(reset=True)
    ms = tot / args.steps
    peak, peak_kind = peaks()
    td_ms, td_n = kt["thick_divide"]
    ab = 8 * blk.n_voxels * blk.ntheta          # each data voxel read and written once
    achieved = ab / (td_ms / max(td_n, 1) / 1000.0) / 1e9
    line = {
        "metric": "non-constant-thickness inversion throughput (data division + inversion)",
        "value": blk.n_voxels / (ms / 1000.0), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"single block {blk.nx}x{blk.ny}x{blk.nz}, {blk.ntheta} angles, {job.nsim} "
                               f"realisations, rel_thick in [0.75, 1.3]"
                               + (", 3D wavelets (dip-adjusted per trace, Halpha damping)" if args.wavelet3d else ""),
                   "l2": "inputs > 126 MB L2"},
        "gpu_launches": launches,
        "kernel_ms_per_step": {c: kt[c][0] / args.steps for c in kt if kt[c][1]},
        "roofline": {"bound": "hbm", "kernel": "thick_divide", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "alg_bytes_per_launch": ab, "peak_kind": peak_kind},
    }
    print(json.dumps(line))
    del keep
    job.close()
    ctx.close()


def kernels_main(args):
    """The auxiliary kernels on the production block (540x540x256, 5 angles, 4 realisations;
    --dims for another size): the local-noise correction, facies probabilities (single volume
    and 4 local-noise corner volumes), the prior-grid generation of a GRIDS job, and the
    general-length transforms of a 250x250x200 block (lengths outside the four-step table).
    Each is timed with the library's CUDA-event timers over `steps` calls after `warmup`;
    achieved GB/s = algorithmic bytes / device time.  One JSON line of its own."""
    import numpy as np
    import torch
    from crava_b200 import api, synth

    dims = tuple(int(v) for v in args.dims.split(",")) if args.dims else None
    peak, peak_kind = peaks()
    ctx = api.Context(0)
    out = {}

    def timed(cls, fn, alg_bytes, note):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ctx.set_profiling(True)
        ctx.kernel_times(reset=True)
        for _ in range(args.steps):
            fn()
        torch.cuda.synchronize()
        ms, n = ctx.kernel_times(reset=True)[cls]
        ctx.set_profiling(False)
        per = ms / max(n, 1)
        gbs = alg_bytes / (per / 1000.0) / 1e9
        return {"ms_per_launch": per, "launches": n, "alg_bytes_per_launch": alg_bytes, "achieved_gbs": gbs,
                "frac": gbs / peak, "bytes_model": note}

    blk = synth.make_block_fast(workload_spec(0, dims))
    nvox = blk.nx * blk.ny * blk.nz
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=5)
    keep = job.upload_block()
    job.run()
    rng = np.random.default_rng(3)
    scales = (1.0 + rng.random((blk.ntheta, blk.ny, blk.nx))).astype(np.float32)
    nsim = job.nsim
    out["local_noise"] = timed("local_noise", lambda: job.local_noise(scales), 4 * nvox * (9 + 6 * nsim),
                               "per voxel: posterior, prior mean and realisations read, posterior and "
                               "realisations written (4 B each)")
    # facies probabilities on the posterior mean
    d_post = [job.device_ptr(api.ROLE_POST_MEAN, a) for a in range(3)]
    nf, nbins = 3, (100, 100, 50)
    rnx = 2 * (blk.nx // 2 + 1)
    probs = [torch.empty((blk.nz, blk.ny, rnx), dtype=torch.float32, device="cuda") for _ in range(nf + 1)]
    mean_host = [job.download(api.ROLE_POST_MEAN, a)[..., :blk.nx] for a in range(3)]
    descs, dkeep, dens = [], [], []
    for c in range(4):
        vmin = [float(m.min()) - 0.05 * (1 + c) for m in mean_host]
        dv = [(float(m.max()) + 0.05 * (1 + c) - vmin[i]) / nbins[i] for i, m in enumerate(mean_host)]
        fd, k = api.facies_desc([0.3, 0.3, 0.4], nbins, vmin, dv, 0.02)
        descs.append(fd)
        dkeep.append(k)
        dens.append(torch.rand((nf, nbins[2], nbins[1], nbins[0]), device="cuda"))
    fbytes = nvox * (12 + 4 * (nf + 1))
    out["facies_single"] = timed("facies", lambda: api.facies_prob(
        ctx, descs[0], dens[0].data_ptr(), nbins[0], d_post, blk.nx, blk.ny, blk.nz, blk.nxp, blk.nyp,
        [t.data_ptr() for t in probs]), fbytes, "per voxel: 3 posterior values read, nf+1 probabilities written")
    sc2 = scales[:2]
    out["facies_corners"] = timed("facies", lambda: api.facies_prob_local_noise(
        ctx, descs, [d.data_ptr() for d in dens], nbins[0], sc2, d_post, blk.nx, blk.ny, blk.nz, blk.nxp, blk.nyp,
        [t.data_ptr() for t in probs]), fbytes, "as facies_single, 4 corner volumes (2 local-noise angles)")
    # the whole run with the facies probabilities: the standalone pass after crava_job_run
    # against crava_job_set_facies (evaluated inside the inverse x transform of the mean)
    def run_classes(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ctx.set_profiling(True)
        ctx.kernel_times(reset=True)
        for _ in range(args.steps):
            fn()
        torch.cuda.synchronize()
        kt = ctx.kernel_times(reset=True)
        ctx.set_profiling(False)
        cl = {c: kt[c][0] / args.steps for c in ("line_inv", "x_c2r", "facies")}
        cl["sum"] = sum(cl.values())
        cl["run_total"] = sum(v[0] for v in kt.values()) / args.steps
        return cl

    def separate():
        job.run()
        api.facies_prob(ctx, descs[0], dens[0].data_ptr(), nbins[0], d_post, blk.nx, blk.ny, blk.nz, blk.nxp,
                        blk.nyp, [t.data_ptr() for t in probs])

    sep = run_classes(separate)
    job.set_facies([descs[0]], [dens[0].data_ptr()], nbins[0], None, [t.data_ptr() for t in probs])
    forms = {}
    for name, v in (("job_two_passes_ms", 0), ("job_one_pass_ms", 1)):
        api.tuning_set("facies_fused", blk.nxp // 2, v)
        forms[name] = run_classes(job.run)
    api.tuning_set("facies_fused", blk.nxp // 2, -1)
    job.set_facies(None, None, 0, None, None)
    out["facies_in_mean_pass"] = dict(
        separate_call_ms=sep, **forms,
        note="ms per run by timer class: crava_job_run then crava_facies_prob (separate call), or "
             "crava_job_set_facies with the evaluation as a pass after the inverse x transform of the mean "
             "(two passes, the default) or inside it (one pass: the 3 mean grids transformed and evaluated by "
             "one kernel, timer class facies); single density volume 100x100x50, 3 facies")
    del keep
    job.close()
    # prior grids of a GRIDS job
    gjob = api.Job(ctx, blk, api.PRIOR_GRIDS, 0, seed=5)
    out["fill_prior"] = timed("fill_prior", lambda: gjob.fill_prior(0.3, -0.2), 28 * blk.nxp * blk.nyp * blk.nzp,
                              "7 grids written (4 B per padded voxel each)")
    gjob.close()
    # general-length transforms
    spec = synth.config1(seed=9)
    spec.nx, spec.ny, spec.nz = 250, 250, 200
    gblk = synth.make_block_fast(spec)
    g = api.Job(ctx, gblk, api.PRIOR_SEPARABLE, 0, seed=5)
    gk = g.upload_block()
    for _ in range(args.warmup):
        g.run()
    torch.cuda.synchronize()
    ctx.set_profiling(True)
    ctx.kernel_times(reset=True)
    for _ in range(args.steps):
        g.run()
    torch.cuda.synchronize()
    kt = ctx.kernel_times(reset=True)
    ctx.set_profiling(False)
    nin, nout = gblk.ntheta + 3, 9 + 3 * g.nsim
    ng = {"x_r2c": nin, "line_fwd": nin, "line_inv": nout, "x_c2r": nout, "zpass": 1}
    gen = {}
    for c in ng:
        ms, n = kt[c]
        per = ms / max(n, 1)
        ab = alg_bytes(gblk, g.nsim, c, ng[c])
        gen[c] = {"ms_per_launch": per, "launches": n, "alg_bytes_per_launch": ab,
                  "achieved_gbs": ab / (per / 1000.0) / 1e9, "frac": ab / (per / 1000.0) / 1e9 / peak}
    out["general_lengths_250x250x200"] = gen
    del gk
    g.close()
    ctx.close()
    print(json.dumps({"metric": "auxiliary kernels: achieved HBM GB/s against algorithmic bytes",
                      "workload": f"{blk.nx}x{blk.ny}x{blk.nz}, {blk.ntheta} angles, {nsim} realisations",
                      "peak_gbs": peak, "peak_kind": peak_kind, "steps": args.steps, "warmup": args.warmup,
                      "kernels": out}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--dims", default=None, help="nx,ny,nz of a smaller block (profiling runs only)")
    ap.add_argument("--no-legs", action="store_true", help="skip the batched and served legs")
    ap.add_argument("--wavelet3d", action="store_true",
                    help="with --nonconst: 3D wavelets (synthetic depth gradients and filter surfaces)")
    ap.add_argument("--nonconst", action="store_true",
                    help="measure the non-constant-thickness path instead (one GPU, its own JSON line)")
    ap.add_argument("--kernels", action="store_true",
                    help="measure the auxiliary kernels instead (one GPU, its own JSON line)")
    args = ap.parse_args()
    if args.nonconst and args.impl == "ours":
        return nonconst_main(args)
    if args.kernels and args.impl == "ours":
        return kernels_main(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_main(args, rank, world)

    # CPU baseline first, in a spawned process, before this process touches the GPU
    cpu = None
    if rank == 0 and not args.no_cpu and cpu_reference_available():
        try:
            vals = run_cpu_sample(nproc=1, steps=1, warmup=0)
            smp = sample_spec()
            cpu = {"value": vals[0], "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"one full inversion (5 angles, 4 realisations) of a {smp.nx}x{smp.ny}x{smp.nz} "
                             f"window of the workload, reference FFTW 2.1.2 float + lib_matr.c, 1 thread"}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {e}"}

    import numpy as np
    import torch
    from crava_b200 import api, synth

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    dims = tuple(int(v) for v in args.dims.split(",")) if args.dims else None
    spec = workload_spec(rank, dims)
    blk = synth.make_block(spec)
    ctx = api.Context(local_rank)
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=1000 + rank)
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    keep = job.upload_block()
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        job.run(sh)
    torch.cuda.synchronize()

    ctx.set_profiling(True)
    ctx.kernel_times(reset=True)
    clk_path = os.path.join(tempfile.gettempdir(), f"crava_clocks_{rank}.csv")
    sampler = start_clock_sampler(clk_path)
    time.sleep(0.3)
    launches0 = ctx.kernel_launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    nv_clocks = NvmlClockSampler(physical_gpu_index(local_rank))
    e0.record(stream)
    for _ in range(args.steps):
        job.run(sh)
    e1.record(stream)
    torch.cuda.synchronize()
    nv_clocks.stop()
    if dist:
        dist.barrier()
    stop_clock_sampler(*sampler)
    launches = ctx.kernel_launches() - launches0
    ms = e0.elapsed_time(e1) / args.steps
    kt = ctx.kernel_times(reset=True)
    ctx.set_profiling(False)
    ms = max_over_ranks(ms, dist)
    value = world * blk.n_voxels / (ms / 1000.0)

    # e2e through the job API with pinned host buffers: a stream of blocks, each uploaded,
    # inverted and downloaded with the C ABI calls; two jobs on two streams alternate so that
    # one block's host<->device copies overlap the other's (the link is full duplex)
    shape = job.shape
    nin = blk.ntheta + 3
    nout = 9 + 3 * job.nsim
    job2 = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=2000 + rank)
    jobs = [job, job2]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    pin_in = [torch.empty(shape, dtype=torch.float32).pin_memory() for _ in range(nin)]
    for l in range(blk.ntheta):
        pin_in[l].numpy()[...] = blk.data[l]
    for a in range(3):
        pin_in[blk.ntheta + a].numpy()[...] = blk.mean[a]
    pin_out = [[torch.empty(shape, dtype=torch.float32).pin_memory() for _ in range(nout)] for _ in range(2)]
    roles_out = [(api.ROLE_POST_MEAN, a) for a in range(3)] + [(api.ROLE_POST_COV, q) for q in range(6)] + \
                [(api.ROLE_SIM, q) for q in range(3 * job.nsim)]
    roles_in = [(api.ROLE_DATA, l) for l in range(blk.ntheta)] + [(api.ROLE_MEAN, a) for a in range(3)]

    def e2e_step(i):
        jb, s = jobs[i % 2], streams[i % 2].cuda_stream
        for (r, q), h in zip(roles_in, pin_in):
            api._check(api.lib().crava_job_upload(jb._h, r, q, h.data_ptr(), s))
        jb.run(s)
        for (r, q), h in zip(roles_out, pin_out[i % 2]):
            api._check(api.lib().crava_job_download(jb._h, r, q, h.data_ptr(), s))

    e2e_steps = max(2, min(args.steps, 4))
    e2e_step(0)
    e2e_step(1)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0.record(stream)
    for st_ in streams:
        st_.wait_stream(stream)
    for i in range(e2e_steps):
        e2e_step(i)
    for st_ in streams:
        stream.wait_stream(st_)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1) / e2e_steps
    ms_e2e = max_over_ranks(ms_e2e, dist)
    bytes_grid = 4 * int(np.prod(shape))

    # roofline of the dominant kernel class
    peak, peak_kind = peaks()
    ngrids = {"x_r2c": nin, "line_fwd": nin, "zpass": 1, "line_inv": nout, "x_c2r": nout, "xy_fwd": nin,
              "xy_inv": nout}
    dom = max(kt, key=lambda c: kt[c][0])
    tot_ms, nl = kt[dom]
    per_launch_ms = tot_ms / max(nl, 1)
    ab = alg_bytes(blk, job.nsim, dom, ngrids[dom])
    achieved = ab / (per_launch_ms / 1000.0) / 1e9
    share = {c: round(kt[c][0] / max(sum(v[0] for v in kt.values()), 1e-9), 4) for c in kt}
    B_alg = 12 * blk.n_voxels * (nin + nout)

    job.close()
    job2.close()
    batched = served = cfg3 = cufft = None
    if rank == 0 and not args.no_legs and not args.dims:
        cfg3 = cfg3_leg(torch, steps=max(3, min(args.steps, 10)), warmup=max(3, args.warmup))
        cufft = cufft_leg(torch)
        batched = batched_leg(ctx, torch)
        served = served_leg(torch)
    clocks = merge_clocks(summarize_clocks(clk_path, physical_gpu_index(local_rank)), nv_clocks)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"single block {blk.nx}x{blk.ny}x{blk.nz}, {blk.ntheta} angles 5..45 deg, "
                                   f"{job.nsim} realisations, separable prior (one block per GPU)",
                       "nx": blk.nx, "ny": blk.ny, "nz": blk.nz, "ntheta": blk.ntheta, "nsim": job.nsim,
                       "parallelism": f"replicas x{world}",
                       "l2": f"no flush: every step reads {nin} input grids and writes {nout} output grids of "
                             f"{bytes_grid / 1e6:.0f} MB each (> 126 MB L2)"},
            "e2e": {"value": world * blk.n_voxels / (ms_e2e / 1000.0), "unit": UNIT,
                    "h2d_bytes_per_step": nin * bytes_grid, "d2h_bytes_per_step": nout * bytes_grid,
                    "ms_per_step": ms_e2e,
                    "pipeline": "stream of blocks on two jobs and two CUDA streams: one block's uploads and "
                                "downloads overlap the next block's, pinned host buffers, crava_job_upload/run/download"},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": read_traffic(dom),
                         "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                         "alg_bytes_per_launch": ab, "ms_per_launch": per_launch_ms},
            "job_roofline": {"alg_bytes": B_alg, "achieved_gbs": B_alg / (ms / 1000.0) / 1e9,
                             "frac": B_alg / (ms / 1000.0) / 1e9 / peak,
                             "model": "12*N*(G_in+G_out): every real grid crosses HBM once plus one write+read of its half-transformed intermediate"},
            "kernel_ms_per_step": {c: kt[c][0] / args.steps for c in kt},
            "kernel_share": share,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "config3": cfg3,
            "cufft_comparator": cufft,
            "batched": batched,
            "served": served,
        }
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
