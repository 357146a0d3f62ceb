"""Autotuner of the schedule table (tile shapes and kernel choices) on the current GPU.

    python -m crava_b200.autotune [--out crava_b200/schedules.txt] [--reps 5] [--workloads prod,cfg3,...]

For each workload block it runs the whole inversion (crava_job_run) with candidate schedule
entries set through crava_tuning_set and times every kernel class with the library's own
CUDA-event timers (crava_ctx_set_profiling / crava_ctx_kernel_times), keeping per key the
fastest value.  The keys swept, with their size key n:

  pencil_kernel  n = nzp*16 + ntheta   1 general kernel (zpass.cu), 2 eigen form (pencil.cu)
  pencil_w       n = nzp*16 + ntheta   eigen form: x-bins per tile (power of two)
  pencil_sb      n = nzp*16 + ntheta   eigen form: realisations per transform batch (0: no
                                       realisation slots, the mean stored first)
  pencil_threads n = nzp*16 + ntheta   eigen form: threads per CTA
  pencil_dense   n = nzp*16 + ntheta   eigen form: 1 = the 80-register instantiation
  pencil_nb      n = nzp*16 + ntheta   eigen form: bins of one z position per thread (1 or 2)
  zpass_w, zpass_sb, zpass_threads     general kernel: tile width, realisations per batch,
                 n = nzp*16 + ntheta   threads per CTA
  line4_w_fwd, line4_w_inv   n = N     four-step column transforms: columns per tile
  line4_threads_fwd, line4_threads_inv  four-step column transforms: threads per CTA (n = N;
                                        at most 256 forward, 512 inverse)
  x4_stage_fwd, x4_stage_inv           four-step row transforms: 1 = twiddle tables staged in
                                        shared memory, 0 = read from global memory (n = nxp/2)
  x4_threads_fwd, x4_threads_inv       four-step row transforms: threads per CTA
                 n = nxp/2
  x4_rpc_fwd, x4_rpc_inv  n = nxp/2    rows per CTA (defaults threads / (N1/2 + 1), threads / N1)
  line4_pf_fwd, line4_pf_inv (n = N),  L2 prefetch of the tiles (rows) that many quarters of
  x4_pf_fwd, x4_pf_inv (n = nxp/2)     the resident CTAs ahead; 0 = off

The file holds one "key n value" line per entry; the library reads it at first use (it
sits beside libcrava_gpu.so) and falls back to built-in defaults for sizes it does not list.
Every candidate runs the same arithmetic, so the choice changes speed only (the parity tests
cover each kernel form).
"""
from __future__ import annotations

import argparse
import datetime
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

WORKLOADS = {
    # the production block (5 angles, 4 realisations)
    "prod": dict(spec="config1"),
    # the precision-study block (6 angles, 1 realisation)
    "cfg3": dict(spec="config3"),
    # mixed-size batch shapes: nzp 128 with 4 angles and 16 realisations, nzp 200 / 6 angles
    "b128": dict(spec="config0", nx=240, ny=192, nz=128, ntheta=4, nsim=16),
    "b200": dict(spec="config0", nx=200, ny=216, nz=200, ntheta=6, nsim=16),
}


def make_spec(w):
    import numpy as np
    from crava_b200 import synth
    spec = getattr(synth, w["spec"])()
    if "nx" in w:
        spec.nx, spec.ny, spec.nz = w["nx"], w["ny"], w["nz"]
    if "ntheta" in w:
        n = w["ntheta"]
        spec.theta_deg = tuple(np.linspace(5.0, 45.0, n))
        spec.peak_hz = (30.0,) * n
        spec.sn = (5.0,) * n
    if "nsim" in w:
        spec.nsim = w["nsim"]
    return spec


def time_classes(ctx, job, stream, reps):
    """Per-class device ms per run of the job (after one warm-up run)."""
    import torch
    job.run(stream)
    torch.cuda.synchronize()
    ctx.set_profiling(True)
    ctx.kernel_times(reset=True)
    for _ in range(reps):
        job.run(stream)
    torch.cuda.synchronize()
    kt = ctx.kernel_times(reset=True)
    ctx.set_profiling(False)
    return {k: v[0] / reps for k, v in kt.items() if v[1]}


def sweep(ctx, job, stream, reps, key, n, values, cls, log):
    """Sets key/n to each value in turn, keeps the fastest for kernel class(es) cls."""
    from crava_b200 import api
    best = None
    for v in values:
        api.tuning_set(key, n, v)
        try:
            t = time_classes(ctx, job, stream, reps)
        except api.CravaError as e:  # a candidate the launcher rejects (e.g. shared memory)
            log.append(f"# {key} {n} {v}: rejected ({e})")
            continue
        ms = sum(t.get(c, 0.0) for c in cls)
        log.append(f"# {key} {n} {v}: {ms:.3f} ms")
        if best is None or ms < best[1]:
            best = (v, ms)
    if best is None:
        api.tuning_set(key, n, -1)
        return None
    api.tuning_set(key, n, best[0])
    return best


def tune_workload(name, w, reps, entries, log):
    import torch
    from crava_b200 import api, synth
    spec = make_spec(w)
    blk = synth.make_block_fast(spec)
    ctx = api.Context(torch.cuda.current_device())
    job = api.Job(ctx, blk, api.PRIOR_SEPARABLE, 0, seed=7)
    keep = job.upload_block()
    stream = torch.cuda.current_stream().cuda_stream
    nxp, nyp, nzp, nth = blk.nxp, blk.nyp, blk.nzp, blk.ntheta
    pk = api.pencil_key(nzp, nth)
    log.append(f"# workload {name}: {nxp}x{nyp}x{nzp}, {nth} angles, {job.nsim} realisations")
    # pencil pass: the eigen form's tile and threads, then the general kernel's, then the form
    eig_best = None
    if nzp in (128, 256, 320):
        api.tuning_set("pencil_kernel", pk, 2)
        sweep(ctx, job, stream, reps, "pencil_w", pk, [1, 2, 4, 8], ["zpass"], log)
        # the realisation batch at the widest tile (without realisation slots a wider tile
        # may fit than with them); the width is swept again below
        w_keep = api.tuning_get("pencil_w", pk)
        api.tuning_set("pencil_w", pk, 8)
        sweep(ctx, job, stream, reps, "pencil_sb", pk, [0, 1, 2, 4], ["zpass"], log)
        api.tuning_set("pencil_w", pk, w_keep)
        eig_best = sweep(ctx, job, stream, reps, "pencil_threads", pk, [64, 128, 256, 384, 512], ["zpass"], log)
        # the tile width again, now with the realisation batch and threads chosen
        sweep(ctx, job, stream, reps, "pencil_w", pk, [2, 4, 8], ["zpass"], log)
        eig_best = sweep(ctx, job, stream, reps, "pencil_threads", pk, [128, 256, 512], ["zpass"], log)
        # one or two bins of a z position per thread in the per-bin step
        eig_best = sweep(ctx, job, stream, reps, "pencil_nb", pk, [1, 2], ["zpass"], log)
        # the 80-register form: two CTAs of up to 384 threads per SM
        if nth <= 6 and nzp in (256, 320):
            keep_w, keep_t, keep_sb = (api.tuning_get(k, pk) for k in ("pencil_w", "pencil_threads", "pencil_sb"))
            api.tuning_set("pencil_dense", pk, 1)
            api.tuning_set("pencil_sb", pk, 1)
            api.tuning_set("pencil_w", pk, 4)
            dense_best = sweep(ctx, job, stream, reps, "pencil_threads", pk, [256, 320, 384], ["zpass"], log)
            if dense_best and dense_best[1] < eig_best[1]:
                eig_best = dense_best
            else:
                api.tuning_set("pencil_dense", pk, -1)
                for k, v in (("pencil_w", keep_w), ("pencil_threads", keep_t), ("pencil_sb", keep_sb)):
                    api.tuning_set(k, pk, v)
    api.tuning_set("pencil_kernel", pk, 1)
    sweep(ctx, job, stream, reps, "zpass_w", pk, [1, 2, 4], ["zpass"], log)
    sweep(ctx, job, stream, reps, "zpass_sb", pk, [1, 2], ["zpass"], log)
    gen_best = sweep(ctx, job, stream, reps, "zpass_threads", pk, [256, 512], ["zpass"], log)
    if eig_best and (not gen_best or eig_best[1] <= gen_best[1]):
        api.tuning_set("pencil_kernel", pk, 2)
    for key in ("pencil_kernel", "pencil_w", "pencil_sb", "pencil_threads", "pencil_dense", "pencil_nb", "zpass_w",
                "zpass_sb", "zpass_threads"):
        v = api.tuning_get(key, pk)
        if v >= 0:
            entries[(key, pk)] = v
    # four-step column (y) and row (x) transforms
    for key, tkey, cls in (("line4_w_fwd", "line4_threads_fwd", ["line_fwd"]),
                           ("line4_w_inv", "line4_threads_inv", ["line_inv"])):
        b = sweep(ctx, job, stream, reps, key, nyp, [4, 8, 16, 32], cls, log)
        if b:
            entries[(key, nyp)] = b[0]
        tv = [128, 160, 192, 224, 256] + ([320, 384, 448, 512] if tkey.endswith("inv") else [])
        b = sweep(ctx, job, stream, reps, tkey, nyp, tv, cls, log)
        if b:
            entries[(tkey, nyp)] = b[0]
        pkey = "line4_pf_fwd" if tkey.endswith("fwd") else "line4_pf_inv"
        b = sweep(ctx, job, stream, reps, pkey, nyp, [0, 2, 4], cls, log)
        if b:
            entries[(pkey, nyp)] = b[0]
    if nxp % 2 == 0:
        h = nxp // 2
        for key, skey, cls in (("x4_threads_fwd", "x4_stage_fwd", ["x_r2c"]),
                               ("x4_threads_inv", "x4_stage_inv", ["x_c2r"])):
            best = None
            for stage in (1, 0):
                api.tuning_set(skey, h, stage)
                b = sweep(ctx, job, stream, reps, key, h, [64, 96, 128, 160, 192, 256], cls, log)
                if b and (best is None or b[1] < best[2]):
                    best = (stage, b[0], b[1])
            if best:
                api.tuning_set(skey, h, best[0])
                api.tuning_set(key, h, best[1])
                entries[(skey, h)] = best[0]
                entries[(key, h)] = best[1]
            rkey = key.replace("threads", "rpc")   # rows per CTA
            b = sweep(ctx, job, stream, reps, rkey, h, [2, 4, 6, 8, 12], cls, log)
            if b:
                entries[(rkey, h)] = b[0]
            pkey = key.replace("threads", "pf")
            b = sweep(ctx, job, stream, reps, pkey, h, [0, 2, 4], cls, log)
            if b:
                entries[(pkey, h)] = b[0]
    total = time_classes(ctx, job, stream, reps)
    log.append(f"# {name} tuned: " + ", ".join(f"{k} {v:.3f}" for k, v in sorted(total.items())) +
               f"; sum {sum(total.values()):.3f} ms")
    del keep
    job.close()
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "schedules.txt"))
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--workloads", default=",".join(WORKLOADS))
    args = ap.parse_args()
    import torch
    from crava_b200 import api
    # start from the built-in defaults: entries of an older file would bias the sweep
    empty = os.path.join(os.path.dirname(os.path.abspath(args.out)), ".schedules_empty")
    open(empty, "w").close()
    api.tuning_load(empty)
    os.remove(empty)
    entries, log = {}, []
    for name in args.workloads.split(","):
        tune_workload(name, WORKLOADS[name], args.reps, entries, log)
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    with open(args.out, "w") as f:
        f.write(f"# crava_b200 schedules: written by crava_b200/autotune.py on {props.name} "
                f"({props.multi_processor_count} SMs), {datetime.datetime.now(datetime.timezone.utc):%Y-%m-%d %H:%M} UTC\n")
        f.write("# key n value   (n: see crava_b200/autotune.py; -1 = every size)\n")
        for (k, n), v in sorted(entries.items()):
            f.write(f"{k} {n} {v}\n")
        f.write("# sweep log (device ms of the kernel class the key controls, per run)\n")
        for l in log:
            f.write(l + "\n")
    print(f"wrote {args.out}: {len(entries)} entries")


if __name__ == "__main__":
    main()
