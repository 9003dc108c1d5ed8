#!/usr/bin/env python
"""Benchmark: SSP-RK3 steps of the Taylor-Green vortex at 512^3 in FP64 (ASTR miniapp setup:
Mach 0.1, Re 1600, Pr 0.72, gamma 1.4, Sutherland, 6th-order compact derivatives, 10th-order
compact filter alpha_f = 0.49 after every stage, dt fixed from CFL 0.5 at t = 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--size 512]
    python bench.py --workload ensemble [--gpus N] [--steps K]   # 48 uneven boxes, batched
    python bench.py --workload adjoint                          # 128^3 gradient, adjoint:forward
    python bench.py --workload gradient                         # 256^3 line operators, GB/s
    python bench.py --workload full                             # full-solver time integration
    python bench.py --workload checkpoint                       # HDF5 flow-field write + restart read

One JSON line on rank 0. `value` = grid-point RK3 updates/s over all ranks (each rank advances
its own 512^3 box: replicas, weak scaling), device-timed with CUDA events on the library's stream,
max over ranks. `e2e` = the same metric through the host-buffer C-ABI call (astr_rk3_step_host:
upload q, one step, download q + diagnostics, every step). `--impl reference` times the CPU
restatement of the reference (the oracle) on all host threads on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK3 grid-point updates/s FP64 TGV 512³ + %HBM peak; adjoint:forward step time"
UNIT = "grid-point RK3 updates/s"
B_ALG_STEP = 2504.0      # algorithmic bytes per unique grid point per RK3 step (pass model)
B_ALG_STEP_FUSED = 2384.0   # the same with the owed filter along A fused into pass A
# fields read + written per stored point by one launch of each pass (B' reads q for the c2 term at
# two of the three stages; the filter along A owed by each stage is its own pass F_A where the
# autotuner found that faster, else pass A filters first and moves 14 fields)
PASS_NAMES = ["A", "B", "C", "A'", "B'", "F", "diag", "F_A"]   # astr_pass_timings order
PASS_FIELDS = {"A": 9, "B": 9, "C": 28, "A'": 15, "B'": 20 + 10 / 3, "F": 10, "F_A": 10}
PASS_PER_STEP = {"A": 3, "B": 3, "C": 3, "A'": 3, "B'": 3, "F": 3, "F_A": 3}
# kernels of one filtered RK3 step in the timed region: 7 passes per stage (6 with filter-A fused
# into pass A) and the diagnostics reduce


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_reference(n, steps, warmup):
    """The oracle (CPU restatement of the reference miniapp) on all host threads."""
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_num_threads(threads)
    o = oracle.TGVOracle(n)
    o.init_tgv()
    o.set_dt(o.cfl_dt(0.5))
    o.steps(warmup)
    t0 = time.perf_counter()
    o.steps(steps)
    dt = time.perf_counter() - t0
    return n ** 3 * steps / dt, dt, oracle.num_threads()


def run_reference(args, ws, rank):
    """The reference's CPU path (the oracle restatement of the miniapp; the Fortran cannot be built
    here) on all host threads, on the same workload as the GPU arm: TGV at --size (512^3), one
    untimed step (it also touches the ~50 GB of arrays), then a bounded number of timed steps
    (--ref-steps, 2 by default: about 30 s each on 16 threads), so the run ends within minutes."""
    if rank != 0:
        return
    n = args.ref_size or args.size
    steps = max(1, min(args.steps, args.ref_steps))
    value, secs, cores = cpu_reference(n, steps, 1)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "steps_requested": args.steps, "warmup": 1, "warmup_requested": args.warmup,
        "ms_per_step": 1e3 * secs / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (analytic Taylor-Green initial field)",
        "config": {"workload": f"TGV {args.size}^3 FP64 SSP-RK3 + compact filter, dt from CFL 0.5",
                   "grid": args.size, "sample_grid": n, "same_config": n == args.size},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"oracle restatement of the reference miniapp (no Fortran compiler on the box), "
                                   f"TGV {n}^3, {steps} timed RK3 steps after 1 untimed, {cores} OpenMP threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, ws, rank, local):
    import numpy as np
    import torch
    import astr_gpu_b200 as ag

    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        pg = dist
    stream = torch.cuda.Stream(device=local)
    ctx = ag.Context(local, stream=stream)
    n = args.size
    s = ag.TGVSolver(ctx, n)
    s.init_tgv()
    dt = s.cfl_dt(0.5)
    s.rk3(dt, args.warmup)
    ctx.synchronize()

    def barrier():
        torch.cuda.synchronize(local)
        if pg:
            pg.barrier()
        torch.cuda.synchronize(local)

    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        s.rk3(dt, args.steps)
        e1.record(stream)
        e1.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
    if pg:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    ms_max = float(t.item())
    ms_step = ms_max / args.steps
    value = ws * n ** 3 * args.steps / (ms_max * 1e-3)

    # live per-pass timing with CUDA events on the library stream (eager launches)
    per = np.zeros(8)
    ctx.check(ctx.L.astr_pass_timings(s._h, dt, 2, per.ctypes.data_as(ag._lib._dp)))
    pk, pk_kind = peaks()
    pts = (n + 1) ** 3
    shares = {nm: per[i] * PASS_PER_STEP[nm] for i, nm in enumerate(PASS_NAMES) if nm in PASS_PER_STEP}
    split_fa = per[PASS_NAMES.index("F_A")] > 0.0   # no F_A launches: filter-A fused into pass A
    fields = dict(PASS_FIELDS, A=PASS_FIELDS["A"] if split_fa else 14)
    dom = max(shares, key=shares.get)
    di = PASS_NAMES.index(dom)
    alg_bytes = fields[dom] * 8.0 * pts
    achieved = alg_bytes / (per[di] * 1e-3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(tf):
        tkey = "A_fused" if dom == "A" and not split_fa else dom
        traffic = json.load(open(tf)).get(str(n), {}).get(tkey)
    roof = {"kernel": f"pass {dom}", "bound": "hbm", "achieved": achieved, "peak": pk, "unit": "GB/s",
            "frac": achieved / pk, "traffic": traffic, "peak_kind": pk_kind,
            "alg_bytes_per_launch": alg_bytes, "ms_per_launch": float(per[di]),
            "per_pass_ms": {nm: float(per[i]) for i, nm in enumerate(PASS_NAMES) if nm != "diag"},
            "diag_reduce_ms": float(per[6])}
    step_bytes = (B_ALG_STEP if split_fa else B_ALG_STEP_FUSED) * n ** 3
    step_roof = {"bytes_per_step": step_bytes, "achieved": step_bytes / (ms_step * 1e-3) / 1e9, "peak": pk,
                 "unit": "GB/s", "frac": step_bytes / (ms_step * 1e-3) / 1e9 / pk, "peak_kind": pk_kind}

    # end to end through the host-buffer C-ABI call: upload, one step, download, every step
    e2e = None
    if not args.no_e2e:
        qh = torch.empty((5, n + 1, n + 1, n + 1), dtype=torch.float64, pin_memory=True)
        q = qh.numpy().transpose(3, 2, 1, 0)          # Fortran-ordered view of pinned memory
        q[...] = s.get_q()
        ne = args.e2e_steps
        s.rk3_host(q, dt, 1)
        barrier()
        t0 = time.perf_counter()
        for _ in range(ne):
            s.rk3_host(q, dt, 1)
        te = time.perf_counter() - t0
        tt = torch.tensor([te], dtype=torch.float64, device=f"cuda:{local}")
        if pg:
            pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        te = float(tt.item())
        qb = 5 * (n + 1) ** 3 * 8
        e2e = {"value": ws * n ** 3 * ne / te, "unit": UNIT, "h2d_bytes_per_step": qb,
               "d2h_bytes_per_step": qb + 24, "steps": ne, "call": "astr_rk3_step_host"}
        # the same call on an ordinary (pageable) host array, as a Python caller or a Fortran caller
        # that does not pin its arrays passes it: the copies go through the library's pinned staging
        qp = np.array(q, order="F", copy=True)
        del q, qh                                     # release the pinned buffer first
        s.rk3_host(qp, dt, 1)
        barrier()
        t0 = time.perf_counter()
        for _ in range(ne):
            s.rk3_host(qp, dt, 1)
        tp = time.perf_counter() - t0
        tt = torch.tensor([tp], dtype=torch.float64, device=f"cuda:{local}")
        if pg:
            pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        tp = float(tt.item())
        e2e["pageable"] = {"value": ws * n ** 3 * ne / tp, "unit": UNIT, "ms_per_step": 1e3 * tp / ne,
                           "memory": "pageable numpy array (not pinned)"}
        del qp

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cn = args.cpu_size
        v, secs, cores = cpu_reference(cn, args.cpu_steps, 0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"oracle restatement of the reference miniapp, TGV {cn}^3, {args.cpu_steps} RK3 steps, "
                         f"{cores} OpenMP threads, {secs:.1f} s"}

    # the metric's second part (adjoint:forward step time, config 4) and the batched ensemble
    # against its boxes one at a time (config 3), on one GPU, after the timed region
    shapes = {k: list(v) for k, v in s.launch_shapes().items()}
    adjoint = ensemble = checkpoint = None
    if ws == 1 and not args.no_extras:
        s.close()
        tl, acfg = measure_adjoint(ctx, stream, local, args.adj_size, args.adj_steps, 20, 3)
        adjoint = dict(adjoint_summary(tl, args.adj_steps), config=acfg, metric=ADJ_METRIC,
                       how="device time, CUDA events on the library stream; reverse = segment recomputation "
                           "+ adjoint stages")
        from astr_gpu_b200.fields import ensemble_specs
        specs = ensemble_specs(48, 48)
        es = args.ens_steps
        ms_b, ms_1, boxes, ens, _ = measure_ensemble(ctx, stream, specs, es, 3, True)
        pts_all = sum(sp.n ** 3 for sp in specs)
        ensemble = {"metric": ENS_METRIC, "steps": es, "batched": pts_all * es / (ms_b * 1e-3),
                    "one_at_a_time": pts_all * es / (ms_1 * 1e-3), "ratio": ms_1 / ms_b,
                    "batched_ms_per_step": ms_b / es, "one_at_a_time_ms_per_step": ms_1 / es, "unit": UNIT,
                    "boxes": len(specs), "points": pts_all}
        ens.close()
        for b in boxes:
            b.close()
        # the restart path: the HDF5 flow field of a 256^3 state written and read back
        import tempfile
        tmp = tempfile.mkdtemp(prefix="astr_ckpt_")
        tw, tr, fbytes, ok = measure_checkpoint(ctx, 256, 2, 1, tmp, rank)
        os.rmdir(tmp)
        checkpoint = {"metric": "flow-field checkpoint write + restart read, file GB/s", "grid": 256,
                      "file_gb": fbytes / 1e9, "write_gbs": 2 * fbytes / tw / 1e9, "read_gbs": 2 * fbytes / tr / 1e9,
                      "round_trip_gbs": 4 * fbytes / (tw + tr) / 1e9, "steps": 2, "density_equal": ok,
                      "how": "wall time; previous file moved aside first (bakupfile); host page cache"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic Taylor-Green initial field)",
            "config": {"workload": f"TGV {n}^3 FP64 SSP-RK3 + compact filter, dt from CFL 0.5",
                       "grid": n, "dt": dt, "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "l2": "inputs larger than L2 (5 x 1.1 GB state per box)", "graph": "one CUDA graph per step",
                       "launch_shapes": shapes},
            "roofline": roof, "step_roofline": step_roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": (3 * (7 if split_fa else 6) + 1) * args.steps, "clocks": clk.summary(),
            "adjoint": adjoint, "ensemble": ensemble, "checkpoint": checkpoint,
        }
        print(json.dumps(line), flush=True)
    s.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


ENS_METRIC = "ensemble grid-point RK3 updates/s FP64 (48 uneven periodic boxes)"


def ensemble_boxes(ctx, specs):
    import astr_gpu_b200 as ag
    from astr_gpu_b200.fields import solenoidal_q
    boxes = []
    for sp in specs:
        b = ag.TGVSolver(ctx, sp.n, params=ag.FlowParams(mach=sp.mach, reynolds=sp.reynolds))
        if sp.kind == "tgv":
            b.init_tgv()
        else:
            b.set_q(solenoidal_q(sp.n, sp.mach, sp.seed))
        boxes.append(b)
    return boxes


def measure_ensemble(ctx, stream, specs, steps, warmup, single, barrier=None):
    """Device time (CUDA events on the library's stream) of `steps` batched ensemble steps of the
    boxes `specs`, and, with `single`, of the same boxes stepped one at a time (each its own
    autotuned shapes and per-step graph). Returns (ms batched, ms one at a time or None, boxes,
    ensemble, time steps); the caller closes the boxes and the ensemble."""
    import torch
    import astr_gpu_b200 as ag
    boxes = ensemble_boxes(ctx, specs)
    dts = [b.cfl_dt(0.5) for b in boxes]
    ens = ag.Ensemble(ctx, boxes)
    ens.step(dts, warmup)
    ctx.synchronize()
    if barrier:
        barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.step(dts, steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    ms_solo = None
    if single:
        solo = ensemble_boxes(ctx, specs)
        sdts = [b.cfl_dt(0.5) for b in solo]
        for b, dt in zip(solo, sdts):
            b.rk3(dt, warmup)
        ctx.synchronize()
        e0.record(stream)
        for b, dt in zip(solo, sdts):
            b.rk3(dt, steps)
        e1.record(stream)
        e1.synchronize()
        ms_solo = e0.elapsed_time(e1)
        for b in solo:
            b.close()
    return ms, ms_solo, boxes, ens, dts


def run_ensemble(args, ws, rank, local):
    """Batched ensemble: every rank advances its LPT share of the 48 boxes (no collective on the
    data path); value = all boxes' grid points x steps / the slowest rank's device time. On one
    GPU the same boxes are also timed one at a time (each box its own per-step graph)."""
    import torch
    import astr_gpu_b200 as ag
    from astr_gpu_b200.fields import ensemble_specs
    from astr_gpu_b200.shard import box_cost, lpt_partition

    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        pg = dist
    specs = ensemble_specs(48, 48)
    mine = lpt_partition([box_cost(sp.n) for sp in specs], ws)[rank]
    stream = torch.cuda.Stream(device=local)
    ctx = ag.Context(local, stream=stream)

    def barrier():
        torch.cuda.synchronize(local)
        if pg:
            pg.barrier()
        torch.cuda.synchronize(local)

    with ClockSampler(local) as clk:
        ms, ms_solo, boxes, ens, dts = measure_ensemble(ctx, stream, [specs[i] for i in mine], args.steps,
                                                        args.warmup, ws == 1 and not args.no_single, barrier)
    barrier()
    t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
    if pg:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    ms_max = float(t.item())
    pts_all = sum(sp.n ** 3 for sp in specs)
    value = pts_all * args.steps / (ms_max * 1e-3)
    single = None
    if ms_solo is not None:
        single = {"value": pts_all * args.steps / (ms_solo * 1e-3), "ms_per_step": ms_solo / args.steps,
                  "how": "each box alone, its own autotuned launch shapes and per-step CUDA graph, boxes in turn"}
    e2e = None
    if not args.no_e2e:
        # end to end: upload every box's state from pinned host memory, step, download, per step
        import numpy as np
        host = []
        for b in boxes:
            qh = torch.empty((5,) + b.shape[::-1], dtype=torch.float64, pin_memory=True)
            q = qh.numpy().transpose(3, 2, 1, 0)
            q[...] = b.get_q()
            host.append((qh, q))
        ne = args.e2e_steps
        barrier()
        t0 = time.perf_counter()
        for _ in range(ne):
            for b, (_, q) in zip(boxes, host):
                b.set_q(q)
            ens.step(dts, 1)
            for b, (_, q) in zip(boxes, host):
                q[...] = b.get_q()
        te = time.perf_counter() - t0
        tt = torch.tensor([te], dtype=torch.float64, device=f"cuda:{local}")
        if pg:
            pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        qb = sum(5 * 8 * int(np.prod(b.shape)) for b in boxes)
        e2e = {"value": pts_all * ne / float(tt.item()), "unit": UNIT, "h2d_bytes_per_step": qb,
               "d2h_bytes_per_step": qb, "steps": ne, "call": "astr_state_upload + astr_ensemble_step + astr_state_download"}
    if rank == 0:
        from collections import Counter
        line = {
            "metric": ENS_METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (24 Taylor-Green, 24 seeded solenoidal k^4 exp(-2(k/4)^2) boxes)",
            "config": {"workload": "48 periodic boxes, sizes seeded from {32,48,64,96,128}^3, Mach U[0.1,0.5], "
                                   "Re U[400,3200], dt per box from CFL 0.5",
                       "sizes": dict(Counter(sp.n for sp in specs)), "points": pts_all,
                       "parallelism": f"LPT box shards x{ws}" if ws > 1 else "single GPU",
                       "graph": "one CUDA graph per ensemble step", "l2": "total state 6 GB > L2"},
            "one_at_a_time": single, "e2e": e2e, "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    ens.close()
    for b in boxes:
        b.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


ADJ_METRIC = "adjoint:forward time ratio, 128^3 decaying turbulence, 200 RK3 steps, checkpoint every 20"


def adjoint_setup(n, seed=2024, mach=0.3):
    """Config-4 initial state: a seeded solenoidal field with E(k) ~ k^4 exp(-2 (k/4)^2) at
    turbulent Mach `mach`, and the Reynolds number that makes Re_lambda = 50 for its spectrum."""
    import numpy as np
    from astr_gpu_b200.fields import solenoidal_q, solenoidal_velocity
    u = solenoidal_velocity(n, seed)
    k = np.fft.fftfreq(n, 1.0 / n)
    d2 = [np.mean(np.fft.ifftn(1j * [k[:, None, None], k[None, :, None], k[None, None, :]][a]
                                * np.fft.fftn(u[a])).real ** 2) for a in range(3)]
    up = np.sqrt(np.mean(u[0] ** 2 + u[1] ** 2 + u[2] ** 2) / 3.0)
    re = 50.0 / (up * up / np.sqrt(np.mean(d2)))
    return solenoidal_q(n, mach, seed), re


def measure_adjoint(ctx, stream, local, n, nsteps, every, warmup, mach=0.3):
    """Device times (CUDA events on the library's stream) of the plain forward (nsteps
    graph-captured steps), the checkpointed forward and the reverse sweep (segment recomputation
    + adjoint stages) of J = final kinetic energy, dJ/dq0 with a checkpoint every `every` steps."""
    import torch
    import astr_gpu_b200 as ag
    from astr_gpu_b200.adjoint import Adjoint, fortran_empty
    q0, re = adjoint_setup(n, mach=mach)
    s = ag.TGVSolver(ctx, n, params=ag.FlowParams(mach=mach, reynolds=re))
    s.set_q(q0)
    dt = s.cfl_dt(0.5)
    s.rk3(dt, warmup)
    ctx.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    g = fortran_empty(s.shape + (5,), f"cuda:{local}")
    s.set_q(q0)
    ev[0].record(stream)
    s.rk3(dt, nsteps)
    ev[1].record(stream)
    s.set_q(q0)
    adj = Adjoint(s, every)
    ev[2].record(stream)
    J = adj.forward(dt, nsteps)
    ev[3].record(stream)
    ev[4].record(stream)
    adj.backward(g)
    ev[5].record(stream)
    ev[5].synchronize()
    t = [ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3]), ev[4].elapsed_time(ev[5])]
    adj.close()
    s.close()
    del g
    return t, {"grid": n, "steps": nsteps, "checkpoint_every": every, "mach_t": mach, "reynolds": re, "dt": dt,
               "J": J}


def adjoint_summary(t, nsteps):
    t_plain, t_fwd, t_bwd = t
    return {"forward_ms_per_step": t_plain / nsteps, "checkpointed_forward_ms_per_step": t_fwd / nsteps,
            "reverse_ms_per_step": t_bwd / nsteps, "ratio": t_bwd / t_plain,
            "ratio_incl_forward": (t_fwd + t_bwd) / t_plain}


def run_adjoint(args, ws, rank, local):
    """Discrete adjoint: 128^3 periodic random solenoidal field (M_t 0.3, Re for Re_lambda = 50),
    200 steps with filter, J = final kinetic energy, dJ/dq0 with a checkpoint every 20 steps.
    Times (device, CUDA events): the plain forward (200 graph-captured steps), the checkpointed
    forward, and the reverse sweep (segment recomputation + adjoint stages). Every rank runs its
    own replica (no collective on the data path)."""
    import torch
    import astr_gpu_b200 as ag

    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        pg = dist
    n, nsteps, every = args.adj_size, args.adj_steps, 20
    stream = torch.cuda.Stream(device=local)
    ctx = ag.Context(local, stream=stream)
    with ClockSampler(local) as clk:
        tl, cfg = measure_adjoint(ctx, stream, local, n, nsteps, every, args.warmup)
    t = torch.tensor(tl, dtype=torch.float64, device=f"cuda:{local}")
    if pg:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    t_plain, t_fwd, t_bwd = (float(x) for x in t.tolist())
    if rank == 0:
        summ = adjoint_summary((t_plain, t_fwd, t_bwd), nsteps)
        line = {
            "metric": ADJ_METRIC, "value": t_bwd / t_plain, "unit": "reverse sweep time / plain forward time",
            "n_gpus": ws, "steps": nsteps, "warmup": args.warmup, "ms_per_step": t_bwd / nsteps,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded solenoidal k^4 exp(-2(k/4)^2) field, uniform rho and p)",
            "config": dict(cfg, workload=f"adjoint {n}^3, {nsteps} steps, checkpoint every {every}"),
            "forward_ms_per_step": summ["forward_ms_per_step"],
            "checkpointed_forward_ms_per_step": summ["checkpointed_forward_ms_per_step"],
            "reverse_ms_per_step": summ["reverse_ms_per_step"],
            "gradient_ratio_incl_forward": summ["ratio_incl_forward"], "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


GRAD_METRIC = "gradient kernel GB/s FP64 256^3 (d/dx, d/dy, d/dz + 3-direction compact filter)"


def run_gradient(args, ws, rank, local):
    """The gradient-kernel workload of the reference's gradient_solver_3d / gradtest setting: a
    256^3 seeded spectral field (x, z periodic, y non-periodic on [0, 2]); one step = the compact
    first derivatives along x, y and z (scaled by 1/dx) and the compact filter along x, then y,
    then z, each a call of the line-level C ABI (astr_deriv_lines / astr_filter_lines) on device
    arrays. Algorithmic bytes: 16 per stored point per call (read f, write the result), 96 per
    step. Every rank runs its own replica (no collective)."""
    import ctypes
    import numpy as np
    import torch
    import astr_gpu_b200 as ag
    from astr_gpu_b200.fields import gradient_input, spectral_field

    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        pg = dist
    n = args.grad_size
    stream = torch.cuda.Stream(device=local)
    ctx = ag.Context(local, stream=stream)
    L = ctx.L
    f = spectral_field(n)
    g, lb = gradient_input(f, periodic=(True, False, True))

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).to(f"cuda:{local}").permute(2, 1, 0)

    G = dev(g)
    ntypes = (3, 4, 3)
    spacing = (2 * np.pi / n, 2.0 / n, 2 * np.pi / n)
    ders = [ag.fd_scheme_initiate(ctx, "643c", ntypes[d], n) for d in range(3)]
    flts = [ag.compact_filter_initiate(ctx, ntypes[d], n, 0.49, 1.11, 0.98) for d in range(3)]
    gshape, glb = list(g.shape), list(lb)
    dshape = [[n + 1 if a == d else gshape[a] for a in range(3)] for d in range(3)]
    dlb = [[0 if a == d else glb[a] for a in range(3)] for d in range(3)]
    dout = [torch.empty(tuple(dshape[d][::-1]), dtype=torch.float64, device=f"cuda:{local}").permute(2, 1, 0)
            for d in range(3)]
    # filter chain x -> y -> z: the x result keeps the z halo lines (filtered like their images),
    # so it feeds y and then z directly
    f1 = torch.empty((gshape[2], n + 1, n + 1), dtype=torch.float64, device=f"cuda:{local}").permute(2, 1, 0)
    f2 = torch.empty((gshape[2], n + 1, n + 1), dtype=torch.float64, device=f"cuda:{local}").permute(2, 1, 0)
    f3 = torch.empty((n + 1, n + 1, n + 1), dtype=torch.float64, device=f"cuda:{local}").permute(2, 1, 0)
    i64 = lambda v: (ctypes.c_int64 * 3)(*[int(x) for x in v])
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    f1s, f1l = [n + 1, n + 1, gshape[2]], [0, 0, glb[2]]
    f3s, f3l = [n + 1, n + 1, n + 1], [0, 0, 0]

    def step(where=ag._lib.ASTR_DEVICE, bufs=None):
        src, d_out, o1, o2, o3 = bufs or (G, dout, f1, f2, f3)
        ptr = (lambda t: ctypes.c_void_p(t.ctypes.data)) if where == ag._lib.ASTR_HOST else vp
        for d in range(3):
            ctx.check(L.astr_deriv_lines(ctx._h, ders[d]._h, d, ptr(src), i64(gshape), i64(glb), ptr(d_out[d]),
                                         i64(dshape[d]), i64(dlb[d]), 1, 1.0 / spacing[d], where))
        ctx.check(L.astr_filter_lines(ctx._h, flts[0]._h, 0, ptr(src), i64(gshape), i64(glb), ptr(o1), i64(f1s),
                                      i64(f1l), 1, where))
        ctx.check(L.astr_filter_lines(ctx._h, flts[1]._h, 1, ptr(o1), i64(f1s), i64(f1l), ptr(o2), i64(f1s),
                                      i64(f1l), 1, where))
        ctx.check(L.astr_filter_lines(ctx._h, flts[2]._h, 2, ptr(o2), i64(f1s), i64(f1l), ptr(o3), i64(f3s),
                                      i64(f3l), 1, where))

    for _ in range(args.warmup):
        step()
    ctx.synchronize()

    def barrier():
        torch.cuda.synchronize(local)
        if pg:
            pg.barrier()
        torch.cuda.synchronize(local)

    # inputs and outputs are 147 MB + 6 x 136-147 MB: larger than L2 between calls
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(7)]
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        e1.synchronize()
    # one more step with events between the calls: per-call times on the library's stream
    ev[0].record(stream)
    for d in range(3):
        ctx.check(L.astr_deriv_lines(ctx._h, ders[d]._h, d, vp(G), i64(gshape), i64(glb), vp(dout[d]),
                                     i64(dshape[d]), i64(dlb[d]), 1, 1.0 / spacing[d], ag._lib.ASTR_DEVICE))
        ev[d + 1].record(stream)
    step_f = [(flts[0], 0, G, gshape, glb, f1, f1s, f1l), (flts[1], 1, f1, f1s, f1l, f2, f1s, f1l),
              (flts[2], 2, f2, f1s, f1l, f3, f3s, f3l)]
    for k, (sch, d, a, ash, alb, o, osh, olb) in enumerate(step_f):
        ctx.check(L.astr_filter_lines(ctx._h, sch._h, d, vp(a), i64(ash), i64(alb), vp(o), i64(osh), i64(olb), 1,
                                      ag._lib.ASTR_DEVICE))
        ev[k + 4].record(stream)
    ev[6].synchronize()
    per_call = [ev[i].elapsed_time(ev[i + 1]) for i in range(6)]
    barrier()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
    if pg:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    ms_max = float(t.item())
    pts = (n + 1) ** 3
    step_bytes = 6 * 16.0 * pts
    value = ws * step_bytes * args.steps / (ms_max * 1e-3) / 1e9
    pk, pk_kind = peaks()
    names = ["d/dx", "d/dy", "d/dz", "filter x", "filter y", "filter z"]
    dom = int(np.argmax(per_call))
    achieved = 16.0 * pts / (per_call[dom] * 1e-3) / 1e9
    roof = {"kernel": f"k_line_api ({names[dom]})", "bound": "hbm", "achieved": achieved, "peak": pk,
            "unit": "GB/s", "frac": achieved / pk, "traffic": None, "peak_kind": pk_kind,
            "alg_bytes_per_launch": 16.0 * pts, "ms_per_launch": per_call[dom],
            "per_call_ms": dict(zip(names, per_call))}
    e2e = None
    if not args.no_e2e:
        # the same calls with host arrays: every call copies its input in and its output back
        hbufs = (g, [np.zeros(dshape[d], order="F") for d in range(3)], np.zeros(f1s, order="F"),
                 np.zeros(f1s, order="F"), np.zeros(f3s, order="F"))
        step(ag._lib.ASTR_HOST, hbufs)
        barrier()
        ne = args.e2e_steps
        t0 = time.perf_counter()
        for _ in range(ne):
            step(ag._lib.ASTR_HOST, hbufs)
        te = time.perf_counter() - t0
        tt = torch.tensor([te], dtype=torch.float64, device=f"cuda:{local}")
        if pg:
            pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        te = float(tt.item())
        h2d = 8 * (3 * g.size + g.size + 2 * int(np.prod(f1s)))
        d2h = 8 * (sum(int(np.prod(s_)) for s_ in dshape) + 2 * int(np.prod(f1s)) + int(np.prod(f3s)))
        e2e = {"value": ws * step_bytes * ne / te / 1e9, "unit": "GB/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": ne, "call": "astr_deriv_lines / astr_filter_lines, host arrays"}
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        import oracle
        oracle.set_num_threads(os.cpu_count() or 1)
        ops = [oracle.fd_scheme_initiate("643c", ntypes[d], n) for d in range(3)]
        t0 = time.perf_counter()
        for d in range(3):
            ops[d].apply3d(g, d, lbound=lb)
        cur = g
        for d in range(3):
            cur = oracle.compact_filter_initiate(ntypes[d], n, 0.49, 1.11, 0.98).apply3d(
                cur, d, lbound=lb if d == 0 else (0, 0, lb[2]))
        secs = time.perf_counter() - t0
        cpu = {"value": step_bytes / secs / 1e9, "unit": "GB/s", "cores": oracle.num_threads(), "kind": "port",
               "sample": f"oracle restatement, the same six calls at {n}^3 once, {oracle.num_threads()} OpenMP threads, "
                         f"{secs:.1f} s"}
    if rank == 0:
        line = {
            "metric": GRAD_METRIC, "value": value, "unit": "GB/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded spectral field, |k| <= 16, |k|^(-5/3), seed 20251203)",
            "config": {"workload": f"gradient kernel {n}^3: x, z periodic (ntype 3), y non-periodic (ntype 4) on "
                                   f"[0, 2]; d/dx, d/dy, d/dz and the filter along x, y, z",
                       "grid": n, "bytes_per_point_per_step": 96, "points": pts,
                       "l2": "input and outputs 136-147 MB each, larger than L2"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": 6 * args.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


FULL_METRIC = "full-solver grid-point RK3 updates/s FP64 (time_integration_rk, periodic TGV)"


def run_full(args, ws, rank, local):
    """The full solver's time integration (astr_full_*, on the reference's halo-extended arrays,
    one kernel per operation of the reference) on the Taylor-Green box of --full-size: device time
    of --steps steps after --warmup. Every rank runs its own replica (no collective)."""
    import torch
    import astr_gpu_b200 as ag
    from astr_gpu_b200.fields import tgv_q

    torch.cuda.set_device(local)
    n = args.full_size
    stream = torch.cuda.Stream(device=local)
    ctx = ag.Context(local, stream=stream)
    ntype = tuple(int(t) for t in args.full_ntype.split(","))
    s = ag.FullSolver(ctx, n, params=ag.FlowParams(sutherland=110.3, beta_bound=0.98, conschm=args.conschm,
                                                   bfacmpld=args.bfac, lchardecomp=args.chardecomp,
                                                   shkcrt=args.shkcrt, ntype=ntype, twall=1.0))
    s.set_q(tgv_q(n, 0.1))
    dt = 1e-3
    s.step(dt, args.warmup)
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        s.step(dt, args.steps)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    if rank == 0:
        line = {"metric": FULL_METRIC, "value": ws * n ** 3 * args.steps / (ms * 1e-3), "unit": UNIT, "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (Taylor-Green initial field)",
                "config": {"workload": f"full-solver mode, TGV {n}^3 (filter first, qswap averaging, metric form), "
                                       f"dt {dt}, " + ("central compact convection (643)" if args.conschm != 543 else
                                                       f"upwind compact flux convection (543, b {args.bfac}"
                                                       + (f", characteristic, shkcrt {args.shkcrt})" if args.chardecomp
                                                          else ")"))
                                       + ("" if ntype == (3, 3, 3) else f", ntype {ntype} with isothermal no-slip walls"),
                           "grid": n},
                "gpu_launches": None, "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    s.close()


def measure_checkpoint(ctx, n, steps, warmup, tmp, rank):
    """Write + restart-read wall times of the flow field of a TGV n^3 state in the directory tmp:
    (total write s, total read s, file bytes, density equal after the round trip). Each step moves
    the previous file aside first, as writeflfed does (bakupfile, src/readwrite.F90:1696-1708), so
    every checkpoint is a new file; the moved copies are deleted outside the timed region."""
    import numpy as np
    import astr_gpu_b200 as ag

    a, b = ag.TGVSolver(ctx, n), ag.TGVSolver(ctx, n)
    a.init_tgv()
    fn = os.path.join(tmp, f"flowfield_r{rank}.h5")
    bak = os.path.join(tmp, "bakup")
    os.makedirs(bak, exist_ok=True)

    def bakupfile():
        if os.path.exists(fn):
            os.rename(fn, os.path.join(bak, os.path.basename(fn)))

    def drop_backups():
        for f in os.listdir(bak):
            os.remove(os.path.join(bak, f))

    for _ in range(max(warmup, 1)):
        bakupfile()
        a.write_flowfield(fn)
        b.read_flowfield(fn)
        drop_backups()
    tw = tr = 0.0
    for _ in range(steps):
        t0 = time.perf_counter()
        bakupfile()
        a.write_flowfield(fn)
        t1 = time.perf_counter()
        b.read_flowfield(fn)
        t2 = time.perf_counter()
        tw += t1 - t0
        tr += t2 - t1
        drop_backups()
    fbytes = os.path.getsize(fn)
    ok = bool(np.array_equal(b.get_q()[..., 0], a.get_q()[..., 0]))
    os.remove(fn)
    os.rmdir(bak)
    a.close()
    b.close()
    return tw, tr, fbytes, ok


def run_checkpoint(args, ws, rank, local):
    """The checkpoint path of the reference's restart (writeflfed's flow field, readcheckpoint +
    updateq): a TGV state of --ckpt-size written to an HDF5 file on the host's disk and read back
    into a second state, through astr_state_write_flowfield / astr_state_read_flowfield (q2fvar and
    fvar2q on the GPU, chunked transfers through pinned slots and host I/O threads, the library's
    HDF5 writer and reader).
    One step = one write and one read of the same file; wall time (the host's file I/O is the
    work), the file in the page cache as right after a checkpoint. CPU baseline: the oracle's
    numpy conversions with its Python HDF5 writer and reader, one write and one read."""
    import tempfile

    import numpy as np
    import torch
    import astr_gpu_b200 as ag

    torch.cuda.set_device(local)
    n = args.ckpt_size
    ctx = ag.Context(local)
    tmp = tempfile.mkdtemp(prefix="astr_ckpt_")
    fn = os.path.join(tmp, f"flowfield_r{rank}.h5")
    with ClockSampler(local) as clk:
        tw, tr, fbytes, ok = measure_checkpoint(ctx, n, args.steps, args.warmup, tmp, rank)
    # the host's own file speed for the same bytes, without the library: a new file written by one
    # thread in 32 MB pwrite calls, then read back by 8 threads in 32 MB pread calls (page cache)
    import threading
    raw = np.ones(fbytes // 8)
    mv = memoryview(raw).cast("B")
    chunk = 32 << 20
    offs = list(range(0, raw.nbytes, chunk))
    fd = os.open(fn, os.O_RDWR | os.O_CREAT | os.O_TRUNC, 0o644)
    t0 = time.perf_counter()
    for o in offs:
        os.pwrite(fd, mv[o:o + chunk], o)
    t1 = time.perf_counter()

    def reader(k):
        for i in range(k, len(offs), 8):
            os.preadv(fd, [mv[offs[i]:offs[i] + chunk]], offs[i])

    ths = [threading.Thread(target=reader, args=(k,)) for k in range(8)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    t2 = time.perf_counter()
    os.close(fd)
    os.remove(fn)
    io_ref = {"write_gbs": raw.nbytes / (t1 - t0) / 1e9, "read_gbs": raw.nbytes / (t2 - t1) / 1e9,
              "what": "the same bytes, no library: a new file by one thread in 32 MB pwrite calls, read back by "
                      "8 threads in 32 MB preads (page cache)"}
    cpu = None
    if rank == 0 and not args.no_cpu:
        import oracle
        from oracle import h5format
        from astr_gpu_b200.fields import tgv_q
        q = tgv_q(n, 0.1)
        t0 = time.perf_counter()
        f = oracle.q2fvar(q, 0.1, 1.4)
        h5format.write(fn, [(nm, np.ascontiguousarray(f[..., m].T)) for m, nm in enumerate(("ro", "u1", "u2", "u3",
                                                                                          "p", "t"))]
                       + [("nstep", np.array([0], np.int32)), ("time", np.array([0.0]))])
        info = h5format.read(fn)
        g = np.stack([info.entries[nm].data.T for nm in ("ro", "u1", "u2", "u3", "p", "t")], axis=-1)
        oracle.fvar2q_temperature(g, 0.1, 1.4)
        tc = time.perf_counter() - t0
        os.remove(fn)
        cpu = {"value": 2 * fbytes / tc / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
               "sample": f"one write + one read of the {n}^3 flow field by the oracle (numpy, Python HDF5)"}
    os.rmdir(tmp)
    if rank == 0:
        total = tw + tr
        line = {"metric": "flow-field checkpoint write + restart read, file GB/s", "value": ws * 2 * fbytes
                * args.steps / total / 1e9, "unit": "GB/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (Taylor-Green initial field)",
                "config": {"workload": f"HDF5 flow field of a TGV {n}^3 state (ro, u1, u2, u3, p, t, nstep, time; "
                                       f"{fbytes / 1e9:.3f} GB): the previous file moved aside (bakupfile), "
                                       "astr_state_write_flowfield, then astr_state_read_flowfield; wall time, "
                                       "host page cache", "grid": n},
                "write_gbs": fbytes * args.steps / tw / 1e9, "read_gbs": fbytes * args.steps / tr / 1e9,
                "round_trip_density_equal": ok, "host_file_io": io_ref, "cpu_baseline": cpu,
                # per step: the state's pack kernel and q2fvar (write), fvar2q and the pack kernel (read)
                "gpu_launches": 4 * args.steps,
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)


def run_profile(args, local):
    """The workload for an ncu capture: `--steps` eager RK3 steps of a TGV box (no graph, no
    timing, no JSON line), with the pass launch shapes pinned by `--shapes`."""
    import astr_gpu_b200 as ag
    ctx = ag.Context(local)
    s = ag.TGVSolver(ctx, args.size)
    if args.shapes:
        for nm, v in json.loads(args.shapes).items():
            s.set_launch_shape(nm, v[0], v[1], v[2], v[4] if len(v) > 4 else 1, v[5] if len(v) > 5 else (1 if len(v) > 4 and v[4] > 1 else 5))
    s.init_tgv()
    dt = s.cfl_dt(0.5)
    s.use_graph(False)
    s.rk3(dt, args.steps)
    ctx.synchronize()
    print(json.dumps({"profiled_steps": args.steps, "grid": args.size, "launch_shapes": s.launch_shapes()}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--ref-size", type=int, default=0, help="grid of the reference arm (default: --size)")
    ap.add_argument("--ref-steps", type=int, default=2, help="timed steps of the reference arm (at most --steps)")
    ap.add_argument("--cpu-size", type=int, default=128, help="grid of the cpu_baseline sample of the GPU arm")
    ap.add_argument("--cpu-steps", type=int, default=25)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="tgv", choices=["tgv", "ensemble", "adjoint", "gradient", "full",
                                                          "checkpoint"])
    ap.add_argument("--ckpt-size", type=int, default=256, help="grid of --workload checkpoint")
    ap.add_argument("--full-size", type=int, default=256)
    ap.add_argument("--conschm", type=int, default=643, choices=[643, 543], help="convection of --workload full")
    ap.add_argument("--bfac", type=float, default=0.3, help="b factor of the upwind compact flux (--conschm 543)")
    ap.add_argument("--chardecomp", action="store_true", help="--conschm 543 in characteristic variables")
    ap.add_argument("--full-ntype", default="3,3,3",
                    help="boundary type per direction of --workload full (3 periodic, 4 no-slip walls at both ends)")
    ap.add_argument("--shkcrt", type=float, default=0.01, help="Ducros sensor threshold (--chardecomp)")
    ap.add_argument("--grad-size", type=int, default=256)
    ap.add_argument("--adj-size", type=int, default=128)
    ap.add_argument("--adj-steps", type=int, default=200)
    ap.add_argument("--no-single", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the adjoint, ensemble and checkpoint keys of the default line")
    ap.add_argument("--ens-steps", type=int, default=10)
    ap.add_argument("--profile", action="store_true", help="eager steps only, for ncu captures")
    ap.add_argument("--shapes", default="", help='pinned launch shapes, e.g. {"A": [9, 2, 8], ...}')
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    ws, rank, local = dist_setup(args)
    if args.profile:
        run_profile(args, local)
    elif args.impl == "reference":
        run_reference(args, ws, rank)
    elif args.workload == "ensemble":
        run_ensemble(args, ws, rank, local)
    elif args.workload == "adjoint":
        run_adjoint(args, ws, rank, local)
    elif args.workload == "gradient":
        run_gradient(args, ws, rank, local)
    elif args.workload == "full":
        run_full(args, ws, rank, local)
    elif args.workload == "checkpoint":
        run_checkpoint(args, ws, rank, local)
    else:
        run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
