#!/usr/bin/env python
"""Benchmark: SSP-RK3 steps of the Taylor-Green vortex at 512^3 in FP64 (ASTR miniapp setup:
Mach 0.1, Re 1600, Pr 0.72, gamma 1.4, Sutherland, 6th-order compact derivatives, 10th-order
compact filter alpha_f = 0.49 after every stage, dt fixed from CFL 0.5 at t = 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--size 512]
    python bench.py --workload ensemble [--gpus N] [--steps K]   # 48 uneven boxes, batched
    python bench.py --workload adjoint                          # 128^3 gradient, adjoint:forward

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
    if rank != 0:
        return
    n = args.ref_size
    value, secs, cores = cpu_reference(n, args.steps, max(args.warmup, 0))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (analytic Taylor-Green initial field)",
        "config": {"workload": f"TGV {args.size}^3 FP64 SSP-RK3 + compact filter (CPU sample {n}^3)",
                   "grid": args.size, "sample_grid": n},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"oracle restatement of the reference miniapp (no Fortran compiler on the box), "
                                   f"TGV {n}^3, one RK3 step per bench step, {cores} OpenMP threads"},
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
        del qh

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cn = args.ref_size
        v, secs, cores = cpu_reference(cn, args.cpu_steps, 0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"oracle restatement of the reference miniapp, TGV {cn}^3, {args.cpu_steps} RK3 steps, "
                         f"{cores} OpenMP threads, {secs:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic Taylor-Green initial field)",
            "config": {"workload": f"TGV {n}^3 FP64 SSP-RK3 + compact filter, dt from CFL 0.5",
                       "grid": n, "dt": dt, "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "l2": "inputs larger than L2 (5 x 1.1 GB state per box)", "graph": "one CUDA graph per step",
                       "launch_shapes": {k: list(v) for k, v in s.launch_shapes().items()}},
            "roofline": roof, "step_roofline": step_roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": (3 * (7 if split_fa else 6) + 1) * args.steps, "clocks": clk.summary(),
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
    boxes = ensemble_boxes(ctx, [specs[i] for i in mine])
    dts = [b.cfl_dt(0.5) for b in boxes]
    ens = ag.Ensemble(ctx, boxes)
    ens.step(dts, args.warmup)
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
        ens.step(dts, args.steps)
        e1.record(stream)
        e1.synchronize()
    barrier()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=f"cuda:{local}")
    if pg:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    ms_max = float(t.item())
    pts_all = sum(sp.n ** 3 for sp in specs)
    value = pts_all * args.steps / (ms_max * 1e-3)
    single = None
    if ws == 1 and not args.no_single:
        solo = ensemble_boxes(ctx, specs)
        sdts = [b.cfl_dt(0.5) for b in solo]
        for b, dt in zip(solo, sdts):
            b.rk3(dt, args.warmup)
        ctx.synchronize()
        e0.record(stream)
        for b, dt in zip(solo, sdts):
            b.rk3(dt, args.steps)
        e1.record(stream)
        e1.synchronize()
        ms_solo = e0.elapsed_time(e1)
        single = {"value": pts_all * args.steps / (ms_solo * 1e-3), "ms_per_step": ms_solo / args.steps,
                  "how": "each box alone, its own autotuned launch shapes and per-step CUDA graph, boxes in turn"}
        for b in solo:
            b.close()
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


def run_adjoint(args, ws, rank, local):
    """Discrete adjoint: 128^3 periodic random solenoidal field (M_t 0.3, Re for Re_lambda = 50),
    200 steps with filter, J = final kinetic energy, dJ/dq0 with a checkpoint every 20 steps.
    Times (device, CUDA events): the plain forward (200 graph-captured steps), the checkpointed
    forward, and the reverse sweep (segment recomputation + adjoint stages). Every rank runs its
    own replica (no collective on the data path)."""
    import torch
    import astr_gpu_b200 as ag
    from astr_gpu_b200.adjoint import Adjoint, fortran_empty
    from astr_gpu_b200.fields import solenoidal_q, solenoidal_velocity
    import numpy as np

    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        pg = dist
    n, nsteps, every, mach, seed = args.adj_size, args.adj_steps, 20, 0.3, 2024
    u = solenoidal_velocity(n, seed)
    k = np.fft.fftfreq(n, 1.0 / n)
    d2 = [np.mean(np.fft.ifftn(1j * [k[:, None, None], k[None, :, None], k[None, None, :]][a]
                                * np.fft.fftn(u[a])).real ** 2) for a in range(3)]
    up = np.sqrt(np.mean(u[0] ** 2 + u[1] ** 2 + u[2] ** 2) / 3.0)
    re = 50.0 / (up * up / np.sqrt(np.mean(d2)))
    stream = torch.cuda.Stream(device=local)
    ctx = ag.Context(local, stream=stream)
    s = ag.TGVSolver(ctx, n, params=ag.FlowParams(mach=mach, reynolds=re))
    q0 = solenoidal_q(n, mach, seed)
    s.set_q(q0)
    dt = s.cfl_dt(0.5)
    s.rk3(dt, args.warmup)
    ctx.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    g = fortran_empty(s.shape + (5,), f"cuda:{local}")
    with ClockSampler(local) as clk:
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
    t_plain, t_fwd, t_bwd = ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3]), ev[4].elapsed_time(ev[5])
    t = torch.tensor([t_plain, t_fwd, t_bwd], dtype=torch.float64, device=f"cuda:{local}")
    if pg:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    t_plain, t_fwd, t_bwd = (float(x) for x in t.tolist())
    if rank == 0:
        line = {
            "metric": ADJ_METRIC, "value": t_bwd / t_plain, "unit": "reverse sweep time / plain forward time",
            "n_gpus": ws, "steps": nsteps, "warmup": args.warmup, "ms_per_step": t_bwd / nsteps,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded solenoidal k^4 exp(-2(k/4)^2) field, uniform rho and p)",
            "config": {"workload": f"adjoint {n}^3, {nsteps} steps, checkpoint every {every}", "grid": n,
                       "mach_t": mach, "reynolds": re, "dt": dt, "J": J},
            "forward_ms_per_step": t_plain / nsteps, "checkpointed_forward_ms_per_step": t_fwd / nsteps,
            "reverse_ms_per_step": t_bwd / nsteps,
            "gradient_ratio_incl_forward": (t_fwd + t_bwd) / t_plain, "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    adj.close()
    s.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


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
    ap.add_argument("--ref-size", type=int, default=128)
    ap.add_argument("--cpu-steps", type=int, default=25)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="tgv", choices=["tgv", "ensemble", "adjoint"])
    ap.add_argument("--adj-size", type=int, default=128)
    ap.add_argument("--adj-steps", type=int, default=200)
    ap.add_argument("--no-single", action="store_true")
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
    else:
        run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
