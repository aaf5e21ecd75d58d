#!/usr/bin/env python
"""Benchmark: Orszag-Tang cell-updates/s, FP32-bulk vs FP64, and HBM % of peak.

Workload (one step = one split time step of the whole grid): the Orszag-Tang
vortex on periodic [0,1]^2 at 4096^2 cells, HLLD, van Leer, CFL 0.4, GLM
c_h = max wave speed, c_r = 0.18 -- deterministic synthetic initial data,
generated by the library (no dataset).  The state (604 MB in FP32, 1.2 GB in
FP64) is larger than the 126 MB L2, so no flush is needed between steps.

Our arm:  `value` = FP32-bulk cell-updates/s of the device-resident, CUDA-graph
step loop (mhd_run) with the state already in HBM, timed with CUDA events on
the launching stream, max over ranks.  `e2e` = the same metric through the C
ABI with pinned FP64 host buffers: every step uploads the state, advances one
step and downloads the state.  The FP64 step is timed the same way and
reported beside it with the FP32/FP64 speed ratio and the density relative L1
between the two after the same steps.

`--impl reference`: the reference's own CPU/OpenMP step (oracle/_ref, built
from the reference sources) on the host cores, rank 0 only.

Multi-GPU (torchrun): one independent instance per rank (weak scaling, no
data-path collective); a barrier brackets the timed region and the time is the
max over ranks.
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

METRIC = "Orszag–Tang cell-updates/s FP32-bulk vs FP64 at L1≤1e-5; HBM % of peak"
UNIT = "cell-updates/s"
BYTES_PER_CELL_SWEEP = {4: 2 * 9 * 4, 8: 2 * 9 * 8}  # read + write 9 fields per sweep


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=4096, help="grid side")
    ap.add_argument("--e2e-steps", type=int, default=16)
    ap.add_argument("--e2e-lanes", type=int, default=3,
                    help="workspaces (each on its own stream) that take e2e steps in turn")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--workload", default="ot", choices=["ot", "batch", "adjoint", "precision", "slabs"],
                    help="ot: Orszag-Tang n^2 (default line); batch: 256 uneven Orszag-Tang instances; "
                         "adjoint: gradient of the Orszag-Tang objective; precision: FP32-bulk vs FP64 "
                         "relative L1 / Linf per field of every configuration, run to t_end; slabs: one "
                         "Orszag-Tang n^2 grid split into y-slabs (--parts on one GPU, or one slab per rank)")
    ap.add_argument("--parts", type=int, default=4, help="slabs workload on one GPU: number of y-slabs")
    ap.add_argument("--precision-max-n", type=int, default=2048,
                    help="largest Orszag-Tang side of the precision workload (512, 2048, 4096)")
    ap.add_argument("--precision-cases", default="",
                    help="comma-separated substrings: run only the precision cases whose names contain one")
    ap.add_argument("--seed", type=int, default=0, help="batch workload seed")
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--xrpw", type=int, default=0,
                    help="x-sweep work per warp: row segments of 128 * xrpw - 4 cells (0: 8 for FP32, 16 for FP64)")
    ap.add_argument("--yband", type=int, default=0,
                    help="y-sweep rows per warp band (0: the precision's default, 28 FP32 / 56 FP64)")
    ap.add_argument("--ystage", type=int, default=0, choices=[0, 1],
                    help="y-sweep rows: 0 per-thread loads, 1 TMA-staged shared-memory boxes")
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("timestamp,index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str | None):
        self.bus_id = (bus_id or "").lower()
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-f", self.path], stdout=subprocess.DEVNULL,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.6)
        except (OSError, FileNotFoundError):
            self.proc = None

    def mark(self, which):
        setattr(self, which, time.time())

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 11:
                    continue
                if self.bus_id and self.bus_id[-12:] not in p[2].lower():
                    continue
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return None

        def ts(s):
            try:
                return time.mktime(time.strptime(s.split(".")[0], "%Y/%m/%d %H:%M:%S"))
            except ValueError:
                return None

        load = [r for r in rows if ts(r[0]) is not None and self.t0 - 1 <= ts(r[0]) <= self.t1 + 1] or rows
        sm = [float(r[3]) for r in load if r[3].replace(".", "").isdigit()]
        mx = [float(r[4]) for r in load if r[4].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in load for k in range(4) if r[7 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(load)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _reduce(x: float, world: int, op: str) -> float:
    """All-reduce of one host float over the ranks (device tensor under NCCL,
    host tensor under gloo); every rank calls it at the same point."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float, world: int) -> float:
    return _reduce(x, world, "max")


def sum_over_ranks(x: float, world: int) -> float:
    return _reduce(x, world, "sum")


def batch_shard(descs, world: int, rank: int) -> list[int]:
    """This rank's instances of the batch: LPT by cells (identical plan on every rank)."""
    from mhd_gpu_acc_b200.batch import lpt_partition

    return lpt_partition([int(d.nx) * int(d.ny) for d in descs], world)[rank]


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# The Orszag-Tang [0,1]^2 configuration: gamma 5/3, CFL 0.4, t_end 0.5, periodic.
OT_EXTENT, OT_GAMMA, OT_CFL, OT_T_END = (0.0, 1.0, 0.0, 1.0), 5.0 / 3.0, 0.4, 0.5


def cpu_reference_run(n: int, steps: int, warmup: int, budget_s: float | None):
    """The reference's CPU step on this host: returns (per-step seconds list, threads).

    Everything on this path -- the initial state included -- comes from the
    reference build (oracle/_ref/libmhdref.so); this repository's library is
    not loaded."""
    import numpy as np

    from oracle.oracle import REF_SO, Reference

    if not os.path.exists(REF_SO):
        return None, 0, "reference CPU build oracle/_ref/libmhdref.so is missing"
    ref = Reference()
    threads = os.cpu_count() or 1
    ref.set_threads(threads)
    U = ref.initialise_orszag_tang_unit(n, n, 2)
    bc = (0, 0, 0, 0)
    if budget_s is not None:  # size the sample from one probe step
        rc, k, secs, ch = ref.run_timed(U, 2, OT_EXTENT, OT_GAMMA, OT_CFL, 2, bc, 1, OT_T_END)
        per = float(secs[0])
        steps = int(max(1, min(steps, budget_s / max(per, 1e-9))))
        warmup = 0
    rc, k, secs, ch = ref.run_timed(U, 2, OT_EXTENT, OT_GAMMA, OT_CFL, 2, bc, warmup + steps, OT_T_END)
    del U
    if rc != 0 or k != warmup + steps:
        return None, threads, f"reference run stopped early (rc {rc}, {k} steps)"
    return list(np.asarray(secs[warmup:])), threads, None


def run_reference_arm(a, world, rank):
    if rank != 0:
        return 0
    n = a.n
    secs, threads, err = cpu_reference_run(n, a.steps, a.warmup, None)
    if err:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return 0
    tot = sum(secs)
    value = n * n * len(secs) / tot
    sample = (f"Orszag-Tang [0,1]^2 {n}x{n}, HLLD, minmod (the reference has no van Leer limiter; "
              f"same cost class), CFL 0.4, {a.warmup} warm-up + {len(secs)} timed steps, FP64 AoS")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": len(secs),
        "warmup": a.warmup, "ms_per_step": 1e3 * tot / len(secs), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (deterministic Orszag-Tang initial data)",
        "config": {"workload": f"orszag_tang_unit_{n}x{n}_hlld_cfl0.4", "nx": n, "ny": n, "solver": "hlld",
                   "limiter": "minmod", "limiter_note": "reference has minmod only (no van Leer); same cost class",
                   "precision": "fp64", "device": "host cpu (OpenMP)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_ours(a, world, rank, local):
    import numpy as np
    import torch

    import mhd_gpu_acc_b200 as m

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.Stream()
    n = a.n
    cfg = m.get_n_case_config(m.CaseId.OrszagTangUnit, 1)
    solver, limiter, bc = m.RiemannSolver.HLLD, m.Limiter.VANLEER, m.BoundaryConfig(0, 0, 0, 0)
    U0 = m.initialise(m.CaseId.OrszagTangUnit, n, n, 2, cfg.extent)
    t_end = cfg.t_end
    res = {}
    states = {}

    def arm(dtype):
        U = m.Grid2DGPU(n, n, 2, *cfg.extent, dtype)
        T = m.Grid2DGPU(n, n, 2, *cfg.extent, dtype)
        ws = m.GpuWorkspace()
        m.init_gpu_workspace(ws, U)
        m.set_gpu_physics_gamma(ws, cfg.gamma)
        m.set_gpu_physics_ch(ws, 0.0)
        ws.set_limiter(limiter)
        ws.set_sweep_shape(a.xrpw, a.yband, a.ystage)
        ws.set_stream(stream.cuda_stream)
        U.upload(U0)
        ws.run(U, T, cfg.cfl, t_end, a.warmup, solver, bc)
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = m.launch_count()
        sampler.mark("t0")
        e0.record(stream)
        info = ws.run(U, T, cfg.cfl, t_end, a.steps, solver, bc)
        e1.record(stream)
        torch.cuda.synchronize()
        sampler.mark("t1")
        launches = m.launch_count() - l0
        barrier(world)
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        assert info.steps == a.steps, info.steps
        prof = ws.profile_sweeps(U, T, cfg.cfl, t_end, solver, bc, 5)
        states[dtype] = U.download()[0]
        ws.destroy()
        return dict(ms=ms, launches=launches, sweeps_ms=prof, t=info.t, fallbacks=info.fallbacks)

    bus = None
    try:
        p = torch.cuda.get_device_properties(local)
        bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}"
    except Exception:
        pass
    sampler = ClockSampler(bus)
    sampler.start()
    res[m.F32] = arm(m.F32)
    clocks = sampler.stop()
    if not a.no_fp64:
        res[m.F64] = arm(m.F64)

    cells = n * n
    v32 = world * cells * a.steps / (res[m.F32]["ms"] / 1e3)
    out_fp64 = None
    l1 = None
    if m.F64 in res:
        v64 = world * cells * a.steps / (res[m.F64]["ms"] / 1e3)
        r64 = states[m.F64][2:-2, 2:-2]
        l1 = float(np.abs(states[m.F32][2:-2, 2:-2] - r64).sum() / np.abs(r64).sum())
        out_fp64 = {"value": v64, "unit": UNIT, "ms_per_step": res[m.F64]["ms"] / a.steps,
                    "sweep_ms": list(res[m.F64]["sweeps_ms"]),
                    "hbm_frac_step": cells * 2 * BYTES_PER_CELL_SWEEP[8] / (res[m.F64]["ms"] / a.steps / 1e3) / 1e9
                    / peaks()[0]}

    # roofline of the dominant FP32 kernel (the slower sweep).  Its bytes are
    # the HBM roofline's (frac against the measured copy bandwidth), but the
    # kernel is bound by instruction issue: `issue` gives its warp instructions
    # per cell (ncu, profiles/traffic.json) and the time those take at one warp
    # instruction per cycle on every SM sub-partition at the sampled SM clock.
    hbm, kind = peaks()
    mx, my = res[m.F32]["sweeps_ms"]
    dom, dom_ms = ("sweep_y", my) if my >= mx else ("sweep_x", mx)
    alg = cells * BYTES_PER_CELL_SWEEP[4]
    achieved = alg / (dom_ms / 1e3) / 1e9
    traffic, issue = None, None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            tj = json.load(f).get(f"fp32_{dom}")
        if tj:
            traffic = tj["bytes_per_cell"] * cells
            wi = tj.get("warp_inst_per_cell")
            clk = (clocks or {}).get("sm_mhz") or 1965.0
            if wi:
                sub = 4 * torch.cuda.get_device_properties(local).multi_processor_count
                ceiling_ms = wi * cells / (sub * clk * 1e6) * 1e3
                issue = {"warp_inst_per_cell": wi, "thread_inst_per_cell": tj.get("thread_inst_per_cell"),
                         "issue_ceiling_ms": ceiling_ms, "issue_frac": ceiling_ms / dom_ms, "sm_mhz": clk,
                         "source": "ncu instruction counts of the same kernel, profiles/traffic.json"}
    roofline = {"bound": "issue", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": traffic, "kernel": dom, "kernel_ms": dom_ms, "algorithmic_bytes": alg,
                "peak_kind": kind, "sweep_ms": [mx, my], "issue": issue,
                "note": "frac is against the measured HBM copy bandwidth; the kernel is issue-bound (issue.issue_frac "
                        "= instruction-issue time at one warp instruction per cycle per SM sub-partition / kernel time)"}

    # e2e through the C ABI with pinned FP32 host buffers (the FP32-bulk step's
    # own state format): every step uploads a state, advances it one FP32-bulk
    # step and downloads the result.  The step is the device-clocked one
    # (mhd_clock_start + the two mhd_sweep_clocked sweeps: dt and c_h stay on
    # the GPU), so the host queues steps without waiting for any.  Steps are
    # independent, so `e2e_lanes` workspaces on their own streams take turns:
    # one lane's upload, another's step and a third's download run at once, and
    # the step is bound by the host <-> device copy rate.
    # Every rank runs the loop (the time is the max over ranks).
    lanes = []
    hin = torch.from_numpy(U0.astype(np.float32)).pin_memory()
    a_in = hin.numpy()
    for _ in range(a.e2e_lanes):
        U = m.Grid2DGPU(n, n, 2, *cfg.extent, m.F32)
        T = m.Grid2DGPU(n, n, 2, *cfg.extent, m.F32)
        ws = m.GpuWorkspace()
        m.init_gpu_workspace(ws, U)
        m.set_gpu_physics_gamma(ws, cfg.gamma)
        ws.set_limiter(limiter)
        ws.set_sweep_shape(a.xrpw, a.yband, a.ystage)
        s = torch.cuda.Stream()
        ws.set_stream(s.cuda_stream)
        hout = torch.empty_like(hin).pin_memory()
        lanes.append((U, T, ws, s, hout.numpy(), hout))

    def e2e_step(k):
        U, T, ws, _, a_out, _ = lanes[k % len(lanes)]
        ws.upload_f32(U, a_in)
        ws.step_async(U, T, cfg.cfl, t_end, solver, bc)
        ws.download_f32(U, a_out)

    for k in range(4):  # warm-up
        e2e_step(k)
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _, _, _, s, _, _ in lanes:
        s.wait_event(e0)
    for k in range(a.e2e_steps):
        e2e_step(k)
    for _, _, _, s, _, _ in lanes:
        ev = torch.cuda.Event()
        ev.record(s)
        stream.wait_event(ev)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    for _, _, ws, _, a_out, _ in lanes:
        # each lane's last step ran (one step on its clock, status OK) and gave a finite state
        info = ws.clock_read()
        if info.steps != 1 or info.status != 0 or not np.isfinite(a_out[0]).all():
            raise RuntimeError(f"e2e step did not complete: steps {info.steps}, status {info.status}")
        ws.destroy()
    nbytes = int(hin.numel() * hin.element_size())
    e2e = {"value": world * cells * a.e2e_steps / (ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
           "d2h_bytes_per_step": nbytes, "steps": a.e2e_steps,
           "what": "per step: H2D of the FP32 SoA state (ghosts included) from pinned memory "
                   "(mhd_upload_f32), one FP32-bulk step with dt and c_h on the GPU (mhd_clock_start, "
                   "mhd_sweep_clocked x and y), D2H of the state (mhd_download_f32); "
                   f"{len(lanes)} workspaces on their own streams take steps in turn, so one step's download "
                   "overlaps the next steps' upload and compute"}

    cpu = None
    if world == 1 and rank == 0 and not a.no_cpu_baseline:
        secs, threads, err = cpu_reference_run(n, 1000, 0, a.cpu_seconds)
        if err is None:
            cpu = {"value": cells * len(secs) / sum(secs), "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"reference CPU/OpenMP step (oracle/_ref), Orszag-Tang {n}x{n}, HLLD, minmod "
                             f"(no van Leer in the reference), {len(secs)} steps after one probe step, FP64"}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": err}

    if rank == 0:
        line = {
            "metric": METRIC, "value": v32, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": res[m.F32]["ms"] / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (deterministic Orszag-Tang initial data)",
            "config": {"workload": f"orszag_tang_unit_{n}x{n}_hlld_vanleer_cfl0.4", "nx": n, "ny": n,
                       "solver": "hlld", "limiter": "vanleer", "precision": "fp32-bulk (fp64 low-beta pressure, "
                       "fp64 dt reduction)", "per_gpu": "one independent instance",
                       "l2": "state 604 MB (fp32) / 1.2 GB (fp64) > 126 MB L2; no flush",
                       "sweep_shape": {"xrpw": a.xrpw or "default (8 fp32, 16 fp64)",
                                       "x_segment_cells": 128 * (a.xrpw or 8) - 4,
                                       "x_tail": "last quarter of each row in segments of a third",
                                       "yband": a.yband or "default (28 fp32, 56 fp64)",
                                       "y_tail": "last eighth of the rows in bands of 1/2, last 1/32 of 1/4",
                                       "y_rows": "tma-staged" if a.ystage else "per-thread loads",
                                       "y_rows_note": "TMA-staged shared-memory boxes are a launch option "
                                                      "(--ystage 1); the per-thread loads measured faster for this "
                                                      "issue-bound kernel"}},
            "fp64": out_fp64,
            "fp32_over_fp64": (v32 / out_fp64["value"]) if out_fp64 else None,
            "rho_rel_l1_fp32_vs_fp64": l1,
            "hbm_frac_step": cells * 2 * BYTES_PER_CELL_SWEEP[4] / (res[m.F32]["ms"] / a.steps / 1e3) / 1e9 / hbm,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": res[m.F32]["launches"],
            "clocks": clocks,
        }
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_batch(a, world, rank, local):
    """256 Orszag-Tang instances of uneven size (sides U{64..1024}), one persistent
    launch per sweep phase, autotuned.  With N ranks the one batch is split over
    the GPUs by LPT on cells (strong scaling, no data-path collective); the time
    is the max over ranks and the value all ranks' cell-updates over it."""
    import numpy as np
    import torch

    import mhd_gpu_acc_b200 as m
    from mhd_gpu_acc_b200.batch import Batch, orszag_tang_batch_spec

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    steps = a.steps
    # t_end far enough that every instance takes all its steps (500 steps of the
    # smallest, 64^2, instance reach t ~ 1)
    all_descs, all_b0, all_gam = orszag_tang_batch_spec(a.seed, n=a.instances, t_end=5.0)
    mine = batch_shard(all_descs, world, rank)
    descs = [all_descs[i] for i in mine]
    b0, gam = all_b0[mine], all_gam[mine]
    stream = torch.cuda.Stream()

    def make(dtype):
        b = Batch(descs, dtype=dtype, solver=m.RiemannSolver.HLLD, limiter=m.Limiter.VANLEER)
        b.set_stream(stream.cuda_stream)
        return b

    def init(b):
        for i in range(len(descs)):
            b.init_orszag_tang(i, b0[i], gam[i])

    b32 = make(m.F32)
    init(b32)
    tuning = b32.tune(2)
    init(b32)
    b32.run(a.warmup)
    init(b32)
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    info = b32.run(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    cells = int(sum_over_ranks(float(b32.cells), world))
    updates = sum_over_ranks(float(sum(int(d.nx) * int(d.ny) * i.steps for d, i in zip(descs, info))), world)
    value = updates / (ms / 1e3)
    steps_min = int(-max_over_ranks(-float(min(i.steps for i in info)), world))
    errs = []
    if not a.no_fp64:
        b64 = make(m.F64)
        init(b64)
        b64.run(steps)
        for i in range(len(descs)):
            r32, r64 = b32.download(i)[0, 2:-2, 2:-2], b64.download(i)[0, 2:-2, 2:-2]
            errs.append(float(np.abs(r32 - r64).sum() / np.abs(r64).sum()))
        b64.destroy()
    b32.destroy()
    err_max = max_over_ranks(max(errs), world) if errs else None
    if rank == 0:
        line = {
            "metric": "batched Orszag-Tang aggregate cell-updates/s (FP32-bulk)", "value": value, "unit": UNIT,
            "n_gpus": world, "steps": steps, "warmup": a.warmup, "ms_per_step": ms / steps,
            "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded Orszag-Tang instances)",
            "config": {"workload": f"orszag_tang_batch_{len(all_descs)}_seed{a.seed}",
                       "instances": len(all_descs), "cells": cells,
                       "sides": [int(d.nx) for d in all_descs][:8] + ["..."],
                       "sharding": f"LPT on cells over {world} GPU(s); rank 0 holds {len(descs)} instances",
                       "solver": "hlld", "limiter": "vanleer",
                       "tuning": {"xrpw": tuning.xrpw, "yseg": tuning.yseg, "ctas_x": tuning.ctas_x,
                                  "ctas_y": tuning.ctas_y}},
            "steps_done_min": steps_min,
            "rho_rel_l1_vs_fp64": ({"max": err_max, "rank0_median": float(np.median(errs)),
                                    "rank0_min": min(errs)} if errs else None),
        }
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_adjoint(a, world, rank, local):
    """Gradient of the Orszag-Tang objective (512^2, 400 steps, HLL + van Leer):
    wall time of the gradient against a forward solve, FP32 and FP64, and the
    FP64 gradient against central differences (h = 1e-6)."""
    import numpy as np
    import torch

    from mhd_gpu_acc_b200 import F32, F64
    from mhd_gpu_acc_b200.adjoint import OTAdjoint, amplitudes

    torch.cuda.set_device(local)
    n, steps = (a.n if a.n != 4096 else 512), (a.steps if a.steps != 100 else 400)
    out = {}
    for name, dt in (("fp32", F32), ("fp64", F64)):
        adj = OTAdjoint(n=n, nsteps=steps, dtype=dt)
        _, target = adj.forward(amplitudes(a.seed + 1), want_rho=True)
        adj.set_target(target)
        amp = amplitudes(a.seed)
        adj.forward(amp)  # warm
        adj.gradient(amp)
        t0 = time.perf_counter()
        J = adj.forward(amp)
        t_fwd = time.perf_counter() - t0
        t0 = time.perf_counter()
        Jg, g = adj.gradient(amp)
        t_grad = time.perf_counter() - t0
        rec = {"J": J, "forward_s": t_fwd, "gradient_s": t_grad, "gradient_over_forward": t_grad / t_fwd,
               "grad": [float(x) for x in g]}
        if dt == F64:
            fd = np.zeros(16)
            for k in range(16):
                e = np.zeros(16)
                e[k] = 1e-6
                fd[k] = (adj.forward(amp + e) - adj.forward(amp - e)) / 2e-6
            rec["rel_err_vs_central_differences"] = float(np.linalg.norm(g - fd) / np.linalg.norm(fd))
        out[name] = rec
        adj.destroy()
    g32, g64 = np.array(out["fp32"]["grad"]), np.array(out["fp64"]["grad"])
    if rank == 0:
        line = {
            "metric": "adjoint gradient cost (gradient wall time / forward wall time)",
            "value": out["fp32"]["gradient_over_forward"], "unit": "x forward", "n_gpus": 1, "steps": steps,
            "higher_is_better": False, "dtype": "f32",
            "config": {"workload": f"orszag_tang_adjoint_{n}x{n}_{steps}steps_hll_vanleer", "seed": a.seed,
                       "checkpoints": "every ~sqrt(N) steps"},
            "fp32": {k: v for k, v in out["fp32"].items() if k != "grad"},
            "fp64": {k: v for k, v in out["fp64"].items() if k != "grad"},
            "fp32_vs_fp64_grad_rel": float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64)),
        }
        print(json.dumps(line))
    return 0


FIELDS = ["rho", "rhou", "rhov", "rhow", "Bx", "By", "Bz", "E", "psi"]


def fp64_with_fp32_state(m, cfg, U0, nx, ny, solver, lim, max_steps):
    """The FP64 step with its state rounded to FP32 after every sweep (the
    x-swept intermediate and the step's result), driven through the per-sweep
    C ABI (mhd_max_speed, mhd_set_ch, mhd_sweep) like the drop-in loop.  FP64
    arithmetic, FP32 storage: the error this run has against the FP64 step is
    the floor of every scheme that stores the state in FP32, whatever its
    arithmetic.  The loop stops as the device loop does (dt not finite, not
    positive or below 1e-8 t_end).  Returns (interior state, steps, t, stop)."""
    import ctypes as C

    import torch

    from mhd_gpu_acc_b200._lib import check, load
    from mhd_gpu_acc_b200.slabs import grid_tensor
    from mhd_gpu_acc_b200.solver import BoundaryConfig

    lib = load()
    U = m.Grid2DGPU(nx, ny, 2, *cfg.extent, m.F64)
    T = m.Grid2DGPU(nx, ny, 2, *cfg.extent, m.F64)
    ws = m.GpuWorkspace()
    m.init_gpu_workspace(ws, U)
    m.set_gpu_physics_gamma(ws, cfg.gamma)
    m.set_gpu_physics_ch(ws, 0.0)
    ws.set_limiter(lim)
    U.upload(U0)
    tu, tt = grid_tensor(U.g), grid_tensor(T.g)

    def to_fp32(t):
        t.copy_(t.float())
        torch.cuda.synchronize()

    to_fp32(tu)
    bc = BoundaryConfig.of(cfg.bc).as_array()
    x0, x1, y0, y1 = cfg.extent
    d = min((x1 - x0) / nx, (y1 - y0) / ny)
    t, steps, M, stop = 0.0, 0, C.c_double(), None
    while t < cfg.t_end and (max_steps == 0 or steps < max_steps):
        check(lib.mhd_max_speed(ws.ptr, C.byref(U.g), C.byref(M)), "mhd_max_speed")
        if not M.value > 0.0:
            stop = "no positive speed"
            break
        check(lib.mhd_set_ch(ws.ptr, M.value), "mhd_set_ch")
        dt = min(cfg.cfl * d / M.value, cfg.t_end - t)
        if not (math.isfinite(dt) and dt > 0.0) or dt < 1e-8 * cfg.t_end:
            stop = f"dt {dt:.3e} at t = {t:.6f}"
            break
        check(lib.mhd_sweep(ws.ptr, C.byref(U.g), C.byref(T.g), dt, int(solver), bc, 0), "mhd_sweep(x)")
        ws.synchronize()
        to_fp32(tt)
        check(lib.mhd_sweep(ws.ptr, C.byref(T.g), C.byref(U.g), dt, int(solver), bc, 1), "mhd_sweep(y)")
        ws.synchronize()
        to_fp32(tu)
        t += dt
        steps += 1
    out = U.download()[:, 2:-2, 2:-2]
    ws.destroy()
    return out, steps, t, stop


def run_precision(a, world, rank, local):
    """Every configuration run with the FP64 step and with the FP32-bulk step
    (device-resident loop); relative L1 (sum|a-b| / sum|b|) and Linf
    (max|a-b| / max|b|) of the interior, per conserved field.  Orszag-Tang and
    Brio-Wu run to t_end.  The Mach-10 shock-bubble runs 500 steps: with the
    reference's scheme (no positivity guard on the update) its pressure turns
    negative once the shock has crossed the dense bubble and the time step
    collapses before t_end -- the reference's own CPU code stops at step 1069 of
    the 512^2 case (t = 0.040), as does the FP64 step here, and at 2048^2 the
    HLLC run stops at step 638.
    Beside each FP32 error stand the FP64 step's own sensitivity -- FP64 from
    initial data perturbed by a relative 1e-12 (seeded), against FP64: where
    that is large, the flow amplifies rounding-level differences -- and the
    FP32-storage floor: the FP64 step with its state rounded to FP32 after
    every sweep (fp64_with_fp32_state), which no scheme storing the state in
    FP32 can beat."""
    import numpy as np
    import torch

    import mhd_gpu_acc_b200 as m

    torch.cuda.set_device(local)
    if rank != 0:
        return 0
    H, HC, VL, MM = m.RiemannSolver.HLLD, m.RiemannSolver.HLLC, m.Limiter.VANLEER, m.Limiter.MINMOD
    cases = [(f"orszag_tang_{n}_hlld_vanleer", m.CaseId.OrszagTangUnit, n, n, H, VL, 0)
             for n in (512, 2048, 4096) if n <= a.precision_max_n]
    cases += [("shock_bubble_2048_hllc_500_steps", m.CaseId.ShockBubbleMHD, 2048, 2048, HC, MM, 500),
              ("shock_bubble_2048_hlld_500_steps", m.CaseId.ShockBubbleMHD, 2048, 2048, H, MM, 500),
              ("brio_wu_800x4_hlld_cfl0.8", m.CaseId.BrioWuCFL08, 800, 4, H, MM, 0)]
    if a.precision_cases:
        keys = [k for k in a.precision_cases.split(",") if k]
        cases = [c for c in cases if any(k in c[0] for k in keys)]
    out = {}
    for name, case, nx, ny, solver, lim, max_steps in cases:
        cfg = m.get_n_case_config(case, 1)
        U0 = m.initialise(case, nx, ny, 2, cfg.extent)
        res = {}
        P0 = U0 * (1.0 + 1e-12 * np.random.default_rng(1).standard_normal(U0.shape))
        for key, dt, init in (("f64", m.F64, U0), ("f32", m.F32, U0), ("f64p", m.F64, P0)):
            U = m.Grid2DGPU(nx, ny, 2, *cfg.extent, dt)
            T = m.Grid2DGPU(nx, ny, 2, *cfg.extent, dt)
            ws = m.GpuWorkspace()
            m.init_gpu_workspace(ws, U)
            m.set_gpu_physics_gamma(ws, cfg.gamma)
            m.set_gpu_physics_ch(ws, 0.0)
            ws.set_limiter(lim)
            U.upload(init)
            info = ws.run(U, T, cfg.cfl, cfg.t_end, max_steps, solver, cfg.bc)
            res[key] = (U.download()[:, 2:-2, 2:-2], info.steps, info.t)
            ws.destroy()
            del U, T
        a64, s64, t64 = res["f64"]
        b_ = np.abs(a64).reshape(9, -1)

        def errs(other):
            d = np.abs(other - a64).reshape(9, -1)
            l1 = [float(d[k].sum() / b_[k].sum()) if b_[k].sum() > 0 else float(d[k].sum()) for k in range(9)]
            li = [float(d[k].max() / b_[k].max()) if b_[k].max() > 0 else float(d[k].max()) for k in range(9)]
            return dict(zip(FIELDS, l1)), dict(zip(FIELDS, li))

        l1, li = errs(res["f32"][0])
        pl1, _ = errs(res["f64p"][0])
        q = fp64_with_fp32_state(m, cfg, U0, nx, ny, solver, lim, max_steps)
        ql1, _ = errs(q[0])
        out[name] = {"steps_fp64": s64, "steps_fp32": res["f32"][1], "t": t64,
                     "rel_l1": l1, "rel_linf": li, "fp64_perturbed_1e-12_rel_l1": pl1,
                     "fp64_fp32_state_rel_l1": ql1, "steps_fp64_fp32_state": q[1], "fp64_fp32_state_stop": q[3]}
        print(f"{name}: rho L1 {l1['rho']:.2e}, FP32-state floor {ql1['rho']:.2e} ({q[3] or 'to the end'})",
              file=sys.stderr, flush=True)
    print(json.dumps({"metric": "FP32-bulk vs FP64 relative error per field of each configuration",
                      "unit": "relative", "n_gpus": 1, "dtype": "f32 vs f64", "data": "synthetic (library initial data)",
                      "config": {"workload": "precision", "cases": list(out)}, "cases": out}))
    return 0


def run_slabs(a, world, rank, local):
    """One Orszag-Tang n^2 grid (FP32-bulk, HLLD + van Leer) split into y-slabs and
    stepped without host round trips (mhd_gpu_acc_b200.slabs): on one GPU as
    `--parts` slabs (halo copies on a second stream), under torchrun as one slab
    per rank (NCCL halo exchange and all-reduce(max)); strong scaling of the one
    grid.  The final state is checked against the single-grid device loop (one
    GPU: bit for bit; ranks: the density sum)."""
    import numpy as np
    import torch

    import mhd_gpu_acc_b200 as m
    from mhd_gpu_acc_b200.slabs import DistSlabRun, SlabGrid

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    n = a.n
    cfg = m.get_n_case_config(m.CaseId.OrszagTangUnit, 1)
    solver, limiter, bc = m.RiemannSolver.HLLD, m.Limiter.VANLEER, (0, 0, 0, 0)
    U0 = m.initialise(m.CaseId.OrszagTangUnit, n, n, 2, cfg.extent)
    if world == 1:
        run = SlabGrid(n, n, 2, cfg.extent, a.parts, m.F32)
        run.upload(U0)
        run.configure(cfg.gamma, limiter)
    else:
        run = DistSlabRun(n, n, 2, cfg.extent, m.F32)
        run.upload(U0)
        m.set_gpu_physics_gamma(run.ws, cfg.gamma)
        m.set_gpu_physics_ch(run.ws, 0.0)
        run.ws.set_limiter(limiter)
    run.start(cfg.cfl, cfg.t_end)
    for _ in range(a.warmup):
        run.step(solver, bc)
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = m.launch_count()
    e0.record(run.stream)
    for _ in range(a.steps):
        run.step(solver, bc)
    e1.record(run.stream)
    torch.cuda.synchronize()
    launches = m.launch_count() - l0
    barrier(world)
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    info = run.info()
    if world == 1:
        got = run.download()
        run.destroy()
        U = m.Grid2DGPU(n, n, 2, *cfg.extent, m.F32)
        T = m.Grid2DGPU(n, n, 2, *cfg.extent, m.F32)
        U.upload(U0)
        ws = m.GpuWorkspace()
        m.init_gpu_workspace(ws, U)
        m.set_gpu_physics_gamma(ws, cfg.gamma)
        ws.set_limiter(limiter)
        ws.run(U, T, cfg.cfl, cfg.t_end, a.warmup + a.steps, solver, bc)
        want = U.download()
        ws.destroy()
        check = {"single_grid_bit_equal": bool(np.array_equal(got[:, 2:-2, :], want[:, 2:-2, :]))}
    else:
        part = float(run.U.download()[0, 2:-2, 2:-2].sum())
        run.destroy()
        check = {"rho_sum": sum_over_ranks(part, world)}
    if rank == 0:
        line = {
            "metric": "Orszag-Tang cell-updates/s, one grid in y-slabs (FP32-bulk)", "unit": UNIT,
            "value": n * n * a.steps / (ms / 1e3), "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (deterministic Orszag-Tang initial data)",
            "config": {"workload": f"orszag_tang_unit_{n}x{n}_slabs", "slabs": a.parts if world == 1 else world,
                       "exchange": "mhd_grid_copy_rows on a second stream" if world == 1 else "NCCL send/recv",
                       "solver": "hlld", "limiter": "vanleer"},
            "steps_done": info.steps, "gpu_launches": launches, "check": check,
        }
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def main():
    a = parse()
    world, rank, local = dist_setup()
    if a.impl == "reference":
        return run_reference_arm(a, world, rank)
    if a.workload == "batch":
        return run_batch(a, world, rank, local)
    if a.workload == "adjoint":
        return run_adjoint(a, world, rank, local)
    if a.workload == "precision":
        return run_precision(a, world, rank, local)
    if a.workload == "slabs":
        return run_slabs(a, world, rank, local)
    return run_ours(a, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
