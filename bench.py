#!/usr/bin/env python
"""Benchmark: LBGK million lattice-cell updates per second (MLUPS) on one or
more B200s, on the porous-channel workload (D3Q19, 512x256x256 cells, seeded
random spheres with solid fraction 0.4, periodic x, no-slip Y/Z walls, body
force 1e-6, tau 0.6; synthetic data generated from a seed).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0. `value` is whole-job MLUPS with populations
resident in HBM; with N > 1 GPUs the channel is N times longer and cut into
x slabs, one per GPU, exchanging faces every step (weak scaling; --replicas
runs independent copies instead);
`e2e` is the same metric through the C ABI with the initial populations
uploaded from pinned host memory and density/velocity downloaded to pinned
host memory inside the timed region; `roofline` describes the dominant
stream-collide kernel; `cpu_baseline` is the CPU oracle on the host cores.
`--impl reference` times that CPU restatement of the reference's algorithm
alone (the reference's own OpenCL build is unavailable here).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "D3Q19/27 MLUPS & % HBM roofline; plain FP32 vs FP16/learned at stated error"
BYTES_PER_CELL = {("f32", 19): 152, ("f16", 19): 76, ("f64", 19): 304, ("f32", 27): 216, ("f16", 27): 108}
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", default="512,256,256")
    ap.add_argument("--storage", default="f32", choices=["f32", "f16"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp16", action="store_true")
    ap.add_argument("--replicas", action="store_true",
                    help="with several GPUs: one independent replica per GPU instead of x slabs")
    ap.add_argument("--slabs", action="store_true",
                    help="the x-slab path even on one GPU (one slab closing its own x-periodic ring)")
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--accuracy-steps", type=int, default=5000,
                    help="steps of the FP16/FP32-against-FP64 accuracy study (0: skip)")
    ap.add_argument("--q27-steps", type=int, default=400,
                    help="timed steps of the D3Q27 vehicle workload (0: skip)")
    ap.add_argument("--q27-size", default="768,384,384")
    ap.add_argument("--vehicle-study-steps", type=int, default=2000,
                    help="steps of the D3Q27 closure / storage study on the downscaled tunnel (0: skip)")
    ap.add_argument("--vehicle-small", default="192,96,96")
    ap.add_argument("--details", default="bench_details.json",
                    help="file for the full results of every leg (the JSON line carries a summary)")
    ap.add_argument("--batch-steps", type=int, default=2000,
                    help="timed steps of the 256-domain batch (0: skip)")
    ap.add_argument("--batch-domains", type=int, default=256)
    ap.add_argument("--fd-steps", type=int, default=100,
                    help="steps of the FD advection-diffusion leg (0 skips it)")
    ap.add_argument("--closure-size", type=int, default=256,
                    help="coarse grid of the learned-closure study (fine = 2x; 0: skip)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profile_traffic(name: str, cells: int):
    """DRAM bytes per launch of `cells` cells from a committed ncu summary
    (line 'traffic_bytes_per_cell: B', measured read + write per cell), or None."""
    p = ROOT / "profiles" / name
    try:
        for line in p.read_text().splitlines():
            if line.strip().startswith("traffic_bytes_per_cell:"):
                return float(line.split(":", 1)[1].split()[0]) * cells
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.tmp = None

    def start(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.tmp.flush()
        rows = [r.split(",") for r in Path(self.tmp.name).read_text().splitlines() if r.strip()]
        os.unlink(self.tmp.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def parse_size(s):
    return tuple(int(v) for v in s.split(","))


# ---------------------------------------------------------------------------
def cpu_baseline(w, steps: int, warm: int = 2):
    """The CPU oracle (a C++ restatement of the reference's LBGK) on the same
    workload, FP32, all host threads, over a bounded number of steps."""
    from oracle import oracle as O
    O.build()
    from asl_b200 import workloads as W
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    o = O.Oracle(w.size, w.q, 4, w.nu, flags=8 if w.periodic[0] else 0)
    if w.body_force:
        o.set_body_force(w.body_force)
    o.init_f(1.0, (0, 0, 0))
    ids = []
    for s in w.bcs:
        if s.kind == "map_noslip":
            ids.append(o.bc_map(10, w.map))
        else:
            ids.append(o.bc_slice(W.SLICE_KIND[s.kind], sum(W.WALL_BITS[x] for x in s.walls), s.p, s.u))

    def one():
        o.step(1)
        for i in ids:
            o.bc_execute(i)

    for _ in range(warm):
        one()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    dt = time.perf_counter() - t0
    return {"value": w.cells * steps / dt / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port",
            "sample": f"{steps} steps (after {warm} warm-up) of the full {w.size[0]}x{w.size[1]}x{w.size[2]} "
                      f"workload, FP32, {threads} OpenMP threads"}


def repo_libraries():
    """Shared libraries of this repository mapped into the process."""
    out = set()
    try:
        for line in Path("/proc/self/maps").read_text().splitlines():
            path = line.split()[-1] if len(line.split()) >= 6 else ""
            if path.endswith(".so") and path.startswith(str(ROOT)):
                out.add(str(Path(path).relative_to(ROOT)))
    except OSError:
        pass
    return sorted(out)


def run_reference(args):
    """The CPU restatement of the reference's LBGK on the host cores. The
    workload is built with the oracle's sphere packer: nothing of the CUDA
    library is loaded (the line lists the repository libraries the process
    mapped)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle as O
    from asl_b200 import workloads as W
    w = W.porous_channel(size=parse_size(args.size), packer=O.pack_spheres)
    steps = max(1, min(args.steps, args.cpu_steps))
    warm = max(0, min(args.warmup, 10))
    cb = cpu_baseline(w, steps, warm=warm)
    # with N GPUs the job is N such slabs along x (weak scaling); the host's
    # rate per cell does not depend on the slab count, so one slab is the
    # bounded sample of it
    n = max(1, world, args.gpus)
    job = w.name if n == 1 else "porous_channel_d3q19_%dx%dx%d" % (w.size[0] * n, w.size[1], w.size[2])
    if n > 1:
        cb["sample"] += "; one %dx%dx%d slab of the %d-slab job" % (*w.size, n)
    job_cells = w.cells * n
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "MLUPS", "n_gpus": args.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": job_cells / (cb["value"] * 1e6) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded random spheres)",
            "config": {"workload": job, "lattice": "D3Q19", "cells": job_cells, "storage": "f32",
                       "implementation": "CPU restatement of the reference LBGK (oracle/lbgk_oracle.cpp); "
                                         "the reference's OpenCL build is unavailable on this box"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "repo_libraries_loaded": repo_libraries()}
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_subprocess(args):
    """The reference arm's CPU measurement, run in a fresh process before this
    process touches the GPU (no CUDA context, no clock sampler, the host's
    threads free), so that the in-arm baseline and the reference arm measure
    the same thing the same way."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR",
                                                            "MASTER_PORT")}
    cmd = [sys.executable, str(Path(__file__).resolve()), "--impl", "reference", "--size", args.size,
           "--steps", str(args.cpu_steps), "--warmup", "2", "--cpu-steps", str(args.cpu_steps)]
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=900)
    for line in reversed(r.stdout.splitlines()):
        if line.startswith("{"):
            return json.loads(line)["cpu_baseline"]
    raise RuntimeError("CPU baseline run failed: " + (r.stderr or r.stdout)[-2000:])


# ---------------------------------------------------------------------------
def storage_accuracy(W, w, steps: int):
    """The porous channel advanced `steps` steps with FP64, FP32 and FP16
    storage (fused no-slip, CUDA graph). FP64 is the reference (the GPU FP64
    kernel matches the FP64 CPU oracle to 1e-12 in the tests). Reports the
    permeability k = nu <u_x> / g (superficial velocity: solid cells count as
    zero) and the relative L2 error of u over the fluid cells."""
    import numpy as np
    g = w.body_force[0]
    fluid = w.map[1:-1, 1:-1, 1:-1] > 0
    out = {"steps": steps, "reference": "FP64 storage on the GPU", "permeability": {}, "permeability_rel_err": {},
           "velocity_rel_l2": {}, "ms_per_step": {}}
    ref = None
    for storage in ("f64", "f32", "f16"):
        import torch
        lb, bcs = W.build_lbgk(w, storage=storage, compVel=False, compRho=False, fuse=True)
        st = torch.cuda.ExternalStream(lb.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        lb.run(steps - 1, bcs, use_graph=True)
        lb.requestMacro()
        lb.run(1, bcs)
        e1.record(st)
        e1.synchronize()
        u = lb.getVelocity(np.float64)[:, 1:-1, 1:-1, 1:-1][:, fluid]
        del lb, bcs
        k = w.nu * float(u[0].sum()) / fluid.size / g
        out["permeability"][storage] = k
        out["ms_per_step"][storage] = e0.elapsed_time(e1) / steps
        if ref is None:
            ref = (u, k)
        else:
            out["permeability_rel_err"][storage] = abs(k - ref[1]) / abs(ref[1])
            out["velocity_rel_l2"][storage] = float(np.sqrt(((u - ref[0]) ** 2).sum() / (ref[0] ** 2).sum()))
    out["unit"] = "lattice units (dx = 1)"
    return out


def vehicle_run(W, size, steps: int, peak: float):
    """D3Q27 vehicle-like channel (seeded boxes and cylinders on the floor):
    MLUPS of the full step (inlet / far-field / moving-floor velocity
    conditions, outlet pressure, fused no-slip obstacles) and a drag / lift
    series from the surface force on the obstacles."""
    import numpy as np
    import torch
    w = W.vehicle_d3q27(size=size, steps=steps)
    lb, bcs = W.build_lbgk(w, storage="f32", compVel=False, compRho=False, fuse=True)
    from asl_b200 import lbgk as A
    force = A.generateComputeSurfaceForce(lb, w.map)
    st = torch.cuda.ExternalStream(lb.stream)
    lb.run(4, bcs, use_graph=True)
    lb.sync()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    lb.run(steps, bcs, use_graph=True)
    e1.record(st)
    e1.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    nk = 20
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k0.record(st)
    lb.execute(nk)
    k1.record(st)
    k1.synchronize()
    tk = k0.elapsed_time(k1) / 1e3 / nk
    series = []
    every = max(1, steps // 8)
    for n in range(8):
        lb.run(every, bcs, use_graph=True)
        fx = force.execute()
        series.append([int(lb.steps), float(fx[0]), float(fx[2])])
    nonslip = sum(b.kernels for b in bcs)
    bpc = BYTES_PER_CELL[("f32", 27)]
    res = {"workload": w.name, "cells": w.cells, "steps": steps, "value": w.cells * steps / t / 1e6,
           "unit": "MLUPS", "ms_per_step": t / steps * 1e3, "kernel_ms": tk * 1e3,
           "kernel_frac_of_peak": bpc * w.cells / tk / 1e9 / peak, "boundary_kernels_per_step": nonslip,
           "obstacles": w.info["obstacles"], "drag_lift_series": series,
           "series_columns": ["step", "drag (sum F_x)", "lift (sum F_z)"]}
    del force, lb, bcs
    return res, w


def closure_run(n: int):
    """Decaying turbulence at n^3 (fine run 2n^3): the learned closure trained
    on the filtered fine run by the library's kernels, judged by the energy
    spectrum against Smagorinsky (Cs 0.17 and the best constant), plus the
    step rates."""
    from asl_b200 import closure as CL
    res = CL.study(n=n, log=lambda *a: None)
    blob = res.pop("blob")
    res["speed"] = CL.closure_speed(n, blob)
    res["metric"] = "relative L2 of log E(k), 2 <= k <= n/4, against the 2x box-filtered fine run"
    return res, blob


def vehicle_series(W, w, storage: str, closure: str, steps: int, every: int, blob=None, period: int = 32):
    """Drag (sum F_x) and lift (sum F_z) of the obstacles every `every` steps
    of a D3Q27 vehicle tunnel, and the step rate (MLUPS, CUDA events around
    the time loop; force evaluations excluded)."""
    import numpy as np
    import torch
    from asl_b200 import _lib as L
    from asl_b200 import lbgk as A
    lb, bcs = W.build_lbgk(w, storage=storage, compVel=False, compRho=False, fuse=True)
    if closure == "smagorinsky":
        lb.setClosure(L.CLOSURE_SMAGORINSKY, 0.17)
    elif closure == "learned":
        lb.setMLP(blob)
        lb.setMLPPeriod(period)
        lb.setClosure(L.CLOSURE_MLP)
    force = A.generateComputeSurfaceForce(lb, w.map)
    st = torch.cuda.ExternalStream(lb.stream)
    out, t = [], 0.0
    for _ in range(max(1, steps // every)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        lb.run(every, bcs, use_graph=True)
        e1.record(st)
        e1.synchronize()
        t += e0.elapsed_time(e1) / 1e3
        f = force.execute()
        out.append([int(lb.steps), float(f[0]), float(f[2])])
    del force, lb, bcs
    return np.array(out), w.cells * every * len(out) / t / 1e6


def vehicle_study(W, blob, small, small_steps: int, full_w, full_steps: int):
    """The D3Q27 vehicle configuration with closures and storage formats: on
    a downscaled tunnel the drag / lift series of FP32 Smagorinsky, FP16
    Smagorinsky and FP16 storage with the learned closure against FP64
    Smagorinsky (the reference), and at full size the step rates of FP32
    Smagorinsky and FP16 + learned closure."""
    import numpy as np

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))
    every = max(1, small_steps // 8)
    ws = W.vehicle_d3q27(size=small, steps=small_steps)
    ref, _ = vehicle_series(W, ws, "f64", "smagorinsky", small_steps, every)
    res = {"small": "%dx%dx%d" % tuple(small), "small_steps": small_steps, "reference": "f64 smagorinsky",
           "vs_reference": {}}
    for storage, closure in (("f32", "smagorinsky"), ("f16", "smagorinsky"), ("f16", "learned")):
        sr, _ = vehicle_series(W, ws, storage, closure, small_steps, every, blob)
        ok = bool(np.isfinite(sr).all())
        res["vs_reference"]["%s_%s" % (storage, closure)] = {
            "drag_rel_l2": rel(sr[:, 1], ref[:, 1]) if ok else None,
            "lift_rel_l2": rel(sr[:, 2], ref[:, 2]) if ok else None}
    res["full_cells"] = full_w.cells
    speed = {}
    for storage, closure in (("f32", "smagorinsky"), ("f16", "learned")):
        _, mlups = vehicle_series(W, full_w, storage, closure, full_steps, full_steps, blob)
        speed["%s_%s" % (storage, closure)] = mlups
    res["full_mlups"] = speed
    res["full_steps"] = full_steps
    res["f16_learned_speedup_vs_f32_smagorinsky"] = speed["f16_learned"] / speed["f32_smagorinsky"]
    return res


def fd_run(W, w, steps: int, peak: float):
    """FD advection-diffusion (aslb_fd) on the porous grid, reading the
    velocity field of the FP32 domain on its stream: device time per step of
    the FD kernel alone, d3q7 and d3q19 stencils. Algorithmic bytes per cell:
    read c (4) and the three velocity components (12), write c (4)."""
    import numpy as np
    import torch
    from asl_b200 import fd as FD
    lb, bcs = W.build_lbgk(w, storage="f32", fuse=True)
    lb.run(2, bcs)
    lb.sync()
    st = torch.cuda.ExternalStream(lb.stream)
    g = tuple(s + 2 for s in w.size)
    c = np.full(g, 0.5, dtype=np.float32)
    out = {}
    for q in (7, 19):
        fd = FD.generateFDAdvectionDiffusion(c, 0.05, lb, q)
        fd.execute(3)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fd.execute(steps)
        e1.record(st)
        e1.synchronize()
        tk = e0.elapsed_time(e1) / 1e3 / steps
        gbs = 20 * w.cells / tk / 1e9
        out["d3q%d" % q] = {"kernel_ms": tk * 1e3, "value": w.cells / tk / 1e6, "unit": "MLUPS",
                            "achieved_gbs": gbs, "frac_of_peak": gbs / peak, "steps": steps}
        fd.close()
    out["bytes_per_cell"] = 20
    out["note"] = ("FP32, velocity read from the LBGK's device field; d3q7: k_fd_step (32 x 8 cell tiles walking 32 "
                   "x planes); d3q19: k_fd_step_rb (64 x 16 tiles, 4 x 2 cells per thread, a ring of four "
                   "shared-memory planes, equal runs of planes per resident block)")
    del lb, bcs
    return out


def batch_run(W, n: int, steps: int, peak: float):
    """Many small domains (seeded channels of random size, viscosity, obstacle
    and inlet velocity): the batch (one persistent stream-collide launch per
    step for all domains plus one link launch per condition position, CUDA
    graph) against ASL's loop over the domains (execute + executeAll of each
    domain, one launch per domain and condition)."""
    import torch
    ws = W.batch_channels(n=n, steps=steps)
    cells = sum(w.cells for w in ws)
    batch, lbs, bcs = W.build_batch(ws, storage="f32", fuse=True)
    st = torch.cuda.ExternalStream(lbs[0].stream)
    batch.run(16, bcs)  # warm-up, long enough for the launch-shape tuner (2 steps per shape)
    batch.sync()
    torch.cuda.synchronize()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)  # the first domain's stream waits for the batch
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    t = timed(lambda: batch.run(steps, bcs))
    nk = min(steps, 200) // 2 * 2
    none = [[] for _ in lbs]
    batch.run(4, none)  # tables and graph for the stream-collide alone
    tk = timed(lambda: batch.run(nk, none)) / nk
    launches = 1 + max(sum(1 for b in bc if not b.fused) for bc in bcs)
    # ASL's loop: every domain and condition launched on its own
    sep_steps = max(2, min(steps, 100))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(sep_steps):
        for lb, bc in zip(lbs, bcs):
            lb.execute()
            for b in bc:
                b.execute()
    for lb in lbs:
        lb.sync()
    t_sep = time.perf_counter() - t0
    bpc = BYTES_PER_CELL[("f32", 19)]
    res = {"domains": n, "cells": cells, "steps": steps, "value": cells * steps / t / 1e6, "unit": "MLUPS",
           "ms_per_step": t / steps * 1e3, "launches_per_step": launches, "tiles_per_step": batch.tiles,
           "layout": "packed rows", "launch_shape": {"chosen": batch.shape,
                                                     "shapes": ["1 cell, 4 blocks/SM", "1 cell, 3", "1 cell, 2",
                                                                "2 cells, 3", "2 cells, 2"],
                                                     "tuning_ms_per_2_steps": batch.shape_times},
           "kernel_ms": tk * 1e3, "kernel_frac_of_peak": bpc * cells / tk / 1e9 / peak,
           "separate_launches": {"value": cells * sep_steps / t_sep / 1e6, "unit": "MLUPS", "steps": sep_steps,
                                 "launches_per_step": sum(1 + sum(b.kernels for b in bc) for bc in bcs),
                                 "timing": "host clock around the loop, device synchronised at both ends"}}
    batch.close()
    del lbs, bcs
    return res


def run_slabs(args):
    """N > 1: one (N x 512) x 256 x 256 porous channel cut into x slabs, one
    512 x 256 x 256 slab per GPU (weak scaling). Every step advances each
    slab's boundary planes, exchanges the faces with NCCL point-to-point
    operations while the interior planes run on a second stream, then unpacks
    (asl_b200.slabs.overlapped_step). Timed with CUDA events on each rank's
    domain stream, max over ranks."""
    import datetime
    import torch
    import torch.distributed as dist
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if "MASTER_ADDR" not in os.environ:  # one GPU without a launcher (--slabs)
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT="29517", RANK="0", WORLD_SIZE="1")
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from asl_b200 import _lib
    from asl_b200 import slabs as SL
    from asl_b200 import workloads as W
    _lib.check(_lib.load().aslb_set_device(local), "set_device")
    sx, sy, sz = parse_size(args.size)
    w = W.porous_channel(size=(sx * world, sy, sz))
    slab = SL.Slab(w, rank, world, storage=args.storage, fuse=True, compVel=False, compRho=False)
    lb = slab.lb
    K, Wm = args.steps, args.warmup
    peak, peak_kind = peak_hbm()

    def max_over_ranks(v: float) -> float:
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(Wm):
        SL.overlapped_step(slab, SL.nccl_transport)
    torch.cuda.synchronize()
    dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(slab.stream)
    for _ in range(K):
        SL.overlapped_step(slab, SL.nccl_transport)
    e1.record(slab.stream)
    e1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    dist.barrier()
    t = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    # the stream-collide alone on each rank's slab (no exchange), for the roofline
    nk = min(K, 200) // 2 * 2
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k0.record(slab.stream)
    lb.execute(nk)
    k1.record(slab.stream)
    k1.synchronize()
    tk = max_over_ranks(k0.elapsed_time(k1) / 1e3 / nk)
    cells_rank = slab.w.cells
    bpc = BYTES_PER_CELL[(args.storage, 19)]
    # end to end: every rank uploads its slab's populations from pinned host
    # memory, runs K steps with the exchange, and reads density and velocity back
    gx, gy, gz = (v + 2 for v in slab.w.size)
    L = gx * gy * gz
    f_host = torch.empty(19 * L, dtype=torch.float32, pin_memory=True)
    rho_host = torch.empty(L, dtype=torch.float32, pin_memory=True)
    u_host = torch.empty(3 * L, dtype=torch.float32, pin_memory=True)
    lib = lb.lib
    _lib.check(lib.aslb_lbgk_read(lb.h, _lib.FIELD_F, _lib.F32, f_host.data_ptr()), "read")
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(slab.stream)
    _lib.check(lib.aslb_lbgk_write(lb.h, _lib.FIELD_F, _lib.F32, f_host.data_ptr()), "write")
    for n in range(K):
        if n == K - 1:
            lb.requestMacro()
        SL.overlapped_step(slab, SL.nccl_transport)
    _lib.check(lib.aslb_lbgk_read(lb.h, _lib.FIELD_RHO, _lib.F32, rho_host.data_ptr()), "read")
    _lib.check(lib.aslb_lbgk_read(lb.h, _lib.FIELD_VELOCITY, _lib.F32, u_host.data_ptr()), "read")
    e1.record(slab.stream)
    e1.synchronize()
    t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    mass = torch.tensor([lb.moments()[0]], dtype=torch.float64, device="cuda")
    dist.all_reduce(mass)
    if rank == 0:
        achieved = bpc * cells_rank / tk / 1e9
        line = {"metric": METRIC, "value": w.cells * K / t / 1e6, "unit": "MLUPS", "n_gpus": world, "steps": K,
                "warmup": Wm, "ms_per_step": t / K * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": args.storage,
                "data": "synthetic (seeded random spheres, base seed 20261203)",
                "config": {"workload": w.name, "lattice": "D3Q19", "cells": w.cells, "storage": args.storage,
                           "cells_per_gpu": cells_rank, "fused_noslip": True,
                           "l2": "populations far exceed L2; no flush needed",
                           "parallelism": "x slabs over %d GPUs, NCCL face exchange overlapped with the interior"
                                          % world},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                             "kernel": "stream-collide of one slab, max over ranks", "bytes_per_cell": bpc,
                             "cells_per_launch": cells_rank, "kernel_ms": tk * 1e3},
                "cpu_baseline": None,
                "e2e": {"value": w.cells * K / t_e2e / 1e6, "unit": "MLUPS",
                        "h2d_bytes_per_step": world * 19 * L * 4 / K, "d2h_bytes_per_step": world * 4 * L * 4 / K,
                        "timed": "every rank: population upload from pinned host memory, K overlapped steps, "
                                 "density and velocity download; max over ranks"},
                "clocks": clk, "gpu_launches": K * 3 * world,
                "summary": {"exchange_overhead": t / K / tk - 1.0, "mass": float(mass.item())}}
        print(json.dumps(line), flush=True)
    del slab, lb
    torch.cuda.synchronize()
    dist.barrier()
    dist.destroy_process_group()
    return 0


def run_ours(args):
    rank, world, local = dist_env()
    if (world > 1 and not args.replicas) or args.slabs:
        return run_slabs(args)
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline_subprocess(args)
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from asl_b200 import _lib
    from asl_b200 import workloads as W

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    _lib.check(_lib.load().aslb_set_device(local), "set_device")
    w = W.porous_channel(size=parse_size(args.size))
    K, Wm = args.steps, args.warmup
    peak, peak_kind = peak_hbm()

    def timed_device_run(storage, fuse, variant=0):
        """Warm up (the two-step CUDA graph is recorded here), then time K
        steps of the whole time loop, then K' back-to-back launches of the
        stream-collide kernel alone, all with CUDA events on the domain's stream."""
        lb, bcs = W.build_lbgk(w, storage=storage, compVel=False, compRho=False, fuse=fuse)
        lb.setKernel(variant)
        st = torch.cuda.ExternalStream(lb.stream)
        lb.run(Wm, bcs, use_graph=True)
        lb.sync()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clocks = ClockSampler(local)
        clocks.start()
        time.sleep(0.3)
        e0.record(st)
        lb.run(K, bcs, use_graph=True)
        e1.record(st)
        e1.synchronize()
        torch.cuda.synchronize()
        clk = clocks.stop()
        barrier()
        t = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        nk = min(K, 200) // 2 * 2
        k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k0.record(st)
        lb.execute(nk)
        k1.record(st)
        k1.synchronize()
        tk = max_over_ranks(k0.elapsed_time(k1) / 1e3 / nk)
        bpc = BYTES_PER_CELL[(storage, 19)]
        res = {"value": w.cells * K * world / t / 1e6, "unit": "MLUPS", "ms_per_step": t / K * 1e3,
               "kernel_ms": tk * 1e3, "kernel_achieved_gbs": bpc * w.cells / tk / 1e9,
               "kernel_frac_of_peak": bpc * w.cells / tk / 1e9 / peak,
               "boundary_kernels_per_step": sum(b.kernels for b in bcs),
               "launches_per_step": 1 + sum(b.kernels for b in bcs)}
        return lb, bcs, res, clk, t, tk

    # Headline: FP32, no-slip walls and map fused into the stream-collide kernel.
    lb, bcs, head, clk, t, tk = timed_device_run(args.storage, True)
    mom = lb.moments()
    links = sum(b.num_links for b in bcs)

    # End to end through the C ABI: initial populations from pinned host memory,
    # the ASL time loop (execute + executeAll per step), rho/u back to pinned host memory.
    q = w.q
    gx, gy, gz = (s + 2 for s in w.size)
    L = gx * gy * gz
    f_host = torch.empty(q * L, dtype=torch.float32, pin_memory=True)
    rho_host = torch.empty(L, dtype=torch.float32, pin_memory=True)
    u_host = torch.empty(3 * L, dtype=torch.float32, pin_memory=True)
    lib = lb.lib
    _lib.check(lib.aslb_lbgk_read(lb.h, _lib.FIELD_F, _lib.F32, f_host.data_ptr()), "read")
    st = torch.cuda.ExternalStream(lb.stream)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    _lib.check(lib.aslb_lbgk_write(lb.h, _lib.FIELD_F, _lib.F32, f_host.data_ptr()), "write")
    for n in range(K):
        if n == K - 1:
            lb.requestMacro()
        lb.execute()
        for b in bcs:
            b.execute()
    _lib.check(lib.aslb_lbgk_read(lb.h, _lib.FIELD_RHO, _lib.F32, rho_host.data_ptr()), "read")
    _lib.check(lib.aslb_lbgk_read(lb.h, _lib.FIELD_VELOCITY, _lib.F32, u_host.data_ptr()), "read")
    e1.record(st)
    e1.synchronize()
    t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    e2e = {"value": w.cells * K * world / t_e2e / 1e6, "unit": "MLUPS",
           "h2d_bytes_per_step": q * L * 4 / K, "d2h_bytes_per_step": 4 * L * 4 / K,
           "timed": "upload of the populations from pinned host memory, K steps of execute()+executeAll(bc) "
                    "through the C ABI, density and velocity download to pinned host memory"}
    rho_np = rho_host.numpy().reshape(gx, gy, gz)
    finite = bool(np.isfinite(rho_np[1:-1, 1:-1, 1:-1]).all())
    del lb, bcs

    lb, bcs, direct, _, _, _ = timed_device_run(args.storage, True, variant=1)
    direct["note"] = "same step with the TMA-staged persistent stream-collide kernel"
    del lb, bcs
    lb, bcs, sep, _, _, _ = timed_device_run(args.storage, False)
    sep["note"] = "every condition as its own kernel after the step (ASL's execution order)"
    del lb, bcs
    fp16 = None
    if not args.no_fp16 and args.storage == "f32":
        lb, bcs, fp16, _, _, _ = timed_device_run("f16", True)
        mom16 = lb.moments()
        fp16["speedup_vs_f32"] = fp16["value"] / head["value"]
        fp16["mass_drift_vs_f32"] = abs(mom16[0] - mom[0]) / abs(mom[0])
        fp16["storage"] = "(f - 1) * 1024 in FP16, FP32 arithmetic"
        del lb, bcs

    accuracy = None
    if world == 1 and args.accuracy_steps > 0:
        accuracy = storage_accuracy(W, w, args.accuracy_steps)
    batched = None
    if world == 1 and args.batch_steps > 0:
        batched = batch_run(W, args.batch_domains, args.batch_steps, peak)
    learned, blob = None, None
    if world == 1 and args.closure_size > 0:
        learned, blob = closure_run(args.closure_size)
    vehicle = None
    if world == 1 and args.q27_steps > 0:
        vehicle, wv = vehicle_run(W, parse_size(args.q27_size), args.q27_steps, peak)
        if blob is not None and args.vehicle_study_steps > 0:
            vehicle["study"] = vehicle_study(W, blob, parse_size(args.vehicle_small), args.vehicle_study_steps, wv,
                                             args.q27_steps)
        del wv
    fdad = None
    if world == 1 and args.fd_steps > 0:
        fdad = fd_run(W, w, args.fd_steps, peak)

    bpc = BYTES_PER_CELL[(args.storage, w.q)]
    achieved = bpc * w.cells / tk / 1e9
    traffic = profile_traffic(f"stream_collide_d3q19_{args.storage}_porous.md", w.cells)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_source": peak_kind,
            "kernel": f"k_stream_collide<19,{args.storage}> (AA pattern, odd/even launches averaged)",
            "bytes_per_cell": bpc, "cells_per_launch": w.cells, "kernel_ms": tk * 1e3,
            "note": "algorithmic bytes: read + write of 19 populations per cell; the 8-byte fused-link "
                    "mask per cell is overhead and not counted"}

    if rank == 0:
        details = {"separate_conditions": sep, "tma_kernel": direct, "fp16": fp16, "accuracy": accuracy,
                   "d3q27_vehicle": vehicle, "batched_domains": batched, "learned_closure": learned,
                   "fd_advection_diffusion": fdad, "finite": finite, "mass": mom[0]}
        try:
            Path(args.details).write_text(json.dumps(details, indent=1))
        except OSError:
            pass
        line = {"metric": METRIC, "value": head["value"], "unit": "MLUPS", "n_gpus": world, "steps": K,
                "warmup": Wm, "ms_per_step": t / K * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": args.storage,
                "data": "synthetic (seeded random spheres, base seed 20261203)",
                "config": {"workload": w.name, "lattice": "D3Q19", "cells": w.cells, "storage": args.storage,
                           "solid_fraction": round(w.info["solid_fraction"], 4), "spheres": w.info["spheres"],
                           "boundary_links": links, "fused_noslip": True,
                           "l2": "populations (%.2f GB) far exceed L2; no flush needed" % (bpc / 2 * w.cells / 1e9),
                           "parallelism": "replica per GPU" if world > 1 else "single GPU",
                           "time_loop": "CUDA graph of two steps, replayed"},
                "roofline": roof, "cpu_baseline": cb, "e2e": e2e, "clocks": clk,
                "gpu_launches": K * head["launches_per_step"],
                "summary": summary(head, sep, fp16, accuracy, batched, learned, vehicle, fdad, finite)}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def _r(v, n=4):
    return None if v is None else float("%.*g" % (n, v))


def summary(head, sep, fp16, acc, batched, learned, vehicle, fdad, finite):
    """The other legs in a few numbers (full results in the details file),
    last in the JSON line so that a tail of it shows them."""
    out = {"f32_kernel_ms": _r(head["kernel_ms"]), "f32_frac": _r(head["kernel_frac_of_peak"], 3),
           "separate_conditions_mlups": _r(sep["value"])}
    if fp16:
        out["fp16"] = {"mlups": _r(fp16["value"]), "kernel_ms": _r(fp16["kernel_ms"]),
                       "frac": _r(fp16["kernel_frac_of_peak"], 3), "speedup_vs_f32": _r(fp16["speedup_vs_f32"], 3)}
    if acc:
        out["accuracy_vs_f64"] = {"steps": acc["steps"],
                                  "perm_err": {k: _r(v, 2) for k, v in acc["permeability_rel_err"].items()},
                                  "u_l2": {k: _r(v, 2) for k, v in acc["velocity_rel_l2"].items()}}
    if batched:
        out["batch"] = {"mlups": _r(batched["value"]), "kernel_frac": _r(batched["kernel_frac_of_peak"], 3),
                        "vs_separate": _r(batched["value"] / batched["separate_launches"]["value"], 3)}
    if learned:
        runs = learned["runs"]
        out["closure"] = {k: [_r(v, 2) for v in runs[k]["spectrum_rel_l2_logE"].values()]
                          for k in ("learned", "smagorinsky", "smagorinsky_fit")}
        out["closure"]["overhead"] = _r(learned["speed"]["learned_overhead_vs_smagorinsky"], 3)
    if vehicle:
        out["d3q27"] = {"mlups": _r(vehicle["value"]), "frac": _r(vehicle["kernel_frac_of_peak"], 3)}
        st = vehicle.get("study")
        if st:
            out["d3q27"]["drag_vs_f64"] = {k: _r(v["drag_rel_l2"], 2) for k, v in st["vs_reference"].items()}
            out["d3q27"]["f16_learned_speedup"] = _r(st["f16_learned_speedup_vs_f32_smagorinsky"], 3)
    if fdad:
        out["fd_frac"] = {k: _r(fdad[k]["frac_of_peak"], 3) for k in ("d3q7", "d3q19")}
    out["finite"] = finite
    return out


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
