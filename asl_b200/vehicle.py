"""The D3Q27 vehicle tunnel with closures and storage formats compared:
drag / lift time series of the seeded obstacles (workloads.vehicle_d3q27)
for

  * FP32 populations with Smagorinsky (Cs 0.17),
  * FP16 populations with the learned closure (network trained by
    closure.study on decaying turbulence),
  * and, on a downscaled tunnel, FP64 Smagorinsky as the reference the
    others' series are measured against.

    python -m asl_b200.vehicle [--steps 10000] [--every 250] [--full 768,384,384] [--small 192,96,96]
"""
from __future__ import annotations

import json
import time

import numpy as np

from . import _lib as L
from . import lbgk as A
from . import workloads as W


def series(w, storage: str, closure: str, steps: int, every: int, blob: bytes | None = None, period: int = 32):
    """Run `steps` steps, recording (step, drag = sum F_x, lift = sum F_z)
    every `every` steps. Returns the series and the step rate (MLUPS, CUDA
    events around the time loop, force evaluations excluded)."""
    import torch
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
    for _ in range(steps // every):
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


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def study(steps=10000, every=250, full=(768, 384, 384), small=(192, 96, 96), blob=None, log=print):
    res = {"steps": steps, "every": every, "full": list(full), "small": list(small)}
    if blob is None:
        from . import closure as CL
        t0 = time.perf_counter()
        r = CL.study(n=128, log=lambda *a: None)
        blob = r["blob"]
        res["network"] = {"trained_on": "decaying turbulence 128^3 / filtered 256^3", "seconds": time.perf_counter() - t0}
    ws = W.vehicle_d3q27(size=small, steps=steps)
    ref, _ = series(ws, "f64", "smagorinsky", steps, every)
    res["small_reference"] = {"storage": "f64", "closure": "smagorinsky", "series": ref.tolist()}
    res["small"] = {}
    for storage, closure in (("f32", "smagorinsky"), ("f16", "smagorinsky"), ("f32", "learned"), ("f16", "learned")):
        s, mlups = series(ws, storage, closure, steps, every, blob)
        fin = bool(np.isfinite(s).all())
        res["small"]["%s_%s" % (storage, closure)] = {
            "finite": fin, "drag_rel_l2": rel_l2(s[:, 1], ref[:, 1]) if fin else None,
            "lift_rel_l2": rel_l2(s[:, 2], ref[:, 2]) if fin else None, "mlups": mlups}
        log(storage, closure, res["small"]["%s_%s" % (storage, closure)])
    wf = W.vehicle_d3q27(size=full, steps=steps)
    res["full_cells"] = wf.cells
    res["full"] = {}
    for storage, closure in (("f32", "smagorinsky"), ("f16", "learned")):
        s, mlups = series(wf, storage, closure, steps, every, blob)
        res["full"]["%s_%s" % (storage, closure)] = {"mlups": mlups, "finite": bool(np.isfinite(s).all()),
                                                    "series": s.tolist()}
        log(storage, closure, "full", mlups)
    a, b = res["full"]["f16_learned"], res["full"]["f32_smagorinsky"]
    if a["finite"] and b["finite"]:
        sa, sb = np.array(a["series"]), np.array(b["series"])
        res["full_f16_learned_vs_f32_smagorinsky"] = {"drag_rel_l2": rel_l2(sa[:, 1], sb[:, 1]),
                                                      "lift_rel_l2": rel_l2(sa[:, 2], sb[:, 2]),
                                                      "speedup": a["mlups"] / b["mlups"]}
    return res


def _main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(prog="python -m asl_b200.vehicle")
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--every", type=int, default=250)
    ap.add_argument("--full", default="768,384,384")
    ap.add_argument("--small", default="192,96,96")
    a = ap.parse_args(argv)
    sz = lambda s: tuple(int(v) for v in s.split(","))
    print(json.dumps(study(a.steps, a.every, sz(a.full), sz(a.small))))


if __name__ == "__main__":
    _main()
