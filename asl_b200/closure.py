"""Learned LBGK closure: decaying periodic turbulence, training data from
filtered fine-grid runs of the solver itself, training with the library's
own kernels (aslb_mlp_grad / aslb_mlp_adam), and the energy-spectrum judge.

Pipeline (D3Q19, FP32):

1. ``turbulence_field``: a random-phase divergence-free field with
   E(k) ~ k^-5/3 on 2 <= k <= 32, scaled to u_rms = Ma c_s per component
   (Ma 0.1), built spectrally so that the same modes can be sampled on the
   coarse grid (n) and the fine grid (2n); the fine samples sit half a fine
   cell off so that a 2x2x2 box average is centred on a coarse cell.
2. The fine run (2n cubed, nu_fine = 2 nu under acoustic scaling, step 2t
   against the coarse step t; Smagorinsky at the fine grid scale, since plain
   BGK at tau = 0.501 does not stay stable for this field) is box-filtered
   by 2 at snapshot times.
3. Targets: the subgrid stress of the box filter, tau_ab = <u_a u_b> -
   <u_a><u_b>, projected on the filtered strain S (3^3-averaged
   least squares), nu_t = max(0, -tau^d : S / (2 S : S)), Cs^2 = nu_t / |S|
   (filter width 1 coarse cell).
4. Features: a coarse LBGK (Smagorinsky) restarted from the filtered
   velocity, advanced a few steps so its non-equilibrium stress settles;
   aslb_lbgk_closure_features gives the nine invariants per cell.
5. Training: mini-batch Adam on the GPU with the library's kernels.
6. Judge: relative L2 of log E(k), 2 <= k <= n/4, of coarse runs (no
   closure, Smagorinsky, learned) against the filtered fine run.

Torch supplies device memory and the FFT diagnostics (cuFFT); the solver,
the feature extraction, the network and its training are the library's.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from . import lbgk as A

OUT_SCALE = 0.05  # Cs^2 = OUT_SCALE * softplus(y)
MA = 0.1
CS_SMAG = 0.17


def _torch():
    import torch
    return torch


def turbulence_modes(n: int, seed: int, kmin: int = 2, kmax: int = 32):
    """Complex half-spectrum (3, n, n, n//2+1) of a solenoidal random-phase
    field with E(k) ~ k^-5/3 on kmin <= |k| <= kmax (unit-less amplitude)."""
    torch = _torch()
    g = torch.Generator().manual_seed(seed)
    kx = torch.fft.fftfreq(n, 1.0 / n)
    kz = torch.fft.rfftfreq(n, 1.0 / n)
    KX, KY, KZ = torch.meshgrid(kx, kx, kz, indexing="ij")
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    kk = torch.sqrt(k2)
    a = torch.randn((3, n, n, n // 2 + 1), generator=g, dtype=torch.float64) \
        + 1j * torch.randn((3, n, n, n // 2 + 1), generator=g, dtype=torch.float64)
    K = torch.stack([KX, KY, KZ])
    kdota = (K * a).sum(0)
    a = a - K * kdota / torch.where(k2 > 0, k2, torch.ones_like(k2))
    norm = torch.sqrt((a.abs() ** 2).sum(0))
    shell = (kk >= kmin) & (kk <= kmax)
    amp = torch.where(shell, kk.clamp(min=1.0) ** (-11.0 / 6.0), torch.zeros_like(kk))
    a = a / torch.where(norm > 0, norm, torch.ones_like(norm)) * amp
    return a


def sample_modes(modes, n_src: int, n: int, shift: float = 0.0):
    """Real field (3, n, n, n) of the modes of an n_src grid on an n grid
    (n >= n_src, zero padding), sampled at x_j = j + shift (grid units of n)."""
    torch = _torch()
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    modes = modes.to(dev)
    h = n_src // 2
    out = torch.zeros((3, n, n, n // 2 + 1), dtype=torch.complex128, device=dev)
    idx = list(range(0, h)) + list(range(n - h, n))
    src = list(range(0, h)) + list(range(n_src - h, n_src))
    ii = torch.tensor(idx, device=dev)
    ss = torch.tensor(src, device=dev)
    hz = torch.arange(h, device=dev)
    out[:, ii[:, None, None], ii[None, :, None], hz[None, None, :]] = \
        modes[:, ss[:, None, None], ss[None, :, None], hz[None, None, :]]
    if shift != 0.0:
        kx = torch.fft.fftfreq(n, 1.0 / n, device=dev)
        kz = torch.fft.rfftfreq(n, 1.0 / n, device=dev)
        ph = torch.exp(1j * 2 * math.pi * shift / n * (kx[:, None, None] + kx[None, :, None] + kz[None, None, :]))
        out = out * ph
    return (torch.fft.irfftn(out, s=(n, n, n), dim=(1, 2, 3)) * (n / n_src) ** 3).cpu()


def turbulence_field(n: int, seed: int, fine: bool = False):
    """Velocity (3, N, N, N) float64 numpy, N = n (coarse) or 2n (fine), with
    u_rms = Ma c_s per component measured on the coarse grid."""
    modes = turbulence_modes(n, seed)
    uc = sample_modes(modes, n, n)
    scale = MA / math.sqrt(3.0) / float(uc.pow(2).mean().sqrt())
    if not fine:
        return (uc * scale).numpy()
    return (sample_modes(modes, n, 2 * n, shift=-0.5) * scale).numpy()


def spectrum(u):
    """Shell-summed kinetic energy E(k), k = 0 .. n/2, of a periodic (3, n, n, n) field."""
    torch = _torch()
    t = u if isinstance(u, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(u))
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = t.to(dev, torch.float32)
    n = t.shape[-1]
    uh = torch.fft.rfftn(t, dim=(1, 2, 3)) / n ** 3
    e = 0.5 * (uh.abs() ** 2).sum(0)
    w = torch.full((n // 2 + 1,), 2.0, device=dev)
    w[0] = 1.0
    if n % 2 == 0:
        w[-1] = 1.0
    e = e * w
    kx = torch.fft.fftfreq(n, 1.0 / n, device=dev)
    kz = torch.fft.rfftfreq(n, 1.0 / n, device=dev)
    kk = torch.sqrt(kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2)
    b = torch.round(kk).long().clamp(max=n // 2)
    E = torch.zeros(n // 2 + 1, device=dev, dtype=torch.float64).index_add_(0, b.ravel(), e.ravel().double())
    return E.cpu().numpy()


def spectrum_error(E, E_ref, kmin=2, kmax=None):
    kmax = kmax or (len(E_ref) - 1) // 2
    a = np.log(E[kmin:kmax + 1])
    b = np.log(E_ref[kmin:kmax + 1])
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def box_filter2(u):
    """2x2x2 average of a (..., 2n, 2n, 2n) torch tensor."""
    s = u.shape
    return u.reshape(*s[:-3], s[-3] // 2, 2, s[-2] // 2, 2, s[-1] // 2, 2).mean(dim=(-5, -3, -1))


def _ghost(u):
    return np.pad(u, ((0, 0), (1, 1), (1, 1), (1, 1)), mode="wrap")


def make_lbgk(n: int, tau: float, u0, closure=L.CLOSURE_NONE, storage="f32", cs=CS_SMAG):
    lb = A.LBGK(A.Block((n, n, n)), (tau - 0.5) / 3.0, A.d3q19(), compVel=False, compRho=False, storage=storage,
                periodic=(True, True, True))
    if closure == L.CLOSURE_SMAGORINSKY:
        lb.setClosure(closure, cs)
    A.LBGKUtilities(lb).initF(_ghost(u0))
    return lb


def velocity(lb):
    """Interior velocity (3, n, n, n) float32 on the device, via one step that
    writes it (the step is taken)."""
    torch = _torch()
    lb.requestMacro()
    lb.run(1, use_graph=False)
    u = lb.getVelocity(np.float32)[:, 1:-1, 1:-1, 1:-1]
    return torch.from_numpy(np.ascontiguousarray(u)).cuda()


def strain(u):
    """Filtered strain S_ab (6, n, n, n), central differences, periodic."""
    torch = _torch()
    d = [[(torch.roll(u[a], -1, b) - torch.roll(u[a], 1, b)) * 0.5 for b in range(3)] for a in range(3)]
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]
    return torch.stack([0.5 * (d[a][b] + d[b][a]) for a, b in pairs])


def targets(uf):
    """Cs^2 per coarse cell from a fine (3, 2n, 2n, 2n) velocity: subgrid
    stress of the 2x box filter projected on the filtered strain."""
    torch = _torch()
    ub = box_filter2(uf)
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]
    tau = torch.stack([box_filter2(uf[a] * uf[b]) - ub[a] * ub[b] for a, b in pairs])
    tr = (tau[0] + tau[1] + tau[2]) / 3.0
    tau[0] -= tr
    tau[1] -= tr
    tau[2] -= tr
    S = strain(ub)
    wgt = torch.tensor([1, 1, 1, 2, 2, 2], device=S.device, dtype=S.dtype).view(6, 1, 1, 1)
    num = -(tau * S * wgt).sum(0)
    den = 2.0 * (S * S * wgt).sum(0)

    def avg3(f):
        f = f[None, None]
        f = torch.nn.functional.pad(f, (1, 1, 1, 1, 1, 1), mode="circular")
        return torch.nn.functional.avg_pool3d(f, 3, stride=1)[0, 0]

    nut = torch.clamp(avg3(num) / (avg3(den) + 1e-20), min=0.0)
    smag = torch.sqrt(den)  # |S| = sqrt(2 S:S)
    return torch.clamp(nut / (smag + 1e-12), 0.0, 0.2), ub


def features(lb):
    """(9, cells) float32 device tensor of the closure features."""
    torch = _torch()
    n = lb.block.size[0] * lb.block.size[1] * lb.block.size[2]
    out = torch.empty((9, n), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    lb.closureFeatures(out.data_ptr())
    return out


@dataclass
class TrainResult:
    params: np.ndarray
    norm: np.ndarray
    blob: bytes
    loss: list
    samples: int


def train(X, T, iters=1500, batch=16384, lr=1e-3, seed=0, init=None):
    """Mini-batch Adam on (X: 9 x N, T: N) device tensors with the library's
    training kernels. Returns the parameters, normalisation and packed net."""
    torch = _torch()
    lib = L.load()
    P = lib.aslb_mlp_param_count()
    mean = X.mean(dim=1)
    std = X.std(dim=1).clamp(min=1e-12)
    norm = torch.cat([mean, 1.0 / std]).float().contiguous()
    g = torch.Generator(device="cuda").manual_seed(seed)
    if init is None:
        rng = np.random.default_rng(seed)
        p = np.zeros(P, dtype=np.float32)
        p[:64 * 9] = rng.normal(0, math.sqrt(2.0 / 9), 64 * 9)
        o = 64 * 9 + 64
        p[o:o + 4096] = rng.normal(0, math.sqrt(2.0 / 64), 4096)
        o += 4096 + 64
        p[o:o + 64] = rng.normal(0, math.sqrt(1.0 / 64), 64)
        init = p
    params = torch.from_numpy(np.asarray(init, dtype=np.float32)).cuda()
    m = torch.zeros(P, device="cuda")
    v = torch.zeros(P, device="cuda")
    grad = torch.zeros(P + 1, device="cuda")
    scratch = torch.zeros(lib.aslb_mlp_grad_scratch_floats(), device="cuda")
    N = X.shape[1]
    st = torch.cuda.current_stream().cuda_stream
    losses = []
    for it in range(iters):
        idx = torch.randint(0, N, (batch,), device="cuda", generator=g)
        xb = X[:, idx].contiguous()
        tb = T[idx].contiguous()
        L.check(lib.aslb_mlp_grad(params.data_ptr(), xb.data_ptr(), tb.data_ptr(), batch, norm.data_ptr(),
                                  OUT_SCALE, scratch.data_ptr(), grad.data_ptr(), C.c_void_p(st)), "mlp_grad")
        L.check(lib.aslb_mlp_adam(params.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(), it + 1, lr, 0.9,
                                  0.999, 1e-8, C.c_void_p(st)), "mlp_adam")
        if it % 100 == 0 or it == iters - 1:
            losses.append((it, float(grad[P].item()) / batch))
    p_host = params.cpu().numpy()
    n_host = norm.cpu().numpy()
    blob = pack(p_host, n_host)
    return TrainResult(p_host, n_host, blob, losses, N)


def pack(params, norm, out_scale=OUT_SCALE) -> bytes:
    lib = L.load()
    buf = C.create_string_buffer(int(lib.aslb_mlp_layout_bytes()))
    p = np.ascontiguousarray(params, dtype=np.float32)
    nm = np.ascontiguousarray(norm, dtype=np.float32)
    L.check(lib.aslb_mlp_pack(p.ctypes.data_as(C.c_void_p), nm.ctypes.data_as(C.c_void_p), float(out_scale),
                              C.cast(buf, C.c_void_p)), "mlp_pack")
    return buf.raw


def study(n=256, seed=20261207, times=(250, 500, 1000), train_times=(200, 400, 600), settle=8, iters=1500,
          period=32, log=print):
    """The whole closure study at coarse size n (fine 2n). Returns a dict."""
    torch = _torch()
    import time
    res = {"n": n, "fine": 2 * n, "seed": seed, "times": list(times)}
    tau_c, tau_f = 0.5005, 0.501
    # fine run: snapshots for training (2 t) and for the judge (2 t)
    t0 = time.perf_counter()
    uf0 = turbulence_field(n, seed, fine=True)
    fine = make_lbgk(2 * n, tau_f, uf0, closure=L.CLOSURE_SMAGORINSKY)
    del uf0
    snap = sorted(set(2 * t for t in times) | set(2 * t for t in train_times))
    ref_E, train_sets = {}, []
    for s in snap:
        fine.run(s - 1 - fine.steps, use_graph=True)
        uf = velocity(fine)
        assert fine.steps == s
        if s // 2 in train_times:
            cs2, ub = targets(uf)
            train_sets.append((s // 2, cs2.reshape(-1).float(), ub.cpu().numpy().astype(np.float64)))
        if s // 2 in times:
            ref_E[s // 2] = spectrum(box_filter2(uf))
        del uf
        torch.cuda.empty_cache()
    del fine
    res["fine_seconds"] = time.perf_counter() - t0
    log("fine run done %.1f s" % res["fine_seconds"])
    # features: coarse Smagorinsky LBGK restarted from the filtered fields
    Xs, Ts = [], []
    for t, cs2, ub in train_sets:
        lb = make_lbgk(n, tau_c, ub, closure=L.CLOSURE_SMAGORINSKY)
        lb.run(settle, use_graph=False)
        Xs.append(features(lb))
        Ts.append(cs2)
        del lb
    X = torch.cat(Xs, dim=1)
    T = torch.cat(Ts)
    del Xs, Ts, train_sets
    ok = torch.isfinite(X).all(0) & torch.isfinite(T)
    X, T = X[:, ok].contiguous(), T[ok].contiguous()
    if T.numel() == 0:
        raise RuntimeError("closure study: no finite training samples (the fine run diverged)")
    res["train_samples"] = int(T.numel())
    res["target_mean_cs2"] = float(T.mean())
    t1 = time.perf_counter()
    tr = train(X, T, iters=iters)
    res["train_seconds"] = time.perf_counter() - t1
    res["train_loss"] = tr.loss
    # a constant-Cs^2 baseline on the same data: the loss the network must beat
    res["const_loss"] = float(((T - T.mean()) ** 2).mean())
    res["smag_loss"] = float(((T - CS_SMAG ** 2) ** 2).mean())
    del X, T
    log("trained: loss %s (constant %.3g, Smagorinsky %.3g)" % (tr.loss[-1], res["const_loss"], res["smag_loss"]))
    # judge: coarse runs from the coarse field. "smagorinsky_fit" uses the
    # constant Cs^2 that best fits the same targets (their mean): what the
    # network adds beyond calibrating one constant.
    uc0 = turbulence_field(n, seed)
    cs_fit = math.sqrt(res["target_mean_cs2"])
    res["cs_fit"] = cs_fit
    runs = {}
    for name in ("none", "smagorinsky", "smagorinsky_fit", "learned"):
        smag = name.startswith("smagorinsky")
        lb = make_lbgk(n, tau_c, uc0, closure=L.CLOSURE_SMAGORINSKY if smag else L.CLOSURE_NONE,
                       cs=cs_fit if name == "smagorinsky_fit" else CS_SMAG)
        if name == "learned":
            lb.setMLP(tr.blob)
            lb.setMLPPeriod(period)
            lb.setClosure(L.CLOSURE_MLP)
        errs = {}
        te = time.perf_counter()
        for t in times:
            lb.run(t - 1 - lb.steps, use_graph=True)
            u = velocity(lb)
            E = spectrum(u)
            errs[t] = spectrum_error(E, ref_E[t]) if np.all(np.isfinite(E)) else float("nan")
        runs[name] = {"spectrum_rel_l2_logE": errs, "seconds": time.perf_counter() - te}
        del lb
    res["runs"] = runs
    res["blob"] = tr.blob
    return res


def closure_speed(n: int, blob: bytes, steps: int = 192, period: int = 32, seed: int = 20261207):
    """MLUPS of the plain, Smagorinsky and learned steps on an n^3 periodic
    turbulence field (CUDA graph, CUDA events on the domain's stream)."""
    torch = _torch()
    u0 = turbulence_field(n, seed)
    out = {}
    for name in ("plain", "smagorinsky", "learned"):
        lb = make_lbgk(n, 0.5005, u0, closure=L.CLOSURE_SMAGORINSKY if name == "smagorinsky" else L.CLOSURE_NONE)
        if name == "learned":
            lb.setMLP(blob)
            lb.setMLPPeriod(period)
            lb.setClosure(L.CLOSURE_MLP)
        st = torch.cuda.ExternalStream(lb.stream)
        lb.run(2 * period, use_graph=True)
        lb.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        lb.run(steps, use_graph=True)
        e1.record(st)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        out[name] = {"mlups": n ** 3 * steps / t / 1e6, "ms_per_step": t / steps * 1e3}
        del lb
    out["learned_overhead_vs_smagorinsky"] = out["smagorinsky"]["mlups"] / out["learned"]["mlups"] - 1.0
    out["period"] = period
    out["steps"] = steps
    return out


def _main(argv=None):
    """python -m asl_b200.closure study [--n N] | speed [--n N] [--steps K]"""
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m asl_b200.closure")
    ap.add_argument("what", choices=["study", "speed"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=192)
    ap.add_argument("--period", type=int, default=32)
    a = ap.parse_args(argv)
    if a.what == "study":
        res = study(n=a.n, period=a.period)
        res.pop("blob")
    else:
        # the step rate does not depend on the weights: a seeded random network
        rng = np.random.default_rng(5)
        p = rng.normal(0, 0.1, L.load().aslb_mlp_param_count()).astype(np.float32)
        blob = pack(p, np.concatenate([np.zeros(9), np.ones(9)]).astype(np.float32))
        res = closure_speed(a.n, blob, steps=a.steps, period=a.period)
    print(json.dumps(res))


if __name__ == "__main__":
    _main()
