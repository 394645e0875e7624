"""CPU oracle of the FD advection-diffusion step (test infrastructure only).

Restates ASL's FDAdvectionDiffusion update for one component
(src/num/aslFDAdvectionDiffusion.cxx:124-160) with the template operators
laplas, div and divProduct (src/math/aslTemplateVE.cxx:164-267) and the
d3q7 / d3q15 / d3q19 coefficients (src/math/aslTemplates.cxx:134-186), in
numpy over the interior of a ghosted field, in the field's precision.
Parity against the reference is unpinned (it cannot be built here); the
oracle is pinned by known answers in the tests (a linear field is a fixed
point of pure diffusion, mass conservation of a closed periodic-free blob
far from the faces, a uniform field advected by a constant velocity).
"""
from __future__ import annotations

import numpy as np

from oracle.oracle import lattice as _lattice


def template(q: int):
    """(vectors (q, 3), laplacian coefficients, gradient coefficients)."""
    c27, _, _ = _lattice(27)
    if q == 15:
        e, _, _ = _lattice(15)
    else:
        e = c27[:q]
    e = np.asarray(e, dtype=np.int64)
    n2 = (e * e).sum(1)
    if q == 7:
        lc = np.where(n2 == 0, -6.0, 1.0)
        gc = np.where(n2 == 0, 0.0, 0.5)
    elif q == 15:
        lc = np.where(n2 == 0, -14.0 / 3.0, np.where(n2 == 1, 2.0 / 3.0, 1.0 / 12.0))
        gc = np.where(n2 == 0, 0.0, np.where(n2 == 1, 1.0 / 3.0, 1.0 / 24.0))
    else:
        lc = np.where(n2 == 0, -4.0, np.where(n2 == 1, 1.0 / 3.0, 1.0 / 6.0))
        gc = np.where(n2 == 0, 0.0, np.where(n2 == 1, 1.0 / 6.0, 1.0 / 12.0))
    return e, lc, gc


def fd_step(c: np.ndarray, D: float, q: int, u: np.ndarray | None = None, cc: bool = False,
            electric=None) -> np.ndarray:
    """One step; returns the new field (ghosts copied unchanged)."""
    T = c.dtype.type
    e, lc, gc = template(q)
    gx, gy, gz = c.shape

    def sh(a, v):
        return a[1 + v[0]:gx - 1 + v[0], 1 + v[1]:gy - 1 + v[1], 1 + v[2]:gz - 1 + v[2]]

    cv = [sh(c, v) for v in e]
    lap = np.zeros_like(cv[0])
    for i in range(q):
        lap = lap + T(lc[i]) * cv[i]
    cnew = T(D) * lap + cv[0]
    if u is not None:
        u0 = [sh(u[d], e[0]) for d in range(3)]
        dp, dv = [], []
        for d in range(3):
            s = np.zeros_like(cv[0])
            v = np.zeros_like(cv[0])
            for i in range(1, q):
                if e[i][d] == 0:
                    continue
                ui = sh(u[d], e[i])
                coef = T(gc[i] * e[i][d])
                s = s + T(0.5) * ((ui + u0[d]) * (cv[i] + cv[0])) * coef
                v = v + coef * ui
            dp.append(s)
            dv.append(v)
        cnew = cnew - (dp[0] + dp[1] + dp[2])
        if cc:
            cnew = cnew / (T(1) - (dv[0] + dv[1] + dv[2]))
            cnew = cnew + lap * (u0[0] * u0[0] + u0[1] * u0[1] + u0[2] * u0[2]) * T(0.5)
    if electric is not None:  # (phi, k, charge): - divAgradB(c q / k, phi)
        phi, kk, qq = electric
        a0 = cv[0] * sh(qq, e[0]) / sh(kk, e[0])
        p0 = sh(phi, e[0])
        s = np.zeros_like(cv[0])
        for i in range(1, q):
            s = s + T(gc[i]) * (cv[i] * sh(qq, e[i]) / sh(kk, e[i]) + a0) * (sh(phi, e[i]) - p0)
        cnew = cnew - s
    out = c.copy()
    out[1:-1, 1:-1, 1:-1] = cnew
    return out


def fd_map_bc(c: np.ndarray, m: np.ndarray, q: int, gradient: bool, value: float) -> np.ndarray:
    """BCConstantValueMap / BCConstantGradientMap (src/num/aslBasicBC.cxx:71-108,
    271-350) on the guard cells -0.9999 < m <= 0: value, or the normal
    gradient ``value`` from fluid neighbours (m > 0, interior) of the
    template, weighted by (n.e/|e| + 1)^2 with n the unit map gradient
    (template gradient coefficients; m is -0.9 off the grid)."""
    T = c.dtype.type
    e, _, gc = template(q)
    g = c.shape
    out = c.copy()

    def mat(p):
        return float(m[p]) if all(0 <= p[a] < g[a] for a in range(3)) else -0.9
    for x in np.ndindex(*g):
        if not (m[x] <= 0 and m[x] > np.float32(-0.9999)):
            continue
        if not gradient:
            out[x] = T(value)
            continue
        nbs = [(k, tuple(x[a] + int(e[k][a]) for a in range(3))) for k in range(1, q)]
        n = sum(gc[k] * e[k].astype(float) * float(np.float32(mat(p))) for k, p in nbs)
        ln = np.linalg.norm(n)
        fluid = [(k, p) for k, p in nbs if all(1 <= p[a] <= g[a] - 2 for a in range(3)) and mat(p) > 0]
        if ln == 0 or not fluid:
            continue
        s = T(0)
        cnt = T(0)
        for k, p in fluid:
            dn = (n @ e[k]) / ln / np.linalg.norm(e[k])
            w = T((dn + 1) ** 2)
            s = s + (c[p] - T(dn) * T(value)) * w
            cnt = cnt + w
        if cnt > T(0.1):
            out[x] = s / cnt
    return out
