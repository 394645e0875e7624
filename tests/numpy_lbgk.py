"""A second, independent restatement of ASL's LBGK step in numpy (test helper).

Used only to cross-check the C++ oracle on tiny domains; written from the
reference formulas (src/num/aslLBGK.cxx:187-235, src/num/aslLBGKBC.cxx:91-432,
691-736, src/num/aslBCond.cxx:373-493 of AvtechScientific/ASL) without
sharing code with the oracle. Ghost-cell semantics match the oracle's: ghost
cells are neither streamed nor collided.
"""
from __future__ import annotations

import numpy as np

V27 = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (-1, 0, 0), (0, -1, 0), (0, 0, -1), (1, 1, 0), (1, -1, 0),
       (-1, -1, 0), (-1, 1, 0), (0, 1, 1), (0, 1, -1), (0, -1, -1), (0, -1, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1),
       (-1, 0, 1), (1, 1, 1), (1, 1, -1), (1, -1, 1), (1, -1, -1), (-1, 1, 1), (-1, 1, -1), (-1, -1, 1),
       (-1, -1, -1)]


def lattice(q):
    c = np.array(V27[:7] + V27[19:] if q == 15 else V27[:q])
    n2 = (c * c).sum(1)
    if q == 15:
        lc = np.where(n2 == 0, -14 / 3, np.where(n2 == 1, 2 / 3, 1 / 12))
        w = lc / 6 + (n2 == 0)
    elif q == 19:
        lc = np.where(n2 == 0, -4.0, np.where(n2 == 1, 1 / 3, 1 / 6))
        w = lc / 6 + (n2 == 0)
    else:
        w = np.select([n2 == 0, n2 == 1, n2 == 2], [8 / 27, 2 / 27, 1 / 54], 1 / 216)
    inv = np.array([int(np.where((c == -c[i]).all(1))[0][0]) for i in range(q)])
    return c, w.astype(float), inv


class NumpyLBGK:
    def __init__(self, size, q, nu, periodic=(False, False, False), compressible=True):
        self.N = tuple(size)
        self.G = tuple(n + 2 for n in size)
        self.q = q
        self.c, self.w, self.inv = lattice(q)
        self.nu = nu
        self.periodic = periodic
        self.compressible = compressible
        self.g = np.zeros(3)
        self.Om = None
        self.closure = 0
        self.cs = 0.17
        self.f = np.ones((q, *self.G))
        self.rho = np.ones(self.G)
        self.u = np.zeros((3, *self.G))

    def wrap(self, v, a):
        if not self.periodic[a]:
            return v
        n = self.N[a]
        return np.where(v < 1, v + n, np.where(v > n, v - n, v))

    def init_f(self, rho, u):
        rho = np.broadcast_to(np.asarray(rho, float), self.G)
        u = np.asarray(u, float)
        u = np.broadcast_to(u.reshape(3, 1, 1, 1) if u.ndim == 1 else u, (3, *self.G))
        for i in range(self.q):
            cu = sum(self.c[i, d] * u[d] for d in range(3))
            self.f[i] = rho * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * (u * u).sum(0))
        self.rho[...] = rho
        self.u[...] = u

    def interior_index(self, shift):
        idx = []
        for a in range(3):
            v = np.arange(1, self.N[a] + 1) + shift[a]
            idx.append(self.wrap(v, a))
        return np.ix_(*idx)

    def step(self):
        q, c, w = self.q, self.c, self.w
        I = self.interior_index((0, 0, 0))
        fo = np.stack([self.f[i][self.interior_index(-c[i])] for i in range(q)])
        m = np.stack([(fo * (w * c[:, d])[:, None, None, None]).sum(0) for d in range(3)])
        rho = (fo * w[:, None, None, None]).sum(0)
        om0 = 1.0 / (3 * self.nu + 0.5)
        om = om0
        if self.Om is not None:
            k = 2.0 / om
            O = self.Om
            m[0] = m[0] + k * (O[1] * m[2] - O[2] * m[1])
            m[1] = m[1] + k * (O[2] * m[0] - O[0] * m[2])
            m[2] = m[2] + k * (O[0] * m[1] - O[1] * m[0])
        if np.any(self.g != 0):
            m = m + 0.5 * rho[None] * self.g.reshape(3, 1, 1, 1)
        self.rho[I] = rho
        self.u[(slice(None),) + I] = m / rho if self.compressible else m
        mm = (m * m).sum(0)
        cm = np.stack([sum(c[i, d] * m[d] for d in range(3)) for i in range(q)])
        if self.compressible:
            feq = rho + 3 * cm + 4.5 * cm * cm / rho - 1.5 * mm / rho
        else:
            feq = rho + 3 * cm + 4.5 * cm * cm - 1.5 * mm
        if self.closure == 1:
            wl = 4 * ((fo - feq) ** 2).sum(0) / (fo * fo).sum(0)
            om = np.where(wl > 1, 1.0 / (3 * np.minimum(self.nu * wl, 0.5) + 0.5), om0)
        elif self.closure == 2:
            d = (fo - feq) * w[:, None, None, None]
            P = np.einsum("i...,ia,ib->ab...", d, c.astype(float), c.astype(float))
            q2 = (P * P).sum((0, 1))
            tau0 = 1 / om0
            tau = 0.5 * (tau0 + np.sqrt(tau0 ** 2 + 18 * np.sqrt(2) * self.cs ** 2 * np.sqrt(q2) / rho))
            om = 1 / tau
        fn = fo * (1 - om) + om * feq
        if np.any(self.g != 0):
            u = m / rho
            for i in range(q):
                cu = sum(c[i, d] * u[d] for d in range(3))
                src = sum((3 * (c[i, d] - u[d]) + 9 * cu * c[i, d]) * self.g[d] for d in range(3))
                fn[i] = fn[i] + (1 - 0.5 * om) * rho * src
        for i in range(q):
            self.f[i][I] = fn[i]

    # --- boundary conditions ---
    def slice_links(self, walls):
        """(p, k) pairs of addSlice* for walls in X0,XE,Y0,YE,Z0,ZE order."""
        normals = {"X0": 1, "XE": 4, "Y0": 2, "YE": 5, "Z0": 3, "ZE": 6}
        out = []
        for wname in ["X0", "XE", "Y0", "YE", "Z0", "ZE"]:
            if wname not in walls:
                continue
            ax = "XYZ".index(wname[0])
            layer = 1 if wname[1] == "0" else self.G[ax] - 2
            n = self.c[normals[wname]]
            t = [a for a in range(3) if a != ax]
            for k in range(1, self.q):
                if self.c[k] @ n <= 0:
                    continue
                for i in range(1, self.G[t[0]] - 1):
                    for j in range(1, self.G[t[1]] - 1):
                        a = [0, 0, 0]
                        a[ax], a[t[0]], a[t[1]] = layer, i, j
                        out.append((tuple(np.array(a) - self.c[k]), k))
        return out

    def apply_slice(self, kind, walls, p=0.0, u=(0, 0, 0)):
        u = np.asarray(u, float)
        for pt, k in self.slice_links(walls):
            q = tuple(np.array(pt) + self.c[k])
            tgt = tuple(int(self.wrap(np.array(pt[a]), a)) for a in range(3))
            cu = self.c[k] @ u
            if kind == "noslip":
                v = self.f[self.inv[k]][q]
            elif kind == "velocity":
                v = self.f[self.inv[k]][q] + 6 * cu
            elif kind == "pressure":
                v = p
            else:
                v = p + 3 * cu
            self.f[k][tgt] = v

    def _map(self, m, x):
        if any(x[a] < 0 or x[a] >= self.G[a] for a in range(3)):
            return -0.9
        return m[x]

    def _interior(self, x):
        return all(1 <= x[a] <= self.N[a] for a in range(3))

    def _nb(self, x, k):
        return tuple(int(self.wrap(np.array(x[a] + self.c[k, a]), a)) for a in range(3))

    def _skip(self, x):
        return any(self.periodic[a] and not (1 <= x[a] <= self.N[a]) for a in range(3))

    def apply_map(self, kind, m, p=0.0, u=(0, 0, 0), lf=0.0, beta=0.0, cd=None):
        m = np.asarray(m, np.float32)
        u = np.asarray(u, float)
        writes = []
        for x in np.ndindex(*self.G):
            if self._skip(x):
                continue
            if not (m[x] <= 0 and m[x] > np.float32(-0.9999)):
                continue
            ks = [k for k in range(1, self.q) if self._interior(self._nb(x, k)) and self._map(m, self._nb(x, k)) > 0
                  and (cd is None or cd[self._nb(x, k)] > 0)]
            if not ks:
                continue
            if kind == "noslip":
                for k in ks:
                    writes.append((k, x, self.f[self.inv[k]][self._nb(x, k)]))
            elif kind == "velocity":
                coef = sum(self.w[k] for k in ks)
                rb = sum(self.f[self.inv[k]][self._nb(x, k)] * self.w[k] for k in ks) / coef
                for k in ks:
                    writes.append((k, x, rb + 3 * rb * (u @ self.c[k])))
            elif kind == "pressure_velocity":
                for k in ks:
                    cu = u @ self.c[k]
                    fe = p + 3 * p * cu + 4.5 * p * cu * cu - 1.5 * p * (u @ u)
                    writes.append((k, x, fe))
            elif kind in ("transport_deposition", "kinetics_deposition"):
                # p is p0: transport limited j = rho - (rho - coef p0) / (1 + coef lf),
                # kinetics limited j = rho - beta (rho / coef - p0) / (1 + lf)
                coef = sum(self.w[k] for k in ks)
                rho = sum(self.f[self.inv[k]][self._nb(x, k)] * self.w[k] for k in ks)
                if kind == "transport_deposition":
                    j = rho - (rho - coef * p) / (1 + coef * lf)
                else:
                    j = rho - beta * (rho / coef - p) / (1 + lf)
                for k in ks:
                    writes.append((k, x, j / coef))
        for k, x, v in writes:
            self.f[k][x] = v

    def flux(self, m):
        """Surface flux field and total (ComputeSurfaceFluxMap)."""
        m = np.asarray(m, np.float32)
        F = np.zeros(self.G)
        for x in np.ndindex(*self.G):
            if self._skip(x) or not (abs(m[x]) < np.float32(0.9999)):
                continue
            for k in range(1, self.q):
                nb = self._nb(x, k)
                mk = self._map(m, nb)
                b0 = m[x] <= 0 and mk > 0 and self._interior(nb)
                bi = mk <= 0 and m[x] > 0 and self._interior(x)
                if b0:
                    F[x] += (self.f[k][x] - self.f[self.inv[k]][nb]) * self.w[k]
                elif bi:
                    F[x] += (self.f[self.inv[k]][nb] - self.f[k][x]) * self.w[k]
        return F, F.sum()

    def force(self, m, r0=(0, 0, 0)):
        m = np.asarray(m, np.float32)
        F = np.zeros((3, *self.G))
        for x in np.ndindex(*self.G):
            if self._skip(x) or not (abs(m[x]) < np.float32(0.9999)):
                continue
            for k in range(1, self.q):
                nb = self._nb(x, k)
                mk = self._map(m, nb)
                b0 = m[x] <= 0 and mk > 0 and self._interior(nb)
                bi = mk <= 0 and m[x] > 0 and self._interior(x)
                if not (b0 or bi):
                    continue
                a = self.f[k][x] + self.f[self.inv[k]][nb] - 2
                F[:, x[0], x[1], x[2]] += (a if b0 else -a) * self.w[k] * self.c[k]
        pos = np.stack(np.meshgrid(*[np.arange(g) - 1.0 for g in self.G], indexing="ij")) - np.asarray(
            r0, float).reshape(3, 1, 1, 1)
        tot = F.reshape(3, -1).sum(1)
        tq = np.cross(pos.reshape(3, -1).T, F.reshape(3, -1).T).sum(0)
        return np.concatenate([tot, tq]), F
