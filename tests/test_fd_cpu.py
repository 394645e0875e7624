"""CPU tests: the FD advection-diffusion oracle against known answers."""
import numpy as np
import pytest

from oracle.fd_oracle import fd_step, template


@pytest.mark.parametrize("q", [7, 15, 19])
def test_template_moments(oracle_mod, q):
    e, lc, gc = template(q)
    assert abs(lc.sum()) < 1e-14                                   # lap(const) = 0
    assert np.allclose((gc[:, None] * e).sum(0), 0)                # grad(const) = 0
    assert np.allclose((gc[:, None, None] * e[:, :, None] * e[:, None, :]).sum(0), np.eye(3))  # grad(x) = 1
    assert np.allclose((lc[:, None, None] * e[:, :, None] * e[:, None, :]).sum(0), 2 * np.eye(3))  # lap(x^2) = 2


@pytest.mark.parametrize("q", [7, 15, 19])
def test_linear_field_known_answers(oracle_mod, q):
    g = (9, 8, 7)
    x, y, z = np.meshgrid(*[np.arange(n, dtype=float) for n in g], indexing="ij")
    c = 0.3 + 0.01 * x - 0.02 * y + 0.005 * z
    # pure diffusion: a linear field is a fixed point
    assert np.allclose(fd_step(c, 0.1, q), c, atol=1e-15)
    # constant velocity U: c' = c - U.grad(c) (central, exact on a linear field)
    U = np.array([0.02, -0.01, 0.03])
    u = np.stack([np.full(g, U[d]) for d in range(3)])
    got = fd_step(c, 0.1, q, u)
    want = c - (U @ np.array([0.01, -0.02, 0.005]))
    assert np.allclose(got[1:-1, 1:-1, 1:-1], want[1:-1, 1:-1, 1:-1], atol=1e-15)
    # a uniform field stays uniform under a constant velocity
    assert np.allclose(fd_step(np.full(g, 0.7), 0.1, q, u), 0.7, atol=1e-15)


def test_diffusion_conserves_mass_away_from_faces(oracle_mod):
    g = (20, 20, 20)
    x, y, z = np.meshgrid(*[np.arange(n, dtype=float) for n in g], indexing="ij")
    c = np.exp(-((x - 10) ** 2 + (y - 9.5) ** 2 + (z - 10.2) ** 2) / 1.0)
    m0 = c.sum()
    for _ in range(5):
        c = fd_step(c, 0.1, 19)
    assert abs(c.sum() - m0) < 1e-10 * m0  # summation rounding only


def test_map_conditions_known_answers(oracle_mod):
    """A flat wall (solid for x <= 3.5): the zero-gradient condition copies
    the fluid neighbours' value when they agree; a gradient condition shifts
    it by the normal component; the value condition sets the guard cells."""
    from oracle.fd_oracle import fd_map_bc
    g = (10, 8, 8)
    x = np.arange(g[0], dtype=float)[:, None, None] * np.ones(g)
    m = np.clip((x - 3.5) / 1.8, -1, 1).astype(np.float32)   # normal +x
    c = np.full(g, 0.4)
    guard = (m <= 0) & (m > -0.9999)
    out = fd_map_bc(c, m, 7, True, 0.0)
    has_fluid = guard & (x == 3)
    assert np.allclose(out[has_fluid & (np.arange(g[1])[None, :, None] > 0) & (np.arange(g[1])[None, :, None] < g[1] - 1)
                           & (np.arange(g[2])[None, None, :] > 0) & (np.arange(g[2])[None, None, :] < g[2] - 1)], 0.4)
    # d3q7: the only fluid neighbour of x = 3 is x = 4 (n . e = 1, W = 4): c = c(4) - value
    out = fd_map_bc(c, m, 7, True, 0.1)
    assert np.allclose(out[3, 1:-1, 1:-1], 0.3)
    out = fd_map_bc(c, m, 19, False, 0.9)
    assert np.all(out[guard] == 0.9) and np.all(out[~guard] == 0.4)
