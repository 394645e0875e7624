"""CPU pins of the closure oracle (oracle/mlp_oracle.py): its gradient
against finite differences, BF16 rounding known answers, and invariants of
known stress tensors. No GPU."""
import numpy as np

from oracle import mlp_oracle as M


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    P = M.param_count()
    p = rng.normal(0, 0.3, P)
    x = rng.normal(0, 1, (9, 40))
    t = rng.uniform(0, 0.05, 40)
    norm = np.concatenate([rng.normal(0, 0.1, 9), rng.uniform(0.5, 2, 9)])
    _, g = M.loss_and_grad(p, x, t, norm, 0.05)

    def mse(q):
        return M.loss_and_grad(q, x, t, norm, 0.05)[0] / x.shape[1]

    for i in list(rng.choice(P, 40, replace=False)) + [P - 1, 0, 64 * 9]:
        e = np.zeros(P)
        e[i] = 1e-6
        fd = (mse(p + e) - mse(p - e)) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_known_answers():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-3, 0.0])
    want = np.array([1.0, 1.0, 1.0 + 4 * 2 ** -8, -2.5, (1 + 3 / 128) * 2.0 ** -10, 0.0])
    assert np.array_equal(M.bf16(vals), want)


def test_features_of_known_stresses():
    rho = np.array([1.0, 2.0])
    u = np.zeros((3, 2))
    c = 0.01
    # isotropic: P = c rho I -> trace 3c, no deviatoric part
    P = [c * rho, c * rho, c * rho, 0 * rho, 0 * rho, 0 * rho]
    f = M.features(rho, *u, P)
    assert np.allclose(f[0], 3 * c) and np.allclose(f[2], 0) and np.allclose(f[4], c)
    # pure shear P01 = s rho: |p| = sqrt(2) s, det = 0, |u| = 0
    s = 0.02
    P = [0 * rho, 0 * rho, 0 * rho, s * rho, 0 * rho, 0 * rho]
    f = M.features(rho, *u, P)
    assert np.allclose(f[1], np.sqrt(2) * s) and np.allclose(f[4], 0, atol=1e-12) and np.allclose(f[8], 0)


def test_adam_first_step_moves_by_lr():
    p = np.zeros(5)
    g = np.array([1.0, -2.0, 0.5, 0.0, 3.0])
    q, m, v = M.adam(p, g, np.zeros(5), np.zeros(5), 1, 0.01)
    assert np.allclose(q[g != 0], -0.01 * np.sign(g[g != 0]), rtol=1e-6) and q[3] == 0
