"""The FP64 adjoint restatement (oracle/adjoint_oracle.py) pinned on CPU:
its forward map is the oracle's real-time RK4 step, and its gradient matches
central finite differences of its own loss."""
import numpy as np

import adjoint_oracle as ad
import oracle_py as orc
from fgpe_b200 import grid_axes, make_config


def small_problem(nsteps=12, n=16, nctrl=4, seed=3):
    cfg = make_config((n, n, 1), (5.0, 5.0, 1.0), dt=2e-3, g=30.0)
    x, y, _ = grid_axes(cfg)
    Y, X = np.meshgrid(y, x, indexing="ij")
    V0 = (0.5 * (X ** 2 + Y ** 2) + 0j).reshape(1, n, n)
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-2, 2, size=(nctrl, 2))
    G = np.stack([np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / 2.0) for cx, cy in centres]).reshape(nctrl, 1, n, n)
    psi0 = np.exp(-(X ** 2 + Y ** 2) / 2.0) * (1 + 0.05j * X)
    psi0 = psi0 / np.sqrt(np.sum(np.abs(psi0) ** 2) * cfg.dx[0] * cfg.dx[1] * cfg.dx[2])
    target = X * np.exp(-(X ** 2 + Y ** 2) / 2.0) + 0j
    target = target / np.sqrt(np.sum(np.abs(target) ** 2) * cfg.dx[0] * cfg.dx[1] * cfg.dx[2])
    u = rng.normal(0.0, 0.1, size=(nsteps, nctrl))
    prob = ad.ControlProblem(cfg, V0, G, psi0.reshape(1, n, n), target.reshape(1, n, n))
    return cfg, prob, u, V0


def test_forward_matches_oracle_real_time_step():
    # with u = 0 the control problem's step is the oracle's real-time RK4 step
    cfg, prob, u, V0 = small_problem()
    o = orc.OracleSolver(cfg)
    o.set_vext(0, V0)
    o.set_psi(0, prob.psi0)
    o.step_real(0, u.shape[0])
    p = prob.forward(np.zeros_like(u))
    ref = o.get_psi(0)
    assert np.linalg.norm(p - ref) <= 1e-13 * np.linalg.norm(ref)


def test_adjoint_gradient_matches_finite_differences():
    cfg, prob, u, _ = small_problem()
    L, grad = prob.gradient(u)
    assert abs(L - prob.loss(u)) < 1e-14
    rng = np.random.default_rng(0)
    h = 1e-5
    for _ in range(8):
        n, k = rng.integers(u.shape[0]), rng.integers(u.shape[1])
        up, um = u.copy(), u.copy()
        up[n, k] += h
        um[n, k] -= h
        fd = (prob.loss(up) - prob.loss(um)) / (2 * h)
        # FD rounding: ~1e-16 / h on a loss of order 1
        assert abs(fd - grad[n, k]) <= 1e-6 * abs(fd) + 1e-10, (n, k, fd, grad[n, k])
