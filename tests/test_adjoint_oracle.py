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


def dipolar_problem(nsteps=10, n=16, nctrl=3, seed=4):
    """The small problem with a dipolar interaction (eps_dd = 0.8, dipoles in
    the plane, no cut-off): the k-space term's Jacobian enters the adjoint."""
    from fgpe_b200 import HAM_DIPOLAR
    a = 30.0 / (4 * ad.PI_REF)
    prms = np.zeros(32)
    prms[0:3] = a
    prms[6] = 0.8 * a
    prms[7:10] = [1.0, 0.5, 0.0]
    cfg = make_config((n, n, 1), (5.0, 5.0, 1.0), dt=2e-3, prms=prms, hamiltonian=HAM_DIPOLAR)
    _, base, u, V0 = small_problem(nsteps=nsteps, n=n, nctrl=nctrl, seed=seed)
    prob = ad.ControlProblem(cfg, V0, base.G, base.psi0, base.target, vtab=ad.dipolar_table(cfg))
    return cfg, prob, u, V0


def test_dipolar_forward_matches_oracle_real_time_step():
    cfg, prob, u, V0 = dipolar_problem()
    o = orc.OracleSolver(cfg)
    o.set_vext(0, V0)
    o.set_psi(0, prob.psi0)
    o.step_real(0, u.shape[0])
    ref = o.get_psi(0)
    p = prob.forward(np.zeros_like(u))
    assert np.linalg.norm(p - ref) <= 1e-13 * np.linalg.norm(ref)
    # the interaction matters at this size: without it the state differs
    plain = ad.ControlProblem(cfg, V0, prob.G, prob.psi0, prob.target)
    assert np.linalg.norm(plain.forward(np.zeros_like(u)) - ref) > 1e-6 * np.linalg.norm(ref)


def test_dipolar_adjoint_gradient_matches_finite_differences():
    cfg, prob, u, _ = dipolar_problem()
    L, grad = prob.gradient(u)
    rng = np.random.default_rng(1)
    h = 1e-5
    for _ in range(6):
        n, k = rng.integers(u.shape[0]), rng.integers(u.shape[1])
        up, um = u.copy(), u.copy()
        up[n, k] += h
        um[n, k] -= h
        fd = (prob.loss(up) - prob.loss(um)) / (2 * h)
        assert abs(fd - grad[n, k]) <= 1e-6 * abs(fd) + 1e-10, (n, k, fd, grad[n, k])
    # the Jacobian term of the interaction is needed: dropping it misses
    no_jac = ad.ControlProblem(cfg, prob.V0, prob.G, prob.psi0, prob.target, vtab=prob.vtab)
    no_jac.JT = lambda mu, p, W: ad.ControlProblem.JT(no_jac, mu, p, W) - 2.0 * no_jac.Phi(np.imag(np.conj(mu) * p)) * p
    _, g2 = no_jac.gradient(u)
    assert np.linalg.norm(g2 - grad) > 1e-4 * np.linalg.norm(grad)
