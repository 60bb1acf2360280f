"""CUDA path (libgpe.so through the C ABI) against the FP64 host oracle.

Tolerances: complex128 form <= 1e-12 relative (the drop-in bar); complex64
form (FP32 fields, FP64 reductions) <= 2e-6 relative per primitive.
"""
import numpy as np
import pytest

import oracle_py as orc
from fgpe_b200 import (C64, C128, HAM_BEC, HAM_BEC2, HAM_DIPOLAR, HAM_SOFT, HAM_TEMPLATE, IMAG_RK4, Solver,
                       grid_axes, make_config)

from test_oracle import PI_REF, gaussian, harmonic

pytestmark = pytest.mark.gpu

TOL = {C128: 1e-12, C64: 2e-6}


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def pair(cfg, V=None, psi=None, seed=1):
    g = Solver(cfg)
    o = orc.OracleSolver(cfg)
    for c in range(cfg.ncomp):
        v = harmonic(cfg, (1.0, 1.2, 1.5)) if V is None else V
        p = gaussian(cfg, seed=seed + c, noise=0.05, npart=cfg.npart[c]) if psi is None else psi
        g.set_vext(c, v)
        o.set_vext(c, v)
        g.set_psi(c, p)
        o.set_psi(c, p)
    return g, o


SHAPES = [(16, 16, 16), (12, 10, 8), (32, 24, 1), (64, 1, 1), (8, 6, 5), (9, 25, 4), (128, 8, 4)]


@pytest.mark.parametrize("prec", [C128, C64])
@pytest.mark.parametrize("shape", SHAPES)
def test_fft_forward_inverse(gpu, prec, shape):
    nx, ny, nz = shape
    cfg = make_config(shape, 4.0, precision=prec)
    rng = np.random.default_rng(7)
    a = rng.standard_normal((nz, ny, nx)) + 1j * rng.standard_normal((nz, ny, nx))
    with Solver(cfg) as s:
        s.set_psi(0, a)
        s.fft(0, -1)
        f = s.get_psi(0)
        assert rel(f, np.fft.fftn(a)) < TOL[prec] * 5
        s.fft(0, +1)
        assert rel(s.get_psi(0) / a.size, a) < TOL[prec] * 5
        assert s.launches > 0


@pytest.mark.parametrize("prec", [C128, C64])
@pytest.mark.parametrize("shape", SHAPES)
def test_laplace(gpu, prec, shape):
    cfg = make_config(shape, (5.0, 4.0, 3.0), precision=prec, hamiltonian=HAM_TEMPLATE)
    g, o = pair(cfg)
    assert rel(g.laplace(0), o.laplace(0)) < TOL[prec]


@pytest.mark.parametrize("prec", [C128, C64])
@pytest.mark.parametrize("shape", [(16, 16, 16), (12, 10, 8), (32, 24, 1)])
def test_apply_h_and_observables(gpu, prec, shape):
    prms = np.zeros(32)
    prms[:6] = [30.0 / (4 * PI_REF), 45.0 / (4 * PI_REF), 40.0 / (4 * PI_REF), 0.01, 0.02, 0.05]
    cfg = make_config(shape, (5.0, 4.0, 3.0), precision=prec, prms=prms)
    g, o = pair(cfg)
    for t in (0.0, 0.005, 0.015, 0.03, 0.1):  # every branch of d_quench_as
        gm, ge = g.apply_h(t, 0)
        om, oe = o.apply_h(t, 0)
        assert rel(gm, om) < TOL[prec]
        assert rel(ge, oe) < TOL[prec]
        assert rel(g.observables(t), o.observables(t)) < TOL[prec]


@pytest.mark.parametrize("prec", [C128, C64])
@pytest.mark.parametrize("shape", [(16, 16, 16), (12, 10, 8), (32, 24, 1), (64, 1, 1)])
def test_real_time_rk4(gpu, prec, shape):
    prms = np.zeros(32)
    prms[:6] = [30.0 / (4 * PI_REF), 33.0 / (4 * PI_REF), 33.0 / (4 * PI_REF), 0.0, 1e300, 1e300]
    cfg = make_config(shape, (5.0, 4.0, 3.0), dt=1e-3, precision=prec, prms=prms)
    g, o = pair(cfg)
    og = g.step_real(0, 20, want_obs=True)
    oo = o.step_real(0, 20, want_obs=True)
    tol = TOL[prec] if prec == C128 else 1e-5
    assert rel(g.get_psi(0), o.get_psi(0)) < tol
    assert rel(og, oo) < tol
    # a second chunk continues the reference's iteration count
    g.step_real(20, 5)
    o.step_real(20, 5)
    assert rel(g.get_psi(0), o.get_psi(0)) < tol


@pytest.mark.parametrize("prec", [C128, C64])
@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 24, 1)])
def test_real_time_call_splitting(gpu, prec, shape):
    # The x-inverse epilogue of each stage also transforms the next stage's
    # input; a later call reuses that transform unless something else ran in
    # between.  One call of 6 steps, 6 calls of 1 step, and calls with other
    # operations (set_psi of the same state, observables) in between must
    # give the same bits.  (complex64 carries the state as float32 high and
    # low parts; get_psi returns their complex128 sum, from which set_psi
    # cannot always recover the same pair of floats, so there the set_psi
    # path agrees to 1e-7 instead of bitwise.)
    prms = np.zeros(32)
    prms[:6] = [30.0 / (4 * PI_REF), 33.0 / (4 * PI_REF), 36.0 / (4 * PI_REF), 0.0, 0.003, 0.006]
    cfg = make_config(shape, (5.0, 4.0, 3.0), dt=1e-3, precision=prec, prms=prms)
    g1, o = pair(cfg)
    g2, _ = pair(cfg)
    g3, _ = pair(cfg)
    g1.step_real(0, 6)
    for k in range(6):
        g2.step_real(k, 1)
    for k in range(6):
        g3.step_real(k, 1)
        if k == 2:
            g3.set_psi(0, g3.get_psi(0))
        if k == 4:
            g3.observables(0.0)
    o.step_real(0, 6)
    p1 = g1.get_psi(0)
    assert np.array_equal(p1, g2.get_psi(0))
    if prec == C128:
        assert np.array_equal(p1, g3.get_psi(0))
    else:
        assert rel(g3.get_psi(0), p1) < 1e-7
    tol = TOL[prec] if prec == C128 else 1e-5
    assert rel(p1, o.get_psi(0)) < tol


@pytest.mark.parametrize("prec", [C128, C64])
def test_logging_observables(gpu, prec):
    # The plugins' status-line reductions on the device against the numpy
    # restatements of the reference kernels, on the state the device holds.
    cfg = make_config((16, 12, 8), (5.0, 4.0, 3.0), precision=prec, hamiltonian=HAM_TEMPLATE)
    g, _ = pair(cfg)
    p = g.get_psi(0)
    tol = TOL[prec]
    want = orc.average_cos(cfg, p)
    assert abs(g.average_cos(0) - want) <= tol * abs(want)
    cfg2 = make_config((16, 12, 8), (5.0, 4.0, 3.0), precision=prec, ncomp=2, hamiltonian=HAM_BEC2,
                       prms=[1.0, 1.0, 0.5], npart=(0.5, 0.5))
    g2, _ = pair(cfg2)
    p1, p2 = g2.get_psi(0), g2.get_psi(1)
    dv = cfg2.dx[0] * cfg2.dx[1] * cfg2.dx[2]
    for sign in (1, -1):
        want = orc.average_cos2(cfg2, p1, p2, sign)
        assert abs(g2.average_cos2(sign) - want) <= tol * abs(want)
    for got, terms in ((g2.relative_phase(), orc.relative_phase_terms(p1, p2)),
                       (g2.dsz_dt(), orc.dsz_dt_terms(p1, p2))):
        # relative to the sum of magnitudes: the signed sums cancel
        assert abs(got - np.sum(terms) * dv) <= tol * np.sum(np.abs(terms)) * dv
    with pytest.raises(Exception):
        g.relative_phase()  # one component


def test_complex64_compensated_state(gpu):
    # complex64 carries the real-time step state as float32 high + low parts
    # (an error-free TwoSum at stage 4), across calls.  Rounding the state to
    # float32 every step would random-walk the norm by ~1e-7 over these 2000
    # steps; compensated, what is left comes from the float32 transforms and
    # pointwise terms (measured 1.5e-9 in the norm, 4e-9 in E on a B200).
    prms = np.zeros(32)
    prms[:3] = 500.0 / (4 * PI_REF)
    cfg64 = make_config((32, 32, 32), 8.0, dt=5e-4, precision=C64, prms=prms)
    cfg128 = make_config((32, 32, 32), 8.0, dt=5e-4, precision=C128, prms=prms)
    psi = gaussian(cfg64, width=1.5, seed=3, noise=1e-3)
    s64, s128 = Solver(cfg64), Solver(cfg128)
    for s in (s64, s128):
        s.set_vext(0, harmonic(cfg64))
        s.set_psi(0, psi)
    # set_psi keeps the complex128 input exactly (rounding residual as the low part)
    assert rel(s64.get_psi(0), psi) < 1e-13
    o0 = s128.observables(0.0)
    for k in range(4):
        ob64 = s64.step_real(500 * k, 500, want_obs=True)
        ob128 = s128.step_real(500 * k, 500, want_obs=True)
    assert abs(ob128[0] / o0[0] - 1) < 1e-9
    assert abs(ob64[0] / o0[0] - 1) < 1e-8
    assert abs(ob64[2] / ob128[2] - 1) < 3e-8
    assert rel(s64.get_psi(0), s128.get_psi(0)) < 2e-6


def test_complex64_low_part_reset(gpu):
    # Any operation that rewrites the state outside the real-time steps drops
    # the low part: after imaginary-time steps, real-time stepping continues
    # exactly as on a fresh handle given the same state.
    prms = np.zeros(32)
    prms[:3] = 30.0 / (4 * PI_REF)
    cfg = make_config((16, 16, 16), 5.0, dt=1e-3, precision=C64, prms=prms)
    g1, _ = pair(cfg)
    g1.step_real(0, 10)
    g1.step_imag(0, 5)
    g2 = Solver(cfg)
    g2.set_vext(0, harmonic(cfg, (1.0, 1.2, 1.5)))
    g2.set_psi(0, g1.get_psi(0))
    g1.step_real(0, 10)
    g2.step_real(0, 10)
    assert np.array_equal(g1.get_psi(0), g2.get_psi(0))


@pytest.mark.parametrize("prec", [C128, C64])
@pytest.mark.parametrize("shape", [(16, 16, 16), (12, 10, 8), (32, 24, 1), (64, 1, 1)])
def test_imag_heavyball(gpu, prec, shape):
    cfg = make_config(shape, (5.0, 4.0, 3.0), dt=2e-3, precision=prec, g=25.0, beta=0.9, epsilon_e=0.0)
    g, o = pair(cfg)
    dg = g.step_imag(0, 30)
    do = o.step_imag(0, 30)
    assert dg == do == (30, False)
    tol = TOL[prec] if prec == C128 else 1e-5
    assert rel(g.get_psi(0), o.get_psi(0)) < tol
    sg, so = g.imag_state(), o.imag_state()
    assert np.allclose(sg, so, rtol=tol, atol=0)
    # continue after get_psi materialised the lazy normalisation
    g.step_imag(30, 10)
    o.step_imag(30, 10)
    assert rel(g.get_psi(0), o.get_psi(0)) < tol
    assert np.allclose(g.imag_state(), o.imag_state(), rtol=tol, atol=0)


def test_imag_heavyball_convergence_iteration(gpu):
    # The device-side convergence test must stop at the same iteration as the
    # reference loop (|dE|/E_prev < eps, src/oneComponentGPSolver.cu:84).
    cfg = make_config((16, 16, 16), 6.0, dt=5e-3, g=10.0, beta=0.5, epsilon_e=1e-7)
    g, o = pair(cfg)
    dg = g.step_imag(0, 2000)
    do = o.step_imag(0, 2000)
    assert dg == do and dg[1]
    assert rel(g.get_psi(0), o.get_psi(0)) < 1e-12


@pytest.mark.parametrize("prec", [C128, C64])
def test_imag_rk4(gpu, prec):
    cfg = make_config((16, 16, 16), 6.0, dt=5e-3, g=10.0, precision=prec, imag_scheme=IMAG_RK4, epsilon_e=0.0)
    g, o = pair(cfg)
    assert g.step_imag(0, 25) == o.step_imag(0, 25)
    tol = TOL[prec] if prec == C128 else 1e-5
    assert rel(g.get_psi(0), o.get_psi(0)) < tol
    assert np.allclose(g.imag_state(), o.imag_state(), rtol=tol, atol=0)


@pytest.mark.parametrize("prec", [C128, C64])
@pytest.mark.parametrize("shape", [(16, 12, 8), (24, 24, 1)])
def test_two_component(gpu, prec, shape):
    prms = [30.0 / (4 * PI_REF), 28.5 / (4 * PI_REF), 27.0 / (4 * PI_REF)]
    cfg = make_config(shape, (5.0, 4.0, 3.0), dt=1e-3, ncomp=2, hamiltonian=HAM_BEC2, prms=prms,
                      npart=(0.5, 0.5), beta=0.5, precision=prec)
    V = harmonic(cfg) + 0.1j * harmonic(cfg)  # complex V exercises the vext1.y quirk
    g, o = pair(cfg, V=V)
    tol = TOL[prec] if prec == C128 else 1e-5
    for c in range(2):
        assert rel(g.apply_h(0.0, c)[1], o.apply_h(0.0, c)[1]) < TOL[prec]
    assert g.step_imag(0, 15) == o.step_imag(0, 15)
    for c in range(2):
        assert rel(g.get_psi(c), o.get_psi(c)) < tol
    assert np.allclose(g.imag_state(), o.imag_state(), rtol=tol, atol=0)
    g.step_real(0, 10)
    o.step_real(0, 10)
    for c in range(2):
        assert rel(g.get_psi(c), o.get_psi(c)) < tol


@pytest.mark.parametrize("prec", [C128, C64])
def test_dipolar(gpu, prec):
    prms = np.zeros(32)
    a = 40.0 / (4 * PI_REF)
    prms[:3] = a
    prms[6] = 0.8 * a
    prms[7:10] = [0.0, 0.0, 1.0]
    prms[10] = 3.0
    cfg = make_config((16, 16, 8), (6.0, 6.0, 3.0), dt=1e-3, precision=prec, prms=prms,
                      hamiltonian=HAM_DIPOLAR, beta=0.5)
    g, o = pair(cfg)
    for c_ in (0,):
        gm, ge = g.apply_h(0.0, c_)
        om, oe = o.apply_h(0.0, c_)
        assert rel(gm, om) < TOL[prec] * 2
        assert rel(ge, oe) < TOL[prec] * 2
    tol = TOL[prec] if prec == C128 else 1e-5
    g.step_imag(0, 10)
    o.step_imag(0, 10)
    assert rel(g.get_psi(0), o.get_psi(0)) < tol
    g.step_real(0, 10)
    o.step_real(0, 10)
    assert rel(g.get_psi(0), o.get_psi(0)) < tol


@pytest.mark.parametrize("prec", [C128, C64])
@pytest.mark.parametrize("shape,box", [((64, 1, 1), (8.0, 1.0, 1.0)), ((24, 20, 1), (6.0, 5.0, 1.0)),
                                       ((16, 16, 8), (6.0, 6.0, 3.0))])
def test_soft_core(gpu, prec, shape, box):
    # soft-core mean field (V~ of SoftCoreInteraction_1D/2D/3D by dimension)
    prms = np.zeros(32)
    prms[0] = 0.9   # a
    prms[1] = 15.0  # U
    cfg = make_config(shape, box, dt=1e-3, precision=prec, prms=prms, hamiltonian=HAM_SOFT, beta=0.5)
    g, o = pair(cfg)
    gm, ge = g.apply_h(0.0, 0)
    om, oe = o.apply_h(0.0, 0)
    assert rel(gm, om) < TOL[prec] * 2
    assert rel(ge, oe) < TOL[prec] * 2
    assert rel(g.observables(0.0), o.observables(0.0)) < TOL[prec] * 2
    tol = TOL[prec] if prec == C128 else 1e-5
    g.step_imag(0, 10)
    o.step_imag(0, 10)
    assert rel(g.get_psi(0), o.get_psi(0)) < tol
    g.step_real(0, 10)
    o.step_real(0, 10)
    assert rel(g.get_psi(0), o.get_psi(0)) < tol


def test_template_hamiltonian(gpu):
    cfg = make_config((16, 16, 16), 5.0, dt=1e-3, hamiltonian=HAM_TEMPLATE)
    g, o = pair(cfg)
    gm, ge = g.apply_h(0.0, 0)
    om, oe = o.apply_h(0.0, 0)
    assert rel(gm, om) < 1e-12 and rel(ge, oe) < 1e-12
    g.step_real(0, 10)
    o.step_real(0, 10)
    assert rel(g.get_psi(0), o.get_psi(0)) < 1e-12


def test_diverged_watchdog(gpu):
    # NaN injected into psi on the host: the device watchdog reports GPE_ERR_DIVERGED.
    from fgpe_b200 import GPEError
    cfg = make_config((16, 16, 16), 5.0, dt=1e-3, g=10.0, beta=0.5)
    s = Solver(cfg)
    p = gaussian(cfg)
    p[3, 4, 5] = np.nan
    s.set_vext(0, harmonic(cfg))
    s.set_psi(0, p)
    with pytest.raises(GPEError) as e:
        s.step_imag(0, 5)
    assert e.value.status == 5


def test_unsupported_length_rejected(gpu):
    from fgpe_b200 import GPEError
    with pytest.raises(GPEError) as e:
        Solver(make_config((14, 8, 8), 4.0))
    assert e.value.status == 2


@pytest.mark.parametrize("prec", [C128, C64])
def test_moving_frame_term(gpu, prec):
    # -lambda P_x psi (the plugins' trotate option) where the reference's
    # alg_calcHpsi adds it: heavy ball, stage 4 of real-time steps, apply-H.
    prms = np.zeros(32)
    prms[:3] = 30.0 / (4 * PI_REF)
    prms[11] = 0.7
    cfg = make_config((16, 12, 8), (5.0, 4.0, 3.0), dt=1e-3, precision=prec, prms=prms, beta=0.5)
    g, o = pair(cfg)
    tol = TOL[prec] if prec == C128 else 1e-5
    gm, ge = g.apply_h(0.0, 0)
    om, oe = o.apply_h(0.0, 0)
    assert rel(gm, om) < TOL[prec] and rel(ge, oe) < TOL[prec]
    assert g.step_imag(0, 12) == o.step_imag(0, 12)
    assert rel(g.get_psi(0), o.get_psi(0)) < tol
    assert np.allclose(g.imag_state(), o.imag_state(), rtol=tol, atol=0)
    og = g.step_real(0, 8, want_obs=True)
    oo = o.step_real(0, 8, want_obs=True)
    assert rel(g.get_psi(0), o.get_psi(0)) < tol and rel(og, oo) < tol
    # the term changes the answer (lambda = 0 does not reproduce it)
    prms[11] = 0.0
    cfg0 = make_config((16, 12, 8), (5.0, 4.0, 3.0), dt=1e-3, precision=prec, prms=prms, beta=0.5)
    z, _ = pair(cfg0)
    assert rel(z.apply_h(0.0, 0)[0], gm) > 1e-6


def test_moving_frame_two_components(gpu):
    prms = np.zeros(32)
    prms[:3] = [30.0 / (4 * PI_REF), 28.5 / (4 * PI_REF), 27.0 / (4 * PI_REF)]
    prms[11], prms[12] = 0.4, -0.6
    cfg = make_config((16, 12, 8), (5.0, 4.0, 3.0), dt=1e-3, ncomp=2, hamiltonian=HAM_BEC2, prms=prms,
                      npart=(0.5, 0.5), beta=0.5)
    g, o = pair(cfg)
    assert g.step_imag(0, 10) == o.step_imag(0, 10)
    for c in range(2):
        assert rel(g.get_psi(c), o.get_psi(c)) < 1e-12
    g.step_real(0, 6)
    o.step_real(0, 6)
    for c in range(2):
        assert rel(g.get_psi(c), o.get_psi(c)) < 1e-12
