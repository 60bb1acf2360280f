"""Full-size checks (the headline and sweep sizes) through properties that do
not need the oracle: transform round trips and Parseval, conservation of the
norm and energy under real-time RK4, agreement of the two precisions, and the
largest supported line length."""
import numpy as np
import pytest

from fgpe_b200 import C64, C128, HAM_BEC2, HAM_DIPOLAR, Solver, grid_axes, make_config

from test_oracle import PI_REF, gaussian, harmonic

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.mark.parametrize("prec,tol", [(C128, 1e-13), (C64, 2e-6)])
@pytest.mark.parametrize("shape", [(128, 128, 128), (1024, 4, 2), (864, 6, 3), (512, 512, 1)])
def test_round_trip_and_parseval(gpu, prec, tol, shape):
    nx, ny, nz = shape
    rng = np.random.default_rng(3)
    a = rng.standard_normal((nz, ny, nx)) + 1j * rng.standard_normal((nz, ny, nx))
    with Solver(make_config(shape, 8.0, precision=prec)) as s:
        s.set_psi(0, a)
        s.fft(0, -1)
        f = s.get_psi(0)
        # the spectrum itself (a consistently permuted or mis-twiddled
        # spectrum would pass the round trip and Parseval below)
        assert rel(f, np.fft.fftn(a)) < 10 * tol
        # Parseval for the unnormalised transform
        assert abs(np.sum(np.abs(f) ** 2) / (a.size * np.sum(np.abs(a) ** 2)) - 1) < 10 * tol
        s.fft(0, +1)
        assert rel(s.get_psi(0) / a.size, a) < 10 * tol


def quench(prec, n=128):
    prms = np.zeros(32)
    prms[0:3] = 1100.0 / (4 * PI_REF)
    cfg = make_config((n, n, n), 10.0, dt=5e-4, precision=prec, prms=prms)
    x, y, z = grid_axes(cfg)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    V = 0.5 * (X ** 2 + Y ** 2 + (2 * Z) ** 2) + 0j
    psi = gaussian(cfg, width=1.5, seed=2, noise=1e-3)
    s = Solver(cfg)
    s.set_vext(0, V)
    s.set_psi(0, psi)
    return s


def test_headline_size_conservation_and_precisions(gpu):
    s128, s64 = quench(C128), quench(C64)
    o0 = s128.observables(0.0)
    ob128 = s128.step_real(0, 200, want_obs=True)
    ob64 = s64.step_real(0, 200, want_obs=True)
    # norm and energy conserved by the complex128 RK4 to its truncation level
    # (an excited, strongly interacting state: 1.7e-9 in norm after 200 steps)
    assert abs(ob128[0] / o0[0] - 1) < 1e-8
    assert abs(ob128[2] / o0[2] - 1) < 1e-7
    # complex64 follows complex128
    assert rel(s64.get_psi(0), s128.get_psi(0)) < 1e-5
    assert abs(ob64[2] / ob128[2] - 1) < 1e-6


def test_dipolar_and_two_component_sizes(gpu):
    a = 1000.0 / (4 * PI_REF)
    prms = np.zeros(32)
    prms[:3] = a
    prms[6] = 0.8 * a
    prms[7:10] = [0.0, 0.0, 1.0]
    prms[10] = 6.0
    cfg = make_config((128, 128, 64), (12.0, 12.0, 6.0), dt=5e-4, precision=C64, prms=prms,
                      hamiltonian=HAM_DIPOLAR, beta=0.9)
    with Solver(cfg) as s:
        s.set_vext(0, harmonic(cfg, (1.0, 1.0, 3.0)))
        s.set_psi(0, gaussian(cfg, seed=4))
        s.step_imag(0, 50)
        st = s.imag_state()
        assert np.all(np.isfinite(st)) and abs(st[0] - 1.0) < 1e-12
        o0 = s.observables(0.0)
        ob = s.step_real(0, 50, want_obs=True)
        assert abs(ob[0] / o0[0] - 1) < 1e-6
    p2 = [1000.0 / (4 * PI_REF), 950.0 / (4 * PI_REF), 900.0 / (4 * PI_REF)]
    cfg2 = make_config((96, 96, 96), 8.0, dt=5e-4, precision=C64, ncomp=2, hamiltonian=HAM_BEC2, prms=p2,
                       npart=(0.5, 0.5), beta=0.9)
    with Solver(cfg2) as s:
        for c in range(2):
            s.set_vext(c, harmonic(cfg2))
            s.set_psi(c, gaussian(cfg2, seed=5 + c, npart=0.5))
        s.step_imag(0, 50)
        assert np.all(np.isfinite(s.imag_state()))
        o0 = s.observables(0.0)
        ob = s.step_real(0, 50, want_obs=True)
        assert abs(ob[0] / o0[0] - 1) < 1e-6 and abs(ob[3] / o0[3] - 1) < 1e-6
