"""Parity at the sizes the benchmark configurations use.

Every grid length is its own template instantiation of the pass kernels, so
the transforms and chains at the configs' lengths are compared here with
independent answers, not only with themselves:

- gpe_fft (forward and inverse) against numpy.fft (pocketfft, FP64) at 128^3,
  64^3, 96^3, 128x128x64 and N x N for every sweep length N;
- complex128 apply-H and RK4 steps of the headline quench (128^3), the dipolar
  ground-state case (128x128x64), the two-component case (96^3) and the 2D
  sweep lengths against the FP64 oracle (a restatement of
  src/oneComponentGPSolver.cu:122-217 and src/parallel.cu:230-302);
- the complex64 form against the same oracle at its own tolerance.

Tolerances: complex128 <= 1e-13 relative for a transform, <= 1e-12 for the
solver chains (the drop-in bar); complex64 <= 2e-6 for a transform or one
primitive, <= 1e-5 over a few steps.
"""
import numpy as np
import pytest

import oracle_py as orc
from fgpe_b200 import C64, C128, HAM_BEC2, HAM_DIPOLAR, IMAG_RK4, Solver, make_config

from test_oracle import PI_REF, gaussian, harmonic

pytestmark = pytest.mark.gpu

FFT_TOL = {C128: 1e-13, C64: 2e-6}
CHAIN_TOL = {C128: 1e-12, C64: 1e-5}
SWEEP_N = (64, 96, 128, 192, 256, 384, 512)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


FFT_SHAPES = [(128, 128, 128), (64, 64, 64), (96, 96, 96), (128, 128, 64)] + [(n, n, 1) for n in SWEEP_N]


@pytest.mark.parametrize("prec", [C128, C64])
@pytest.mark.parametrize("shape", FFT_SHAPES)
def test_fft_matches_numpy_at_config_sizes(gpu, prec, shape):
    nx, ny, nz = shape
    rng = np.random.default_rng(nx * 7 + ny * 3 + nz)
    a = rng.standard_normal((nz, ny, nx)) + 1j * rng.standard_normal((nz, ny, nx))
    with Solver(make_config(shape, 8.0, precision=prec)) as s:
        s.set_psi(0, a)
        s.fft(0, -1)
        f = s.get_psi(0)
        assert rel(f, np.fft.fftn(a)) < FFT_TOL[prec], "forward"
        # inverse of a spectrum (a fresh input, so the inverse is checked on its own)
        b = rng.standard_normal((nz, ny, nx)) + 1j * rng.standard_normal((nz, ny, nx))
        s.set_psi(0, b)
        s.fft(0, +1)
        assert rel(s.get_psi(0), np.fft.ifftn(b) * b.size) < FFT_TOL[prec], "inverse"


def pair(cfg, V, psis):
    g = Solver(cfg)
    o = orc.OracleSolver(cfg)
    for c in range(cfg.ncomp):
        for s in (g, o):
            s.set_vext(c, V)
            s.set_psi(c, psis[c])
    return g, o


def quench_cfg(prec):
    prms = np.zeros(32)
    prms[0:3] = 1100.0 / (4 * PI_REF)
    return make_config((128, 128, 128), 10.0, dt=5e-4, precision=prec, prms=prms, beta=0.9)


@pytest.fixture(scope="module")
def quench_start():
    """A state near the g = 1000 ground state of the headline trap: 150
    heavy-ball iterations (complex128, the reference's scheme) from the
    seeded Gaussian."""
    prms = np.zeros(32)
    prms[0:3] = 1000.0 / (4 * PI_REF)
    cfg = make_config((128, 128, 128), 10.0, dt=2e-3, precision=C128, prms=prms, beta=0.9)
    V = harmonic(cfg, (1.0, 1.0, 2.0))
    with Solver(cfg) as s:
        s.set_vext(0, V)
        s.set_psi(0, gaussian(cfg, width=1.5, seed=1))
        s.step_imag(0, 150)
        return V, s.get_psi(0)


@pytest.mark.parametrize("prec", [C128, C64])
def test_headline_quench_steps_match_oracle(gpu, prec, quench_start):
    """Config 2 (128^3, g 1000 -> 1100 at t = 0, dt = 5e-4): 4 real-time RK4
    steps with the observables of the last one."""
    V, psi0 = quench_start
    g, o = pair(quench_cfg(prec), V, [psi0])
    og = g.step_real(0, 4, want_obs=True)
    oo = o.step_real(0, 4, want_obs=True)
    assert rel(g.get_psi(0), o.get_psi(0)) < CHAIN_TOL[prec]
    for q in range(3):  # norm, sum Re(psi* h_mu), sum Re(psi* h_en)
        assert abs(og[q] / oo[q] - 1) < CHAIN_TOL[prec], q
    g.close()


@pytest.mark.parametrize("prec", [C128, C64])
def test_headline_apply_h_matches_oracle(gpu, prec, quench_start):
    V, psi0 = quench_start
    g, o = pair(quench_cfg(prec), V, [psi0])
    gm, ge = g.apply_h(0.0, 0)
    om, oe = o.apply_h(0.0, 0)
    # complex64: the FP32 transforms of a 128^3 grid (21 radix stages forward
    # and back) leave about 2e-6 of H psi.  The Laplacian alone of this smooth
    # state is another matter: the transform's FP32 rounding (about 1e-7 of
    # the spectrum, spread over all k) is weighted by k^2 up to the grid's
    # cut-off while the Laplacian itself lives at small k, so its relative
    # error is about 5e-5.
    tol = 1e-12 if prec == C128 else 5e-6
    assert rel(gm, om) < tol and rel(ge, oe) < tol
    assert rel(g.laplace(0), o.laplace(0)) < (1e-12 if prec == C128 else 2e-4)
    g.close()


def dipolar_cfg(prec, scheme=IMAG_RK4):
    a = 1000.0 / (4 * PI_REF)
    prms = np.zeros(32)
    prms[:3] = a
    prms[6] = 0.8 * a
    prms[7:10] = [0.0, 0.0, 1.0]
    prms[10] = 6.0
    return make_config((128, 128, 64), (12.0, 12.0, 6.0), dt=5e-4, precision=prec, prms=prms,
                       hamiltonian=HAM_DIPOLAR, imag_scheme=scheme, beta=0.9, epsilon_e=1e-8)


@pytest.mark.parametrize("prec", [C128, C64])
def test_dipolar_config_matches_oracle(gpu, prec):
    """Config 3a (128x128x64, eps_dd = 0.8 along z, cut-off R = 6): 3 RK4
    imaginary-time iterations, then 2 real-time steps."""
    cfg = dipolar_cfg(prec)
    V = harmonic(cfg, (1.0, 1.0, 3.0))
    g, o = pair(cfg, V, [gaussian(cfg, seed=4)])
    for s in (g, o):
        s.step_imag(0, 3)
    sg, so = g.imag_state(), o.imag_state()
    assert rel(g.get_psi(0), o.get_psi(0)) < CHAIN_TOL[prec]
    assert abs(sg[1] / so[1] - 1) < CHAIN_TOL[prec] and abs(sg[2] / so[2] - 1) < CHAIN_TOL[prec]
    og = g.step_real(0, 2, want_obs=True)
    oo = o.step_real(0, 2, want_obs=True)
    assert rel(g.get_psi(0), o.get_psi(0)) < CHAIN_TOL[prec]
    assert abs(og[2] / oo[2] - 1) < CHAIN_TOL[prec]
    g.close()


@pytest.mark.parametrize("prec", [C128, C64])
def test_two_component_config_matches_oracle(gpu, prec):
    """Config 3b (96^3, g11 = 1000, g22 = 950, g12 = 900, norms 0.5 each):
    3 heavy-ball iterations of the reference's two-component loop, then 2
    real-time steps."""
    p2 = np.zeros(32)
    p2[:3] = [1000.0 / (4 * PI_REF), 950.0 / (4 * PI_REF), 900.0 / (4 * PI_REF)]
    cfg = make_config((96, 96, 96), 8.0, dt=5e-4, precision=prec, ncomp=2, hamiltonian=HAM_BEC2, prms=p2,
                      npart=(0.5, 0.5), beta=0.9, epsilon_e=1e-8)
    V = harmonic(cfg)
    psis = [gaussian(cfg, seed=5 + c, npart=0.5) for c in range(2)]
    g, o = pair(cfg, V, psis)
    for s in (g, o):
        s.step_imag(0, 3)
    sg, so = g.imag_state(), o.imag_state()
    for c in range(2):
        assert rel(g.get_psi(c), o.get_psi(c)) < CHAIN_TOL[prec]
        assert abs(sg[4 * c + 2] / so[4 * c + 2] - 1) < CHAIN_TOL[prec]
    g.step_real(1, 2)
    o.step_real(1, 2)
    for c in range(2):
        assert rel(g.get_psi(c), o.get_psi(c)) < CHAIN_TOL[prec]
    g.close()


@pytest.mark.parametrize("prec", [C128, C64])
@pytest.mark.parametrize("n", SWEEP_N)
def test_sweep_lengths_match_oracle(gpu, prec, n):
    """Config 4's 2D instances: box [-L, L]^2 with L = 8 sqrt(N/64), an
    anisotropic trap, RK4 in imaginary time (dt = 4e-4): 4 iterations."""
    L = 8.0 * np.sqrt(n / 64.0)
    cfg = make_config((n, n, 1), (L, L, 1.0), dt=4e-4, precision=prec, g=700.0, imag_scheme=IMAG_RK4,
                      epsilon_e=1e-8)
    V = harmonic(cfg, (1.0, 2.5, 0.0))
    g, o = pair(cfg, V, [gaussian(cfg, seed=n)])
    for s in (g, o):
        s.step_imag(0, 4)
    sg, so = g.imag_state(), o.imag_state()
    assert rel(g.get_psi(0), o.get_psi(0)) < CHAIN_TOL[prec]
    assert abs(sg[1] / so[1] - 1) < CHAIN_TOL[prec] and abs(sg[2] / so[2] - 1) < CHAIN_TOL[prec]
    g.close()


def test_imaginary_time_stops_issuing_after_convergence(gpu):
    """A call asked for many more iterations than convergence needs issues
    kernels for at most a few chunks past the converging iteration."""
    cfg = make_config((32, 32, 32), 6.0, dt=2e-3, g=50.0, beta=0.9, epsilon_e=1e-6)
    with Solver(cfg) as s:
        s.set_vext(0, harmonic(cfg))
        s.set_psi(0, gaussian(cfg))
        l0 = s.launches
        s.step_imag(0, 1)
        l1 = s.launches
        s.step_imag(1, 2)
        l2 = s.launches
        per_iter = (l2 - l1) - (l1 - l0)  # the per-call set-up cancels
        setup = (l1 - l0) - per_iter
        assert per_iter > 0
        done, conv = s.step_imag(3, 100000)
        assert conv and done < 5000
        issued = (s.launches - l2 - setup) // per_iter
        assert done <= issued <= done + 2 * 64, (issued, done)
