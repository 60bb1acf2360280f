"""The FP64 host oracle against numpy.fft and against physics known answers.

The reference (fGPE v0.3) ships no numerical tests and no golden data; the
oracle is pinned by (1) numpy's pocketfft for the transform, (2) analytic
answers of the discrete operators, (3) golden outputs of the reference's own
CUDA build (test_golden.py).
"""
import numpy as np
import pytest

import oracle_py as orc
from fgpe_b200 import HAM_BEC, HAM_BEC2, HAM_TEMPLATE, IMAG_HEAVYBALL, IMAG_RK4, grid_axes, make_config

PI_REF = 3.141592653589793

SHAPES = [(8, 8, 8), (16, 12, 10), (64, 1, 1), (96, 1, 1), (7, 11, 13), (128, 32, 1), (6, 10, 12),
          (1, 1, 1), (2, 3, 5), (25, 9, 27), (48, 20, 3), (1, 16, 8)]


@pytest.mark.parametrize("shape", SHAPES)
def test_fft_matches_numpy(shape):
    nx, ny, nz = shape
    rng = np.random.default_rng(nx * 1000 + ny * 10 + nz)
    a = rng.standard_normal((nz, ny, nx)) + 1j * rng.standard_normal((nz, ny, nx))
    f = orc.fft3d(a, -1)
    ref = np.fft.fftn(a)
    assert np.linalg.norm(f - ref) <= 1e-14 * np.linalg.norm(ref)
    b = orc.fft3d(f, +1) / a.size
    assert np.linalg.norm(b - a) <= 1e-14 * np.linalg.norm(a)


def harmonic(cfg, w=(1.0, 1.0, 1.0)):
    x, y, z = grid_axes(cfg)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return 0.5 * ((w[0] * X) ** 2 + (w[1] * Y) ** 2 + (w[2] * Z) ** 2) + 0j


def gaussian(cfg, width=1.0, seed=1, noise=1e-3, npart=1.0):
    x, y, z = grid_axes(cfg)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    rng = np.random.default_rng(seed)
    g = np.exp(-(X ** 2 + Y ** 2 + Z ** 2) / (2 * width ** 2))
    psi = g * (1 + noise * (rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)))
    dv = cfg.dx[0] * cfg.dx[1] * cfg.dx[2]
    return psi * np.sqrt(npart / (np.sum(np.abs(psi) ** 2) * dv))


def test_axes_match_reference_formula():
    # src/baseHamiltonian.cu:43-45,61-68 and src/params.cu:206-211 (odd-N k formula kept)
    cfg = make_config((16, 5, 8), (4.0, 3.0, 2.0))
    x, y, z, kx, ky, kz = orc.axes(cfg)
    assert np.allclose(x, -4.0 + (np.arange(16) + 0.5) * 0.5)
    dk = 1.0 / (16 * 0.5)
    assert np.allclose(kx, np.r_[np.arange(9), np.arange(9, 16) - 16] * dk)
    dky = 1.0 / (5 * cfg.dx[1])
    assert np.allclose(ky, np.r_[0, 1, 2, -2.5 + 1, -2.5 + 2] * dky)  # reference's odd-N values


def test_plane_wave_is_kinetic_eigenvector():
    # A discrete plane wave exp(2 pi i m x/L) has T psi = 2 pi^2 (m/L)^2 psi,
    # up to the scale literal 19.739208802 of src/parallel.cu:199.
    cfg = make_config((32, 16, 8), (5.0, 4.0, 3.0))
    x, y, z = grid_axes(cfg)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    m = (3, -2, 1)
    L = [2 * cfg.xmax[d] for d in range(3)]
    psi = np.exp(2j * np.pi * (m[0] * X / L[0] + m[1] * Y / L[1] + m[2] * Z / L[2]))
    s = orc.OracleSolver(make_config((32, 16, 8), (5.0, 4.0, 3.0), hamiltonian=HAM_TEMPLATE))
    s.set_psi(0, psi)
    T = s.laplace(0)
    lam = 19.739208802 * sum((m[d] / L[d]) ** 2 for d in range(3))
    assert np.allclose(T, lam * psi, rtol=0, atol=1e-12 * lam)


def test_harmonic_ground_state_g0():
    # g = 0 isotropic oscillator: mu = E = 3/2 (3D) at convergence.
    cfg = make_config((32, 32, 32), 8.0, dt=5e-3, g=0.0, beta=0.5, epsilon_e=1e-13)
    s = orc.OracleSolver(cfg)
    s.set_vext(0, harmonic(cfg))
    s.set_psi(0, gaussian(cfg, width=1.4, noise=0.0))
    done, conv = s.step_imag(0, 3000)
    st = s.imag_state()
    assert abs(st[1] - 1.5) < 1e-6 and abs(st[2] - 1.5) < 1e-6


def test_harmonic_ground_state_g0_rk4_imag():
    cfg = make_config((24, 24, 24), 7.0, dt=1e-2, g=0.0, epsilon_e=1e-12, imag_scheme=IMAG_RK4)
    s = orc.OracleSolver(cfg)
    s.set_vext(0, harmonic(cfg))
    s.set_psi(0, gaussian(cfg, width=1.3, noise=0.0))
    done, conv = s.step_imag(0, 4000)
    assert conv
    st = s.imag_state()
    assert abs(st[1] - 1.5) < 1e-6 and abs(st[2] - 1.5) < 1e-6


def test_real_time_norm_and_energy_conservation():
    cfg = make_config((32, 32, 16), (8.0, 8.0, 6.0), dt=1e-3, g=50.0)
    s = orc.OracleSolver(cfg)
    s.set_vext(0, harmonic(cfg))
    s.set_psi(0, gaussian(cfg, width=1.2, noise=1e-2))
    o0 = s.observables(0.0)
    s.step_real(0, 200)
    o1 = s.observables(200 * 1e-3)
    assert abs(o1[0] - o0[0]) < 1e-9
    assert abs(o1[2] - o0[2]) / abs(o0[2]) < 1e-7


def test_displaced_gaussian_oscillates():
    # g = 0 harmonic trap: <x>(t) = x0 cos t.
    cfg = make_config((64, 1, 1), 10.0, dt=2e-3, g=0.0, dim=1)
    x = grid_axes(cfg)[0]
    x0 = 1.5
    psi = (np.exp(-(x - x0) ** 2 / 2) + 0j).reshape(1, 1, -1)
    s = orc.OracleSolver(cfg)
    s.set_vext(0, (0.5 * x ** 2 + 0j).reshape(1, 1, -1))
    s.set_psi(0, psi)
    n = 500
    s.step_real(0, n)
    p = s.get_psi(0).reshape(-1)
    xm = np.sum(x * np.abs(p) ** 2) / np.sum(np.abs(p) ** 2)
    assert abs(xm - x0 * np.cos(n * 2e-3)) < 1e-6


def reference_heavyball_numpy(cfg, psi0, V, niter):
    """Pure-numpy restatement of src/oneComponentGPSolver.cu:46-95 (1 component),
    used to cross-check the C++ oracle loop on a tiny grid."""
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    kx, ky, kz = orc.axes(cfg)[3:]
    K2 = (kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2)
    N = nx * ny * nz
    dv = cfg.dx[0] * cfg.dx[1] * cfg.dx[2]
    a = cfg.prms[0]
    psi = psi0.copy()
    old = psi0.copy()
    E = 0.0
    hist = []
    for it in range(niter):
        Eprev = E
        T = np.fft.ifftn(19.739208802 / N * K2 * np.fft.fftn(psi)) * N
        n = np.abs(psi) ** 2
        hmu = T + (V.real + 4 * PI_REF * a * n + 1j * V.imag) * psi
        hen = T + (V.real + 2 * PI_REF * a * n + 1j * V.imag) * psi
        new = psi - cfg.dt * hmu + cfg.beta * (psi - old)
        norm = np.sum(np.abs(new) ** 2) * dv
        old = psi
        psi = new * np.sqrt(cfg.npart[0] / norm)
        mu = np.sum((psi.conj() * hmu).real) * dv / cfg.npart[0]
        E = np.sum((psi.conj() * hen).real) * dv / cfg.npart[0]
        hist.append((mu, E))
        if abs(E - Eprev) / Eprev < cfg.epsilon_e:
            break
    return psi, hist


def test_heavyball_loop_matches_numpy_restatement():
    cfg = make_config((12, 10, 8), (5.0, 4.0, 3.5), dt=2e-3, g=20.0, beta=0.9, epsilon_e=0.0)
    V = harmonic(cfg, (1.0, 1.3, 1.7))
    psi0 = gaussian(cfg, noise=0.05)
    s = orc.OracleSolver(cfg)
    s.set_vext(0, V)
    s.set_psi(0, psi0)
    s.step_imag(0, 25)
    st = s.imag_state()
    ref, hist = reference_heavyball_numpy(cfg, psi0, V, 25)
    assert np.linalg.norm(s.get_psi(0) - ref) <= 1e-13 * np.linalg.norm(ref)
    assert abs(st[1] - hist[-1][0]) <= 1e-13 * abs(hist[-1][0])
    assert abs(st[2] - hist[-1][1]) <= 1e-13 * abs(hist[-1][1])


def test_two_component_runs_and_conserves():
    cfg = make_config((16, 16, 8), (6.0, 6.0, 4.0), dt=1e-3, ncomp=2, hamiltonian=HAM_BEC2,
                      prms=[10.0 / (4 * PI_REF), 9.5 / (4 * PI_REF), 9.0 / (4 * PI_REF)],
                      npart=(0.5, 0.5), beta=0.5)
    s = orc.OracleSolver(cfg)
    for c in range(2):
        s.set_vext(c, harmonic(cfg))
        s.set_psi(c, gaussian(cfg, seed=3 + c, noise=0.01, npart=0.5))
    s.step_imag(0, 50)
    st = s.imag_state()
    assert np.all(np.isfinite(st))
    o0 = s.observables()
    s.step_real(0, 50)
    o1 = s.observables()
    assert abs(o1[0] - o0[0]) < 1e-10 and abs(o1[3] - o0[3]) < 1e-10


def test_oracle_rejects_bad_configs():
    with pytest.raises(ValueError):
        orc.OracleSolver(make_config((8, 8, 8), 4.0, ncomp=2, hamiltonian=HAM_BEC))
    with pytest.raises(ValueError):
        orc.OracleSolver(make_config((8, 8, 8), 4.0, ncomp=1, hamiltonian=HAM_BEC2))


def test_moving_frame_term_matches_numpy():
    # alg_addVPx (src/baseHamiltonian.cu:198-211): h += -(lambda/N) IFFT(kx FFT psi)
    # with the unnormalised inverse, i.e. -lambda * ifftn(kx * fftn(psi)) in numpy.
    prms = np.zeros(32)
    prms[:3] = 20.0 / (4 * PI_REF)
    prms[11] = 0.9
    cfg = make_config((12, 10, 8), (5.0, 4.0, 3.5), dt=2e-3, prms=prms)
    V = harmonic(cfg, (1.0, 1.3, 1.7))
    psi = gaussian(cfg, noise=0.05)
    s = orc.OracleSolver(cfg)
    s.set_vext(0, V)
    s.set_psi(0, psi)
    hm, he = s.apply_h(0.0, 0)
    kx, ky, kz = orc.axes(cfg)[3:]
    K2 = kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2
    N = psi.size
    T = np.fft.ifftn(19.739208802 / N * K2 * np.fft.fftn(psi)) * N
    P = np.fft.ifftn(kx[None, None, :] * np.fft.fftn(psi))
    n = np.abs(psi) ** 2
    a = prms[2]
    want_mu = T + (V.real + 4 * PI_REF * a * n + 1j * V.imag) * psi - 0.9 * P
    want_en = T + (V.real + 2 * PI_REF * a * n + 1j * V.imag) * psi - 0.9 * P
    assert np.linalg.norm(hm - want_mu) <= 1e-13 * np.linalg.norm(want_mu)
    assert np.linalg.norm(he - want_en) <= 1e-13 * np.linalg.norm(want_en)


@pytest.mark.parametrize("shape,box", [((32, 1, 1), (6.0, 1.0, 1.0)), ((16, 12, 1), (5.0, 4.0, 1.0)),
                                       ((12, 10, 8), (5.0, 4.0, 3.5))])
def test_soft_core_matches_numpy(shape, box):
    # GPE_HAM_SOFT: h_mu = T + (V + Phi) psi, h_en = T + (V + Phi/2) psi, with
    # Phi = ifftn(V~ fftn|psi|^2) and V~ the SoftCoreInteraction_1D/2D/3D
    # formulas of src/parallel.cu:360-477 for the grid's dimension.
    from scipy.special import j1
    from fgpe_b200 import HAM_SOFT
    prms = np.zeros(32)
    prms[0], prms[1] = 0.8, 12.0
    cfg = make_config(shape, box, dt=2e-3, prms=prms, hamiltonian=HAM_SOFT)
    V = harmonic(cfg, (1.0, 1.3, 1.7))
    psi = gaussian(cfg, noise=0.05)
    s = orc.OracleSolver(cfg)
    s.set_vext(0, V)
    s.set_psi(0, psi)
    hm, he = s.apply_h(0.0, 0)
    kx, ky, kz = orc.axes(cfg)[3:]
    K2 = kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2
    N = psi.size
    T = np.fft.ifftn(19.739208802 / N * K2 * np.fft.fftn(psi)) * N
    a, U = prms[0], prms[1]
    k = 2 * PI_REF * np.sqrt(K2)
    ks = np.where(k < 1e-6, 1.0, k)
    if cfg.dim == 1:
        vt = np.where(k < 1e-6, U * 2 * a * (1 - (a * k) ** 2 / 6.0), U * 2 * np.sin(a * ks) / ks)
    elif cfg.dim == 2:
        vt = np.where(k < 1e-6, U * PI_REF * a * a, 2 * PI_REF * a * U * j1(ks * a) / ks)
    else:
        vt = np.where(k < 1e-6, U * 4.0 / 3.0 * PI_REF * a ** 3,
                      4 * PI_REF * U * a ** 3 * (np.sin(ks * a) - ks * a * np.cos(ks * a)) / (ks * a) ** 3)
    phi = np.fft.ifftn(vt * np.fft.fftn(np.abs(psi) ** 2)).real
    want_mu = T + (V.real + phi + 1j * V.imag) * psi
    want_en = T + (V.real + 0.5 * phi + 1j * V.imag) * psi
    assert np.linalg.norm(hm - want_mu) <= 1e-12 * np.linalg.norm(want_mu)
    assert np.linalg.norm(he - want_en) <= 1e-12 * np.linalg.norm(want_en)
