"""User Hamiltonian plug-point (include/gpe_plugin.cuh, gpe_set_user_hamiltonian):
the example plugin fgpe_b200/plugins/user_bec.cu re-implements the
one-component BEC term (hamiltonians/BEC_oneComponent.cu:128-178) as a user
functor compiled in its own library; a GPE_HAM_USER handle with it must
reproduce the built-in GPE_HAM_BEC handle to the rounding of the precision
(1e-13 relative in complex128, 1e-6 in complex64)."""
import ctypes
import os

import numpy as np
import pytest

from fgpe_b200 import C64, C128, HAM_BEC, HAM_USER, IMAG_RK4, GPEError, Solver, make_config

from test_oracle import PI_REF, gaussian, harmonic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PLUGIN = os.path.join(ROOT, "fgpe_b200", "plugins", "libgpe_user_bec.so")


def plugin_ops():
    L = ctypes.CDLL(PLUGIN)
    L.gpe_user_bec.restype = ctypes.c_void_p
    return L, L.gpe_user_bec()


def test_plugin_library_exports_its_table():
    """Host only: the plugin's table carries the ABI version and both launchers."""
    assert os.path.exists(PLUGIN), "plugin not built (make -C fgpe_b200)"
    L, ops = plugin_ops()
    assert ops
    tab = ctypes.cast(ops, ctypes.POINTER(ctypes.c_int))
    assert tab[0] == 2  # GPE_ABI_VERSION
    ptrs = ctypes.cast(ops + 8, ctypes.POINTER(ctypes.c_void_p))
    assert ptrs[0] and ptrs[1]


def cfg_of(shape, prec, ham, scheme=0):
    prms = np.zeros(32)
    prms[:6] = [30.0 / (4 * PI_REF), 45.0 / (4 * PI_REF), 40.0 / (4 * PI_REF), 0.01, 0.02, 0.05]  # quench
    return make_config(shape, (5.0, 4.0, 3.0), dt=1e-3, precision=prec, prms=prms, hamiltonian=ham, beta=0.9,
                       imag_scheme=scheme, epsilon_e=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [C128, C64])
@pytest.mark.parametrize("shape", [(64, 32, 16), (128, 128, 1), (32, 24, 20)])
def test_user_plugin_reproduces_builtin_bec(gpu, prec, shape):
    _, ops = plugin_ops()
    out = {}
    for ham in (HAM_BEC, HAM_USER):
        for scheme in (0, IMAG_RK4):
            cfg = cfg_of(shape, prec, ham, scheme)
            V = harmonic(cfg, (1.0, 1.3, 1.7)) + 0.05j * harmonic(cfg)
            psi = gaussian(cfg, seed=3, noise=0.05)
            with Solver(cfg) as s:
                if ham == HAM_USER:
                    s.set_user_hamiltonian(ops)
                s.set_vext(0, V)
                s.set_psi(0, psi)
                r = [s.apply_h(0.015, 0)[0], s.apply_h(0.015, 0)[1], s.observables(0.03)]
                s.step_imag(0, 6)
                r += [s.get_psi(0), s.imag_state()]
                s.set_psi(0, psi)
                r += [s.step_real(0, 5, want_obs=True), s.get_psi(0)]
                out[(ham, scheme)] = r
    # The plugin runs the same arithmetic, compiled in another translation
    # unit: the compiler may fuse a multiply-add differently there, so the
    # results agree to the last bits of the precision, not bit for bit.
    tol = 1e-13 if prec == C128 else 1e-6
    for scheme in (0, IMAG_RK4):
        for a, b in zip(out[(HAM_BEC, scheme)], out[(HAM_USER, scheme)]):
            a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
            assert np.linalg.norm(a - b) <= tol * np.linalg.norm(a)


@pytest.mark.gpu
def test_user_handle_needs_its_plugin(gpu):
    cfg = cfg_of((64, 32, 16), C128, HAM_USER)
    with Solver(cfg) as s:
        s.set_vext(0, harmonic(cfg))
        s.set_psi(0, gaussian(cfg))
        with pytest.raises(GPEError):
            s.step_real(0, 1)
    # a length the plugin was not built for
    cfg = cfg_of((96, 32, 16), C128, HAM_USER)
    _, ops = plugin_ops()
    with Solver(cfg) as s:
        s.set_user_hamiltonian(ops)
        s.set_vext(0, harmonic(cfg))
        s.set_psi(0, gaussian(cfg))
        with pytest.raises(GPEError):
            s.step_real(0, 1)
