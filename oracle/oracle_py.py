"""ctypes loader for the FP64 host oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker or the timed CPU baseline.  The
interface mirrors fgpe_b200.Solver method for method so a parity test runs the
same calls on both.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, byref, c_double, c_int, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = ctypes.CDLL(LIB_PATH)
    P = POINTER(c_double)
    S = c_void_p
    from fgpe_b200 import GPEConfig  # the shared config struct layout
    sig = {
        "orc_set_threads": (None, [c_int]),
        "orc_get_threads": (c_int, []),
        "orc_create": (S, [POINTER(GPEConfig)]),
        "orc_destroy": (None, [S]),
        "orc_set_params": (c_int, [S, P]),
        "orc_set_psi": (c_int, [S, c_int, P]),
        "orc_get_psi": (c_int, [S, c_int, P]),
        "orc_set_vext": (c_int, [S, c_int, P]),
        "orc_step_real": (c_int, [S, c_int, c_int, P]),
        "orc_step_imag": (c_int, [S, c_int, c_int, POINTER(c_int), POINTER(c_int)]),
        "orc_imag_state": (c_int, [S, P]),
        "orc_reset_imag_state": (c_int, [S]),
        "orc_laplace": (c_int, [S, c_int, P]),
        "orc_apply_h": (c_int, [S, c_double, c_int, P, P]),
        "orc_observables": (c_int, [S, c_double, P]),
        "orc_fft": (c_int, [S, c_int, c_int]),
        "orc_fft3d": (None, [c_int, c_int, c_int, P, c_int]),
        "orc_axes": (None, [POINTER(GPEConfig), P, P, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(POINTER(c_double))


def set_threads(n: int) -> None:
    lib().orc_set_threads(n)


def get_threads() -> int:
    return lib().orc_get_threads()


def fft3d(a: np.ndarray, sign: int) -> np.ndarray:
    """Unnormalised DFT of a (nz, ny, nx) complex array, sign -1 / +1."""
    b = np.ascontiguousarray(a, dtype=np.complex128).copy()
    nz, ny, nx = b.shape
    lib().orc_fft3d(nx, ny, nz, _dp(b.view(np.float64)), sign)
    return b


def axes(cfg):
    out = [np.zeros(n) for n in (cfg.nx, cfg.ny, cfg.nz, cfg.nx, cfg.ny, cfg.nz)]
    lib().orc_axes(byref(cfg), *[_dp(o) for o in out])
    return out


# ---- logging-cadence observables: numpy restatements -----------------------------
# x[ix] = -XMAX + (ix + 1/2) DX (src/baseHamiltonian.cu:25-51), L = 2 XMAX[0];
# each returns the grid sum times DV, as the reference's reduction does
# (src/baseHamiltonian.cu:112-150).  psi arrays are (nz, ny, nx).
PI_REF = 3.141592653589793  # hpp/header.hpp:28


def _cos_weight(cfg):
    x = -cfg.xmax[0] + (np.arange(cfg.nx, dtype=np.float64) + 0.5) * cfg.dx[0]
    return np.cos(2 * PI_REF * x / (2 * cfg.xmax[0]))


def _dv(cfg):
    return cfg.dx[0] * cfg.dx[1] * cfg.dx[2]


def average_cos(cfg, psi):
    """CalcAverageCos (src/parallel.cu:535-561): sum cos(2 pi x/L) |psi|^2 DV."""
    return float(np.sum(_cos_weight(cfg) * np.abs(psi) ** 2) * _dv(cfg))


def average_cos2(cfg, psi1, psi2, sign):
    """CalcAverageCos for psi1 + sign psi2 (src/parallel.cu:739-771)."""
    return float(np.sum(_cos_weight(cfg) * np.abs(psi1 + sign * psi2) ** 2) * _dv(cfg))


def relative_phase_terms(psi1, psi2):
    """CalculateRelativePhase (src/parallel.cu:774-802), per point."""
    return np.arctan2(psi1.imag, psi1.real) - np.arctan2(psi2.imag, psi2.real)


def dsz_dt_terms(psi1, psi2):
    """CalculateDszDt (src/parallel.cu:805-839), per point."""
    ph = relative_phase_terms(psi1, psi2)
    return np.sqrt(np.abs(psi1) ** 2 * np.abs(psi2) ** 2) * np.sin(ph)


class OracleSolver:
    """Same methods as fgpe_b200.Solver, computed on the host in FP64."""

    def __init__(self, cfg):
        self.cfg = cfg.copy()
        self.shape = (cfg.nz, cfg.ny, cfg.nx)
        self.N = cfg.nx * cfg.ny * cfg.nz
        s = lib().orc_create(byref(self.cfg))
        if not s:
            raise ValueError("oracle rejected the configuration")
        self._s = c_void_p(s)

    def close(self):
        if getattr(self, "_s", None):
            lib().orc_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c128(self, arr):
        a = np.ascontiguousarray(arr, dtype=np.complex128).reshape(-1)
        assert a.size == self.N
        return a

    def set_params(self, prms):
        p = np.zeros(32)
        p[: len(prms)] = prms
        lib().orc_set_params(self._s, _dp(p))

    def set_psi(self, comp, psi):
        a = self._c128(psi)
        assert lib().orc_set_psi(self._s, comp, _dp(a.view(np.float64))) == 0

    def get_psi(self, comp=0):
        out = np.empty(self.N, np.complex128)
        assert lib().orc_get_psi(self._s, comp, _dp(out.view(np.float64))) == 0
        return out.reshape(self.shape)

    def set_vext(self, comp, v):
        a = self._c128(v)
        assert lib().orc_set_vext(self._s, comp, _dp(a.view(np.float64))) == 0

    def step_real(self, first_iteration, nsteps, want_obs=False):
        if want_obs:
            obs = np.zeros(6)
            lib().orc_step_real(self._s, first_iteration, nsteps, _dp(obs))
            return obs[: 3 * self.cfg.ncomp]
        lib().orc_step_real(self._s, first_iteration, nsteps, None)
        return None

    def step_imag(self, first_iteration, nsteps):
        done, conv = c_int(0), c_int(0)
        lib().orc_step_imag(self._s, first_iteration, nsteps, byref(done), byref(conv))
        return done.value, bool(conv.value)

    def imag_state(self):
        out = np.zeros(8)
        lib().orc_imag_state(self._s, _dp(out))
        return out[: 4 * self.cfg.ncomp]

    def reset_imag_state(self):
        lib().orc_reset_imag_state(self._s)

    def laplace(self, comp=0):
        out = np.empty(self.N, np.complex128)
        lib().orc_laplace(self._s, comp, _dp(out.view(np.float64)))
        return out.reshape(self.shape)

    def apply_h(self, t, comp=0):
        hmu = np.empty(self.N, np.complex128)
        hen = np.empty(self.N, np.complex128)
        lib().orc_apply_h(self._s, t, comp, _dp(hmu.view(np.float64)), _dp(hen.view(np.float64)))
        return hmu.reshape(self.shape), hen.reshape(self.shape)

    def observables(self, t=0.0):
        out = np.zeros(6)
        lib().orc_observables(self._s, t, _dp(out))
        return out[: 3 * self.cfg.ncomp]

    def fft(self, comp, sign):
        lib().orc_fft(self._s, comp, sign)
