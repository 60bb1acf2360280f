"""fgpe_b200 -- B200-native Gross-Pitaevskii solver (Python side of the C ABI).

The product is ``libgpe.so`` (hand-written sm_100a CUDA kernels behind the C
ABI of ``include/gpe.h``) plus the ``gpe`` command-line driver.  This module is
a thin ctypes mirror of that ABI for tests, the benchmark and Python users; it
loads the in-tree library and fails loudly when it is missing -- there is no
CPU fallback.

Grid arrays are numpy complex128 of shape (nz, ny, nx) (x fastest, the
reference's index z*NX*NY + y*NX + x, hpp/header.hpp:20).
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, byref, c_double, c_int, c_longlong, c_void_p

import numpy as np

__all__ = [
    "GPEConfig", "GPEError", "Solver", "Batch", "lib", "make_config", "grid_axes", "kspace_kernel", "tune",
    "set_tune_cache", "pass_variant_exists",
    "C128", "C64", "HAM_BEC", "HAM_BEC2", "HAM_TEMPLATE", "HAM_DIPOLAR",
    "IMAG_HEAVYBALL", "IMAG_RK4", "NO_HAMIL_PARAMS",
]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpe.so")

NO_HAMIL_PARAMS = 32
C128, C64 = 0, 1
HAM_BEC, HAM_BEC2, HAM_TEMPLATE, HAM_DIPOLAR, HAM_SOFT, HAM_USER = 0, 1, 2, 3, 4, 5
IMAG_HEAVYBALL, IMAG_RK4 = 0, 1
# gpe_batch_mode (include/gpe.h)
BATCH_PER_GROUP, BATCH_PERSISTENT, BATCH_GROUPED = 0, 1, 2
# gpe_lattice (include/gpe.h): Psi::force*Lattice seeds
LATTICE_1D, LATTICE_2D_TRIANGULAR, LATTICE_2D_SQUARE, LATTICE_3D_HEX, LATTICE_3D_FCC, LATTICE_3D_BCC, \
    LATTICE_3D_SC = 1, 2, 3, 4, 5, 6, 7
ABI_VERSION = 2

STATUS = {0: "ok", 1: "invalid argument", 2: "unsupported", 3: "CUDA error",
          4: "out of memory", 5: "diverged", 6: "timeout", 7: "I/O error"}


class GPEError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"gpe status {status} ({STATUS.get(status, '?')}): {msg}")
        self.status = status


class GPEConfig(ctypes.Structure):
    """ctypes image of ``gpe_config`` (include/gpe.h)."""
    _fields_ = [
        ("abi_version", c_int), ("nx", c_int), ("ny", c_int), ("nz", c_int), ("dim", c_int),
        ("xmax", c_double * 3), ("dx", c_double * 3),
        ("ncomp", c_int), ("precision", c_int), ("hamiltonian", c_int), ("imag_scheme", c_int),
        ("prms", c_double * NO_HAMIL_PARAMS), ("dt", c_double), ("beta", c_double),
        ("npart", c_double * 2), ("epsilon_e", c_double), ("reserved", c_int * 8),
    ]

    def copy(self) -> "GPEConfig":
        c = GPEConfig()
        ctypes.memmove(byref(c), byref(self), ctypes.sizeof(GPEConfig))
        return c


_lib = None


def lib() -> ctypes.CDLL:
    """Load libgpe.so from the package directory (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} not found: build it with `make -C fgpe_b200` "
                           "(or __graft_entry__.build()); there is no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    H = c_void_p
    P = POINTER(c_double)
    sig = {
        "gpe_abi_version": (c_int, []),
        "gpe_last_error_string": (ctypes.c_char_p, []),
        "gpe_status_string": (ctypes.c_char_p, [c_int]),
        "gpe_config_init": (c_int, [POINTER(GPEConfig)]),
        "gpe_fft_length_supported": (c_int, [c_int]),
        "gpe_kspace_kernel": (c_int, [POINTER(GPEConfig), P]),
        "gpe_create": (c_int, [POINTER(GPEConfig), POINTER(H)]),
        "gpe_destroy": (c_int, [H]),
        "gpe_set_stream": (c_int, [H, c_void_p]),
        "gpe_set_params": (c_int, [H, P]),
        "gpe_set_psi": (c_int, [H, c_int, P]),
        "gpe_get_psi": (c_int, [H, c_int, P]),
        "gpe_set_vext": (c_int, [H, c_int, P]),
        "gpe_set_psi_device": (c_int, [H, c_int, c_void_p]),
        "gpe_imprint_vortex_tube": (c_int, [H, c_int, c_double]),
        "gpe_seed_lattice": (c_int, [H, c_int, c_int, c_double, c_double, P, c_double, c_double]),
        "gpe_get_psi_device": (c_int, [H, c_int, c_void_p]),
        "gpe_step_real": (c_int, [H, c_int, c_int, P]),
        "gpe_step_imag": (c_int, [H, c_int, c_int, POINTER(c_int), POINTER(c_int)]),
        "gpe_imag_state": (c_int, [H, P]),
        "gpe_reset_imag_state": (c_int, [H]),
        "gpe_laplace": (c_int, [H, c_int, P]),
        "gpe_apply_h": (c_int, [H, c_double, c_int, P, P]),
        "gpe_observables": (c_int, [H, c_double, P]),
        "gpe_fft": (c_int, [H, c_int, c_int]),
        "gpe_momentum_x": (c_int, [H, c_int, P]),
        "gpe_average_cos": (c_int, [H, c_int, P]),
        "gpe_average_cos2": (c_int, [H, c_int, P]),
        "gpe_relative_phase": (c_int, [H, P]),
        "gpe_dsz_dt": (c_int, [H, P]),
        "gpe_sync": (c_int, [H]),
        "gpe_kernel_launches": (c_longlong, [H]),
        "gpe_profile_enable": (c_int, [H, c_int]),
        "gpe_profile_read": (c_int, [H, P, POINTER(c_longlong)]),
        "gpe_control_set_basis": (c_int, [H, c_int, P]),
        "gpe_control_gradient": (c_int, [H, P, c_int, P, c_int, P, P]),
        "gpe_batch_create": (c_int, [POINTER(GPEConfig), c_int, POINTER(H)]),
        "gpe_batch_destroy": (c_int, [H]),
        "gpe_batch_set_stream": (c_int, [H, c_void_p]),
        "gpe_batch_set_psi": (c_int, [H, c_int, P]),
        "gpe_batch_set_vext": (c_int, [H, c_int, P]),
        "gpe_batch_get_psi": (c_int, [H, c_int, P]),
        "gpe_batch_step_imag": (c_int, [H, c_int, POINTER(c_int), POINTER(c_int)]),
        "gpe_batch_imag_state": (c_int, [H, c_int, P]),
        "gpe_batch_kernel_launches": (c_longlong, [H]),
        "gpe_tune": (c_int, [POINTER(GPEConfig), c_int, ctypes.c_char_p, P]),
        "gpe_set_tune_cache": (c_int, [ctypes.c_char_p]),
        "gpe_batch_tune": (c_int, [H, ctypes.c_char_p, P]),
        "gpe_batch_groups": (c_int, [H]),
        "gpe_batch_set_persistent": (c_int, [H, c_int, ctypes.c_uint]),
        "gpe_batch_persistent": (c_int, [H]),
        "gpe_batch_set_launch_mode": (c_int, [H, c_int, ctypes.c_uint]),
        "gpe_batch_launch_mode": (c_int, [H]),
        "gpe_batch_persistent_info": (c_int, [H, POINTER(c_longlong)]),
        "gpe_get_pass_variants": (c_int, [H, POINTER(c_int)]),
        "gpe_set_pass_variants": (c_int, [H, POINTER(c_int)]),
        "gpe_pass_variant_exists": (c_int, [POINTER(GPEConfig), c_int, c_int]),
        "gpe_set_user_hamiltonian": (c_int, [H, c_void_p]),
        "gpe_set_flow": (c_int, [H, c_int, ctypes.c_uint]),
        "gpe_flow_active": (c_int, [H]),
        "gpe_flow_status": (c_int, [H, POINTER(c_int)]),
        "gpe_set_x_staging": (c_int, [H, c_int]),
        "gpe_x_staging": (c_int, [H]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    if L.gpe_abi_version() != ABI_VERSION:
        raise RuntimeError("libgpe ABI version mismatch")
    _lib = L
    return L


def _check(status: int) -> None:
    if status != 0:
        msg = lib().gpe_last_error_string()
        raise GPEError(status, msg.decode() if msg else "")


def _dp(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_double))


def grid_axes(cfg: GPEConfig):
    """Cell-centred x, y, z axes (src/baseHamiltonian.cu:25-51)."""
    out = []
    for d, n in enumerate((cfg.nx, cfg.ny, cfg.nz)):
        zero = (cfg.dim == 1 and d > 0) or (cfg.dim == 2 and d == 2)
        i = np.arange(n, dtype=np.float64)
        out.append(np.zeros(n) if zero else -cfg.xmax[d] + i * cfg.dx[d] + 0.5 * cfg.dx[d])
    return out


def make_config(shape, xmax, *, dt=1e-3, ncomp=1, precision=C128, hamiltonian=HAM_BEC,
                imag_scheme=IMAG_HEAVYBALL, g=0.0, prms=None, beta=0.0, npart=(1.0, 1.0),
                epsilon_e=0.0, dim=None) -> GPEConfig:
    """Config in code units.  shape = (nx, ny, nz); xmax = half box widths.

    ``g`` sets a constant contact coupling g = 4 pi a for the BEC plugin
    (d_h_params = {a, a, a, 0, 0, 0}); ``prms`` overrides d_h_params entirely.
    """
    c = GPEConfig()  # zero-initialised, as gpe_config_init does
    c.abi_version = ABI_VERSION
    nx, ny, nz = shape
    c.nx, c.ny, c.nz = nx, ny, nz
    if dim is None:
        dim = 3 if nz > 1 else (2 if ny > 1 else 1)
    c.dim = dim
    xm = list(xmax) if np.ndim(xmax) else [xmax] * 3
    for d in range(3):
        c.xmax[d] = xm[d]
        c.dx[d] = 2.0 * xm[d] / (nx, ny, nz)[d]
    c.ncomp = ncomp
    c.precision = precision
    c.hamiltonian = hamiltonian
    c.imag_scheme = imag_scheme
    if prms is None:
        prms = np.zeros(NO_HAMIL_PARAMS)
        a = g / (4.0 * 3.141592653589793)
        prms[0:3] = a
    for i in range(NO_HAMIL_PARAMS):
        c.prms[i] = float(prms[i]) if i < len(prms) else 0.0
    c.dt = dt
    c.beta = beta
    c.npart[0], c.npart[1] = npart
    c.epsilon_e = epsilon_e
    return c


NSVAR = 12  # strided-pass variants per axis and mode (include/gpe.h, gpe_pass_variant_exists)


def tune(cfg: GPEConfig, workload: int = 0, cache_path: str | None = None) -> dict:
    """Autotune the pass variants of cfg's grid (gpe_tune): workload 0 =
    real-time RK4 steps, 1 = imaginary-time iterations.  Stores the result
    in the JSON-lines cache_path when given."""
    rep = np.zeros(13)
    _check(lib().gpe_tune(byref(cfg), workload, cache_path.encode() if cache_path else None, _dp(rep)))
    return {"default_us": float(rep[0]), "tuned_us": float(rep[1]), "timed": int(rep[2]),
            "variants": [int(x) for x in rep[3:9]], "xrows": int(rep[9]), "yz": int(rep[10]),
            "flow": int(rep[11]), "xstage": int(rep[12])}


def set_tune_cache(path: str | None) -> None:
    """Process-wide cache that new handles and batches apply (None: $GPE_TUNE_CACHE)."""
    _check(lib().gpe_set_tune_cache(path.encode() if path else None))


def pass_variant_exists(cfg: GPEConfig, axis: int, v: int) -> bool:
    return bool(lib().gpe_pass_variant_exists(byref(cfg), axis, v))


def kspace_kernel(cfg: GPEConfig) -> np.ndarray:
    """V~(k) of a GPE_HAM_DIPOLAR / GPE_HAM_SOFT config as libgpe builds it
    (host arithmetic, gpe_kspace_kernel), shape (nz, ny, nx)."""
    out = np.zeros((cfg.nz, cfg.ny, cfg.nx))
    _check(lib().gpe_kspace_kernel(byref(cfg), _dp(out)))
    return out


class Solver:
    """One libgpe handle (owns its device buffers)."""

    def __init__(self, cfg: GPEConfig):
        self.cfg = cfg.copy()
        self.shape = (cfg.nz, cfg.ny, cfg.nx)
        self.N = cfg.nx * cfg.ny * cfg.nz
        h = c_void_p()
        _check(lib().gpe_create(byref(self.cfg), byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().gpe_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr: int) -> None:
        _check(lib().gpe_set_stream(self._h, c_void_p(stream_ptr)))

    def set_params(self, prms) -> None:
        p = np.zeros(NO_HAMIL_PARAMS)
        p[: len(prms)] = prms
        _check(lib().gpe_set_params(self._h, _dp(p)))

    def _c128(self, arr) -> np.ndarray:
        a = np.ascontiguousarray(arr, dtype=np.complex128).reshape(-1)
        if a.size != self.N:
            raise ValueError(f"expected {self.N} points, got {a.size}")
        return a

    def set_psi(self, comp: int, psi) -> None:
        a = self._c128(psi)
        _check(lib().gpe_set_psi(self._h, comp, _dp(a.view(np.float64))))

    def get_psi(self, comp: int = 0) -> np.ndarray:
        out = np.empty(self.N, np.complex128)
        _check(lib().gpe_get_psi(self._h, comp, _dp(out.view(np.float64))))
        return out.reshape(self.shape)

    def set_vext(self, comp: int, v) -> None:
        a = self._c128(v)
        _check(lib().gpe_set_vext(self._h, comp, _dp(a.view(np.float64))))

    def set_psi_device(self, comp: int, ptr: int) -> None:
        _check(lib().gpe_set_psi_device(self._h, comp, c_void_p(ptr)))

    def get_psi_device(self, comp: int, ptr: int) -> None:
        _check(lib().gpe_get_psi_device(self._h, comp, c_void_p(ptr)))

    def imprint_vortex_tube(self, comp: int, ncirc: float) -> None:
        """psi *= exp(i ncirc 2 pi x / (2 xmax_x)) on the device (gpe_imprint_vortex_tube)."""
        _check(lib().gpe_imprint_vortex_tube(self._h, comp, float(ncirc)))

    def seed_lattice(self, comp: int, lattice: int, amp: float, k: float, off=(0.0, 0.0, 0.0),
                     seed_npart: float = 1.0, norm_npart: float = 1.0) -> None:
        """Add a Psi::force*Lattice seed and renormalise, on the device (gpe_seed_lattice)."""
        o = np.ascontiguousarray(off, dtype=np.float64)
        if o.size != 3:
            raise ValueError("off needs 3 offsets")
        _check(lib().gpe_seed_lattice(self._h, comp, int(lattice), float(amp), float(k), _dp(o), float(seed_npart),
                                      float(norm_npart)))

    def step_real(self, first_iteration: int, nsteps: int, want_obs: bool = False):
        if want_obs:
            obs = np.zeros(6)
            _check(lib().gpe_step_real(self._h, first_iteration, nsteps, _dp(obs)))
            return obs[: 3 * self.cfg.ncomp]
        _check(lib().gpe_step_real(self._h, first_iteration, nsteps, None))
        return None

    def step_imag(self, first_iteration: int, nsteps: int):
        done, conv = c_int(0), c_int(0)
        _check(lib().gpe_step_imag(self._h, first_iteration, nsteps, byref(done), byref(conv)))
        return done.value, bool(conv.value)

    def control_set_basis(self, G) -> None:
        """Control basis functions G_k (real, shape (nctrl, nz, ny, nx))."""
        g = np.ascontiguousarray(G, dtype=np.float64).reshape(-1)
        if g.size % self.N:
            raise ValueError("basis size is not a multiple of the grid size")
        _check(lib().gpe_control_set_basis(self._h, g.size // self.N, _dp(g)))
        self._nctrl = g.size // self.N

    def control_gradient(self, u, target, checkpoint_every: int = 50, want_grad: bool = True):
        """Infidelity 1 - |<target|psi(T)>|^2 after u.shape[0] controlled RK4
        steps from the current state, and its gradient with respect to u
        (shape (nsteps, nctrl)) by the adjoint.  The state is left unchanged."""
        un = np.ascontiguousarray(u, dtype=np.float64)
        if un.ndim != 2 or un.shape[1] != getattr(self, "_nctrl", -1):
            raise ValueError("u must have shape (nsteps, nctrl)")
        t = self._c128(target)
        loss = c_double()
        grad = np.zeros_like(un) if want_grad else None
        _check(lib().gpe_control_gradient(self._h, _dp(un), un.shape[0], _dp(t.view(np.float64)),
                                          int(checkpoint_every), byref(loss),
                                          _dp(grad) if want_grad else None))
        return loss.value, grad

    def imag_state(self) -> np.ndarray:
        out = np.zeros(8)
        _check(lib().gpe_imag_state(self._h, _dp(out)))
        return out[: 4 * self.cfg.ncomp]

    def reset_imag_state(self) -> None:
        _check(lib().gpe_reset_imag_state(self._h))

    def laplace(self, comp: int = 0) -> np.ndarray:
        out = np.empty(self.N, np.complex128)
        _check(lib().gpe_laplace(self._h, comp, _dp(out.view(np.float64))))
        return out.reshape(self.shape)

    def apply_h(self, t: float, comp: int = 0):
        hmu = np.empty(self.N, np.complex128)
        hen = np.empty(self.N, np.complex128)
        _check(lib().gpe_apply_h(self._h, t, comp, _dp(hmu.view(np.float64)), _dp(hen.view(np.float64))))
        return hmu.reshape(self.shape), hen.reshape(self.shape)

    def observables(self, t: float = 0.0) -> np.ndarray:
        out = np.zeros(6)
        _check(lib().gpe_observables(self._h, t, _dp(out)))
        return out[: 3 * self.cfg.ncomp]

    def fft(self, comp: int, sign: int) -> None:
        _check(lib().gpe_fft(self._h, comp, sign))

    def _scalar(self, name: str, *args) -> float:
        out = c_double(0.0)
        _check(getattr(lib(), name)(self._h, *args, byref(out)))
        return out.value

    def momentum_x(self, comp: int = 0) -> float:
        """sum Re(conj(psi) P_x psi) DV before the plugin's division (alg_calcPx)."""
        return self._scalar("gpe_momentum_x", comp)

    def average_cos(self, comp: int = 0) -> float:
        """sum cos(2 pi x/L) |psi_comp|^2 DV (alg_calcCos; divide by the norm for <cos>)."""
        return self._scalar("gpe_average_cos", comp)

    def average_cos2(self, sign: int = 1) -> float:
        """sum cos(2 pi x/L) |psi_0 + sign psi_1|^2 DV."""
        return self._scalar("gpe_average_cos2", sign)

    def relative_phase(self) -> float:
        """sum (arg psi_0 - arg psi_1) DV."""
        return self._scalar("gpe_relative_phase")

    def dsz_dt(self) -> float:
        """sum sqrt(n_0 n_1) sin(arg psi_0 - arg psi_1) DV."""
        return self._scalar("gpe_dsz_dt")

    def sync(self) -> None:
        _check(lib().gpe_sync(self._h))

    @property
    def launches(self) -> int:
        return int(lib().gpe_kernel_launches(self._h))

    PROF_KINDS = ("x_fwd", "x_inv", "x_full", "s_fwd", "s_inv", "s_fki", "flow", "s_flow")

    def set_flow(self, mode, wait_bound: int = 0) -> None:
        """Persistent launches (gpe_set_flow): True / 1 = one launch per
        real-time RK4 step, 2 = the three strided passes of each stage in
        one launch, False / 0 = the per-pass chain; wait_bound 0 keeps the
        current bound."""
        _check(lib().gpe_set_flow(self._h, int(mode), int(wait_bound)))

    def set_x_staging(self, on: bool) -> None:
        """Stage the fused real-time x pass's epilogue inputs in shared memory
        (gpe_set_x_staging; complex64 one-field chains)."""
        _check(lib().gpe_set_x_staging(self._h, 1 if on else 0))

    @property
    def x_staging(self) -> bool:
        return bool(lib().gpe_x_staging(self._h))

    @property
    def flow_active(self) -> int:
        """1 (whole step), 2 (strided stages) or 0 (per-pass chain)."""
        return int(lib().gpe_flow_active(self._h))

    def flow_status(self) -> int:
        """0, or GPE_ERR_TIMEOUT when a persistent step gave up since the last
        call (the step's counters are then re-armed)."""
        st = c_int(0)
        _check(lib().gpe_flow_status(self._h, byref(st)))
        return int(st.value)

    def set_user_hamiltonian(self, ops_ptr: int) -> None:
        """Install a user Hamiltonian plugin (the gpe_user_hamiltonian table a
        plugin built with include/gpe_plugin.cuh returns) on a HAM_USER handle."""
        _check(lib().gpe_set_user_hamiltonian(self.handle, c_void_p(ops_ptr)))

    def pass_variants(self) -> list:
        """[s(y, fwd), s(y, fki), s(y, inv), s(z, fwd), s(z, fki), s(z, inv), x rows, fused y-z]."""
        out = (c_int * 8)()
        _check(lib().gpe_get_pass_variants(self.handle, out))
        return list(out)

    def set_pass_variants(self, v) -> None:
        v = list(v) + [0] * (8 - len(v))
        arr = (c_int * 8)(*[int(x) for x in v])
        _check(lib().gpe_set_pass_variants(self.handle, arr))

    def profile(self, enable: bool) -> None:
        _check(lib().gpe_profile_enable(self._h, 1 if enable else 0))

    def profile_read(self) -> dict:
        """{kind: (summed ms, launches)} since the previous read (syncs)."""
        ms = np.zeros(len(self.PROF_KINDS))
        cnt = (c_longlong * len(self.PROF_KINDS))()
        _check(lib().gpe_profile_read(self._h, _dp(ms), cnt))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.PROF_KINDS)}


class Batch:
    """Independent one-component instances advanced together (gpe_batch):
    instances of equal geometry share every pass launch, one iteration of
    all groups is a CUDA graph on a non-default stream."""

    def __init__(self, cfgs):
        self.cfgs = [c.copy() for c in cfgs]
        arr = (GPEConfig * len(cfgs))(*self.cfgs)
        h = c_void_p()
        _check(lib().gpe_batch_create(arr, len(cfgs), byref(h)))
        self._h = h
        self.n = len(cfgs)

    def close(self):
        if getattr(self, "_h", None):
            lib().gpe_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _c128(self, i, arr):
        c = self.cfgs[i]
        a = np.ascontiguousarray(arr, dtype=np.complex128).reshape(-1)
        if a.size != c.nx * c.ny * c.nz:
            raise ValueError(f"instance {i}: expected {c.nx * c.ny * c.nz} points, got {a.size}")
        return a

    def set_stream(self, stream_ptr: int) -> None:
        _check(lib().gpe_batch_set_stream(self._h, c_void_p(stream_ptr)))

    def set_psi(self, i: int, psi) -> None:
        a = self._c128(i, psi)
        _check(lib().gpe_batch_set_psi(self._h, i, _dp(a.view(np.float64))))

    def set_vext(self, i: int, v) -> None:
        a = self._c128(i, v)
        _check(lib().gpe_batch_set_vext(self._h, i, _dp(a.view(np.float64))))

    def get_psi(self, i: int) -> np.ndarray:
        c = self.cfgs[i]
        out = np.empty(c.nx * c.ny * c.nz, np.complex128)
        _check(lib().gpe_batch_get_psi(self._h, i, _dp(out.view(np.float64))))
        return out.reshape(c.nz, c.ny, c.nx)

    def step_imag(self, nsteps: int):
        """Returns (iterations done per instance, converged flag per instance)."""
        it = (c_int * self.n)()
        cv = (c_int * self.n)()
        _check(lib().gpe_batch_step_imag(self._h, nsteps, it, cv))
        return np.array(it[:], dtype=np.int64), np.array(cv[:], dtype=bool)

    def imag_state(self, i: int) -> np.ndarray:
        out = np.zeros(4)
        _check(lib().gpe_batch_imag_state(self._h, i, _dp(out)))
        return out

    def tune(self, cache_path: str | None = None) -> list:
        """Tune every geometry group in place (gpe_batch_tune): per group
        (default, tuned) microseconds per imaginary-time iteration."""
        ng = lib().gpe_batch_groups(self._h)
        rep = np.zeros(2 * max(ng, 1))
        _check(lib().gpe_batch_tune(self._h, cache_path.encode() if cache_path else None, _dp(rep)))
        return [(float(rep[2 * g]), float(rep[2 * g + 1])) for g in range(ng)]

    def set_persistent(self, enable: bool = True, wait_bound: int = 0) -> None:
        """One cooperative launch per RK4 stage for every instance
        (gpe_batch_set_persistent); wait_bound: iterations a grid-barrier
        wait may spin, 0 for the default (about a second)."""
        _check(lib().gpe_batch_set_persistent(self._h, 1 if enable else 0, int(wait_bound)))

    def set_launch_mode(self, mode: int, wait_bound: int = 0) -> None:
        """BATCH_PER_GROUP, BATCH_PERSISTENT or BATCH_GROUPED (gpe_batch_set_launch_mode)."""
        _check(lib().gpe_batch_set_launch_mode(self._h, int(mode), int(wait_bound)))

    @property
    def launch_mode(self) -> int:
        return int(lib().gpe_batch_launch_mode(self._h))

    @property
    def persistent(self) -> bool:
        return bool(lib().gpe_batch_persistent(self._h))

    def persistent_info(self) -> dict:
        """Resources of the persistent stage kernel (gpe_batch_persistent_info)."""
        out = (c_longlong * 9)()
        _check(lib().gpe_batch_persistent_info(self._h, out))
        keys = ("registers", "static_smem", "max_threads", "local_bytes", "ctas_per_sm", "sms", "cooperative",
                "dynamic_smem", "last_grid")
        return dict(zip(keys, (int(v) for v in out)))

    @property
    def launches(self) -> int:
        return int(lib().gpe_batch_kernel_launches(self._h))
