"""gpe_norm_noalloc (the allocation-free norm over a caller-owned device
array, block partials in a fixed device array inside libgpe) against the
handle-based gpe_observables norm, through the C ABI.

Named to be collected last, so that it also runs after every other GPU test
has used the device and the library.
"""
import ctypes

import numpy as np
import pytest

from fgpe_b200 import C128, Solver, lib, make_config

from test_oracle import gaussian, harmonic

pytestmark = pytest.mark.gpu

MAX_POINTS = 134217728  # GPE_NORM_NOALLOC_MAX_POINTS, 512^3
TOL = 1e-12


def entry():
    f = lib().gpe_norm_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    return f


@pytest.mark.parametrize("shape", [(32, 24, 16), (128, 128, 64), (96, 40, 27), (1, 1, 1)])
def test_norm_noalloc_matches_observables(gpu, shape):
    import torch
    cfg = make_config(shape, (5.0, 4.0, 3.0), precision=C128, g=10.0)
    psi = gaussian(cfg, seed=5, noise=0.05, npart=2.5)
    with Solver(cfg) as s:
        s.set_vext(0, harmonic(cfg))
        s.set_psi(0, psi)
        want = s.observables(0.0)[0]
    dv = cfg.dx[0] * cfg.dx[1] * cfg.dx[2]
    dev_psi = torch.from_numpy(np.ascontiguousarray(psi).reshape(-1)).to("cuda")
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    f = entry()
    # two calls in a row on one stream: the second reuses the scratch the first left
    assert f(dev_psi.data_ptr(), psi.size, dv, out.data_ptr(), stream) == 0
    assert f(dev_psi.data_ptr(), psi.size, dv, out.data_ptr() + 8, stream) == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert abs(got[0] - want) <= TOL * abs(want), (got[0], want)
    assert abs(got[1] - want) <= TOL * abs(want), (got[1], want)
    assert got[0] == got[1]  # fixed reduction order: same bits
    assert abs(got[0] - np.sum(np.abs(psi) ** 2) * dv) <= TOL * abs(want)


def test_norm_noalloc_empty_input(gpu):
    import torch
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    assert entry()(None, 0, 1.0, out.data_ptr(), torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    assert out.item() == 0.0


def test_norm_noalloc_rejects_bad_arguments(gpu):
    import torch
    f = entry()
    L = lib()
    buf = torch.zeros(8, dtype=torch.complex128, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    assert f(buf.data_ptr(), MAX_POINTS + 1, 1.0, out.data_ptr(), st) == 2  # GPE_ERR_UNSUPPORTED
    assert b"limit" in L.gpe_last_error_string()
    assert f(buf.data_ptr(), -1, 1.0, out.data_ptr(), st) == 1
    assert f(buf.data_ptr() + 8, 4, 1.0, out.data_ptr(), st) == 1  # not 16-byte aligned
    assert f(buf.data_ptr(), 4, 1.0, None, st) == 1


def test_norm_noalloc_first_call_on_a_side_stream(gpu, tmp_path):
    """The one-time set-up of a device (scratch address lookup and a
    synchronous zeroing of the completion counter) must also be right when
    the very first call of the process is issued on a non-default stream:
    run that first call in a fresh process."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    prog = (
        "import ctypes, numpy as np, torch, sys\n"
        f"sys.path.insert(0, {root!r})\n"
        "from fgpe_b200 import lib\n"
        "f = lib().gpe_norm_noalloc\n"
        "f.restype = ctypes.c_int\n"
        "f.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]\n"
        "rng = np.random.default_rng(3)\n"
        "a = rng.standard_normal(300000) + 1j * rng.standard_normal(300000)\n"
        "d = torch.from_numpy(a).to('cuda')\n"
        "out = torch.full((2,), float('nan'), dtype=torch.float64, device='cuda')\n"
        "s = torch.cuda.Stream()\n"
        "torch.cuda.synchronize()\n"
        "with torch.cuda.stream(s):\n"
        "    assert f(d.data_ptr(), a.size, 0.5, out.data_ptr(), s.cuda_stream) == 0\n"
        "    assert f(d.data_ptr(), a.size, 0.5, out.data_ptr() + 8, s.cuda_stream) == 0\n"
        "s.synchronize()\n"
        "got = out.cpu().numpy()\n"
        "want = np.sum(np.abs(a) ** 2) * 0.5\n"
        "assert abs(got[0] - want) <= 1e-12 * want and got[0] == got[1], (got, want)\n"
        "print('ok')\n"
    )
    r = subprocess.run([sys.executable, "-c", prog], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr
