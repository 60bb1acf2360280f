"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "fgpe_b200", "libgpe.so")


def declared_functions():
    names = []
    inc = os.path.join(ROOT, "include")
    for fn in sorted(os.listdir(inc)):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(inc, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(gpe[a-z_0-9]*)\s*\(", src):
            if not m.group(1).startswith("gpe_status") and m.group(1) not in names:
                names.append(m.group(1))
    return names


def test_library_exists():
    assert os.path.exists(LIB), "libgpe.so not built (make -C fgpe_b200)"


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 20
    lib = ctypes.CDLL(LIB)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    assert not [n for n in names if n not in exported]


def test_host_only_entry_points_work_without_gpu():
    import fgpe_b200 as g
    L = g.lib()
    assert L.gpe_abi_version() == 2
    cfg = g.GPEConfig()
    assert L.gpe_config_init(ctypes.byref(cfg)) == 0
    assert cfg.abi_version == 2 and cfg.ncomp == 1 and cfg.nx == 1
    for n in (1, 2, 3, 5, 8, 96, 128, 192, 384, 512, 768, 1024, 25, 27, 864):
        assert L.gpe_fft_length_supported(n) == 1, n
    for n in (0, 7, 14, 2048, 15, 1536):
        assert L.gpe_fft_length_supported(n) == 0, n
    assert L.gpe_status_string(5) == b"diverged"
    h = ctypes.c_void_p()
    assert L.gpe_create(None, ctypes.byref(h)) == 1  # null config -> invalid argument
    assert b"null" in L.gpe_last_error_string()
    bad = g.make_config((14, 8, 8), 4.0)
    assert L.gpe_create(ctypes.byref(bad), ctypes.byref(h)) == 2  # no FFT plan for 14


def test_launch_form_entry_points_reject_bad_arguments_without_gpu():
    """The persistent-launch and x-staging switches validate their arguments
    on the host before any device work (null handle, mode out of range)."""
    import fgpe_b200 as g
    L = g.lib()
    st = ctypes.c_int(-1)
    assert L.gpe_set_flow(None, 1, 0) == 1
    assert L.gpe_flow_status(None, ctypes.byref(st)) == 1
    assert L.gpe_flow_active(None) == 0
    assert L.gpe_set_x_staging(None, 1) == 1
    assert L.gpe_x_staging(None) == 0
    assert b"null handle" in L.gpe_last_error_string()


def test_config_struct_layout():
    import fgpe_b200 as g
    # int abi, nx, ny, nz, dim; pad; 3+3 doubles; 4 ints; 32 doubles; dt, beta, npart[2], eps; 8 ints
    assert ctypes.sizeof(g.GPEConfig) == 5 * 4 + 4 + 6 * 8 + 4 * 4 + 32 * 8 + 5 * 8 + 8 * 4
