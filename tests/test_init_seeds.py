"""Initial-state seeds on the device (gpe_seed_lattice, gpe_imprint_vortex_tube)
against the host mirror's Psi class (gpeh_init_psi_lattice), which
test_host_mirror pins bit for bit to the reference's own Psi class
(src/psi.cu:155-374).

The device seeds keep the reference's expression order without fused
multiply-adds; they differ from the host only by the device cosine/sine
(a few ulp) and the order of the norm's sum: tolerance 1e-14 relative."""
import ctypes

import numpy as np
import pytest

from fgpe_b200 import C64, C128, Solver, make_config

from test_host_mirror import dp, materialise, ours

pytestmark = pytest.mark.gpu

TOL = 1e-14
D = ctypes.c_double


def host_lattice(f, lattice, amp, k, off, typ=1):
    L = ours()
    L.gpeh_init_psi_lattice.argtypes = [ctypes.c_char_p, ctypes.c_int, D, D, D, D, D, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_double)]
    p = np.zeros(47)
    L.gpeh_params(f, dp(p))
    out = np.zeros(int(p[4]), np.complex128)
    assert L.gpeh_init_psi_lattice(f, lattice, amp, k, *off, typ, dp(out.view(np.float64))) == 0
    base = np.zeros(int(p[4]), np.complex128)
    assert L.gpeh_init_psi(f, 0, dp(base.view(np.float64))) == 0
    return p, base, out


def solver_for(p, prec):
    nx, ny, nz = int(p[0]), int(p[1]), int(p[2])
    cfg = make_config((nx, ny, nz), (p[5], p[6], p[7]), precision=prec)
    for d in range(3):  # the host's own grid numbers, not recomputed
        cfg.xmax[d] = p[5 + d]
        cfg.dx[d] = p[8 + d]
    return Solver(cfg), (nz, ny, nx)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("lattice", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("case", ["bec_harmonic_3d.txt", "bec_2d.txt"])
def test_lattice_seed_matches_host_psi_class(gpu, case, lattice, tmp_path):
    f = materialise(case, tmp_path)
    amp, k, off = 0.7, 1.9, (0.3, -0.2, 0.1)
    p, base, want = host_lattice(f, lattice, amp, k, off)
    npart = p[33]
    s, shape = solver_for(p, C128)
    with s:
        s.set_psi(0, base.reshape(shape))
        s.seed_lattice(0, lattice, amp, k, off, npart, npart)
        got = s.get_psi(0).reshape(-1)
    assert rel(got, want) < TOL, (lattice, rel(got, want))
    # complex64 handles seed in FP64 and keep the result as high + low parts
    s, shape = solver_for(p, C64)
    with s:
        s.set_psi(0, base.reshape(shape))
        s.seed_lattice(0, lattice, amp, k, off, npart, npart)
        assert rel(s.get_psi(0).reshape(-1), want) < TOL


def test_vortex_tube_imprint_matches_restatement(gpu, tmp_path):
    f = materialise("bec_harmonic_3d.txt", tmp_path)
    p, base, _ = host_lattice(f, 1, 0.0, 1.0, (0.0, 0.0, 0.0))
    s, shape = solver_for(p, C128)
    ncirc = 2.0
    with s:
        s.set_psi(0, base.reshape(shape))
        s.imprint_vortex_tube(0, ncirc)
        got = s.get_psi(0)
    # Psi::imprintVortexTube: x = -XMAX + i DX + DX/2, phase Ncirc 2 pi x / (2 XMAX)
    nx = int(p[0])
    x = -p[5] + np.arange(nx) * p[8] + 0.5 * p[8]
    ph = ncirc * 2 * np.pi / (2 * p[5]) * x
    want = base.reshape(shape) * (np.cos(ph) + 1j * np.sin(ph))[None, None, :]
    assert rel(got, want) < TOL
    assert np.allclose(np.abs(got), np.abs(base.reshape(shape)), rtol=1e-14, atol=0)


def test_seed_arguments_are_checked(gpu):
    from fgpe_b200 import GPEError
    cfg = make_config((16, 16, 16), 4.0)
    with Solver(cfg) as s:
        with pytest.raises(GPEError):
            s.seed_lattice(0, 9, 1.0, 1.0)
        with pytest.raises(GPEError):
            s.seed_lattice(0, 1, 1.0, 1.0, seed_npart=0.0)
        with pytest.raises(ValueError):
            s.seed_lattice(0, 1, 1.0, 1.0, off=(0.0, 0.0))
