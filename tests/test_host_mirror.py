"""Host mirror (fgpe_b200/host, via include/gpe_host.h) against the reference's
own host classes compiled from its sources (oracle/_ref/libref_host.so, see
oracle/ref.mk): input parsing, unit conversion, initial psi (including the
seeded noise), Vext and info.wtxt must be bit-identical.  Runs on CPU."""
import ctypes
import os
import shutil

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
INPUTS = os.path.join(ROOT, "tests", "inputs")
CASES = ["bec_harmonic_3d.txt", "bec_tube_3d.txt", "bec_2d.txt", "bec2_3d.txt", "bec2_tube.txt"]

needs_ref = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference host library not built (oracle/ref.mk)")


def ours():
    import fgpe_b200 as gp
    L = gp.lib()
    P = ctypes.POINTER(ctypes.c_double)
    L.gpeh_params.argtypes = [ctypes.c_char_p, P]
    L.gpeh_init_psi.argtypes = [ctypes.c_char_p, ctypes.c_int, P]
    L.gpeh_init_vext.argtypes = [ctypes.c_char_p, ctypes.c_int, P]
    L.gpeh_write_info.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, P, ctypes.c_void_p]
    L.gpeh_last_error.restype = ctypes.c_char_p
    return L


def ref():
    L = ctypes.CDLL(REF_LIB)
    P = ctypes.POINTER(ctypes.c_double)
    L.ref_params.argtypes = [ctypes.c_char_p, P]
    L.ref_init_psi.argtypes = [ctypes.c_char_p, ctypes.c_int, P]
    L.ref_init_vext.argtypes = [ctypes.c_char_p, ctypes.c_int, P]
    L.ref_write_info.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, P, ctypes.c_void_p]
    return L


def materialise(case, tmp_path):
    src = open(os.path.join(INPUTS, case)).read().replace("@OUT@", str(tmp_path) + "/run_")
    fn = tmp_path / case
    fn.write_text(src)
    return str(fn).encode()


def dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@needs_ref
@pytest.mark.parametrize("case", CASES)
def test_params_bit_identical(case, tmp_path):
    f = materialise(case, tmp_path)
    a = np.zeros(47)
    b = np.zeros(47)
    na = ours().gpeh_params(f, dp(a))
    nb = ref().ref_params(f, dp(b))
    assert na == nb
    assert np.array_equal(a, b), np.nonzero(a != b)


@needs_ref
@pytest.mark.parametrize("lattice", ["triangular", "HEX", "BCC", "SC", "FCC", "other", None])
@pytest.mark.parametrize("case", ["bec_harmonic_3d.txt", "bec_2d.txt"])
def test_soft_lattice_redefinition_bit_identical(case, lattice, tmp_path):
    # hamiltonian "soft": the domain is rounded to whole inter-droplet
    # distances (Params::RedefineLatticeSoft).  Without its keys the
    # reference exits (status 3, so it is not called in-process here) and the
    # mirror reports an error.
    src = open(os.path.join(INPUTS, case)).read().replace("@OUT@", str(tmp_path) + "/run_")
    src = src.replace('hamiltonian     "bec"', 'hamiltonian     "soft"')
    if lattice is not None:
        src += f'akrot           7.3\na_soft          1.37\nLatticetype     "{lattice}"\n'
    fn = tmp_path / ("soft_" + case)
    fn.write_text(src)
    f = str(fn).encode()
    a = np.zeros(47)
    if lattice is None:
        assert ours().gpeh_params(f, dp(a)) != 1
        assert b"akrot" in ours().gpeh_last_error()
        return
    b = np.zeros(47)
    assert ours().gpeh_params(f, dp(a)) == ref().ref_params(f, dp(b)) == 1
    assert np.array_equal(a, b), np.nonzero(a != b)
    base = np.zeros(47)
    ours().gpeh_params(materialise(case, tmp_path), dp(base))
    assert not np.array_equal(a[5:8], base[5:8])  # the domain changed


@needs_ref
@pytest.mark.parametrize("case", CASES)
def test_initial_psi_and_vext_bit_identical(case, tmp_path):
    f = materialise(case, tmp_path)
    p = np.zeros(47)
    nc = ours().gpeh_params(f, dp(p))
    n = int(p[4])
    types = [0] if nc == 1 else [1, 2]
    for t in types:
        for fn_o, fn_r in (("gpeh_init_psi", "ref_init_psi"), ("gpeh_init_vext", "ref_init_vext")):
            a = np.zeros(n, np.complex128)
            b = np.zeros(n, np.complex128)
            assert getattr(ours(), fn_o)(f, t, dp(a.view(np.float64))) == 0
            getattr(ref(), fn_r)(f, t, dp(b.view(np.float64)))
            assert np.array_equal(a.view(np.float64), b.view(np.float64)), (fn_o, t)


@needs_ref
@pytest.mark.parametrize("case", CASES)
def test_info_wtxt_identical(case, tmp_path):
    f = materialise(case, tmp_path)
    names = (ctypes.c_char_p * 3)(b"en", b"mu", b"convergence")
    units = (ctypes.c_char_p * 3)(b"code", b"code", b"code")
    vals = np.array([1.2345678901, -0.5, 3e-9])
    ref().ref_write_info(f, 7, 3, names, dp(vals), units)
    info = tmp_path / "run_info.wtxt"
    want = info.read_bytes()
    info.unlink()
    assert ours().gpeh_write_info(f, 7, 3, names, dp(vals), units) == 0
    assert info.read_bytes() == want


def test_info_wtxt_lengths_key(tmp_path):
    """ly/lz of info.wtxt: NX[0]*DX[1]*aho and NX[0]*DX[2]*aho as the reference
    writes them (src/output.cu:42-44) unless `wtxt_ref_lengths false`."""
    names = (ctypes.c_char_p * 1)(b"en")
    units = (ctypes.c_char_p * 1)(b"code")
    vals = np.array([1.0])
    lines = {}
    for flag in (None, "true", "false"):
        src = open(os.path.join(INPUTS, "bec_harmonic_3d.txt")).read().replace("@OUT@", str(tmp_path) + "/run_")
        if flag is not None:
            src += f"\nwtxt_ref_lengths {flag}\n"
        fn = tmp_path / "in.txt"
        fn.write_text(src)
        assert ours().gpeh_write_info(str(fn).encode(), 1, 1, names, dp(vals), units) == 0
        txt = (tmp_path / "run_info.wtxt").read_text()
        lines[flag] = {l.split()[0]: float(l.split()[1]) for l in txt.splitlines()
                       if l.split() and l.split()[0] in ("nx", "ny", "nz", "dx", "dy", "dz", "lx", "ly", "lz")}
    assert lines[None] == lines["true"]
    d = lines["false"]
    p = np.zeros(47)
    assert ours().gpeh_params(str(tmp_path / "in.txt").encode(), dp(p)) == 1
    aho = p[24]
    for ax, n, DX in (("ly", "ny", p[9]), ("lz", "nz", p[10])):
        assert d[n] != d["nx"]
        assert abs(d[ax] - d[n] * DX * aho) < 1e-5 * max(1.0, d[ax])
        assert abs(lines[None][ax] - d["nx"] * DX * aho) < 1e-5 * max(1.0, d[ax])


def test_missing_key_is_an_error_not_exit(tmp_path):
    src = open(os.path.join(INPUTS, "bec_2d.txt")).read().replace("@OUT@", str(tmp_path) + "/run_")
    src = "\n".join(l for l in src.splitlines() if not l.startswith("mass"))
    fn = tmp_path / "bad.txt"
    fn.write_text(src)
    out = np.zeros(47)
    assert ours().gpeh_params(str(fn).encode(), dp(out)) == -1
    assert b"mass" in ours().gpeh_last_error()


def test_missing_file_is_an_error(tmp_path):
    out = np.zeros(47)
    assert ours().gpeh_params(str(tmp_path / "nope.txt").encode(), dp(out)) == -1


def test_input_typing_rules(tmp_path):
    # "1E-7" parses as int 1 and double 1e-7 (stoi/stod prefixes,
    # src/input_variables.cu:55-74); later duplicates override earlier lines.
    src = open(os.path.join(INPUTS, "bec_2d.txt")).read().replace("@OUT@", str(tmp_path) + "/run_")
    src += "\nniter 1E-7 # int prefix\nnx 32\n"
    fn = tmp_path / "t.txt"
    fn.write_text(src)
    out = np.zeros(47)
    assert ours().gpeh_params(str(fn).encode(), dp(out)) == 1
    assert out[22] == 1 and out[0] == 32


@needs_ref
@pytest.mark.parametrize("lattice", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("case", ["bec_harmonic_3d.txt", "bec_2d.txt"])
def test_lattice_seed_bit_identical(case, lattice, tmp_path):
    # Psi::force*Lattice seeds (1D, 2D triangular/square, 3D HEX/FCC/BCC/SC)
    # added to the plugin's initial psi, against the reference's Psi class.
    f = materialise(case, tmp_path)
    p = np.zeros(47)
    ours().gpeh_params(f, dp(p))
    n = int(p[4])
    a = np.zeros(n, np.complex128)
    b = np.zeros(n, np.complex128)
    args = (lattice, 0.7, 1.9, 0.3, -0.2, 0.1, 1)
    L = ours()
    R = ref()
    D = ctypes.c_double
    sig = [ctypes.c_char_p, ctypes.c_int, D, D, D, D, D, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.gpeh_init_psi_lattice.argtypes = sig
    R.ref_init_psi_lattice.argtypes = sig
    assert L.gpeh_init_psi_lattice(f, *args, dp(a.view(np.float64))) == 0
    assert R.ref_init_psi_lattice(f, *args, dp(b.view(np.float64))) == 0
    assert np.array_equal(a, b), np.max(np.abs(a - b))
    base = np.zeros(n, np.complex128)
    L.gpeh_init_psi(f, 0, dp(base.view(np.float64)))
    assert not np.array_equal(a, base)  # the seed changed psi
