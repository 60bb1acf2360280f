"""Helpers shared by the golden-fixture tests: load a fixture, rebuild the
solver configuration of its input file through the host mirror
(include/gpe_host.h), and replay it on a solver (oracle or libgpe)."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")

TRACE_CASES = ["g_hb_bec", "g_hb_conv", "g_rt_quench", "g_hb_bec2", "g_rt_bec2", "g_hb_template", "g_cfg1_hb64"]
STOCK_CASES = ["g_stock_2d", "g_stock_rt", "g_stock_rot", "g_stock_rot_rt"]
# real-time stock cases start from the psi_final of an imaginary-time case
PREREQ = {"g_stock_rt": "g_stock_2d", "g_stock_rot_rt": "g_stock_rot"}


# Cases whose initial state and trap are regenerated from a seed instead of
# being stored (their inputs would be most of the fixture): the fixture keeps
# checksums of the inputs the reference read, and load() checks them.
GENERATED = ["g_cfg1_hb64"]


def available(case):
    return os.path.exists(os.path.join(GOLDEN, case + ".npz"))


def cfg1_inputs(o):
    """Config 1 inputs on the grid of the parameter dump o (gpeh_params):
    V = (x^2 + y^2 + z^2)/2 and psi0 = exp(-r^2/2) (1 + 1e-3 (n1 + i n2)) with
    n1, n2 standard normal from numpy's legacy RandomState(1) (a frozen
    stream), normalised to 1.  Cell-centred axes x_i = -XMAX + (i + 1/2) DX
    (src/baseHamiltonian.cu:25-51)."""
    n = [int(o[0]), int(o[1]), int(o[2])]
    ax = [-o[5 + d] + np.arange(n[d]) * o[8 + d] + 0.5 * o[8 + d] for d in range(3)]
    Z, Y, X = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    r2 = X * X + Y * Y + Z * Z
    V = (0.5 * r2 + 0j).reshape(-1)
    rng = np.random.RandomState(1)
    n1 = rng.standard_normal(r2.shape)
    n2 = rng.standard_normal(r2.shape)
    psi = np.exp(-r2 / 2.0) * (1.0 + 1e-3 * (n1 + 1j * n2))
    dv = o[8] * o[9] * o[10]
    psi = psi / np.sqrt(np.sum(np.abs(psi) ** 2) * dv)
    return psi.reshape(-1), V


def input_checksums(psi, V):
    """Norms and leading values of the regenerated inputs."""
    return {"psi_init_norm2": np.array(np.sum(np.abs(psi) ** 2)), "psi_init_head": psi[:1024].copy(),
            "vext_norm2": np.array(np.sum(np.abs(V) ** 2)), "vext_head": V[:1024].copy()}


def regenerate(fx, tmpdir=None):
    """psi_init and vext of a GENERATED case, checked against the checksums
    stored with the fixture (to 1e-14: the arrays come from libm exp, which
    may differ in the last bit between hosts)."""
    import tempfile
    d = tmpdir or tempfile.mkdtemp()
    _, o = params_dump(str(fx["input"]), d)
    psi, V = cfg1_inputs(o)
    want = input_checksums(psi, V)
    for k, v in want.items():
        ref = fx[k]
        assert np.max(np.abs(v - ref)) <= 1e-14 * max(np.max(np.abs(ref)), 1e-300), k
    return psi, V


def load(case):
    fx = dict(np.load(os.path.join(GOLDEN, case + ".npz"), allow_pickle=False))
    if case in GENERATED and "psi_init" not in fx:
        fx["psi_init"], fx["vext"] = regenerate(fx)
    return fx


def keys(text):
    out = {}
    for line in text.splitlines():
        line = line.split("#", 1)[0].split()
        if len(line) >= 2:
            out[line[0]] = line[1]
    return out


def params_dump(input_text, tmpdir):
    import fgpe_b200 as gp
    fn = os.path.join(str(tmpdir), "golden_input.txt")
    with open(fn, "w") as f:
        f.write(input_text.replace("@OUT@", str(tmpdir) + "/"))
    L = gp.lib()
    L.gpeh_params.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
    o = np.zeros(47)
    nc = L.gpeh_params(fn.encode(), o.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert nc in (1, 2), L.gpeh_last_error()
    return nc, o


def config(fx, tmpdir, precision=0, stock=False):
    """gpe_config of a fixture's input (code units, plugin d_h_params)."""
    import fgpe_b200 as gp
    text = str(fx["input"])
    k = keys(text)
    nc, o = params_dump(text, tmpdir)
    cfg = gp.GPEConfig()
    cfg.abi_version = gp.ABI_VERSION
    cfg.nx, cfg.ny, cfg.nz = int(o[0]), int(o[1]), int(o[2])
    cfg.dim = int(o[3])
    for d in range(3):
        cfg.xmax[d] = o[5 + d]
        cfg.dx[d] = o[8 + d]
    cfg.ncomp = nc
    cfg.precision = precision
    cfg.dt = o[19] * o[25] / 1000  # p.dt * p.omho / 1000 (src/oneComponentGPSolver.cu:39)
    cfg.beta = float(k.get("beta", 0.0))
    cfg.epsilon_e = o[20]
    cfg.npart[0] = o[33]
    cfg.npart[1] = o[46] if nc == 2 else 0.0
    prms = np.zeros(32)
    ham = k.get("hamiltonian", '"bec"').strip('"')
    if nc == 2:
        cfg.hamiltonian = gp.HAM_BEC2
        prms[0:3] = o[34:37]
    elif ham == "template":
        cfg.hamiltonian = gp.HAM_TEMPLATE
    else:
        cfg.hamiltonian = gp.HAM_BEC
        a = o[34]
        if stock:
            prms[0] = a  # hamiltonians/BEC_oneComponent.cu:14
            if k.get("trotate", "false") == "true":  # :98-101, lambda = 2 pi omega / (omho aho)
                prms[11] = 2 * 3.141592653589793 * float(k["omega"]) / (o[25] * o[24])
        else:
            prms[0:3] = [a * float(k.get(f"quench_f{i}", 1.0)) for i in range(3)]
            prms[3:6] = [float(k.get(f"quench_t{i}", 0.0)) for i in (1, 2, 3)]
    for i in range(32):
        cfg.prms[i] = prms[i]
    return cfg, k


def initial_state(fx, nc):
    if nc == 1:
        return [fx["psi_init"]], [fx["vext"]]
    return [fx["psi_init1"], fx["psi_init2"]], [fx["vext1"], fx["vext2"]]


def final_state(fx, nc):
    return [fx["psi_final"]] if nc == 1 else [fx["psi_final1"], fx["psi_final2"]]


def replay(solver, fx, k, nc, psi_from=None):
    """Run the fixture's loop on `solver`; returns the list of PARS rows
    (iteration, NORM, MU, EN, EN_PREV [, comp 2...]) comparable with fx['trace']."""
    psis, vexts = initial_state(fx, nc)
    if psi_from is not None:
        psis = psi_from
    for c in range(nc):
        solver.set_vext(c, vexts[c])
        solver.set_psi(c, psis[c])
    niter = int(k["niter"])
    rows = []
    if k["treal"] == "false":
        for it in range(niter):
            done, conv = solver.step_imag(it, 1)
            st = solver.imag_state()
            row = [1.0 if conv else 0.0, it] + list(st)
            rows.append(row)
            if conv:
                break
    else:
        every = int(k.get("trace_every", k.get("itStatMod", "1")))
        if nc == 2:
            solver.step_real(1, niter - 1)  # src/twoComponentGPSolver.cu:142
        else:
            it = 0  # steps done; the trace line after step `it` carries ITER = it
            while it < niter:
                n = min(every - (it % every), niter - it)
                want = (it + n) % every == 0
                obs = solver.step_real(it, n, want_obs=want)
                it += n
                if want:
                    norm = obs[0]
                    rows.append([2.0, it, norm, obs[1] / norm, obs[2] / norm])
    return rows
