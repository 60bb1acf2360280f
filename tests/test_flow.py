"""The persistent RK4 step (gpe_set_flow: one launch per real-time step, whose
CTAs run the tiles of the step's sixteen axis passes in one ordered list with
per-tile dependency counters) against the per-pass chain it replaces.

The tiles are the pass kernels' own bodies, so the persistent step must equal
the chain bit for bit (psi, the compensated low part, the observables), and
through the chain the FP64 oracle.  Handles it does not serve keep the chain.
A dependency wait that runs out records GPE_ERR_TIMEOUT; after
gpe_flow_status re-arms it the handle steps exactly again.
"""
import numpy as np
import pytest

import oracle_py as orc
from fgpe_b200 import C64, C128, HAM_TEMPLATE, GPEError, Solver, make_config

from test_oracle import gaussian, harmonic

pytestmark = pytest.mark.gpu

GPE_ERR_TIMEOUT = 6
PI_REF = 3.141592653589793


def quench_cfg(n, prec=C64, ham=None):
    prms = np.zeros(32)
    prms[0:3] = 1100.0 / (4 * PI_REF)
    kw = {} if ham is None else {"hamiltonian": ham}
    return make_config((n, n, n), 10.0, dt=5e-4, precision=prec, prms=prms, beta=0.9, **kw)


def start(cfg):
    V = harmonic(cfg, (1.0, 1.0, 2.0))
    return V, gaussian(cfg, width=1.5, seed=3, noise=1e-2)


def run(cfg, V, psi, flow, calls, bound=0):
    """calls: list of (nsteps, want_obs); returns psi and the observables."""
    with Solver(cfg) as s:
        s.set_vext(0, V)
        s.set_psi(0, psi)
        s.set_flow(flow, bound)
        obs, it = [], 0
        for n, want in calls:
            obs.append(s.step_real(it, n, want_obs=want))
            it += n
        return s.get_psi(0), obs, s.flow_active, s.launches


@pytest.mark.parametrize("n", [128, 256])
def test_flow_step_equals_the_chain_bit_for_bit(gpu, n):
    cfg = quench_cfg(n)
    V, psi = start(cfg)
    calls = [(3, False), (2, True), (1, True), (2, False)]
    a, oa, active, la = run(cfg, V, psi, True, calls)
    b, ob, _, lb = run(cfg, V, psi, False, calls)
    assert active
    assert np.array_equal(a, b)  # get_psi returns high + low part: both compared
    for x, y in zip(oa, ob):
        assert (x is None and y is None) or np.array_equal(x, y)
    # one launch per step (and an x-forward pass after each observables step)
    assert la < lb


def test_flow_step_matches_oracle(gpu):
    cfg = quench_cfg(128)
    V, psi = start(cfg)
    got, og, active, _ = run(cfg, V, psi, True, [(2, False), (1, True)])
    assert active
    o = orc.OracleSolver(quench_cfg(128, C128))
    o.set_vext(0, V)
    o.set_psi(0, psi)
    o.step_real(0, 2)
    oo = o.step_real(2, 1, want_obs=True)
    want = o.get_psi(0)
    o.close()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-5
    for q in range(3):
        assert abs(og[-1][q] / oo[q] - 1) < 1e-5, q


def test_flow_template_hamiltonian_equals_the_chain(gpu):
    cfg = quench_cfg(128, ham=HAM_TEMPLATE)
    V, psi = start(cfg)
    a, _, active, _ = run(cfg, V, psi, True, [(2, True)])
    b, _, _, _ = run(cfg, V, psi, False, [(2, True)])
    assert active and np.array_equal(a, b)


@pytest.mark.parametrize("shape,prec", [((128, 128, 128), C128), ((96, 96, 96), C64), ((128, 128, 64), C64)])
def test_flow_leaves_other_handles_on_the_chain(gpu, shape, prec):
    prms = np.zeros(32)
    prms[0:3] = 500.0 / (4 * PI_REF)
    cfg = make_config(shape, 8.0, dt=5e-4, precision=prec, prms=prms, beta=0.9)
    V, psi = start(cfg)
    a, _, active, _ = run(cfg, V, psi, True, [(2, True)])
    b, _, _, _ = run(cfg, V, psi, False, [(2, True)])
    assert not active
    assert np.array_equal(a, b)


def test_flow_timeout_is_reported_and_rearmed(gpu):
    """A bound of one 32 ns sleep: the first tile of the z pass finds the y
    pass of its x block unfinished and gives up; the launch ends, the status
    is reported, and after the re-arm the same steps are exact again."""
    cfg = quench_cfg(128)
    V, psi = start(cfg)
    ref, _, _, _ = run(cfg, V, psi, False, [(2, False)])
    with Solver(cfg) as s:
        s.set_vext(0, V)
        s.set_psi(0, psi)
        s.set_flow(True, 1)
        s.step_real(0, 2)
        assert s.flow_status() == GPE_ERR_TIMEOUT
        assert s.flow_status() == 0  # re-armed
        with pytest.raises(GPEError):  # the sticky handle status of a step with observables
            s.set_flow(True, 1)
            s.step_real(0, 1, want_obs=True)
        assert s.flow_status() == GPE_ERR_TIMEOUT
        s.set_flow(True, 1 << 22)
        s.set_psi(0, psi)
        s.step_real(0, 2)
        assert s.flow_status() == 0
        assert np.array_equal(s.get_psi(0), ref)


def run_mode2(cfg, V, psi, mode, bound=0):
    """Real-time steps (with and without observables), then imaginary-time
    iterations of cfg's scheme, through one handle; psi and observables."""
    with Solver(cfg) as s:
        s.set_vext(0, V)
        s.set_psi(0, psi)
        s.set_flow(mode, bound)
        o1 = s.step_real(0, 3, want_obs=True)
        s.step_real(3, 2)
        p1 = s.get_psi(0)
        o2 = s.observables(0.0)
        s.step_imag(0, 5)
        return p1, o1, o2, s.get_psi(0), s.flow_active


@pytest.mark.parametrize("n", [128, 256])
@pytest.mark.parametrize("scheme", ["heavyball", "rk4"])
def test_strided_stage_equals_the_chain_bit_for_bit(gpu, n, scheme):
    from fgpe_b200 import IMAG_HEAVYBALL, IMAG_RK4
    prms = np.zeros(32)
    prms[0:3] = 1100.0 / (4 * PI_REF)
    cfg = make_config((n, n, n), 10.0, dt=5e-4, precision=C64, prms=prms, beta=0.9,
                      imag_scheme=IMAG_HEAVYBALL if scheme == "heavyball" else IMAG_RK4)
    V, psi = start(cfg)
    a = run_mode2(cfg, V, psi, 2)
    b = run_mode2(cfg, V, psi, 0)
    assert a[4] == 2 and b[4] == 0
    for x, y in zip(a[:4], b[:4]):
        assert np.array_equal(x, y)


def test_strided_stage_timeout_is_reported_and_rearmed(gpu):
    cfg = quench_cfg(128)
    V, psi = start(cfg)
    ref, _, _, _ = run(cfg, V, psi, False, [(2, False)])
    with Solver(cfg) as s:
        s.set_vext(0, V)
        s.set_psi(0, psi)
        s.set_flow(2, 1)
        s.step_real(0, 2)
        assert s.flow_status() == GPE_ERR_TIMEOUT
        assert s.flow_status() == 0
        s.set_flow(2, 1 << 22)
        s.set_psi(0, psi)
        s.step_real(0, 2)
        assert s.flow_status() == 0
        assert np.array_equal(s.get_psi(0), ref)
