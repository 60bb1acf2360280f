"""Persistent batch launches (gpe_batch_set_persistent): one cooperative
kernel per RK4 stage runs the three passes of that stage for every instance
of every geometry group, with a bounded grid-wide barrier between passes.

- The 2D sweep lengths (64 ... 512, uneven group sizes) against the per-group
  launches of the same batch and against the FP64 oracle (a restatement of
  src/oneComponentGPSolver.cu:122-217 and src/parallel.cu:230-302);
- 4 kernel launches per iteration (the per-group path: 12 per group);
- a wait bound that cannot be met ends the call with GPE_ERR_TIMEOUT, the
  context stays usable, and the next call with the default bound is exact
  again;
- grids the kernel is not compiled for are refused on the host.

Tolerances: against the per-group launches (the same line transforms and
epilogues, other tile shapes) 1e-13 complex128 / 1e-6 complex64; against
the oracle the chain tolerances of test_config_sizes.
"""
import numpy as np
import pytest

import oracle_py as orc
from fgpe_b200 import (BATCH_GROUPED, BATCH_PER_GROUP, BATCH_PERSISTENT, C64, C128, IMAG_RK4, Batch, GPEError, Solver,
                       make_config)

from test_oracle import gaussian, harmonic

pytestmark = pytest.mark.gpu

SAME_TOL = {C128: 1e-13, C64: 1e-6}
CHAIN_TOL = {C128: 1e-12, C64: 1e-5}
GPE_ERR_UNSUPPORTED = 2
GPE_ERR_TIMEOUT = 6


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def sweep_cfgs(prec, sizes, eps=1e-8, dt=4e-4):
    cfgs = []
    for k, n in enumerate(sizes):
        L = 8.0 * np.sqrt(n / 64.0)
        cfgs.append(make_config((n, n, 1), (L, L, 1.0), dt=dt, precision=prec, g=300.0 + 50.0 * k,
                                imag_scheme=IMAG_RK4, epsilon_e=eps))
    return cfgs


def fill(b, cfgs):
    inits = []
    for i, c in enumerate(cfgs):
        V = harmonic(c, (1.0, 2.0 + 0.1 * i, 0.0))
        p = gaussian(c, seed=10 + i)
        b.set_vext(i, V)
        b.set_psi(i, p)
        inits.append((V, p))
    return inits


# two instances of 64 and of 96 (groups of two), one of each other length
SIZES = [64, 96, 64, 128, 192, 96, 256, 384, 512]


@pytest.mark.parametrize("mode", [BATCH_PERSISTENT, BATCH_GROUPED])
@pytest.mark.parametrize("prec", [C64, C128])
def test_persistent_matches_per_group_and_oracle(gpu, prec, mode):
    """Both all-group modes (one cooperative launch per stage; one launch per
    pass over every group's tiles) against the per-group launches and the
    oracle."""
    cfgs = sweep_cfgs(prec, SIZES)
    nit = 5
    out = {}
    for m in (BATCH_PER_GROUP, mode):
        with Batch(cfgs) as b:
            if m != BATCH_PER_GROUP:
                b.set_launch_mode(m)
                assert b.launch_mode == m and b.persistent == (m == BATCH_PERSISTENT)
            fill(b, cfgs)
            it, cv = b.step_imag(nit)
            out[m != BATCH_PER_GROUP] = ([b.get_psi(i) for i in range(len(cfgs))],
                                         [b.imag_state(i) for i in range(len(cfgs))], it, cv)
    for i in range(len(cfgs)):
        assert rel(out[True][0][i], out[False][0][i]) < SAME_TOL[prec], i
        assert np.allclose(out[True][1][i], out[False][1][i], rtol=SAME_TOL[prec], atol=0), i
    assert np.array_equal(out[True][2], out[False][2]) and np.array_equal(out[True][3], out[False][3])
    # the oracle, on three of the instances (one per group size class)
    for i in (0, 3, 8):
        c = cfgs[i]
        c128 = c.copy()
        c128.precision = C128
        o = orc.OracleSolver(c128)
        V = harmonic(c, (1.0, 2.0 + 0.1 * i, 0.0))
        o.set_vext(0, V)
        o.set_psi(0, gaussian(c, seed=10 + i))
        o.step_imag(0, nit)
        assert rel(out[True][0][i], o.get_psi(0)) < CHAIN_TOL[prec], i
        so = o.imag_state()
        assert abs(out[True][1][i][2] / so[2] - 1) < CHAIN_TOL[prec], i


def test_persistent_launches_four_kernels_per_iteration(gpu):
    cfgs = sweep_cfgs(C64, [64, 128, 256])
    with Batch(cfgs) as b:
        fill(b, cfgs)
        b.step_imag(1)  # set-up launches and graph capture
        l0 = b.launches
        b.step_imag(3)
        per_group = b.launches - l0
        b.set_persistent(True)
        fill(b, cfgs)
        b.step_imag(1)
        l1 = b.launches
        b.step_imag(3)
        per_stage = b.launches - l1
        b.set_launch_mode(BATCH_GROUPED)
        fill(b, cfgs)
        b.step_imag(1)
        l2 = b.launches
        b.step_imag(3)
        grouped = b.launches - l2
    # per call one iteration-counter reset per group; per iteration 4 stage
    # kernels, or 3 passes x 4 stages for all groups, or per group the
    # x-forward of stage 1 and 2 passes a stage (stages 1-3 fuse the next
    # stage's x-forward into their x-inverse pass)
    assert per_stage == len(cfgs) + 4 * 3
    assert grouped == len(cfgs) + 12 * 3
    assert per_group == len(cfgs) + (1 + 2 * 4) * 3 * len(cfgs)


def test_persistent_rk4_convergence_stops_each_instance(gpu):
    """Instances converge at different iterations; each stops on its own
    (its tiles skip on the device) exactly as under per-group launches."""
    cfgs = sweep_cfgs(C128, [64, 96, 128], eps=1e-5, dt=5e-3)
    res = {}
    for persistent in (False, True):
        with Batch(cfgs) as b:
            if persistent:
                b.set_persistent(True)
            fill(b, cfgs)
            it, cv = b.step_imag(3000)
            res[persistent] = (it, cv, [b.get_psi(i) for i in range(len(cfgs))])
    assert res[False][1].all() and res[True][1].all()
    assert np.array_equal(res[True][0], res[False][0])
    for i in range(len(cfgs)):
        assert rel(res[True][2][i], res[False][2][i]) < 1e-12


def test_persistent_wait_bound_expires_with_timeout_status(gpu):
    """A bound of one sleep cannot be met by a grid of hundreds of CTAs: the
    call returns GPE_ERR_TIMEOUT after every CTA has left the kernel, the
    device stays usable, and the next call with the default bound is exact."""
    cfgs = sweep_cfgs(C64, [256, 512, 384])
    with Batch(cfgs) as b:
        b.set_persistent(True, wait_bound=1)
        fill(b, cfgs)
        with pytest.raises(GPEError) as ei:
            b.step_imag(2)
        assert ei.value.status == GPE_ERR_TIMEOUT
        # the same batch again, default bound, fresh state
        b.set_persistent(True)
        fill(b, cfgs)
        b.step_imag(3)
        got = [b.get_psi(i) for i in range(len(cfgs))]
    with Batch(cfgs) as b:
        fill(b, cfgs)
        b.step_imag(3)
        for i in range(len(cfgs)):
            assert rel(got[i], b.get_psi(i)) < SAME_TOL[C64], i
    # an unrelated handle still runs on this context
    cfg = make_config((32, 32, 32), 6.0, precision=C128)
    with Solver(cfg) as s:
        s.set_psi(0, gaussian(cfg))
        s.fft(0, -1)


def test_persistent_refused_where_it_does_not_apply(gpu):
    """Host-side checks (no kernel runs): 3D grids, lengths the kernel is not
    compiled for and the heavy-ball scheme are refused with
    GPE_ERR_UNSUPPORTED, and the batch keeps its per-group launches."""
    bad = [
        [make_config((64, 64, 64), 8.0, precision=C64, imag_scheme=IMAG_RK4)],
        [make_config((80, 80, 1), (8.0, 8.0, 1.0), precision=C64, imag_scheme=IMAG_RK4)],
        [make_config((64, 64, 1), (8.0, 8.0, 1.0), precision=C64)],
    ]
    for cfgs in bad:
        with Batch(cfgs) as b:
            with pytest.raises(GPEError) as ei:
                b.set_persistent(True)
            assert ei.value.status == GPE_ERR_UNSUPPORTED
            assert not b.persistent
