"""Batched independent instances (gpe_batch) against single handles and the
FP64 oracle: every instance of a batch must reproduce, bit for bit, the same
instance run alone (same kernels, same reduction order), including the
iteration at which its convergence test fires."""
import numpy as np
import pytest

import oracle_py as orc
from fgpe_b200 import C64, C128, IMAG_HEAVYBALL, IMAG_RK4, Batch, GPEError, Solver, grid_axes, make_config

pytestmark = pytest.mark.gpu


def sweep_configs(prec, scheme, eps=0.0, dt=1e-3):
    """Mixed 2D grids (two share a geometry) with different couplings and
    trap anisotropies, as in a parameter sweep."""
    specs = [(32, 1.0, 40.0, 1.0), (24, 0.8, 120.0, 2.0), (32, 1.0, 400.0, 3.5), (64, 1.3, 900.0, 1.5),
             (96, 1.6, 1500.0, 2.5)]
    cfgs, traps = [], []
    for n, scale, g, aniso in specs:
        L = 6.0 * scale
        cfg = make_config((n, n, 1), (L, L, 1.0), dt=dt, precision=prec, g=g, imag_scheme=scheme, beta=0.6,
                          epsilon_e=eps)
        x, y, _ = grid_axes(cfg)
        Y, X = np.meshgrid(y, x, indexing="ij")
        traps.append((0.5 * (X ** 2 + (aniso * Y) ** 2) + 0j).reshape(1, n, n))
        cfgs.append(cfg)
    return cfgs, traps


def initial(cfg, seed):
    x, y, _ = grid_axes(cfg)
    Y, X = np.meshgrid(y, x, indexing="ij")
    rng = np.random.default_rng(seed)
    g = np.exp(-(X ** 2 + Y ** 2) / 2.0)
    p = g * (1 + 1e-3 * (rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)))
    dv = cfg.dx[0] * cfg.dx[1] * cfg.dx[2]
    return (p / np.sqrt(np.sum(np.abs(p) ** 2) * dv)).reshape(1, *g.shape)


@pytest.mark.parametrize("prec", [C64, C128])
@pytest.mark.parametrize("scheme", [IMAG_RK4, IMAG_HEAVYBALL])
def test_batch_matches_single_handles(gpu, prec, scheme):
    import torch
    cfgs, traps = sweep_configs(prec, scheme)
    stream = torch.cuda.Stream()
    with Batch(cfgs) as b:
        b.set_stream(stream.cuda_stream)  # non-default stream: one CUDA graph per iteration
        for i, c in enumerate(cfgs):
            b.set_vext(i, traps[i])
            b.set_psi(i, initial(c, 10 + i))
        it1, cv1 = b.step_imag(7)
        it2, cv2 = b.step_imag(8)  # graph replays continue the state
        assert np.all(it1 == 7) and np.all(it2 == 8) and not cv1.any() and not cv2.any()
        assert b.launches > 0
        for i, c in enumerate(cfgs):
            s = Solver(c)
            s.set_vext(0, traps[i])
            s.set_psi(0, initial(c, 10 + i))
            s.step_imag(0, 7)
            s.step_imag(7, 8)
            assert np.array_equal(b.get_psi(i), s.get_psi(0)), i
            assert np.array_equal(b.imag_state(i), s.imag_state()), i
            s.close()


def test_batch_default_stream_and_oracle(gpu):
    # legacy default stream: direct launches instead of a graph
    cfgs, traps = sweep_configs(C128, IMAG_RK4)
    with Batch(cfgs) as b:
        for i, c in enumerate(cfgs):
            b.set_vext(i, traps[i])
            b.set_psi(i, initial(c, 10 + i))
        b.step_imag(12)
        for i in (1, 4):
            o = orc.OracleSolver(cfgs[i])
            o.set_vext(0, traps[i])
            o.set_psi(0, initial(cfgs[i], 10 + i))
            o.step_imag(0, 12)
            ref = o.get_psi(0)
            got = b.get_psi(i)
            assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)
            assert np.allclose(b.imag_state(i), o.imag_state(), rtol=1e-12, atol=0)


def test_batch_convergence_per_instance(gpu):
    import torch
    cfgs, traps = sweep_configs(C64, IMAG_RK4, eps=1e-5, dt=5e-3)
    stream = torch.cuda.Stream()
    want = []
    for i, c in enumerate(cfgs):
        s = Solver(c)
        s.set_vext(0, traps[i])
        s.set_psi(0, initial(c, 10 + i))
        done, conv = s.step_imag(0, 3000)
        assert conv
        want.append(done)
        s.close()
    with Batch(cfgs) as b:
        b.set_stream(stream.cuda_stream)
        for i, c in enumerate(cfgs):
            b.set_vext(i, traps[i])
            b.set_psi(i, initial(c, 10 + i))
        total = np.zeros(len(cfgs), dtype=np.int64)
        for _ in range(30):
            it, cv = b.step_imag(100)
            total += it
            if cv.all():
                break
        assert cv.all()
        assert list(total) == want
    assert len(set(want)) > 1  # the instances converge at different iterations


def test_batch_stops_issuing_after_every_instance_converged(gpu):
    """A call asked for far more iterations than convergence needs issues at
    most a few chunks (64 iterations each) past the last instance's
    convergence."""
    import torch
    cfgs, traps = sweep_configs(C64, IMAG_RK4, eps=1e-5, dt=5e-3)
    stream = torch.cuda.Stream()
    with Batch(cfgs) as b:
        b.set_stream(stream.cuda_stream)
        for i, c in enumerate(cfgs):
            b.set_vext(i, traps[i])
            b.set_psi(i, initial(c, 10 + i))
        b.step_imag(1)  # graph capture
        l0 = b.launches
        b.step_imag(2)
        per_iter = (b.launches - l0 - len(set((c.nx, c.ny) for c in cfgs))) // 2  # minus the per-call resets
        for i, c in enumerate(cfgs):
            b.set_vext(i, traps[i])
            b.set_psi(i, initial(c, 10 + i))
        l1 = b.launches
        it, cv = b.step_imag(1000000)
        assert cv.all() and it.max() < 3000
        issued = (b.launches - l1) / per_iter
        assert it.max() <= issued <= it.max() + 3 * 64, (issued, it.max())


def test_batch_rejects_mixed_settings(gpu):
    a = make_config((32, 32, 1), (6.0, 6.0, 1.0), precision=C64, g=10.0, imag_scheme=IMAG_RK4)
    b = make_config((32, 32, 1), (6.0, 6.0, 1.0), precision=C128, g=10.0, imag_scheme=IMAG_RK4)
    with pytest.raises(GPEError) as e:
        Batch([a, b])
    assert e.value.status == 1
    prms = np.zeros(32)
    prms[:6] = [1.0, 1.1, 1.2, 0.0, 0.5, 1.0]
    q = make_config((32, 32, 1), (6.0, 6.0, 1.0), precision=C64, prms=prms, imag_scheme=IMAG_RK4)
    with pytest.raises(GPEError) as e:
        Batch([a, q])
    assert e.value.status == 2
