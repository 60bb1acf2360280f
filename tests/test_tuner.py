"""Autotuner: the pass variants it chooses between (strided-pass
implementation, tile, resident CTAs, radix order; x-pass rows per CTA) all
compute the same transforms, a tuning result round-trips through the cache
file, and tuned handles stay within the tolerances of the default ones.

Tolerances: complex128 variants <= 1e-13 relative for a transform; complex64
<= 2e-6 (their rounding differs from the default's: other radix orders and
packed FP32x2 arithmetic)."""
import json
import os

import numpy as np
import pytest

import oracle_py as orc
from fgpe_b200 import (C64, C128, IMAG_RK4, NSVAR, Batch, Solver, make_config, pass_variant_exists, set_tune_cache,
                       tune)

from test_oracle import PI_REF, gaussian, harmonic

FFT_TOL = {C128: 1e-13, C64: 2e-6}


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def test_variant_table_host_only():
    """Which variants exist (no GPU needed): the default everywhere, the
    paired and tuned ones for complex64 at the tuned lengths, a few scalar
    ones for complex128, none beyond the default at untuned lengths."""
    c64 = make_config((128, 128, 128), 8.0, precision=C64)
    c128 = make_config((128, 128, 128), 8.0, precision=C128)
    odd = make_config((27, 20, 40), 8.0, precision=C64)
    for axis in (1, 2):
        assert pass_variant_exists(c64, axis, 0) and pass_variant_exists(c128, axis, 0)
        assert pass_variant_exists(c64, axis, 1)  # paired lines at the default tile
        assert not pass_variant_exists(c128, axis, 1 + 5)  # complex128 has variants 0..5 at most
        assert sum(pass_variant_exists(c64, axis, v) for v in range(NSVAR)) >= 8
        assert not pass_variant_exists(c64, axis, NSVAR)
    # odd nx: no paired lines; 20 and 40 are not tuned lengths
    assert not pass_variant_exists(odd, 1, 1)
    assert [pass_variant_exists(odd, 2, v) for v in range(NSVAR)] == [True] + [False] * (NSVAR - 1)


SHAPES = [(128, 128, 128), (96, 96, 96), (128, 128, 64), (512, 512, 1), (192, 192, 1), (64, 64, 64)]


def variants_of(cfg, axis):
    return [v for v in range(NSVAR) if pass_variant_exists(cfg, axis, v)]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [C64, C128])
@pytest.mark.parametrize("shape", SHAPES)
def test_every_variant_transforms_like_numpy(gpu, prec, shape):
    nx, ny, nz = shape
    cfg = make_config(shape, 8.0, precision=prec)
    rng = np.random.default_rng(nx + 3 * ny + 7 * nz)
    a = rng.standard_normal((nz, ny, nx)) + 1j * rng.standard_normal((nz, ny, nx))
    want_f = np.fft.fftn(a)
    want_i = np.fft.ifftn(a) * a.size
    with Solver(cfg) as s:
        axes = [ax for ax, n in ((1, ny), (2, nz)) if n > 1]
        for ax in axes:
            for v in variants_of(cfg, ax):
                sv = [0] * 8
                for m in range(3):
                    sv[(ax - 1) * 3 + m] = v
                s.set_pass_variants(sv)
                s.set_psi(0, a)
                s.fft(0, -1)
                assert rel(s.get_psi(0), want_f) < FFT_TOL[prec], (ax, v, "forward")
                s.set_psi(0, a)
                s.fft(0, +1)
                assert rel(s.get_psi(0), want_i) < FFT_TOL[prec], (ax, v, "inverse")
        # x rows per CTA
        for rows in (1, 3, 7, 15):
            s.set_pass_variants([0] * 6 + [rows, 0])
            s.set_psi(0, a)
            s.fft(0, -1)
            assert rel(s.get_psi(0), want_f) < FFT_TOL[prec], ("rows", rows)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [C64, C128])
def test_every_variant_of_the_kspace_pass_matches_oracle(gpu, prec):
    """The forward*k-space*inverse mode (last strided axis) in the Laplacian,
    against the FP64 oracle, for every variant of the headline grid."""
    cfg = make_config((128, 128, 128), 10.0, precision=prec, g=1000.0)
    psi = gaussian(cfg, width=1.5, seed=3, noise=1e-2)
    o = orc.OracleSolver(cfg)
    o.set_psi(0, psi)
    want = o.laplace(0)
    # complex64: the Laplacian of a smooth state carries the transform's FP32
    # rounding weighted by k^2 (see test_config_sizes)
    tol = 1e-12 if prec == C128 else 2e-4
    with Solver(cfg) as s:
        s.set_psi(0, psi)
        for v in variants_of(cfg, 2):
            s.set_pass_variants([0, 0, 0, 0, v, 0, 0, 0])
            assert rel(s.laplace(0), want) < tol, v


@pytest.mark.gpu
def test_tune_cache_round_trip_and_tuned_steps_match_oracle(gpu, tmp_path):
    prms = np.zeros(32)
    prms[0:3] = 1100.0 / (4 * PI_REF)
    cfg = make_config((64, 64, 64), 8.0, dt=5e-4, precision=C64, prms=prms)
    cache = str(tmp_path / "tune.jsonl")
    rep = tune(cfg, 0, cache)
    assert rep["default_us"] > 0 and rep["tuned_us"] > 0 and rep["timed"] >= 4
    lines = [json.loads(l) for l in open(cache)]
    assert len(lines) == 1 and lines[0]["nx"] == 64 and lines[0]["prec"] == C64 and lines[0]["nb"] == 1
    # a second tuning of the same key replaces its line; another key appends
    tune(cfg, 0, cache)
    cfg2 = make_config((64, 64, 32), 8.0, dt=5e-4, precision=C64, prms=prms)
    tune(cfg2, 0, cache)
    assert len(open(cache).read().splitlines()) == 2
    want = rep["variants"] + [rep["xrows"]]
    V = harmonic(cfg, (1.0, 1.0, 2.0))
    psi = gaussian(cfg, seed=2)
    try:
        set_tune_cache(cache)
        with Solver(cfg) as s:
            got = s.pass_variants()
            line = [l for l in map(json.loads, open(cache)) if l["nz"] == 64][0]
            assert got == [line[k] for k in ("s10", "s11", "s12", "s20", "s21", "s22", "xrows", "yz")]
            s.set_vext(0, V)
            s.set_psi(0, psi)
            s.step_real(0, 3)
            o = orc.OracleSolver(cfg)
            o.set_vext(0, V)
            o.set_psi(0, psi)
            o.step_real(0, 3)
            assert rel(s.get_psi(0), o.get_psi(0)) < 1e-5
    finally:
        set_tune_cache(None)
    with Solver(cfg) as s:  # no cache: defaults
        assert s.pass_variants() == [0] * 8
    assert len(want) == 7


@pytest.mark.gpu
def test_batch_tune_matches_oracle(gpu, tmp_path):
    cfgs = []
    for n, g in ((64, 300.0), (64, 900.0), (96, 500.0)):
        L = 8.0 * np.sqrt(n / 64.0)
        cfgs.append(make_config((n, n, 1), (L, L, 1.0), dt=4e-4, precision=C64, g=g, imag_scheme=IMAG_RK4,
                                epsilon_e=1e-8))
    b = Batch(cfgs)
    rep = b.tune(str(tmp_path / "batch.jsonl"))
    assert len(rep) == 2 and all(d > 0 and t > 0 for d, t in rep)
    assert len(open(tmp_path / "batch.jsonl").read().splitlines()) == 2
    inits = []
    for i, c in enumerate(cfgs):
        V = harmonic(c, (1.0, 2.0, 0.0))
        p = gaussian(c, seed=i)
        b.set_vext(i, V)
        b.set_psi(i, p)
        inits.append((V, p))
    b.step_imag(5)
    for i, c in enumerate(cfgs):
        c128 = c.copy()
        c128.precision = C128
        o = orc.OracleSolver(c128)
        o.set_vext(0, inits[i][0])
        o.set_psi(0, inits[i][1])
        o.step_imag(0, 5)
        assert rel(b.get_psi(i), o.get_psi(0)) < 1e-5, i
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(128, 128, 128), (128, 128, 64), (64, 64, 64), (32, 64, 128)])
def test_fused_yz_kernel_matches_oracle(gpu, shape):
    """The fused y-z cluster kernel (the three strided passes of a 3D
    complex64 stage in one launch) against the FP64 oracle: the Laplacian,
    H psi, and real- and imaginary-time steps, beside the three-pass chain."""
    prms = np.zeros(32)
    prms[0:3] = 800.0 / (4 * PI_REF)
    prms[11] = 0.3  # moving-frame term: the k-space factor's FP64 branch
    cfg = make_config(shape, (9.0, 8.0, 7.0), dt=5e-4, precision=C64, prms=prms, beta=0.9,
                      imag_scheme=IMAG_RK4, epsilon_e=1e-12)
    V = harmonic(cfg, (1.0, 1.2, 1.5))
    psi = gaussian(cfg, width=1.5, seed=8, noise=1e-2)
    o = orc.OracleSolver(cfg)
    o.set_vext(0, V)
    o.set_psi(0, psi)
    lap, (hm, he) = o.laplace(0), o.apply_h(0.0, 0)
    o.step_real(0, 3)
    p_rt = o.get_psi(0)
    o.set_psi(0, psi)
    o.step_imag(0, 3)
    p_im = o.get_psi(0)
    results = {}
    for yz in (0, 1):
        with Solver(cfg) as s:
            s.set_pass_variants([0] * 7 + [yz])
            assert s.pass_variants()[7] == yz
            s.set_vext(0, V)
            s.set_psi(0, psi)
            l0 = s.launches
            got = [s.laplace(0), *s.apply_h(0.0, 0)]
            s.step_real(0, 3)
            got.append(s.get_psi(0))
            s.set_psi(0, psi)
            s.step_imag(0, 3)
            got.append(s.get_psi(0))
            results[yz] = (got, s.launches - l0)
    # the Laplacian of a smooth state carries the FP32 transform rounding
    # weighted by k^2 (see test_config_sizes); H psi and the steps do not
    for g, w, tol in zip(results[1][0], (lap, hm, he, p_rt, p_im), (2e-4, 5e-6, 5e-6, 1e-5, 1e-5)):
        assert rel(g, w) < tol
    # the fused kernel runs the scalar passes' line transforms and k-space
    # factor operation for operation: the two chains agree bit for bit
    for a, b in zip(results[0][0], results[1][0]):
        assert np.array_equal(a, b)
    assert results[1][1] < results[0][1]  # fewer launches: one kernel in place of three


@pytest.mark.gpu
def test_fused_yz_kernel_rejected_where_it_does_not_fit(gpu):
    from fgpe_b200 import GPEError
    for shape, prec in (((96, 96, 96), C64), ((128, 128, 128), C128), ((50, 64, 64), C64)):
        with Solver(make_config(shape, 8.0, precision=prec)) as s:
            with pytest.raises(GPEError):
                s.set_pass_variants([0] * 7 + [1])


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(128, 128, 128), (64, 64, 64), (96, 96, 96), (256, 256, 1)])
@pytest.mark.parametrize("rows", [0, 4])
def test_x_staging_equals_the_unstaged_pass_bit_for_bit(gpu, shape, rows):
    """gpe_set_x_staging: the fused real-time x pass copies its epilogue
    inputs into shared memory before its wait instead of loading them after
    the inverse transform; same arithmetic, so psi (high and low part) and
    the observables must not change by a bit."""
    prms = np.zeros(32)
    prms[0:3] = 800.0 / (4 * PI_REF)
    cfg = make_config(shape, 8.0, dt=5e-4, precision=C64, prms=prms, beta=0.9)
    V = harmonic(cfg, (1.0, 1.5, 2.0))
    psi = gaussian(cfg, width=1.3, seed=7, noise=1e-2)
    out = {}
    for on in (0, 1):
        with Solver(cfg) as s:
            s.set_vext(0, V)
            s.set_psi(0, psi)
            if rows:
                v = s.pass_variants()
                v[6] = rows
                s.set_pass_variants(v)
            s.set_x_staging(bool(on))
            assert s.x_staging == bool(on)
            s.step_real(0, 3)
            o = s.step_real(3, 2, want_obs=True)
            out[on] = (s.get_psi(0), o)
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
