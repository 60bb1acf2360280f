"""The k-space interaction tables libgpe uploads (gpe_kspace_kernel, host
arithmetic, no GPU) against restatements that do not share its formula.

Dipolar (GPE_HAM_DIPOLAR): the reference's DipoleDipoleInteraction kernel
(src/parallel.cu:326-352) is 12 pi a_dd ((k.d)^2/k^2 - 1/3) with 0 for
|k| < 1e-6.  The spherical real-space cut-off at radius R multiplies it by the
factor c(q), q = 2 pi |k| R.  Here c(q) is not taken from its closed form but
from the radial integral that defines it: projecting exp(-i k.r) on the l = 2
angular dependence of the dipole potential leaves
    V~_R(k) / V~_inf(k) = int_0^{kR} j2(x)/x dx / int_0^inf j2(x)/x dx
                        = 3 int_0^q j2(x)/x dx,
evaluated by adaptive quadrature (scipy).  The q -> 0 limit is q^2/10, so the
k = 0 entry is 0.  The coupling convention of the configs,
(4 pi/3) g_dd (3 cos^2 - 1) with g_dd = 3 g eps_dd / (4 pi), is checked to be
the same table.

Soft core (GPE_HAM_SOFT): the 3D kernel 4 pi U a^3 (sin ka - ka cos ka)/(ka)^3
(SoftCoreInteraction_3D, src/parallel.cu:453-477) is the Fourier transform of
a step of height U and radius a; it is checked against a radial quadrature of
that transform, and the 2D one (2 pi a U J1(ka)/k) likewise.
"""
import numpy as np
import pytest
from scipy import integrate, special

from fgpe_b200 import HAM_DIPOLAR, HAM_SOFT, kspace_kernel, make_config

PI = 3.141592653589793


def kaxis(n, dx):
    """k axis in cycles per length from numpy's frequency helper, with the
    k = N/2 entry of an even length made positive as the reference's
    InitializeKspace has it (src/baseHamiltonian.cu:61-68)."""
    k = np.fft.fftfreq(n, d=dx)
    if n % 2 == 0:
        k[n // 2] = -k[n // 2]
    return k


def kgrid(cfg):
    ks = [kaxis(n, dx) if n > 1 else np.zeros(1) for n, dx in zip((cfg.nx, cfg.ny, cfg.nz), cfg.dx)]
    if cfg.dim == 2:
        ks[2] = np.zeros(cfg.nz)
    KZ, KY, KX = np.meshgrid(ks[2], ks[1], ks[0], indexing="ij")
    return KX, KY, KZ


def cutoff_quadrature(q):
    """3 int_0^q j2(x)/x dx by adaptive quadrature."""
    if q == 0.0:
        return 0.0
    f = lambda x: special.spherical_jn(2, x) / x if x > 0 else 0.0
    v, err = integrate.quad(f, 0.0, q, limit=400, epsabs=1e-15, epsrel=1e-13)
    return 3.0 * v


def test_cutoff_integral_limits():
    # int_0^inf j2(x)/x dx = 1/3, so the factor tends to 1 for R -> inf
    assert abs(cutoff_quadrature(400.0) - 1.0) < 5e-3
    # q -> 0: c(q) = q^2/10 - q^4/280 + q^6/15120 - ... (from j2(x) = x^2/15 - x^4/210 + x^6/7560)
    for q in (1e-3, 1e-2, 0.1):
        assert abs(cutoff_quadrature(q) / (q * q / 10.0 - q ** 4 / 280.0 + q ** 6 / 15120.0) - 1.0) < 1e-9


def dipolar_cfg(R, direction=(0.0, 0.0, 1.0), shape=(128, 128, 64), box=(12.0, 12.0, 6.0), g=1000.0, edd=0.8):
    a = g / (4 * PI)
    prms = np.zeros(32)
    prms[0:3] = a
    prms[6] = edd * a
    prms[7:10] = direction
    prms[10] = R
    return make_config(shape, box, prms=prms, hamiltonian=HAM_DIPOLAR)


@pytest.mark.parametrize("direction", [(0.0, 0.0, 1.0), (1.0, 1.0, 0.5)])
def test_dipolar_without_cutoff_is_the_reference_kernel(direction):
    cfg = dipolar_cfg(0.0, direction, shape=(32, 24, 16), box=(6.0, 5.0, 4.0))
    got = kspace_kernel(cfg)
    KX, KY, KZ = kgrid(cfg)
    d = np.array(direction) / np.linalg.norm(direction)
    num = KX * d[0] + KY * d[1] + KZ * d[2]
    den = np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
    a_dd = cfg.prms[6]
    safe = np.where(den < 1e-6, 1.0, den)
    want = np.where(den < 1e-6, 0.0, 12.0 * PI * a_dd * ((num / safe) ** 2 - 1.0 / 3.0))
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


def test_dipolar_cutoff_against_radial_quadrature():
    """Config 3a: 128x128x64 on [-12,12]^2 x [-6,6], g = 1000, eps_dd = 0.8 along z, R = 6."""
    R = 6.0
    cfg = dipolar_cfg(R)
    got = kspace_kernel(cfg)
    bare = kspace_kernel(dipolar_cfg(0.0))
    KX, KY, KZ = kgrid(cfg)
    kk = np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
    assert got[0, 0, 0] == 0.0 and bare[0, 0, 0] == 0.0
    # seeded sample of grid points plus the three axes and the corner of k-space
    rng = np.random.default_rng(11)
    pts = [tuple(rng.integers(0, s) for s in got.shape) for _ in range(60)]
    pts += [(0, 0, i) for i in range(1, 64)] + [(0, i, 0) for i in range(1, 64)] + [(i, 0, 0) for i in range(1, 32)]
    pts += [(32, 64, 64), (1, 1, 1)]
    for p in pts:
        q = 2 * PI * kk[p] * R
        c = cutoff_quadrature(q)
        assert abs(got[p] - bare[p] * c) <= 1e-11 * max(abs(bare[p]), 1e-300) + 1e-13, (p, q, got[p], bare[p] * c)
    # the configs' convention: (4 pi/3) g_dd (3 cos^2 theta - 1) with g_dd = 3 g eps_dd / (4 pi)
    g, edd = 1000.0, 0.8
    gdd = 3 * g * edd / (4 * PI)
    safe = np.where(kk == 0, 1.0, kk)
    conv = np.where(kk == 0, 0.0, (4 * PI / 3) * gdd * (3 * (KZ / safe) ** 2 - 1))
    assert np.max(np.abs(bare - conv)) <= 1e-12 * np.max(np.abs(conv))


def test_dipolar_cutoff_small_q_limit():
    """A box large against R puts the first k points at small q: the table
    must follow c(q) -> q^2/10 there without cancellation trouble."""
    R = 0.05
    cfg = dipolar_cfg(R, shape=(16, 16, 16), box=(20.0, 20.0, 20.0))
    got = kspace_kernel(cfg)
    bare = kspace_kernel(dipolar_cfg(0.0, shape=(16, 16, 16), box=(20.0, 20.0, 20.0)))
    KX, KY, KZ = kgrid(cfg)
    kk = np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
    m = (kk > 0) & (np.abs(bare) > 1e-3 * np.abs(bare).max())
    q = 2 * PI * kk[m] * R
    assert q.max() < 0.8
    ratio = got[m] / bare[m]
    quad = np.array([cutoff_quadrature(x) for x in q])
    assert np.max(np.abs(ratio / quad - 1)) < 1e-8


def step_transform_3d(k, a, U):
    """int_{|r|<a} U exp(-i k.r) d^3r = 4 pi U int_0^a r^2 sin(kr)/(kr) dr."""
    if k == 0:
        return 4 * PI * U * a ** 3 / 3
    v, _ = integrate.quad(lambda r: r * r * np.sinc(k * r / PI), 0.0, a, epsabs=1e-15, epsrel=1e-13)
    return 4 * PI * U * v


def step_transform_2d(k, a, U):
    """int_{|r|<a} U exp(-i k.r) d^2r = 2 pi U int_0^a r J0(kr) dr."""
    v, _ = integrate.quad(lambda r: r * special.j0(k * r), 0.0, a, epsabs=1e-15, epsrel=1e-13)
    return 2 * PI * U * v


@pytest.mark.parametrize("shape,box", [((24, 20, 16), (5.0, 4.0, 3.5)), ((32, 24, 1), (6.0, 5.0, 1.0))])
def test_soft_core_is_the_step_transform(shape, box):
    prms = np.zeros(32)
    prms[0], prms[1] = 0.8, 12.0
    cfg = make_config(shape, box, prms=prms, hamiltonian=HAM_SOFT)
    got = kspace_kernel(cfg)
    KX, KY, KZ = kgrid(cfg)
    k = 2 * PI * np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
    rng = np.random.default_rng(5)
    pts = [tuple(rng.integers(0, s) for s in got.shape) for _ in range(40)] + [(0, 0, 0), (0, 0, 1), (0, 1, 0)]
    f = step_transform_3d if cfg.dim == 3 else step_transform_2d
    for p in pts:
        want = f(k[p], 0.8, 12.0)
        assert abs(got[p] - want) <= 1e-10 * abs(f(0.0, 0.8, 12.0)), (p, got[p], want)
