"""FP64 restatement of the real-time RK4 step with a time-dependent control
potential, its final-state infidelity and the discrete adjoint gradient
(numpy; TEST INFRASTRUCTURE: used only by tests/ as the checker).

Forward model (the reference's real-time step, src/oneComponentGPSolver.cu:150-208
with the BECHamiltonianMU term of hamiltonians/BEC_oneComponent.cu:152-165 and
the Laplace operator of src/baseHamiltonian.cu:86-96 / src/parallel.cu:194-205):

    h(psi) = T psi + (W_n + 4 pi a |psi|^2) psi,  T = IFFT[(19.739208802/N) k^2 FFT]
    W_n    = V0 + sum_k u[n, k] G_k,              G_k(x) = exp(-|x - c_k|^2 / 2)
    f(psi) = -i h(psi)
    k1 = f(psi_n), psi_a = psi_n + dt/2 k1, k2 = f(psi_a), psi_b = psi_n + dt/2 k2,
    k3 = f(psi_b), psi_c = psi_n + dt k3, k4 = f(psi_c),
    psi_{n+1} = psi_n + dt/6 (k1 + 2 k2 + 2 k3 + k4)

Loss: L = 1 - |o|^2, o = sum conj(psi_target) psi_T DV.

With a k-space interaction (the dipolar term of GPE_HAM_DIPOLAR without the
cut-off: the reference's DipoleDipoleInteraction kernel, src/parallel.cu:326-352)
h gains Phi[|psi|^2] psi, Phi[n] = IFFT[V~(k) FFT n] (real for real n: V~ is
real and even in k).

Adjoint (gradients as complex numbers d/dRe + i d/dIm, real inner product
Re sum conj(a) b):
    J^T mu = i (T mu + (W + 2 g |psi|^2 + Phi[|psi|^2]) mu) - i g psi^2 conj(mu)
             + 2 Phi[Im(conj(mu) psi)] psi
(W.imag enters as - i W.imag mu inside the bracket) with g = 4 pi a; the last
term is the transpose of psi Phi[2 Re(conj(psi) d)], Phi being symmetric.
dL/du[n, k] = sum_s sum_x G_k(x) Im(conj(lam_ks(x)) psi_s(x)).
"""
from __future__ import annotations

import numpy as np

LAP = 19.739208802  # src/parallel.cu:199
PI_REF = 3.141592653589793


def k_axes(cfg):
    """k axes in cycles per length (src/baseHamiltonian.cu:53-82 with the
    odd-N formula); axes beyond the dimension are zero."""
    ks = []
    for d, n in enumerate((cfg.nx, cfg.ny, cfg.nz)):
        dx = cfg.dx[d]
        dk = 1.0 / (n * dx)
        kmax = 1.0 / (2.0 * dx)
        k = np.zeros(n)
        for i in range(n):
            k[i] = i * dk if i <= n // 2 else -kmax + (i - n // 2) * dk
        zero = (cfg.dim == 1 and d > 0) or (cfg.dim == 2 and d == 2)
        ks.append(np.zeros(n) if zero else k)
    return ks


def k_squared(cfg):
    """k^2 on the grid."""
    kx, ky, kz = k_axes(cfg)
    return kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2


def dipolar_table(cfg):
    """V~(k) = 12 pi a_dd ((k.d)^2 / k^2 - 1/3), 0 for |k| < 1e-6, a_dd =
    prms[6], d = prms[7:10] normalised (src/parallel.cu:326-352); only
    without the real-space cut-off (prms[10] = 0)."""
    if cfg.prms[10] != 0:
        raise ValueError("dipolar_table restates the kernel without the cut-off (prms[10] = 0)")
    kx, ky, kz = k_axes(cfg)
    KZ, KY, KX = np.meshgrid(kz, ky, kx, indexing="ij")
    d = np.array([cfg.prms[7], cfg.prms[8], cfg.prms[9]], dtype=np.float64)
    d = d / np.linalg.norm(d)
    kk = np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
    kd = KX * d[0] + KY * d[1] + KZ * d[2]
    safe = np.where(kk < 1e-6, 1.0, kk)
    return np.where(kk < 1e-6, 0.0, 12.0 * PI_REF * cfg.prms[6] * ((kd / safe) ** 2 - 1.0 / 3.0))


class ControlProblem:
    def __init__(self, cfg, V0, G, psi0, target, vtab=None):
        self.cfg = cfg
        self.N = cfg.nx * cfg.ny * cfg.nz
        self.shape = (cfg.nz, cfg.ny, cfg.nx)
        self.K2 = k_squared(cfg)
        self.scale = LAP / self.N
        self.V0 = np.asarray(V0, np.complex128).reshape(self.shape)
        self.G = np.asarray(G, np.float64).reshape((-1,) + self.shape)
        self.psi0 = np.asarray(psi0, np.complex128).reshape(self.shape)
        self.target = np.asarray(target, np.complex128).reshape(self.shape)
        self.g = 4 * PI_REF * cfg.prms[2]
        self.dt = cfg.dt
        self.DV = cfg.dx[0] * cfg.dx[1] * cfg.dx[2]
        self.vtab = None if vtab is None else np.asarray(vtab, np.float64).reshape(self.shape)

    def Phi(self, n):
        """The k-space interaction's potential of a real density (0 without one)."""
        if self.vtab is None:
            return 0.0
        return np.real(np.fft.ifftn(self.vtab * np.fft.fftn(n)))

    def T(self, p):
        return np.fft.ifftn(self.scale * self.K2 * np.fft.fftn(p)) * self.N

    def W(self, u_n):
        return self.V0 + np.tensordot(u_n, self.G, axes=(0, 0))

    def f(self, p, W):
        n = np.abs(p) ** 2
        return -1j * (self.T(p) + (W.real + self.g * n + self.Phi(n)) * p + 1j * W.imag * p)

    def step(self, p, W, keep=False):
        dt = self.dt
        k1 = self.f(p, W)
        pa = p + 0.5 * dt * k1
        k2 = self.f(pa, W)
        pb = p + 0.5 * dt * k2
        k3 = self.f(pb, W)
        pc = p + dt * k3
        k4 = self.f(pc, W)
        nxt = p + dt / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)
        return (nxt, (p, pa, pb, pc)) if keep else nxt

    def JT(self, mu, p, W):
        n = np.abs(p) ** 2
        jt = 1j * (self.T(mu) + (W.real + 2 * self.g * n + self.Phi(n)) * mu - 1j * W.imag * mu) \
            - 1j * self.g * p ** 2 * np.conj(mu)
        if self.vtab is not None:
            jt = jt + 2.0 * self.Phi(np.imag(np.conj(mu) * p)) * p
        return jt

    def forward(self, u):
        p = self.psi0.copy()
        for n in range(u.shape[0]):
            p = self.step(p, self.W(u[n]))
        return p

    def loss(self, u):
        p = self.forward(u)
        o = np.sum(np.conj(self.target) * p) * self.DV
        return 1.0 - abs(o) ** 2

    def gradient(self, u):
        """Loss and dL/du (nsteps x nctrl) by the discrete adjoint (all states kept)."""
        nsteps = u.shape[0]
        states = [self.psi0.copy()]
        for n in range(nsteps):
            states.append(self.step(states[-1], self.W(u[n])))
        o = np.sum(np.conj(self.target) * states[-1]) * self.DV
        L = 1.0 - abs(o) ** 2
        lam = -2.0 * o * self.target * self.DV
        grad = np.zeros_like(u)
        dt = self.dt
        for n in range(nsteps - 1, -1, -1):
            W = self.W(u[n])
            _, (pn, pa, pb, pc) = self.step(states[n], W, keep=True)
            m4 = dt / 6.0 * lam
            a = self.JT(m4, pc, W)
            m3 = dt / 3.0 * lam + dt * a
            b = self.JT(m3, pb, W)
            m2 = dt / 3.0 * lam + 0.5 * dt * b
            c = self.JT(m2, pa, W)
            m1 = dt / 6.0 * lam + 0.5 * dt * c
            d = self.JT(m1, pn, W)
            q = (np.imag(np.conj(m1) * pn) + np.imag(np.conj(m2) * pa) + np.imag(np.conj(m3) * pb)
                 + np.imag(np.conj(m4) * pc))
            grad[n] = np.tensordot(self.G, q, axes=([1, 2, 3], [0, 1, 2]))
            lam = lam + a + b + c + d
        return L, grad
