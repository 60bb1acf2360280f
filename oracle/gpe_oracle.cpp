// gpe_oracle.cpp -- FP64 host oracle (test infrastructure; see gpe_oracle.h).
//
// Every numerical routine below restates a routine of the reference (fGPE v0.3)
// and cites it.  The reference runs these on the GPU with cuFFT; this file runs
// them on the host in double precision with its own FFT.
#include "gpe_oracle.h"

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::complex<double> cplx;

// hpp/header.hpp:27 -- the reference's pi literal.
const double PI_REF = 3.141592653589793;

// ---------------------------------------------------------------------------
// Neumaier-compensated accumulator.
struct Acc {
    double s = 0.0, c = 0.0;
    void add(double v) {
        double t = s + v;
        if (std::fabs(s) >= std::fabs(v)) c += (s - t) + v;
        else c += (v - t) + s;
        s = t;
    }
    void merge(const Acc& o) { add(o.s); add(o.c); }
    double value() const { return s + c; }
};

// ---------------------------------------------------------------------------
// 1D FFT plan: mixed-radix Stockham autosort, radices 4, 2, 3, 5 and a direct
// DFT for any remaining prime factor.  Twiddle table tw[m] = exp(-2 pi i m/n)
// from long double trigonometry.
struct Plan1D {
    int n = 1;
    std::vector<int> rad;
    std::vector<cplx> tw;               // forward roots of unity, length n
    std::vector<std::vector<cplx>> dft; // per generic radix: exp(-2 pi i m/R)

    explicit Plan1D(int n_) : n(n_) {
        int m = n;
        while (m % 4 == 0) { rad.push_back(4); m /= 4; }
        while (m % 2 == 0) { rad.push_back(2); m /= 2; }
        while (m % 3 == 0) { rad.push_back(3); m /= 3; }
        while (m % 5 == 0) { rad.push_back(5); m /= 5; }
        for (int p = 7; m > 1; p += 2)
            while (m % p == 0) { rad.push_back(p); m /= p; }
        tw.resize(n);
        const long double two_pi = 6.283185307179586476925286766559005768L;
        for (int k = 0; k < n; ++k) {
            long double a = -two_pi * (long double)k / (long double)n;
            tw[k] = cplx((double)cosl(a), (double)sinl(a));
        }
        for (int r : rad) {
            std::vector<cplx> t(r);
            for (int k = 0; k < r; ++k) {
                long double a = -two_pi * (long double)k / (long double)r;
                t[k] = cplx((double)cosl(a), (double)sinl(a));
            }
            dft.push_back(t);
        }
    }

    // In-place transform of x (length n) using work (length n).  sign -1 is the
    // forward transform exp(-i...), +1 the unnormalised inverse, as cuFFT's
    // CUFFT_FORWARD / CUFFT_INVERSE used at src/baseHamiltonian.cu:89,95.
    void exec(cplx* x, cplx* work, int sign) const {
        if (n == 1) return;
        cplx* src = x;
        cplx* dst = work;
        int Ns = 1;
        cplx v[64];
        cplx o[64];
        std::vector<cplx> vbig, obig;
        for (size_t p = 0; p < rad.size(); ++p) {
            const int R = rad[p];
            const int m = n / R;
            cplx* vv = v;
            cplx* oo = o;
            if (R > 64) { vbig.resize(R); obig.resize(R); vv = vbig.data(); oo = obig.data(); }
            const int tstride = n / (Ns * R);
            for (int j = 0; j < m; ++j) {
                const int k = j % Ns;
                for (int r = 0; r < R; ++r) {
                    cplx a = src[j + r * m];
                    if (r && k) {
                        cplx w = tw[(size_t)r * k * tstride];
                        if (sign > 0) w = std::conj(w);
                        a *= w;
                    }
                    vv[r] = a;
                }
                butterfly(R, (int)p, vv, oo, sign);
                const int idxD = (j / Ns) * Ns * R + k;
                for (int r = 0; r < R; ++r) dst[idxD + r * Ns] = oo[r];
            }
            std::swap(src, dst);
            Ns *= R;
        }
        if (src != x) std::memcpy((void*)x, (const void*)src, sizeof(cplx) * n);
    }

    void butterfly(int R, int p, const cplx* v, cplx* o, int sign) const {
        const double s = (double)sign;
        if (R == 2) {
            o[0] = v[0] + v[1];
            o[1] = v[0] - v[1];
        } else if (R == 4) {
            cplx a0 = v[0] + v[2], a1 = v[0] - v[2];
            cplx b0 = v[1] + v[3], b1 = v[1] - v[3];
            cplx ib1 = cplx(-s * b1.imag(), s * b1.real());  // sign*i*b1
            o[0] = a0 + b0;
            o[2] = a0 - b0;
            o[1] = a1 + ib1;
            o[3] = a1 - ib1;
        } else if (R == 3) {
            const double c = -0.5;
            const double sn = 0.86602540378443864676372317075293618;  // sqrt(3)/2
            cplx t1 = v[1] + v[2];
            cplx t2 = v[0] + c * t1;
            cplx d = v[1] - v[2];
            cplx it = cplx(-s * sn * d.imag(), s * sn * d.real());
            o[0] = v[0] + t1;
            o[1] = t2 + it;
            o[2] = t2 - it;
        } else {
            const std::vector<cplx>& t = dft[p];
            for (int q = 0; q < R; ++q) {
                cplx acc(0.0, 0.0);
                for (int r = 0; r < R; ++r) {
                    cplx w = t[(size_t)(r * q) % R];
                    if (sign > 0) w = std::conj(w);
                    acc += v[r] * w;
                }
                o[q] = acc;
            }
        }
    }
};

// 3D unnormalised DFT over a field with x fastest: the cufftPlan3d(NZ,NY,NX)
// transform of src/parallel.cu:97-102.
struct Plan3D {
    int nx, ny, nz;
    Plan1D px, py, pz;
    Plan3D(int nx_, int ny_, int nz_) : nx(nx_), ny(ny_), nz(nz_), px(nx_), py(ny_), pz(nz_) {}

    void exec(cplx* a, int sign) const {
        const long nxy = (long)nx * ny;
        const int nmax = std::max(nx, std::max(ny, nz));
        if (nx > 1) {
#pragma omp parallel
            {
                std::vector<cplx> w(nmax);
#pragma omp for schedule(static)
                for (long l = 0; l < (long)ny * nz; ++l) px.exec(a + l * nx, w.data(), sign);
            }
        }
        if (ny > 1) {
#pragma omp parallel
            {
                std::vector<cplx> line(nmax), w(nmax);
#pragma omp for schedule(static)
                for (long l = 0; l < (long)nx * nz; ++l) {
                    long ix = l % nx, iz = l / nx;
                    cplx* base = a + iz * nxy + ix;
                    for (int i = 0; i < ny; ++i) line[i] = base[(long)i * nx];
                    py.exec(line.data(), w.data(), sign);
                    for (int i = 0; i < ny; ++i) base[(long)i * nx] = line[i];
                }
            }
        }
        if (nz > 1) {
#pragma omp parallel
            {
                std::vector<cplx> line(nmax), w(nmax);
#pragma omp for schedule(static)
                for (long l = 0; l < nxy; ++l) {
                    cplx* base = a + l;
                    for (int i = 0; i < nz; ++i) line[i] = base[(long)i * nxy];
                    pz.exec(line.data(), w.data(), sign);
                    for (int i = 0; i < nz; ++i) base[(long)i * nxy] = line[i];
                }
            }
        }
    }
};

// ---------------------------------------------------------------------------
// Grid axes.  src/baseHamiltonian.cu:25-51 (x cell-centred) and :53-82 (k in
// cycles per length, reference formula kept for odd N), with DKX and KXMAX of
// src/params.cu:206-211.
void make_axes(const gpe_config& c, std::vector<double>* xs, std::vector<double>* ks) {
    const int NX[3] = {c.nx, c.ny, c.nz};
    for (int d = 0; d < 3; ++d) {
        const int n = NX[d];
        const double DX = c.dx[d];
        const double XMAX = c.xmax[d];
        const double DKX = 1.0 / (n * DX);
        const double KXMAX = 1.0 / (2.0 * DX);
        xs[d].assign(n, 0.0);
        ks[d].assign(n, 0.0);
        bool zero_x = (c.dim == 1 && d > 0) || (c.dim == 2 && d == 2);
        for (int i = 0; i < n; ++i) xs[d][i] = zero_x ? 0.0 : (-XMAX + (i)*DX + 0.5 * DX);
        for (int ik = 0; ik <= n / 2 && ik < n; ++ik) ks[d][ik] = (ik)*DKX;
        for (int ik = n / 2 + 1; ik < n; ++ik) ks[d][ik] = -KXMAX + (ik - (n / 2)) * DKX;
        if (zero_x) for (int i = 0; i < n; ++i) ks[d][i] = 0.0;
    }
}

}  // namespace

// ===========================================================================
struct orc_solver {
    gpe_config cfg;
    int N;            // Npoints
    double DV;        // src/params.cu:213
    int ncomp;
    Plan3D plan;
    std::vector<double> x[3], k[3];
    std::vector<double> k2;     // kx^2+ky^2+kz^2 per point (Laplace, src/parallel.cu:203)
    std::vector<double> vdd;    // dipolar kernel per point (GPE_HAM_DIPOLAR)
    // Reference device buffers per component (src/parallel.cu:37-56).
    std::vector<cplx> psi[2], psi_old[2], psi_new[2], hpsi[2], hpsi_en[2], vext[2], aux[2];
    // PARS of the imaginary-time loops (hpp/oneComponentGPSolver.hpp:20-39,
    // hpp/twoComponentGPSolver.hpp:23-24).
    double EN[2] = {0, 0}, EN_PREV[2] = {0, 0}, MU[2] = {0, 0}, NORM[2] = {0, 0};
    double MU_PREV_RK[2] = {0, 0};
    bool have_mu_prev = false;
    bool converged = false;

    explicit orc_solver(const gpe_config& c)
        : cfg(c), N(c.nx * c.ny * c.nz), DV(c.dx[0] * c.dx[1] * c.dx[2]), ncomp(c.ncomp),
          plan(c.nx, c.ny, c.nz) {
        make_axes(cfg, x, k);
        k2.resize(N);
        for (int iz = 0; iz < c.nz; ++iz)
            for (int iy = 0; iy < c.ny; ++iy)
                for (int ix = 0; ix < c.nx; ++ix) {
                    long idx = ((long)iz * c.ny + iy) * c.nx + ix;
                    k2[idx] = k[0][ix] * k[0][ix] + k[1][iy] * k[1][iy] + k[2][iz] * k[2][iz];
                }
        for (int cc = 0; cc < ncomp; ++cc) {
            psi[cc].assign(N, 0.0); psi_old[cc].assign(N, 0.0); psi_new[cc].assign(N, 0.0);
            hpsi[cc].assign(N, 0.0); hpsi_en[cc].assign(N, 0.0); vext[cc].assign(N, 0.0);
            aux[cc].assign(N, 0.0);
        }
        NORM[0] = cfg.npart[0];
        NORM[1] = cfg.npart[1];
        build_vdd();
    }

    // Spherical cut-off factor c(q) = 1 + 3cos(q)/q^2 - 3sin(q)/q^3
    // = 3 int_0^q j2(x)/x dx; for q < 0.5, where the closed form cancels, the
    // power series 3 sum_n (-1)^n q^(2n+2) / ((2n+2) 2^n n! (2n+5)!!).
    static double cutoff_factor(double q) {
        if (q >= 0.5) return 1.0 + 3.0 * std::cos(q) / (q * q) - 3.0 * std::sin(q) / (q * q * q);
        double sum = 0.0;
        for (int n = 0; n < 8; ++n) {
            double den = 2.0 * n + 2.0;
            for (int i = 1; i <= n; ++i) den *= 2.0 * i;       // 2^n n!
            for (int i = 1; i <= 2 * n + 5; i += 2) den *= i;  // (2n+5)!!
            sum += ((n % 2) ? -1.0 : 1.0) * std::pow(q, 2 * n + 2) / den;
        }
        return 3.0 * sum;
    }

    // Dipolar kernel 12 pi a_dd ((k.d)^2/k^2 - 1/3), src/parallel.cu:326-352
    // (0 for |k| < 1e-6 as there), times the spherical cut-off factor
    // 1 + 3cos(q)/q^2 - 3sin(q)/q^3, q = 2 pi |k| R (its q -> 0 limit is 0).
    void build_vdd() {
        if (cfg.hamiltonian == GPE_HAM_SOFT) {
            build_vsoft();
            return;
        }
        if (cfg.hamiltonian != GPE_HAM_DIPOLAR) return;
        vdd.assign(N, 0.0);
        const double add = cfg.prms[6];
        double d[3] = {cfg.prms[7], cfg.prms[8], cfg.prms[9]};
        double dn = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        if (dn > 0) for (double& v : d) v /= dn;
        const double R = cfg.prms[10];
        for (int iz = 0; iz < cfg.nz; ++iz)
            for (int iy = 0; iy < cfg.ny; ++iy)
                for (int ix = 0; ix < cfg.nx; ++ix) {
                    long idx = ((long)iz * cfg.ny + iy) * cfg.nx + ix;
                    double kx = k[0][ix], ky = k[1][iy], kz = k[2][iz];
                    double num = kx * d[0] + ky * d[1] + kz * d[2];
                    double den = std::sqrt(kx * kx + ky * ky + kz * kz);
                    double v = 0.0;
                    if (den >= 1e-6) {
                        v = 12.0 * PI_REF * add * ((num / den) * (num / den) - 1.0 / 3.0);
                        if (R > 0) {
                            double q = 2.0 * PI_REF * den * R;
                            v *= cutoff_factor(q);
                        }
                    }
                    vdd[idx] = v;
                }
    }

    // Soft-core kernel by dimension: SoftCoreInteraction_1D (src/parallel.cu:371-398),
    // _2D (:412-439), _3D (:453-477); a = prms[0], U = prms[1], k = 2 pi |k|.
    void build_vsoft() {
        vdd.assign(N, 0.0);
        const double a = cfg.prms[0], U = cfg.prms[1];
        for (int iz = 0; iz < cfg.nz; ++iz)
            for (int iy = 0; iy < cfg.ny; ++iy)
                for (int ix = 0; ix < cfg.nx; ++ix) {
                    long idx = ((long)iz * cfg.ny + iy) * cfg.nx + ix;
                    double kx = k[0][ix], ky = k[1][iy], kz = k[2][iz];
                    double kk = 2 * PI_REF * std::sqrt(kx * kx + ky * ky + kz * kz);
                    double v;
                    if (cfg.dim == 1) {
                        if (kk < 1E-6) v = U * 2 * a * (1 - (a * kk) * (a * kk) / 6.0);
                        else v = U * 2 * std::sin(a * kk) / (kk);
                    } else if (cfg.dim == 2) {
                        if (kk < 1E-6) v = U * PI_REF * a * a;
                        else v = 2 * PI_REF * a * U * std::cyl_bessel_j(1.0, kk * a) / kk;
                    } else {
                        if (kk < 1E-6) v = U * (4. / 3.) * PI_REF * std::pow(a, 3);
                        else v = 4 * PI_REF * U * std::pow(a, 3) * (std::sin(kk * a) - kk * a * std::cos(kk * a)) / (std::pow(kk * a, 3));
                    }
                    vdd[idx] = v;
                }
    }

    // BaseHamiltonian::alg_Laplace, src/baseHamiltonian.cu:86-96 with the kernel
    // Laplace of src/parallel.cu:194-205 (scale literal 19.739208802/N kept).
    void laplace(const cplx* in, cplx* out) {
        std::memcpy((void*)out, (const void*)in, sizeof(cplx) * N);
        plan.exec(out, -1);
        const double scale = 19.739208802 / N;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) {
            cplx v = out[i];
            out[i] = cplx(v.real() * scale * k2[i], v.imag() * scale * k2[i]);
        }
        plan.exec(out, +1);
    }

    // BaseHamiltonian::alg_addVPx, src/baseHamiltonian.cu:198-211 with BECVPx
    // (src/parallel.cu:283-292) and AppendArray: aux = IFFT(kx FFT psi)
    // (unnormalised, kx in cycles/length), then h += (-lambda/N) aux and
    // h_en += (-lambda/N) aux.  The plugins add it inside alg_calcHpsi when
    // trotate is set (hamiltonians/BEC_oneComponent.cu:98-101,
    // hamiltonians/BEC_twoComponent.cu:125-129); lambda is prms[11 + c].
    void add_vpx(int c, double lambda) {
        std::vector<cplx>& a = aux[c];
        std::memcpy((void*)a.data(), (const void*)psi[c].data(), sizeof(cplx) * N);
        plan.exec(a.data(), -1);
        const int nx = cfg.nx;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) {
            const double kx = k[0][i % nx];
            a[i] = cplx(a[i].real() * kx, a[i].imag() * kx);
        }
        plan.exec(a.data(), +1);
        const double f = (-1) * lambda / N;
        cplx* hm = hpsi[c].data();
        cplx* he = hpsi_en[c].data();
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) {
            hm[i] = cplx(hm[i].real() + f * a[i].real(), hm[i].imag() + f * a[i].imag());
            he[i] = cplx(he[i].real() + f * a[i].real(), he[i].imag() + f * a[i].imag());
        }
    }

    // Dipolar mean field Phi = IFFT(vdd * FFT(|psi|^2)) / N (new; see build_vdd).
    void dipolar_field(const cplx* p, std::vector<cplx>& phi) {
        phi.resize(N);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) phi[i] = cplx(p[i].real() * p[i].real() + p[i].imag() * p[i].imag(), 0.0);
        plan.exec(phi.data(), -1);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) phi[i] *= vdd[i];
        plan.exec(phi.data(), +1);
        const double inv = 1.0 / N;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) phi[i] *= inv;
    }

    // d_quench_as, hamiltonians/BEC_oneComponent.cu:167-178.
    static double quench_as(double time, const double* prms) {
        double a0 = prms[0], a1 = prms[1], a2 = prms[2];
        double t1 = prms[3], t2 = prms[4], t3 = prms[5];
        if (0 < time && time <= t1) return a0 + (a1 - a0) / (t1)*time;
        if (t1 < time && time <= t2) return a1;
        if (t2 < time && time <= t3) return a1 + (a2 - a1) / (t3 - t2) * (time - t2);
        return a2;
    }

    // Plugin alg_calcHpsi (want_en) / alg_calcHpsiMU: kinetic part then the
    // pointwise kernel, writing hpsi (h_mu) and, if want_en, hpsi_en.
    //  BEC:      hamiltonians/BEC_oneComponent.cu:92-111,128-165
    //  BEC2:     hamiltonians/BEC_twoComponent.cu:120-142,168-244 (vext1.y typo kept)
    //  TEMPLATE: hamiltonians/single_template.cu:313-373
    void calc_hpsi(double t, bool want_en) {
        for (int c = 0; c < ncomp; ++c) laplace(psi[c].data(), hpsi[c].data());
        const int ham = cfg.hamiltonian;
        if (ham == GPE_HAM_BEC || ham == GPE_HAM_DIPOLAR || ham == GPE_HAM_SOFT) {
            // soft core: no contact term, the mean field of the soft kernel
            const double a = (ham == GPE_HAM_SOFT) ? 0.0 : quench_as(t, cfg.prms);
            const bool field = ham == GPE_HAM_DIPOLAR || ham == GPE_HAM_SOFT;
            std::vector<cplx> phi;
            if (field) dipolar_field(psi[0].data(), phi);
            const cplx* p = psi[0].data();
            const cplx* V = vext[0].data();
            cplx* hm = hpsi[0].data();
            cplx* he = hpsi_en[0].data();
#pragma omp parallel for schedule(static)
            for (long i = 0; i < N; ++i) {
                const double px = p[i].real(), py = p[i].imag();
                const double n = px * px + py * py;
                const double Tx = hm[i].real(), Ty = hm[i].imag();
                const double phid = field ? phi[i].real() : 0.0;
                double rX, rY;
                if (want_en) {
                    rX = (V[i].real() + 2 * PI_REF * a * n) + 0.5 * phid;
                    rY = V[i].imag();
                    he[i] = cplx(Tx + rX * px - rY * py, Ty + rX * py + rY * px);
                }
                rX = (V[i].real() + 4 * PI_REF * a * n) + phid;
                rY = V[i].imag();
                hm[i] = cplx(Tx + rX * px - rY * py, Ty + rX * py + rY * px);
            }
        } else if (ham == GPE_HAM_BEC2) {
            const double a11 = cfg.prms[0], a22 = cfg.prms[1], a12 = cfg.prms[2];
            const cplx *p1 = psi[0].data(), *p2 = psi[1].data();
            const cplx *V1 = vext[0].data(), *V2 = vext[1].data();
            cplx *h1 = hpsi[0].data(), *h2 = hpsi[1].data();
            cplx *e1 = hpsi_en[0].data(), *e2 = hpsi_en[1].data();
#pragma omp parallel for schedule(static)
            for (long i = 0; i < N; ++i) {
                const double x1 = p1[i].real(), y1 = p1[i].imag();
                const double x2 = p2[i].real(), y2 = p2[i].imag();
                const double n1 = x1 * x1 + y1 * y1, n2 = x2 * x2 + y2 * y2;
                double aX, aY;
                if (want_en) {
                    aX = (V1[i].real() + 2 * PI_REF * a11 * n1 + 2 * PI_REF * a12 * n2);
                    aY = V1[i].imag();
                    e1[i] = cplx(h1[i].real() + aX * x1 - aY * y1, h1[i].imag() + aX * y1 + aY * x1);
                }
                aX = (V1[i].real() + 4 * PI_REF * a11 * n1 + 4 * PI_REF * a12 * n2);
                aY = V1[i].imag();
                h1[i] = cplx(h1[i].real() + (aX * x1 - aY * y1), h1[i].imag() + (aX * y1 + aY * x1));
                if (want_en) {
                    aX = (V2[i].real() + 2 * PI_REF * a22 * n2 + 2 * PI_REF * a12 * n1);
                    aY = V2[i].imag();
                    e2[i] = cplx(h2[i].real() + aX * x2 - aY * y2, h2[i].imag() + aX * y2 + aY * x2);
                    aX = (V2[i].real() + 4 * PI_REF * a22 * n2 + 4 * PI_REF * a12 * n1);
                    aY = V1[i].imag();  // BEC_twoComponent.cu:208 reads vext1 here
                } else {
                    aX = (V2[i].real() + 4 * PI_REF * a22 * n2 + 4 * PI_REF * a12 * n1);
                    aY = V2[i].imag();
                }
                h2[i] = cplx(h2[i].real() + (aX * x2 - aY * y2), h2[i].imag() + (aX * y2 + aY * x2));
            }
        } else {  // GPE_HAM_TEMPLATE: h_en = h_mu = T
            for (int c = 0; c < ncomp; ++c)
                if (want_en) hpsi_en[c] = hpsi[c];
        }
        if (want_en && ham != GPE_HAM_TEMPLATE)
            for (int c = 0; c < ncomp; ++c)
                if (cfg.prms[11 + c] != 0.0) add_vpx(c, cfg.prms[11 + c]);
    }

    // UpdateRKStep complex overload, src/parallel.cu:238-244.
    static void rk_update(cplx* out, const cplx* old, const cplx* h, cplx c, long n) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i)
            out[i] = cplx(old[i].real() + (c.real() * h[i].real() - c.imag() * h[i].imag()),
                          old[i].imag() + (c.real() * h[i].imag() + c.imag() * h[i].real()));
    }
    // UpdateRKStep real overload, src/parallel.cu:230-236 (k = k + 2 h).
    static void rk_accum(cplx* k, const cplx* h, double sc, long n) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i)
            k[i] = cplx(k[i].real() + sc * h[i].real(), k[i].imag() + sc * h[i].imag());
    }
    // FinalRKStep, src/parallel.cu:261-271.
    static void rk_final(cplx* out, const cplx* old, const cplx* k, const cplx* h, cplx c, long n) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) {
            double aX = k[i].real() + h[i].real();
            double aY = k[i].imag() + h[i].imag();
            out[i] = cplx(old[i].real() + (c.real() * aX - c.imag() * aY) / 6.0,
                          old[i].imag() + (c.real() * aY + c.imag() * aX) / 6.0);
        }
    }

    Acc sum_norm(const cplx* p) const {
        std::vector<Acc> part(omp_threads());
#pragma omp parallel
        {
            Acc a;
#pragma omp for schedule(static)
            for (long i = 0; i < N; ++i) a.add(p[i].real() * p[i].real() + p[i].imag() * p[i].imag());
            part[tid()] = a;
        }
        Acc t;
        for (auto& a : part) t.merge(a);
        return t;
    }
    // sum Re(conj(p) o): Calculate2Observables, src/parallel.cu:613-645.
    Acc sum_dot(const cplx* p, const cplx* o) const {
        std::vector<Acc> part(omp_threads());
#pragma omp parallel
        {
            Acc a;
#pragma omp for schedule(static)
            for (long i = 0; i < N; ++i) a.add(p[i].real() * o[i].real() + p[i].imag() * o[i].imag());
            part[tid()] = a;
        }
        Acc t;
        for (auto& a : part) t.merge(a);
        return t;
    }
    static int omp_threads() {
#ifdef _OPENMP
        return omp_get_max_threads();
#else
        return 1;
#endif
    }
    static int tid() {
#ifdef _OPENMP
        return omp_get_thread_num();
#else
        return 0;
#endif
    }

    // ---- real time -------------------------------------------------------
    // One iteration of OneComponentGPSolver::runRealTimeEvol,
    // src/oneComponentGPSolver.cu:150-188 (per component for 2 components,
    // src/twoComponentGPSolver.cu:142-177, which always uses alg_calcHpsiMU).
    void real_step(int iteration) {
        const double dt = cfg.dt;
        const cplx m05Idt(0.0, -0.5 * dt), mIdt(0.0, -1.0 * dt);
        const bool two = (ncomp == 2);
        for (int c = 0; c < ncomp; ++c) psi_old[c] = psi[c];
        double t = (double)iteration * dt;  // PARS[T] left by the previous iteration
        calc_hpsi(t, false);
        for (int c = 0; c < ncomp; ++c) {
            psi_new[c] = hpsi[c];  // d_k = d_psi_new
            rk_update(psi[c].data(), psi_old[c].data(), hpsi[c].data(), m05Idt, N);
        }
        t = (iteration + 0.5) * dt;
        calc_hpsi(t, false);
        for (int c = 0; c < ncomp; ++c) {
            rk_accum(psi_new[c].data(), hpsi[c].data(), 2.0, N);
            rk_update(psi[c].data(), psi_old[c].data(), hpsi[c].data(), m05Idt, N);
        }
        calc_hpsi(t, false);
        for (int c = 0; c < ncomp; ++c) {
            rk_accum(psi_new[c].data(), hpsi[c].data(), 2.0, N);
            rk_update(psi[c].data(), psi_old[c].data(), hpsi[c].data(), mIdt, N);
        }
        t = (iteration + 1) * dt;
        calc_hpsi(t, !two);
        for (int c = 0; c < ncomp; ++c)
            rk_final(psi[c].data(), psi_old[c].data(), psi_new[c].data(), hpsi[c].data(), mIdt, N);
    }

    // ---- imaginary time: heavy ball ----------------------------------------
    // BECUpdatePsi, src/parallel.cu:294-302.
    void hb_update(int c, double mu, double dt, double beta) {
        const cplx* p = psi[c].data();
        const cplx* o = psi_old[c].data();
        const cplx* h = hpsi[c].data();
        cplx* nw = psi_new[c].data();
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i)
            nw[i] = cplx((1.0 + mu * dt) * p[i].real() - dt * h[i].real() + beta * (p[i].real() - o[i].real()),
                         (1.0 + mu * dt) * p[i].imag() - dt * h[i].imag() + beta * (p[i].imag() - o[i].imag()));
    }
    // alg_updateWavefunctions, src/baseHamiltonian.cu:217-226.
    void update_wavefunctions(int c, double s) {
        psi_old[c] = psi[c];
        cplx* p = psi[c].data();
        const cplx* nw = psi_new[c].data();
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; ++i) p[i] = cplx(nw[i].real() * s, nw[i].imag() * s);
    }

    // One iteration of OneComponentGPSolver::runImagTimeEvol
    // (src/oneComponentGPSolver.cu:51-88) or of TwoComponentGPSolver's
    // (src/twoComponentGPSolver.cu:39-98).  Returns true when it converged.
    bool hb_iteration(int iteration) {
        const double dt = cfg.dt, beta = cfg.beta;
        if (ncomp == 1) {
            EN_PREV[0] = EN[0];
            calc_hpsi(iteration * dt, true);
            hb_update(0, 0 * MU[0], dt, beta);
            NORM[0] = sum_norm(psi_new[0].data()).value() * DV;
            update_wavefunctions(0, std::pow(cfg.npart[0] / NORM[0], 0.5));
            NORM[0] = cfg.npart[0];
            MU[0] = sum_dot(psi[0].data(), hpsi[0].data()).value() * DV / NORM[0];
            EN[0] = sum_dot(psi[0].data(), hpsi_en[0].data()).value() * DV / NORM[0];
            return std::fabs(EN[0] - EN_PREV[0]) / EN_PREV[0] < cfg.epsilon_e;
        }
        EN_PREV[0] = EN[0];
        EN_PREV[1] = EN[1];
        calc_hpsi(0.0, true);
        hb_update(0, MU[0], dt, beta);
        hb_update(1, MU[1], dt, beta);
        NORM[0] = sum_norm(psi_new[0].data()).value() * DV;
        NORM[1] = sum_norm(psi_new[1].data()).value() * DV;
        update_wavefunctions(0, std::pow(cfg.npart[0] / NORM[0], 0.5));
        update_wavefunctions(1, std::pow(cfg.npart[1] / NORM[1], 0.5));
        for (int c = 0; c < 2; ++c) {
            MU[c] = sum_dot(psi[c].data(), hpsi[c].data()).value() * DV / NORM[c];
            EN[c] = sum_dot(psi[c].data(), hpsi_en[c].data()).value() * DV / NORM[c];
        }
        return (std::fabs(EN[0] - EN_PREV[0]) < cfg.epsilon_e) && (std::fabs(EN[1] - EN_PREV[1]) < cfg.epsilon_e);
    }

    // ---- imaginary time: RK4 (new scheme, not in the reference) -------------
    // d psi/d tau = -H psi, classic RK4, then renormalise each component to
    // npart.  mu and E of the normalised state come from stage 1 of the next
    // step; converged when |mu_n - mu_{n-1}| < epsilon_e for every component.
    // Returns true (and leaves psi untouched) when stage 1 detects convergence.
    bool rk4_imag_iteration(int iteration) {
        const double dt = cfg.dt;
        const double t = iteration * dt;
        for (int c = 0; c < ncomp; ++c) psi_old[c] = psi[c];
        calc_hpsi(t, true);
        bool conv = have_mu_prev;
        for (int c = 0; c < ncomp; ++c) {
            EN_PREV[c] = EN[c];
            MU_PREV_RK[c] = MU[c];
            MU[c] = sum_dot(psi[c].data(), hpsi[c].data()).value() * DV / cfg.npart[c];
            EN[c] = sum_dot(psi[c].data(), hpsi_en[c].data()).value() * DV / cfg.npart[c];
            NORM[c] = cfg.npart[c];
            if (!(std::fabs(MU[c] - MU_PREV_RK[c]) < cfg.epsilon_e)) conv = false;
        }
        have_mu_prev = true;
        if (conv) return true;
        const cplx h05(-0.5 * dt, 0.0), h1(-dt, 0.0);
        for (int c = 0; c < ncomp; ++c) {
            psi_new[c] = hpsi[c];
            rk_update(psi[c].data(), psi_old[c].data(), hpsi[c].data(), h05, N);
        }
        calc_hpsi(t, false);
        for (int c = 0; c < ncomp; ++c) {
            rk_accum(psi_new[c].data(), hpsi[c].data(), 2.0, N);
            rk_update(psi[c].data(), psi_old[c].data(), hpsi[c].data(), h05, N);
        }
        calc_hpsi(t, false);
        for (int c = 0; c < ncomp; ++c) {
            rk_accum(psi_new[c].data(), hpsi[c].data(), 2.0, N);
            rk_update(psi[c].data(), psi_old[c].data(), hpsi[c].data(), h1, N);
        }
        calc_hpsi(t, false);
        for (int c = 0; c < ncomp; ++c) {
            rk_final(psi[c].data(), psi_old[c].data(), psi_new[c].data(), hpsi[c].data(), h1, N);
            double nrm = sum_norm(psi[c].data()).value() * DV;
            double s = std::sqrt(cfg.npart[c] / nrm);
            cplx* p = psi[c].data();
#pragma omp parallel for schedule(static)
            for (long i = 0; i < N; ++i) p[i] = cplx(p[i].real() * s, p[i].imag() * s);
        }
        return false;
    }
};

// ===========================================================================
extern "C" {

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

orc_solver* orc_create(const gpe_config* cfg) {
    if (!cfg || cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1) return nullptr;
    if (cfg->ncomp < 1 || cfg->ncomp > 2) return nullptr;
    if (cfg->ncomp == 2 && cfg->hamiltonian != GPE_HAM_BEC2 && cfg->hamiltonian != GPE_HAM_TEMPLATE) return nullptr;
    if (cfg->ncomp == 1 && cfg->hamiltonian == GPE_HAM_BEC2) return nullptr;
    return new orc_solver(*cfg);
}

void orc_destroy(orc_solver* s) { delete s; }

int orc_set_params(orc_solver* s, const double* prms) {
    std::memcpy(s->cfg.prms, prms, sizeof(double) * GPE_NO_HAMIL_PARAMS);
    s->build_vdd();
    return 0;
}

int orc_set_psi(orc_solver* s, int comp, const double* c128) {
    if (comp < 0 || comp >= s->ncomp) return 1;
    std::memcpy((void*)s->psi[comp].data(), c128, sizeof(cplx) * s->N);
    s->psi_old[comp] = s->psi[comp];
    return 0;
}

int orc_get_psi(orc_solver* s, int comp, double* c128) {
    if (comp < 0 || comp >= s->ncomp) return 1;
    std::memcpy(c128, (const void*)s->psi[comp].data(), sizeof(cplx) * s->N);
    return 0;
}

int orc_set_vext(orc_solver* s, int comp, const double* c128) {
    if (comp < 0 || comp >= s->ncomp) return 1;
    std::memcpy((void*)s->vext[comp].data(), c128, sizeof(cplx) * s->N);
    return 0;
}

int orc_step_real(orc_solver* s, int first_iteration, int nsteps, double* obs_out) {
    for (int j = 0; j < nsteps; ++j) s->real_step(first_iteration + j);
    if (obs_out && nsteps > 0) {
        for (int c = 0; c < s->ncomp; ++c) {
            obs_out[3 * c + 0] = s->sum_norm(s->psi[c].data()).value() * s->DV;
            obs_out[3 * c + 1] = s->sum_dot(s->psi[c].data(), s->hpsi[c].data()).value() * s->DV;
            obs_out[3 * c + 2] = s->sum_dot(s->psi[c].data(), s->hpsi_en[c].data()).value() * s->DV;
        }
    }
    return 0;
}

int orc_step_imag(orc_solver* s, int first_iteration, int nsteps, int* iters_done, int* converged) {
    int done = 0;
    int conv = 0;
    if (!s->converged) {
        for (int j = 0; j < nsteps; ++j) {
            bool c;
            if (s->cfg.imag_scheme == GPE_IMAG_RK4) {
                c = s->rk4_imag_iteration(first_iteration + j);
                if (c) { conv = 1; break; }
                ++done;
            } else {
                c = s->hb_iteration(first_iteration + j);
                ++done;
                if (c) { conv = 1; break; }
            }
        }
    }
    if (conv) s->converged = true;
    if (iters_done) *iters_done = done;
    if (converged) *converged = s->converged ? 1 : 0;
    return 0;
}

int orc_imag_state(orc_solver* s, double* out) {
    for (int c = 0; c < s->ncomp; ++c) {
        out[4 * c + 0] = s->NORM[c];
        out[4 * c + 1] = s->MU[c];
        out[4 * c + 2] = s->EN[c];
        out[4 * c + 3] = s->EN_PREV[c];
    }
    return 0;
}

int orc_reset_imag_state(orc_solver* s) {
    for (int c = 0; c < 2; ++c) {
        s->EN[c] = s->EN_PREV[c] = s->MU[c] = 0.0;
        s->NORM[c] = s->cfg.npart[c];
    }
    s->have_mu_prev = false;
    s->converged = false;
    return 0;
}

int orc_laplace(orc_solver* s, int comp, double* out_c128) {
    if (comp < 0 || comp >= s->ncomp) return 1;
    std::vector<cplx> out(s->N);
    s->laplace(s->psi[comp].data(), out.data());
    std::memcpy(out_c128, (const void*)out.data(), sizeof(cplx) * s->N);
    return 0;
}

int orc_apply_h(orc_solver* s, double t, int comp, double* hmu_c128, double* hen_c128) {
    if (comp < 0 || comp >= s->ncomp) return 1;
    s->calc_hpsi(t, true);
    if (hmu_c128) std::memcpy(hmu_c128, (const void*)s->hpsi[comp].data(), sizeof(cplx) * s->N);
    if (hen_c128) std::memcpy(hen_c128, (const void*)s->hpsi_en[comp].data(), sizeof(cplx) * s->N);
    return 0;
}

int orc_observables(orc_solver* s, double t, double* out) {
    s->calc_hpsi(t, true);
    for (int c = 0; c < s->ncomp; ++c) {
        out[3 * c + 0] = s->sum_norm(s->psi[c].data()).value() * s->DV;
        out[3 * c + 1] = s->sum_dot(s->psi[c].data(), s->hpsi[c].data()).value() * s->DV;
        out[3 * c + 2] = s->sum_dot(s->psi[c].data(), s->hpsi_en[c].data()).value() * s->DV;
    }
    return 0;
}

int orc_fft(orc_solver* s, int comp, int sign) {
    if (comp < 0 || comp >= s->ncomp) return 1;
    s->plan.exec(s->psi[comp].data(), sign < 0 ? -1 : +1);
    return 0;
}

void orc_fft3d(int nx, int ny, int nz, double* c128, int sign) {
    Plan3D p(nx, ny, nz);
    p.exec(reinterpret_cast<cplx*>(c128), sign < 0 ? -1 : +1);
}

void orc_axes(const gpe_config* cfg, double* x, double* y, double* z, double* kx, double* ky, double* kz) {
    std::vector<double> xs[3], ks[3];
    make_axes(*cfg, xs, ks);
    std::memcpy(x, xs[0].data(), sizeof(double) * cfg->nx);
    std::memcpy(y, xs[1].data(), sizeof(double) * cfg->ny);
    std::memcpy(z, xs[2].data(), sizeof(double) * cfg->nz);
    std::memcpy(kx, ks[0].data(), sizeof(double) * cfg->nx);
    std::memcpy(ky, ks[1].data(), sizeof(double) * cfg->ny);
    std::memcpy(kz, ks[2].data(), sizeof(double) * cfg->nz);
}

}  // extern "C"
