// gpe_kernels_impl.cuh -- bodies of the axis-pass kernels (included by the
// per-length instantiation units gpe_inst_*.cu).
#pragma once

#include "gpe_kernels.cuh"

namespace gpe {

// ---- psi source ---------------------------------------------------------------
template <typename R>
__device__ __forceinline__ typename Cx<R>::T load_psi(const PassArgs<R>& a, int c, long long gi, int cur) {
    typedef typename Cx<R>::T C;
    if (a.pro == PRO_PIN) return a.pin[c][gi];
    const C* src = (a.pro == PRO_CUR) ? a.buf[cur][c] : a.buf[0][c];
    const double s = a.sc->scale[cur][c];
    const C x = src[gi];
    return from_d<C>(make_double2((double)x.x * s, (double)x.y * s));
}

// ---- k-space multiply ---------------------------------------------------------
// Kinetic: the Laplace kernel of src/parallel.cu:194-205, scale*v*(kx^2+ky^2+kz^2)
// with scale = 19.739208802/N; dipolar density: times vdd (already / N).
template <typename R, int NF>
__device__ __forceinline__ void spec_point(const PassArgs<R>& a, typename Cx<R>::T (&v)[NF], int ix, int iy, int iz,
                                           long long gi) {
    const double k2 = a.kx[ix] * a.kx[ix] + a.ky[iy] * a.ky[iy] + a.kz[iz] * a.kz[iz];
    const int npsi = NF - a.dens;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        if (f < npsi) {
            if constexpr (sizeof(R) == 8) {
                v[f].x = (v[f].x * a.lap_scale) * k2;
                v[f].y = (v[f].y * a.lap_scale) * k2;
            } else {
                const R fac = (R)(a.lap_scale * k2);
                v[f].x *= fac;
                v[f].y *= fac;
            }
        } else {
            const R d = a.vdd[gi];
            v[f].x *= d;
            v[f].y *= d;
        }
    }
}

// ---- finalize (last block, thread 0) --------------------------------------------
template <typename R>
__device__ void finalize_scalars(const PassArgs<R>& a, const double* S) {
    DevScalars* sc = a.sc;
    const int nc = a.ncomp;
    bool bad = false;
    if (a.epi == EPI_HB) {
        const int cur = sc->cur_slot, nxt = 1 - cur;
        bool conv;
        if (nc == 1) {
            // src/oneComponentGPSolver.cu:68-73,84
            const double NORM = S[0] * a.DV;
            const double s = pow(a.npart[0] / NORM, 0.5);
            const double npart = a.npart[0];
            sc->en_prev[0] = sc->en[0];
            sc->mu[0] = (s * S[1]) * a.DV / npart;
            sc->en[0] = (s * S[2]) * a.DV / npart;
            sc->norm[0] = npart;
            sc->scale[nxt][0] = s;
            bad = !isfinite(s) || !isfinite(sc->mu[0]) || !isfinite(sc->en[0]);
            conv = fabs(sc->en[0] - sc->en_prev[0]) / sc->en_prev[0] < a.eps;
        } else {
            // src/twoComponentGPSolver.cu:64-94 (observables divided by the
            // pre-renormalisation norm, absolute energy test)
            conv = true;
            for (int c = 0; c < 2; ++c) {
                const double NORM = S[3 * c] * a.DV;
                const double s = pow(a.npart[c] / NORM, 0.5);
                sc->en_prev[c] = sc->en[c];
                sc->mu[c] = (s * S[3 * c + 1]) * a.DV / NORM;
                sc->en[c] = (s * S[3 * c + 2]) * a.DV / NORM;
                sc->norm[c] = NORM;
                sc->scale[nxt][c] = s;
                bad = bad || !isfinite(s) || !isfinite(sc->mu[c]) || !isfinite(sc->en[c]);
                conv = conv && (fabs(sc->en[c] - sc->en_prev[c]) < a.eps);
            }
        }
        sc->cur_slot = nxt;
        sc->iters_done += 1;
        if (conv) {
            sc->converged = 1;
            sc->done = 1;
        }
    } else if (a.epi == EPI_OBS || a.epi == EPI_RK) {
        for (int q = 0; q < 3 * nc; ++q) sc->obs[q] = S[q] * a.DV;
        for (int q = 0; q < 3 * nc; ++q) bad = bad || !isfinite(sc->obs[q]);
    } else if (a.epi == EPI_RKI) {
        if (a.stage == 1) {
            bool conv = sc->have_mu_prev != 0;
            for (int c = 0; c < nc; ++c) {
                const double mu = (S[3 * c + 1] * a.DV) / a.npart[c];
                const double en = (S[3 * c + 2] * a.DV) / a.npart[c];
                sc->en_prev[c] = sc->en[c];
                sc->mu_prev[c] = sc->mu[c];
                sc->mu[c] = mu;
                sc->en[c] = en;
                sc->norm[c] = a.npart[c];
                if (!(fabs(mu - sc->mu_prev[c]) < a.eps)) conv = false;
                bad = bad || !isfinite(mu) || !isfinite(en);
            }
            sc->have_mu_prev = 1;
            if (conv) {
                sc->converged = 1;
                sc->done = 1;
            }
        } else {
            const int cur = sc->cur_slot, nxt = 1 - cur;
            for (int c = 0; c < nc; ++c) {
                const double NORM = S[3 * c] * a.DV;
                const double s = sqrt(a.npart[c] / NORM);
                sc->scale[nxt][c] = s;
                bad = bad || !isfinite(s);
            }
            sc->cur_slot = nxt;
            sc->iters_done += 1;
        }
    }
    if (bad) {
        sc->status = GPE_ERR_DIVERGED;
        sc->done = 1;
    }
}

template <typename R, int NQ>
__device__ void reduce_and_finalize(const PassArgs<R>& a, DD (&acc)[NQ], DD* red) {
    __shared__ int is_last;
    block_reduce<NQ>(acc, red);
    if (threadIdx.x == 0) {
        double* p = a.partials + (size_t)blockIdx.x * NQ * 2;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            p[2 * q] = acc[q].s;
            p[2 * q + 1] = acc[q].c;
        }
        __threadfence();
        const unsigned int ticket = atomicAdd(&a.sc->counter, 1u);
        is_last = (ticket == gridDim.x * gridDim.y - 1) ? 1 : 0;
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        DD s[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) s[q] = DD{0.0, 0.0};
        const unsigned int nb = gridDim.x * gridDim.y;
        for (unsigned int i = threadIdx.x; i < nb; i += blockDim.x) {
            const double* p = a.partials + (size_t)i * NQ * 2;
#pragma unroll
            for (int q = 0; q < NQ; ++q) s[q] = dd_merge(s[q], DD{__ldcg(p + 2 * q), __ldcg(p + 2 * q + 1)});
        }
        block_reduce<NQ>(s, red);
        if (threadIdx.x == 0) {
            double S[NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q) S[q] = s[q].s + s[q].c;
            finalize_scalars(a, S);
            a.sc->counter = 0;
            __threadfence();
        }
    }
}

// ---- epilogue for one grid point ------------------------------------------------
// v: the NF inverse-transformed fields at this point (kinetic part per psi
// component, dipolar potential field last).
template <typename R, int NF>
__device__ __forceinline__ void epilogue_point(const PassArgs<R>& a, const HamCoef<R>& hc, const typename Cx<R>::T* v,
                                               long long gi, int cur, DD* acc) {
    typedef typename Cx<R>::T C;
    const int nc = a.ncomp;
    const int epi = a.epi;
    if (epi == EPI_STORE) {
#pragma unroll
        for (int f = 0; f < NF; ++f) a.w[f][gi] = v[f];
        return;
    }
    C T[2], psi[2], V[2], hmu[2], hen[2];
    const R phi = a.dens ? v[NF - 1].x : (R)0;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        if (c < nc) {
            T[c] = v[c];
            V[c] = a.vext[c][gi];
        }
    }
    if (epi == EPI_RK) {
        const int stage = a.stage;
        const bool want_en = (stage == 4) && a.want_obs;
#pragma unroll
        for (int c = 0; c < 2; ++c)
            if (c < nc) psi[c] = a.pin[c][gi];
        ham_point<R, C>(a.ham, nc, hc, psi, T, V, phi, want_en, hmu, hen);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (c >= nc) continue;
            const double2 h = to_d(hmu[c]);
            C* A = a.buf[0][c];
            C* B = a.buf[1][c];
            C* K = a.kacc[c];
            if (stage == 1) {
                K[gi] = hmu[c];
                B[gi] = from_d<C>(rk_axpy(to_d(psi[c]), a.c_re, a.c_im, h));
            } else if (stage < 4) {
                const double2 k = to_d(K[gi]);
                K[gi] = from_d<C>(make_double2(k.x + 2.0 * h.x, k.y + 2.0 * h.y));
                B[gi] = from_d<C>(rk_axpy(to_d(A[gi]), a.c_re, a.c_im, h));
            } else {
                const C nv = from_d<C>(rk_final(to_d(A[gi]), a.c_re, a.c_im, to_d(K[gi]), h));
                A[gi] = nv;
                if (a.want_obs) {
                    const double2 n = to_d(nv);
                    const double2 he = to_d(hen[c]);
                    acc[3 * c + 0] = dd_add(acc[3 * c + 0], n.x * n.x + n.y * n.y);
                    acc[3 * c + 1] = dd_add(acc[3 * c + 1], n.x * h.x + n.y * h.y);
                    acc[3 * c + 2] = dd_add(acc[3 * c + 2], n.x * he.x + n.y * he.y);
                }
            }
        }
        return;
    }
    if (epi == EPI_HB) {
        // BECUpdatePsi (src/parallel.cu:294-302) on psi = s_cur*X_cur and
        // psi_old = s_old*X_old; psi~ is written over X_old.
        double2 pd[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (c >= nc) continue;
            const double s = a.sc->scale[cur][c];
            const C x = a.buf[cur][c][gi];
            pd[c] = make_double2((double)x.x * s, (double)x.y * s);
            psi[c] = from_d<C>(pd[c]);
        }
        ham_point<R, C>(a.ham, nc, hc, psi, T, V, phi, true, hmu, hen);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (c >= nc) continue;
            const double so = a.sc->scale[1 - cur][c];
            C* Xo = a.buf[1 - cur][c];
            const C xo = Xo[gi];
            const double ox = (double)xo.x * so, oy = (double)xo.y * so;
            const double mu = (nc == 1) ? 0 * a.sc->mu[0] : a.sc->mu[c];
            const double dt = a.dt, beta = a.beta;
            const double2 p = to_d(psi[c]);
            const double2 h = to_d(hmu[c]);
            const double2 nw = make_double2((1.0 + mu * dt) * p.x - dt * h.x + beta * (p.x - ox),
                                            (1.0 + mu * dt) * p.y - dt * h.y + beta * (p.y - oy));
            const C ns = from_d<C>(nw);
            Xo[gi] = ns;
            const double2 n = to_d(ns);
            const double2 he = to_d(hen[c]);
            acc[3 * c + 0] = dd_add(acc[3 * c + 0], n.x * n.x + n.y * n.y);
            acc[3 * c + 1] = dd_add(acc[3 * c + 1], n.x * h.x + n.y * h.y);
            acc[3 * c + 2] = dd_add(acc[3 * c + 2], n.x * he.x + n.y * he.y);
        }
        return;
    }
    if (epi == EPI_RKI) {
        const int stage = a.stage;
        double2 p0[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (c >= nc) continue;
            const double s = a.sc->scale[cur][c];
            const C x = a.buf[0][c][gi];
            p0[c] = make_double2((double)x.x * s, (double)x.y * s);
            psi[c] = (stage == 1) ? from_d<C>(p0[c]) : a.pin[c][gi];
        }
        ham_point<R, C>(a.ham, nc, hc, psi, T, V, phi, stage == 1, hmu, hen);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (c >= nc) continue;
            const double2 h = to_d(hmu[c]);
            C* A = a.buf[0][c];
            C* B = a.buf[1][c];
            C* K = a.kacc[c];
            if (stage == 1) {
                const double2 p = to_d(psi[c]);
                const double2 he = to_d(hen[c]);
                acc[3 * c + 0] = dd_add(acc[3 * c + 0], p.x * p.x + p.y * p.y);
                acc[3 * c + 1] = dd_add(acc[3 * c + 1], p.x * h.x + p.y * h.y);
                acc[3 * c + 2] = dd_add(acc[3 * c + 2], p.x * he.x + p.y * he.y);
                K[gi] = hmu[c];
                B[gi] = from_d<C>(rk_axpy(p0[c], a.c_re, a.c_im, h));
            } else if (stage < 4) {
                const double2 k = to_d(K[gi]);
                K[gi] = from_d<C>(make_double2(k.x + 2.0 * h.x, k.y + 2.0 * h.y));
                B[gi] = from_d<C>(rk_axpy(p0[c], a.c_re, a.c_im, h));
            } else {
                const C nv = from_d<C>(rk_final(p0[c], a.c_re, a.c_im, to_d(K[gi]), h));
                A[gi] = nv;
                const double2 n = to_d(nv);
                acc[3 * c + 0] = dd_add(acc[3 * c + 0], n.x * n.x + n.y * n.y);
            }
        }
        return;
    }
    // EPI_APPLYH / EPI_OBS
#pragma unroll
    for (int c = 0; c < 2; ++c)
        if (c < nc) psi[c] = load_psi<R>(a, c, gi, cur);
    ham_point<R, C>(a.ham, nc, hc, psi, T, V, phi, true, hmu, hen);
    if (epi == EPI_APPLYH) {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (c >= nc) continue;
            if (a.out[2 * c]) a.out[2 * c][gi] = hmu[c];
            if (a.out[2 * c + 1]) a.out[2 * c + 1][gi] = hen[c];
        }
        return;
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        if (c >= nc) continue;
        const double2 p = to_d(psi[c]), h = to_d(hmu[c]), he = to_d(hen[c]);
        acc[3 * c + 0] = dd_add(acc[3 * c + 0], p.x * p.x + p.y * p.y);
        acc[3 * c + 1] = dd_add(acc[3 * c + 1], p.x * h.x + p.y * h.y);
        acc[3 * c + 2] = dd_add(acc[3 * c + 2], p.x * he.x + p.y * he.y);
    }
}

template <typename R>
__device__ __forceinline__ bool epi_reduces(const PassArgs<R>& a) {
    return a.epi == EPI_HB || a.epi == EPI_OBS || (a.epi == EPI_RK && a.stage == 4 && a.want_obs) ||
           (a.epi == EPI_RKI && (a.stage == 1 || a.stage == 4));
}

// ---- X pass -----------------------------------------------------------------------
template <typename R, int L, int NF>
__global__ void __launch_bounds__(256) k_xpass(PassArgs<R> a) {
    typedef typename Cx<R>::T C;
    constexpr int E = Plan<L>::E;
    constexpr int T = Plan<L>::T;
    constexpr int B = XCfg<R, L>::B;
    constexpr int RinF = Plan<L>::in_radix(false);
    constexpr int RoutF = Plan<L>::out_radix(false);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ DD red[32 * MAXQ];
    if (a.check_done && a.sc->done) return;

    C* S = reinterpret_cast<C*>(smem_raw);
    const int tid = threadIdx.x;
    const int b = tid / T, t = tid % T;
    const int row = blockIdx.x * B + b;
    const bool valid = row < a.nrows;
    const long long base = (long long)(valid ? row : 0) * L;
    const RowAddr<C> addr{S + b * L};
    const int mode = a.mode;
    const int cur = (a.pro != PRO_PIN || a.epi == EPI_HB || a.epi == EPI_RKI) ? a.sc->cur_slot : 0;
    C v[NF][E];

    if (mode == XM_FWD || mode == XM_FULL) {
        const int npsi = NF - a.dens;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long long gi = base + reg_pos<L, E, T, RinF>(t, e);
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                if (f < npsi) {
                    v[f][e] = valid ? load_psi<R>(a, f, gi, cur) : mk((R)0, (R)0);
                } else {
                    const C p = v[0][e];
                    v[f][e] = mk(p.x * p.x + p.y * p.y, (R)0);
                }
            }
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) line_fft_fwd<L>(v[f], addr, a.tw, t);
        if (mode == XM_FWD) {
            if (valid) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const long long gi = base + reg_pos<L, E, T, RoutF>(t, e);
#pragma unroll
                    for (int f = 0; f < NF; ++f) a.w[f][gi] = v[f][e];
                }
            }
            return;
        }
        // XM_FULL: x is the only transformed axis.
        const int iy = row % a.ny, iz = row / a.ny;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int pos = reg_pos<L, E, T, RoutF>(t, e);
            C tmp[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) tmp[f] = v[f][e];
            if (valid) spec_point<R, NF>(a, tmp, pos, iy, iz, base + pos);
#pragma unroll
            for (int f = 0; f < NF; ++f) v[f][e] = tmp[f];
        }
    } else {
        // XM_INV: registers in the inverse input pattern.
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long long gi = base + reg_pos<L, E, T, RoutF>(t, e);
#pragma unroll
            for (int f = 0; f < NF; ++f) v[f][e] = valid ? a.w[f][gi] : mk((R)0, (R)0);
        }
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) line_fft_inv<L>(v[f], addr, a.tw, t);

    // Epilogue: registers at positions of pattern RinF.
    const HamCoef<R> hc = make_coef<R>(a);
    DD acc[MAXQ];
#pragma unroll
    for (int q = 0; q < MAXQ; ++q) acc[q] = DD{0.0, 0.0};
    if (valid) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long long gi = base + reg_pos<L, E, T, RinF>(t, e);
            C tmp[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) tmp[f] = v[f][e];
            epilogue_point<R, NF>(a, hc, tmp, gi, cur, acc);
        }
    }
    if (epi_reduces(a)) reduce_and_finalize<R, MAXQ>(a, acc, red);
}

// ---- strided pass -----------------------------------------------------------------
template <typename R, int L, int NF>
__global__ void __launch_bounds__(512) k_spass(PassArgs<R> a) {
    typedef typename Cx<R>::T C;
    constexpr int E = Plan<L>::E;
    constexpr int T = Plan<L>::T;
    constexpr int RinF = Plan<L>::in_radix(false);
    constexpr int RoutF = Plan<L>::out_radix(false);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.check_done && a.sc->done) return;

    C* S = reinterpret_cast<C*>(smem_raw);
    const int tx = a.tx;
    const int b = threadIdx.x % tx, t = threadIdx.x / tx;
    const int x = blockIdx.x * tx + b;
    const bool valid = x < a.nx;
    const long long base = (long long)blockIdx.y * a.ostride + (valid ? x : 0);
    const long long ss = a.sstride;
    const ColAddr<C> addr{S + b, tx};
    const int mode = a.mode;
    C v[NF][E];

    if (mode == SM_INV) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long long gi = base + (long long)reg_pos<L, E, T, RoutF>(t, e) * ss;
#pragma unroll
            for (int f = 0; f < NF; ++f) v[f][e] = valid ? a.w[f][gi] : mk((R)0, (R)0);
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) line_fft_inv<L>(v[f], addr, a.tw, t);
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long long gi = base + (long long)reg_pos<L, E, T, RinF>(t, e) * ss;
#pragma unroll
            for (int f = 0; f < NF; ++f) v[f][e] = valid ? a.w[f][gi] : mk((R)0, (R)0);
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) line_fft_fwd<L>(v[f], addr, a.tw, t);
        if (mode == SM_FWD) {
            if (valid) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const long long gi = base + (long long)reg_pos<L, E, T, RoutF>(t, e) * ss;
#pragma unroll
                    for (int f = 0; f < NF; ++f) a.w[f][gi] = v[f][e];
                }
            }
            return;
        }
        // SM_FKI: k-space multiply at the forward output positions, then inverse.
        if (a.spec == SPEC_KIN) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int pos = reg_pos<L, E, T, RoutF>(t, e);
                C tmp[NF];
#pragma unroll
                for (int f = 0; f < NF; ++f) tmp[f] = v[f][e];
                if (valid) {
                    const int iy = (a.sax == 2) ? (int)blockIdx.y : pos;
                    const int iz = (a.sax == 2) ? pos : (int)blockIdx.y;
                    spec_point<R, NF>(a, tmp, x, iy, iz, base + (long long)pos * ss);
                }
#pragma unroll
                for (int f = 0; f < NF; ++f) v[f][e] = tmp[f];
            }
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) line_fft_inv<L>(v[f], addr, a.tw, t);
    }
    if (valid) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long long gi = base + (long long)reg_pos<L, E, T, RinF>(t, e) * ss;
#pragma unroll
            for (int f = 0; f < NF; ++f) a.w[f][gi] = v[f][e];
        }
    }
}

// ---- launchers ----------------------------------------------------------------------
template <typename R, int L, int NF>
cudaError_t launch_xpass(const PassArgs<R>& a, cudaStream_t st) {
    typedef typename Cx<R>::T C;
    constexpr int B = XCfg<R, L>::B;
    constexpr int THR = XCfg<R, L>::THREADS;
    const size_t smem = (size_t)B * L * sizeof(C);
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_xpass<R, L, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const int grid = (a.nrows + B - 1) / B;
    k_xpass<R, L, NF><<<grid, THR, smem, st>>>(a);
    return cudaGetLastError();
}

template <typename R, int L, int NF>
cudaError_t launch_spass(const PassArgs<R>& a, int nouter, cudaStream_t st) {
    typedef typename Cx<R>::T C;
    constexpr int T = Plan<L>::T;
    const size_t smem = (size_t)L * a.tx * sizeof(C);
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_spass<R, L, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    dim3 grid((a.nx + a.tx - 1) / a.tx, nouter);
    k_spass<R, L, NF><<<grid, a.tx * T, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace gpe
