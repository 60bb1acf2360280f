// gpe_kernels_impl.cuh -- bodies of the axis-pass kernels (included by the
// per-length instantiation units gpe_inst_*.cu).
#pragma once

#include "gpe_kernels.cuh"

namespace gpe {

// ---- staged inputs ----------------------------------------------------------------
// psi of component c at slot-local index li (prologue and epilogue source):
// PRO_PIN as staged, PRO_CUR / PRO_A_SCALED times the lazy normalisation
// factor of the current slot.
template <typename R>
__device__ __forceinline__ typename Cx<R>::T psi_at(const PassArgs<R>& a, const typename Cx<R>::T* slots, int tile,
                                                    int c, int li, int cur) {
    typedef typename Cx<R>::T C;
    const C x = slots[a.s_psi[c] * tile + li];
    if (a.pro == PRO_PIN) return x;
    const double s = a.sc->scale[cur][c];
    return from_d<C>(make_double2((double)x.x * s, (double)x.y * s));
}

template <typename R>
__device__ __forceinline__ const typename Cx<R>::T* stage_source(const PassArgs<R>& a, int s, int cur) {
    const int k = a.stage_kind[s], c = a.stage_comp[s];
    if (k == SK_CUR) return a.buf[cur][c];
    if (k == SK_OLD) return a.buf[1 - cur][c];
    return a.stage_ptr[s];
}

// ---- tile staging pipeline ---------------------------------------------------------------
// Inputs of a tile are copied asynchronously into one of two shared-memory
// buffers while the CTA computes the previous tile.  x pass: one bulk copy
// (TMA engine) per staged field when rows are 16-byte aligned, completing on
// an mbarrier; strided pass (and unaligned rows): cp.async of 16-byte chunks
// (8-byte elements when a chunk would straddle alignment) by all threads.

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Copy nseg segments of seg elements (segment q: global g0 + q*gstride ->
// slot offset q*sstride) of every staged field with cp.async; commits one group.
template <typename R>
__device__ __forceinline__ void issue_cp_async(const PassArgs<R>& a, typename Cx<R>::T* slots, int tile, long long g0,
                                               int nseg, int seg, long long gstride, int sstride, int cur,
                                               bool chunk16) {
    typedef typename Cx<R>::T C;
    const int ns = a.nstage;
    if (chunk16) {
        constexpr int EPC = 16 / sizeof(C);  // elements per 16-byte chunk
        const int nch = seg / EPC;
        if (nch > 0 && blockDim.x % nch == 0) {
            // each thread keeps one chunk column j and walks segments q0, q0+qs, ...
            const int j = threadIdx.x % nch, q0 = threadIdx.x / nch, qs = blockDim.x / nch;
            for (int f = 0; f < ns; ++f) {
                const C* src = stage_source(a, f, cur) + g0 + j * EPC;
                C* dst = slots + (size_t)f * tile + j * EPC;
                for (int q = q0; q < nseg; q += qs)
                    cp_async16(dst + q * sstride, src + (unsigned)q * (unsigned)gstride);
            }
            cp_async_commit();
            return;
        }
        const int total = ns * nseg * nch;
        for (int k = threadIdx.x; k < total; k += blockDim.x) {
            const int f = k / (nseg * nch);
            const int r = k - f * (nseg * nch);
            const int q = r / nch, j = r - q * nch;
            cp_async16(slots + (size_t)f * tile + (size_t)q * sstride + j * EPC,
                       stage_source(a, f, cur) + g0 + q * gstride + j * EPC);
        }
    } else {
        const int total = ns * nseg * seg;
        for (int k = threadIdx.x; k < total; k += blockDim.x) {
            const int f = k / (nseg * seg);
            const int r = k - f * (nseg * seg);
            const int q = r / seg, j = r - q * seg;
            C* d = slots + (size_t)f * tile + (size_t)q * sstride + j;
            const C* sp = stage_source(a, f, cur) + g0 + q * gstride + j;
            if (sizeof(C) == 16) cp_async16(d, sp);
            else cp_async8(d, sp);
        }
    }
    cp_async_commit();
}

// x pass: nvalid contiguous rows of L elements per staged field.
template <typename R>
__device__ __forceinline__ void issue_rows(const PassArgs<R>& a, typename Cx<R>::T* slots, int tile, long long g0,
                                           int nelems, int cur, uint64_t* mbar) {
    typedef typename Cx<R>::T C;
    if (a.nstage == 0) return;
    if (a.tma) {
        if (threadIdx.x == 0) {
            fence_proxy_async_smem();
            const uint32_t bytes = (uint32_t)(nelems * sizeof(C));
            mbar_arrive_expect_tx(mbar, bytes * (uint32_t)a.nstage);
            for (int f = 0; f < a.nstage; ++f) bulk_g2s(slots + (size_t)f * tile, stage_source(a, f, cur) + g0, bytes, mbar);
        }
    } else {
        issue_cp_async<R>(a, slots, tile, g0, 1, nelems, 0, 0, cur, false);
    }
}

// Wait for the x-pass tile in buffer s (use count u); `more` = a later tile
// was issued after this one.  Uniform across the CTA; false after a timeout.
template <typename R>
__device__ __forceinline__ bool wait_rows(const PassArgs<R>& a, uint64_t* mbar, uint32_t parity, bool more) {
    if (a.nstage == 0) return true;
    if (a.tma) {
        const bool ok = mbar_wait_bounded(mbar, parity, 2000000000ull);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                a.sc->status = GPE_ERR_TIMEOUT;
                a.sc->done = 1;
            }
            return false;
        }
        return true;
    }
    if (more) cp_async_wait_1();
    else cp_async_wait_0();
    __syncthreads();
    return true;
}

// ---- k-space multiply ---------------------------------------------------------
// Kinetic: the Laplace kernel of src/parallel.cu:194-205, scale*v*(kx^2+ky^2+kz^2)
// with scale = 19.739208802/N; dipolar density: times vdd (already / N).
template <typename R, int NF>
__device__ __forceinline__ void spec_point(const PassArgs<R>& a, typename Cx<R>::T (&v)[NF], int ix, int iy, int iz,
                                           long long gi) {
    const int npsi = NF - a.dens;
    if (a.spec == SPEC_PX) {  // v * kx (BECVPx, src/parallel.cu:289-290)
        const double kxv = a.kx[ix];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            v[f].x = (R)(v[f].x * kxv);
            v[f].y = (R)(v[f].y * kxv);
        }
        return;
    }
    const double k2 = a.kx[ix] * a.kx[ix] + a.ky[iy] * a.ky[iy] + a.kz[iz] * a.kz[iz];
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
// component, dipolar potential field last).  Inputs are read from the staged
// slots at li, outputs written to global memory at gi.
template <typename R, int NF, int EPI>
__device__ __forceinline__ void epilogue_point(const PassArgs<R>& a, const HamCoef<R>& hc, const typename Cx<R>::T* v,
                                               const typename Cx<R>::T* slots, int tile, int li, long long gi,
                                               int cur, DD* acc) {
    typedef typename Cx<R>::T C;
    const int nc = a.ncomp;
    const int epi = (EPI >= 0) ? EPI : a.epi;
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
            V[c] = slots[a.s_v[c] * tile + li];
        }
    }
    if (epi == EPI_RK) {
        const int stage = a.stage;
        const bool want_en = (stage == 4) && a.want_obs;
#pragma unroll
        for (int c = 0; c < 2; ++c)
            if (c < nc) psi[c] = slots[a.s_psi[c] * tile + li];
        ham_point<R, C>(a.ham, nc, hc, psi, T, V, phi, want_en, hmu, hen);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (c >= nc) continue;
            const double2 h = to_d(hmu[c]);
            if (stage == 1) {
                a.kacc[c][gi] = hmu[c];
                a.buf[1][c][gi] = from_d<C>(rk_axpy(to_d(psi[c]), a.c_re, a.c_im, h));
            } else if (stage < 4) {
                const double2 k = to_d(slots[a.s_k[c] * tile + li]);
                a.kacc[c][gi] = from_d<C>(make_double2(k.x + 2.0 * h.x, k.y + 2.0 * h.y));
                a.buf[1][c][gi] = from_d<C>(rk_axpy(to_d(slots[a.s_a[c] * tile + li]), a.c_re, a.c_im, h));
            } else {
                const C nv = from_d<C>(rk_final(to_d(slots[a.s_a[c] * tile + li]), a.c_re, a.c_im,
                                                to_d(slots[a.s_k[c] * tile + li]), h));
                a.buf[0][c][gi] = nv;
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
#pragma unroll
        for (int c = 0; c < 2; ++c)
            if (c < nc) psi[c] = psi_at<R>(a, slots, tile, c, li, cur);
        ham_point<R, C>(a.ham, nc, hc, psi, T, V, phi, true, hmu, hen);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (c >= nc) continue;
            const double so = a.sc->scale[1 - cur][c];
            const C xo = slots[a.s_xo[c] * tile + li];
            const double ox = (double)xo.x * so, oy = (double)xo.y * so;
            const double mu = (nc == 1) ? 0 * a.sc->mu[0] : a.sc->mu[c];
            const double dt = a.dt, beta = a.beta;
            const double2 p = to_d(psi[c]);
            const double2 h = to_d(hmu[c]);
            const double2 nw = make_double2((1.0 + mu * dt) * p.x - dt * h.x + beta * (p.x - ox),
                                            (1.0 + mu * dt) * p.y - dt * h.y + beta * (p.y - oy));
            const C ns = from_d<C>(nw);
            a.buf[1 - cur][c][gi] = ns;
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
            const C x = slots[a.s_a[c] * tile + li];
            p0[c] = make_double2((double)x.x * s, (double)x.y * s);
            psi[c] = (stage == 1) ? from_d<C>(p0[c]) : slots[a.s_psi[c] * tile + li];
        }
        ham_point<R, C>(a.ham, nc, hc, psi, T, V, phi, stage == 1, hmu, hen);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (c >= nc) continue;
            const double2 h = to_d(hmu[c]);
            if (stage == 1) {
                const double2 p = to_d(psi[c]);
                const double2 he = to_d(hen[c]);
                acc[3 * c + 0] = dd_add(acc[3 * c + 0], p.x * p.x + p.y * p.y);
                acc[3 * c + 1] = dd_add(acc[3 * c + 1], p.x * h.x + p.y * h.y);
                acc[3 * c + 2] = dd_add(acc[3 * c + 2], p.x * he.x + p.y * he.y);
                a.kacc[c][gi] = hmu[c];
                a.buf[1][c][gi] = from_d<C>(rk_axpy(p0[c], a.c_re, a.c_im, h));
            } else if (stage < 4) {
                const double2 k = to_d(slots[a.s_k[c] * tile + li]);
                a.kacc[c][gi] = from_d<C>(make_double2(k.x + 2.0 * h.x, k.y + 2.0 * h.y));
                a.buf[1][c][gi] = from_d<C>(rk_axpy(p0[c], a.c_re, a.c_im, h));
            } else {
                const C nv = from_d<C>(rk_final(p0[c], a.c_re, a.c_im, to_d(slots[a.s_k[c] * tile + li]), h));
                a.buf[0][c][gi] = nv;
                const double2 n = to_d(nv);
                acc[3 * c + 0] = dd_add(acc[3 * c + 0], n.x * n.x + n.y * n.y);
            }
        }
        return;
    }
    // EPI_APPLYH / EPI_OBS
#pragma unroll
    for (int c = 0; c < 2; ++c)
        if (c < nc) psi[c] = psi_at<R>(a, slots, tile, c, li, cur);
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
// One tile = `rows` rows of the x axis (T threads per row).  Persistent CTAs
// loop over tiles with the inputs of the next tile in flight.  Shared memory:
// two buffers of a.nstage slots of rows*L elements, then the FFT exchange
// buffer of rows*L elements.
template <typename R, int L, int NF, int KIND>
__device__ __forceinline__ void xpass_tile(const PassArgs<R>& a, const HamCoef<R>& hc, const typename Cx<R>::T* slots,
                                           typename Cx<R>::T* X, int tile, int row0, int cur, DD* acc) {
    typedef typename Cx<R>::T C;
    constexpr int E = Plan<L>::E;
    constexpr int T = Plan<L>::T;
    constexpr int RinF = Plan<L>::in_radix(false);
    constexpr int RoutF = Plan<L>::out_radix(false);
    const int b = threadIdx.x / T, t = threadIdx.x % T;
    const bool valid = row0 + b < a.nrows;
    const long long gbase = (long long)(row0 + (valid ? b : 0)) * L;
    const int lbase = b * L;
    const RowAddr<C> addr{X + b * xpad(L)};
    constexpr int EPI = (KIND == XK_STORE) ? EPI_STORE
                      : (KIND == XK_RK || KIND == XK_RKO) ? EPI_RK
                      : (KIND == XK_HB)    ? EPI_HB
                      : (KIND == XK_RKI)   ? EPI_RKI
                      : (KIND == XK_AH)    ? EPI_APPLYH
                                           : -1;
    C v[NF][E];

    if constexpr (KIND == XK_FWD || KIND == XK_FULL) {
        const int npsi = NF - a.dens;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int li = lbase + reg_pos<L, E, T, RinF>(t, e);
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                if (f < npsi) {
                    v[f][e] = valid ? psi_at<R>(a, slots, tile, f, li, cur) : mk((R)0, (R)0);
                } else {
                    const C p = v[0][e];
                    v[f][e] = mk(p.x * p.x + p.y * p.y, (R)0);
                }
            }
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) line_fft_fwd<L>(v[f], addr, a.tw, t);
        if constexpr (KIND == XK_FWD) {
            if (valid) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const long long gi = gbase + reg_pos<L, E, T, RoutF>(t, e);
#pragma unroll
                    for (int f = 0; f < NF; ++f) a.w[f][gi] = v[f][e];
                }
            }
            return;
        }
        // XM_FULL: x is the only transformed axis.
        const int row = row0 + b;
        const int iy = row % a.ny, iz = row / a.ny;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int pos = reg_pos<L, E, T, RoutF>(t, e);
            C tmp[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) tmp[f] = v[f][e];
            if (valid) spec_point<R, NF>(a, tmp, pos, iy, iz, gbase + pos);
#pragma unroll
            for (int f = 0; f < NF; ++f) v[f][e] = tmp[f];
        }
    } else {
        // XM_INV: registers in the inverse input pattern, from the staged W slots.
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int li = lbase + reg_pos<L, E, T, RoutF>(t, e);
#pragma unroll
            for (int f = 0; f < NF; ++f) v[f][e] = valid ? slots[a.s_w[f] * tile + li] : mk((R)0, (R)0);
        }
    }
    // Inverse transform of each field; the results go to the exchange
    // buffers (one per field, natural order) so that the epilogue can walk the
    // points with consecutive threads on consecutive points and few live
    // registers.
    const int rows = blockDim.x / T;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        line_fft_inv<L>(v[f], RowAddr<C>{X + (size_t)f * rows * xpad(L) + b * xpad(L)}, a.tw, t);
        __syncthreads();
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int pos = reg_pos<L, E, T, RinF>(t, e);
            X[(size_t)f * rows * xpad(L) + b * xpad(L) + pos + (pos >> 3)] = v[f][e];
        }
    }
    __syncthreads();
    const int nvalid = min(rows, a.nrows - row0);
    for (int i = threadIdx.x; i < nvalid * L; i += blockDim.x) {
        const int bb = i / L, pos = i - bb * L;
        C tmp[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) tmp[f] = X[(size_t)f * rows * xpad(L) + bb * xpad(L) + pos + (pos >> 3)];
        const int li = bb * L + pos;
        const long long gi = (long long)(row0 + bb) * L + pos;
        if constexpr (EPI == EPI_APPLYH) {
            // the apply-H kernel serves both EPI_APPLYH and EPI_OBS
            if (a.epi == EPI_OBS) epilogue_point<R, NF, EPI_OBS>(a, hc, tmp, slots, tile, li, gi, cur, acc);
            else epilogue_point<R, NF, EPI_APPLYH>(a, hc, tmp, slots, tile, li, gi, cur, acc);
        } else {
            epilogue_point<R, NF, EPI>(a, hc, tmp, slots, tile, li, gi, cur, acc);
        }
    }
}

template <typename R, int L, int NF, int KIND>
__global__ void __launch_bounds__(256, 1) k_xpass(PassArgs<R> a, int rows, int ntiles) {
    typedef typename Cx<R>::T C;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ DD red[32 * MAXQ];
    __shared__ __align__(8) uint64_t mbar[2];
    if (a.check_done && a.sc->done) return;

    const int tile = rows * L;
    const int ns = a.nstage;
    C* bufs = reinterpret_cast<C*>(smem_raw);
    C* X = bufs + (size_t)2 * ns * tile;
    const int cur = a.sc->cur_slot;
    const HamCoef<R> hc = make_coef<R>(a);
    DD acc[MAXQ];
#pragma unroll
    for (int q = 0; q < MAXQ; ++q) acc[q] = DD{0.0, 0.0};
    if (threadIdx.x == 0 && a.tma) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto nrow = [&](int tl) { return min(rows, a.nrows - tl * rows); };
    int tl = blockIdx.x;
    if (tl < ntiles) issue_rows<R>(a, bufs, tile, (long long)tl * rows * L, nrow(tl) * L, cur, &mbar[0]);
    if (tl + (int)gridDim.x < ntiles)
        issue_rows<R>(a, bufs + (size_t)ns * tile, tile, (long long)(tl + gridDim.x) * rows * L,
                      nrow(tl + gridDim.x) * L, cur, &mbar[1]);
    for (int i = 0; tl < ntiles; ++i, tl += gridDim.x) {
        const int sb = i & 1;
        C* slots = bufs + (size_t)sb * ns * tile;
        if (!wait_rows<R>(a, &mbar[sb], (uint32_t)((i >> 1) & 1), tl + (int)gridDim.x < ntiles)) return;
        xpass_tile<R, L, NF, KIND>(a, hc, slots, X, tile, tl * rows, cur, acc);
        __syncthreads();
        const int nx2 = tl + 2 * (int)gridDim.x;
        if (nx2 < ntiles) issue_rows<R>(a, slots, tile, (long long)nx2 * rows * L, nrow(nx2) * L, cur, &mbar[sb]);
    }
    // Only the epilogue-bearing passes reduce (the forward pass carries the
    // chain's epilogue op but runs no epilogue).
    if constexpr (KIND != XK_FWD && KIND != XK_STORE && KIND != XK_RK)
        if (epi_reduces(a)) reduce_and_finalize<R, MAXQ>(a, acc, red);
}

// ---- strided pass -----------------------------------------------------------------
// One tile = tx consecutive x values x the whole line along y or z
// (ntx = ceil(nx/tx) tiles per outer index).  Shared memory: two buffers of
// a.nstage (= NF) W slots of L*tx elements ([pos][b]), then the exchange buffer.
template <typename R, int L, int NF>
__device__ __forceinline__ void spass_tile(const PassArgs<R>& a, const typename Cx<R>::T* slots,
                                           typename Cx<R>::T* X, int tile, int x0, int outer) {
    typedef typename Cx<R>::T C;
    constexpr int E = Plan<L>::E;
    constexpr int T = Plan<L>::T;
    constexpr int RinF = Plan<L>::in_radix(false);
    constexpr int RoutF = Plan<L>::out_radix(false);
    const int tx = a.tx;
    const int b = threadIdx.x % tx, t = threadIdx.x / tx;
    const bool valid = x0 + b < a.nx;
    const long long base0 = (long long)outer * a.ostride + x0;
    const long long ss = a.sstride;
    const ColAddr<C> addr{X + b, tx};
    const int mode = a.mode;
    C v[NF][E];

    if (mode == SM_INV) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int li = reg_pos<L, E, T, RoutF>(t, e) * tx + b;
#pragma unroll
            for (int f = 0; f < NF; ++f) v[f][e] = valid ? slots[a.s_w[f] * tile + li] : mk((R)0, (R)0);
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) line_fft_inv<L>(v[f], addr, a.tw, t);
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int li = reg_pos<L, E, T, RinF>(t, e) * tx + b;
#pragma unroll
            for (int f = 0; f < NF; ++f) v[f][e] = valid ? slots[a.s_w[f] * tile + li] : mk((R)0, (R)0);
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) line_fft_fwd<L>(v[f], addr, a.tw, t);
        if (mode == SM_FWD) {
            if (valid) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const long long gi = base0 + b + (long long)reg_pos<L, E, T, RoutF>(t, e) * ss;
#pragma unroll
                    for (int f = 0; f < NF; ++f) a.w[f][gi] = v[f][e];
                }
            }
            return;
        }
        // SM_FKI: k-space multiply at the forward output positions, then inverse.
        if (a.spec != SPEC_NONE) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int pos = reg_pos<L, E, T, RoutF>(t, e);
                C tmp[NF];
#pragma unroll
                for (int f = 0; f < NF; ++f) tmp[f] = v[f][e];
                if (valid) {
                    const int iy = (a.sax == 2) ? outer : pos;
                    const int iz = (a.sax == 2) ? pos : outer;
                    spec_point<R, NF>(a, tmp, x0 + b, iy, iz, base0 + b + (long long)pos * ss);
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
            const long long gi = base0 + b + (long long)reg_pos<L, E, T, RinF>(t, e) * ss;
#pragma unroll
            for (int f = 0; f < NF; ++f) a.w[f][gi] = v[f][e];
        }
    }
}

template <typename R, int L, int NF>
__global__ void __launch_bounds__(512, 1) k_spass(PassArgs<R> a, int ntx, int ntiles) {
    typedef typename Cx<R>::T C;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    if (a.check_done && a.sc->done) return;

    const int tx = a.tx;
    const int tile = L * tx;
    const int ns = a.nstage;
    C* bufs = reinterpret_cast<C*>(smem_raw);
    C* X = bufs + (size_t)2 * ns * tile;
    const bool chunk16 = a.tma != 0;
    auto issue = [&](int tl, C* slots) {
        const int xb = tl % ntx, outer = tl / ntx;
        const int x0 = xb * tx;
        const int nxv = min(tx, a.nx - x0);
        issue_cp_async<R>(a, slots, tile, (long long)outer * a.ostride + x0, L, nxv, a.sstride, tx, 0, chunk16);
    };
    int tl = blockIdx.x;
    if (tl < ntiles) issue(tl, bufs);
    if (tl + (int)gridDim.x < ntiles) issue(tl + gridDim.x, bufs + (size_t)ns * tile);
    for (int i = 0; tl < ntiles; ++i, tl += gridDim.x) {
        const int sb = i & 1;
        C* slots = bufs + (size_t)sb * ns * tile;
        if (tl + (int)gridDim.x < ntiles) cp_async_wait_1();
        else cp_async_wait_0();
        __syncthreads();
        spass_tile<R, L, NF>(a, slots, X, tile, (tl % ntx) * tx, tl / ntx);
        __syncthreads();
        const int nx2 = tl + 2 * (int)gridDim.x;
        if (nx2 < ntiles) issue(nx2, slots);
    }
}

// ---- launchers ----------------------------------------------------------------------
inline int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 1;
    }
    return n;
}

// rows: rows per tile (x pass), smem bytes per CTA, both chosen by the host.
// The grid is persistent: min(tiles, resident CTAs).
template <typename R, int L, int NF, int KIND>
cudaError_t launch_xpass_kind(const PassArgs<R>& a, int rows, size_t smem, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e =
            cudaFuncSetAttribute(k_xpass<R, L, NF, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const int threads = rows * Plan<L>::T;
    const int ntiles = (a.nrows + rows - 1) / rows;
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_xpass<R, L, NF, KIND>, threads, smem);
    if (occ < 1) occ = 1;
    const int grid = min(ntiles, occ * sm_count());
    k_xpass<R, L, NF, KIND><<<grid, threads, smem, st>>>(a, rows, ntiles);
    return cudaGetLastError();
}

// Kernel role from the pass mode and epilogue op.
__host__ __device__ inline int xkind_of(int mode, int epi) {
    if (mode == XM_FWD) return XK_FWD;
    if (mode == XM_FULL) return XK_FULL;
    switch (epi) {
        case EPI_STORE: return XK_STORE;
        case EPI_RK: return XK_RK;  // XK_RKO when the logging reductions are wanted (see launch_xpass)
        case EPI_HB: return XK_HB;
        case EPI_RKI: return XK_RKI;
        default: return XK_AH;
    }
}

template <typename R, int L, int NF>
cudaError_t launch_xpass(const PassArgs<R>& a, int rows, size_t smem, cudaStream_t st) {
    int kind = xkind_of(a.mode, a.epi);
    if (kind == XK_RK && a.want_obs && a.stage == 4) kind = XK_RKO;
    switch (kind) {
        case XK_FWD: return launch_xpass_kind<R, L, NF, XK_FWD>(a, rows, smem, st);
        case XK_STORE: return launch_xpass_kind<R, L, NF, XK_STORE>(a, rows, smem, st);
        case XK_RK: return launch_xpass_kind<R, L, NF, XK_RK>(a, rows, smem, st);
        case XK_RKO: return launch_xpass_kind<R, L, NF, XK_RKO>(a, rows, smem, st);
        case XK_HB: return launch_xpass_kind<R, L, NF, XK_HB>(a, rows, smem, st);
        case XK_RKI: return launch_xpass_kind<R, L, NF, XK_RKI>(a, rows, smem, st);
        case XK_AH: return launch_xpass_kind<R, L, NF, XK_AH>(a, rows, smem, st);
        default: return launch_xpass_kind<R, L, NF, XK_FULL>(a, rows, smem, st);
    }
}

template <typename R, int L, int NF>
cudaError_t launch_spass(const PassArgs<R>& a, int nouter, size_t smem, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_spass<R, L, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const int threads = a.tx * Plan<L>::T;
    const int ntx = (a.nx + a.tx - 1) / a.tx;
    const int ntiles = ntx * nouter;
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_spass<R, L, NF>, threads, smem);
    if (occ < 1) occ = 1;
    const int grid = min(ntiles, occ * sm_count());
    k_spass<R, L, NF><<<grid, threads, smem, st>>>(a, ntx, ntiles);
    return cudaGetLastError();
}

// Threads per line for a length (host side).
inline int plan_threads(int L) { return L / make_plan(L).E; }

}  // namespace gpe
