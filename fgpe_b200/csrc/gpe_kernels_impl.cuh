// gpe_kernels_impl.cuh -- bodies of the axis-pass kernels (included by the
// per-length instantiation units gpe_inst_*.cu).
//
// Every pass loads its lines straight from global memory into registers in
// the FFT's register pattern (consecutive threads of a line hold consecutive
// points, so each warp load is one or two 128-byte segments), runs the
// Stockham passes with shared-memory exchanges, and stores from registers.
// The x-inverse epilogue runs on the registers too: the other fields it needs
// (psi, V, the RK4 stage fields) are loaded at the same positions.  One CTA
// takes one tile; with no staging buffers the CTAs are small and many are
// resident per SM, which is what hides the memory latency.
#pragma once

#include <atomic>

#include "gpe_kernels.cuh"

namespace gpe {

// Programmatic dependent launch: the pass kernels are launched so that the
// next pass's CTAs may be scheduled while the last CTAs of this pass run.
// Each pass waits for the previous grid (and its memory) before touching
// any field, then lets the following grid start launching.
__device__ __forceinline__ void pass_prologue_sync() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// The members of one instance: for a batched launch (gpe_batch) instance
// blockIdx.y's scalars, parameters, partial sums and field offset.  The kernel
// parameter block itself is never modified (a modified parameter struct would
// be copied to local memory by every thread).
struct InstPtr {
    DevScalars* sc;
    const double* prms;
    double* partials;
    long long boff;
};

template <typename R>
__device__ __forceinline__ InstPtr select_instance_at(const PassArgs<R>& a, unsigned inst) {
    InstPtr p{a.sc, a.prms, a.partials, 0};
    if (a.nbatch > 1) {
        p.sc += inst;
        p.prms += (size_t)inst * GPE_NO_HAMIL_PARAMS;
        p.partials += (size_t)inst * a.pstride;
        p.boff = (long long)inst * a.bstride;
    }
    return p;
}
template <typename R>
__device__ __forceinline__ InstPtr select_instance(const PassArgs<R>& a) {
    return select_instance_at(a, a.nbatch > 1 ? blockIdx.y : 0u);
}

// Lazy normalisation factors of the current / previous heavy-ball slot.
template <typename R>
struct PsiScale {
    double cur[2], old[2];
    double mu[2];  // chemical potentials of the last heavy-ball step
};

template <typename R>
__device__ __forceinline__ PsiScale<R> load_scales(const DevScalars* sc, int cur) {
    PsiScale<R> s;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        s.cur[c] = sc->scale[cur][c];
        s.old[c] = sc->scale[1 - cur][c];
        s.mu[c] = sc->mu[c];
    }
    return s;
}

template <typename C>
__device__ __forceinline__ C scaled(C x, double s) {
    return from_d<C>(make_double2((double)x.x * s, (double)x.y * s));
}

// psi of component c at global index gi (prologue and epilogue source):
// PRO_PIN as stored, PRO_CUR / PRO_A_SCALED times the lazy normalisation
// factor of the current slot.
template <typename R>
__device__ __forceinline__ typename Cx<R>::T load_psi(const PassArgs<R>& a, const PsiScale<R>& ps, int c, long long gi,
                                                      int cur) {
    if (a.pro == PRO_PIN) return a.pin[c][gi];
    if (a.pro == PRO_CUR) return scaled(a.buf[cur][c][gi], ps.cur[c]);
    return scaled(a.buf[0][c][gi], ps.cur[c]);
}

// The host launches a pass with NF = ncomp + dens fields, so a one-field pass
// always serves one component without the dipolar density field: its
// component counts are compile-time constants.
template <int NF>
__host__ __device__ constexpr int maxc_of() {
    return NF == 1 ? 1 : 2;
}
template <int NF, typename R>
__device__ __forceinline__ int ncomp_of(const PassArgs<R>& a) {
    return NF == 1 ? 1 : a.ncomp;
}
template <int NF, typename R>
__device__ __forceinline__ int npsi_of(const PassArgs<R>& a) {
    return NF == 1 ? 1 : NF - a.dens;
}

// ---- k-space multiply ---------------------------------------------------------
// Kinetic: the Laplace kernel of src/parallel.cu:194-205, scale*v*(kx^2+ky^2+kz^2)
// with scale = 19.739208802/N; dipolar density: times vdd (already / N).
template <typename R, int NF>
__device__ __forceinline__ void spec_point(const PassArgs<R>& a, typename Cx<R>::T (&v)[NF], int ix, int iy, int iz,
                                           long long gi) {
    const int npsi = npsi_of<NF>(a);
    if (a.spec == SPEC_PX) {  // v * kx (BECVPx, src/parallel.cu:289-290)
        const double kxv = a.kx[ix];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            v[f].x = (R)(v[f].x * kxv);
            v[f].y = (R)(v[f].y * kxv);
        }
        return;
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        if (f < npsi) {
            // kinetic multiplier; with the moving-frame term (alg_addVPx,
            // src/baseHamiltonian.cu:198-211) also - (lambda/N) kx
            const double rl = a.rot[f < 2 ? f : 0];
            if constexpr (sizeof(R) == 8) {
                const double k2 = a.kx[ix] * a.kx[ix] + a.ky[iy] * a.ky[iy] + a.kz[iz] * a.kz[iz];
                double x = (v[f].x * a.lap_scale) * k2, y = (v[f].y * a.lap_scale) * k2;
                if (rl != 0.0) {
                    const double kr = a.kx[ix] * rl;
                    x -= v[f].x * kr;
                    y -= v[f].y * kr;
                }
                v[f].x = x;
                v[f].y = y;
            } else {
                // complex64: the per-axis float tables of lap_scale * k^2
                // (FP64 only with the moving-frame term)
                R fac;
                if (rl == 0.0) {
                    fac = (a.k2s[0][ix] + a.k2s[1][iy]) + a.k2s[2][iz];
                } else {
                    const double k2 = a.kx[ix] * a.kx[ix] + a.ky[iy] * a.ky[iy] + a.kz[iz] * a.kz[iz];
                    fac = (R)(a.lap_scale * k2 - a.kx[ix] * rl);
                }
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
__device__ void finalize_scalars(const PassArgs<R>& a, DevScalars* sc, const double* S) {
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

// Block-reduction scratch: one array per kernel, however many tile bodies
// (lengths, kinds) the kernel inlines.
__device__ __forceinline__ DD* reduce_scratch() {
    __shared__ DD red[32 * MAXQ];
    return red;
}

// bidx: this tile's partial slot; nblk: the tiles of the instance (the last
// of them to arrive finalises).
template <typename R, int NQ>
__device__ void reduce_and_finalize(const PassArgs<R>& a, const InstPtr& ip, DD (&acc)[NQ], DD* red, unsigned bidx,
                                    unsigned nblk) {
    __shared__ int is_last;
    block_reduce<NQ>(acc, red);
    if (threadIdx.x == 0) {
        double* p = ip.partials + (size_t)bidx * NQ * 2;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            p[2 * q] = acc[q].s;
            p[2 * q + 1] = acc[q].c;
        }
        __threadfence();
        const unsigned int ticket = atomicAdd(&ip.sc->counter, 1u);
        is_last = (ticket == nblk - 1) ? 1 : 0;
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        DD s[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) s[q] = DD{0.0, 0.0};
        const unsigned int nb = nblk;
        for (unsigned int i = threadIdx.x; i < nb; i += blockDim.x) {
            const double* p = ip.partials + (size_t)i * NQ * 2;
#pragma unroll
            for (int q = 0; q < NQ; ++q) s[q] = dd_merge(s[q], DD{__ldcg(p + 2 * q), __ldcg(p + 2 * q + 1)});
        }
        block_reduce<NQ>(s, red);
        if (threadIdx.x == 0) {
            double S[MAXQ];  // quantities past NQ (one-field kernels: 3) are 0
#pragma unroll
            for (int q = 0; q < MAXQ; ++q) S[q] = q < NQ ? s[q].s + s[q].c : 0.0;
            finalize_scalars(a, ip.sc, S);
            ip.sc->counter = 0;
            __threadfence();
        }
    }
}

// ---- Hamiltonian policies ------------------------------------------------------------
// The x-inverse epilogues evaluate the pointwise Hamiltonian through a policy
// type H: coef() builds, once per CTA, what the pointwise term needs from
// d_h_params and the time; point() evaluates h_mu (and h_en) at one grid
// point.  BuiltinHam is the library's plugins (ham_point); UserHam<U> adapts
// a user functor compiled in the user's own translation unit
// (include/gpe_plugin.cuh), the counterpart of the reference's user-written
// Hamiltonian kernels (hamiltonians/BEC_oneComponent.hpp:8-22,
// hamiltonians/single_template.cu:333-373).
struct BuiltinHam {
    template <typename R> using Coef = HamCoef<R>;
    static constexpr bool builtin = true;
    template <typename R>
    __device__ __forceinline__ static HamCoef<R> coef(const PassArgs<R>& a, const double* prms) {
        return make_coef<R>(a, prms);
    }
    template <typename R, typename C, int MC>
    __device__ __forceinline__ static void point(const PassArgs<R>& a, int nc, const HamCoef<R>& hc, const C* psi,
                                                 const C* T, const C* V, R phi, bool want_en, C* hmu, C* hen) {
        ham_point<R, C, MC>(a.ham, nc, hc, psi, T, V, phi, want_en, hmu, hen);
    }
};

// U provides (one component, R = float or double, C = float2 or double2):
//   template <typename R> struct Coef { ... };
//   template <typename R> __device__ static Coef<R> coef(const double* prms, double t);
//   template <typename R, typename C> __device__ static void point(const Coef<R>& k, C psi, C T, C V,
//                                                                   bool want_en, C& hmu, C& hen);
// with T the kinetic part (the reference's KEpsi) at the point.
template <class U>
struct UserHam {
    template <typename R> using Coef = typename U::template Coef<R>;
    static constexpr bool builtin = false;
    template <typename R>
    __device__ __forceinline__ static Coef<R> coef(const PassArgs<R>& a, const double* prms) {
        return U::template coef<R>(prms, a.t);
    }
    template <typename R, typename C, int MC>
    __device__ __forceinline__ static void point(const PassArgs<R>& a, int nc, const Coef<R>& hc, const C* psi,
                                                 const C* T, const C* V, R phi, bool want_en, C* hmu, C* hen) {
        (void)a;
        (void)nc;
        (void)phi;
        C e = T[0];
        U::template point<R, C>(hc, psi[0], T[0], V[0], want_en, hmu[0], e);
        if (want_en) hen[0] = e;
    }
};

// ---- epilogue for one grid point ------------------------------------------------
// The epilogue of a chunk of points first loads every input it needs
// (load_inputs), then computes and stores (epilogue_point).  Loading first
// lets all loads of the chunk be in flight together: a load that followed a
// store of the previous point could not be moved above it, because the state
// buffers are updated in place (the stage state is read from and written to
// the same array, each point by the thread that owns it).
template <typename C>
struct EpiIn {
    C V[2], psi[2], k[2], p0[2], xo[2];
    C aux;  // EPI_ADJ: running control-gradient density
};

// STG: the RK stage when the caller fixed it at compile time (1; 2 for
// stages 2-3; 4), 0 for the run-time a.stage.
template <typename R, int EPI, int NF, int STG>
__device__ __forceinline__ EpiIn<typename Cx<R>::T> load_inputs(const PassArgs<R>& a, const PsiScale<R>& ps,
                                                                long long gi, int cur) {
    typedef typename Cx<R>::T C;
    if constexpr (EPI == EPI_STORE) {
        return EpiIn<C>{};  // the store epilogue reads no inputs
    } else {
        EpiIn<C> in;
        const int nc = ncomp_of<NF>(a);
        const int stage = STG ? STG : a.stage;
        if constexpr (EPI != EPI_STORE) {
#pragma unroll
            for (int c = 0; c < maxc_of<NF>(); ++c) {
                if (c >= nc) continue;
                in.V[c] = a.vext[c][gi];
                if constexpr (EPI == EPI_RK) {
                    in.psi[c] = a.pin[c][gi];
                    if (stage > 1) {
                        in.k[c] = a.kacc[c][gi];
                        in.p0[c] = a.buf[0][c][gi];
                    }
                    if constexpr (sizeof(R) == 4)
                        if (stage == 4 && a.lo[0] != nullptr) in.xo[c] = a.lo[c][gi];
                } else if constexpr (EPI == EPI_HB) {
                    in.psi[c] = scaled(a.buf[cur][c][gi], ps.cur[c]);
                    in.xo[c] = a.buf[1 - cur][c][gi];
                } else if constexpr (EPI == EPI_RKI) {
                    in.p0[c] = a.buf[0][c][gi];
                    if (stage > 1) {
                        in.psi[c] = a.pin[c][gi];
                        in.k[c] = a.kacc[c][gi];
                    }
                } else if constexpr (EPI == EPI_ADJ) {
                    in.psi[c] = a.pin[c][gi];     // mu, the stage adjoint being applied
                    in.p0[c] = a.buf[0][c][gi];   // psi_s, the stage argument
                    in.k[c] = a.out[0][gi];       // lambda_{n+1}
                    if (stage < 4) {
                        in.xo[c] = a.kacc[c][gi];  // running sum of J^T terms
                        in.aux = mk(reinterpret_cast<const R*>(a.out[1])[gi], (R)0);
                    }
                } else {
                    in.psi[c] = load_psi<R>(a, ps, c, gi, cur);
                }
            }
        }
        return in;
    }
}

// XK_RKS: where a tile's staged epilogue inputs start in shared memory
// (after the exchange rows, 16-byte aligned), and the inputs of register e
// read back from this thread's slots (field f of register e at
// stg[(f * E + e) * blockDim.x + threadIdx.x]; fields V, the stage state,
// the accumulator, psi0, the low part, as stage_rk_inputs copies them).
template <typename C>
__host__ __device__ constexpr size_t xstage_offset(int rows, int L) {
    return ((size_t)rows * xpad(L) * sizeof(C) + 15) / 16 * 16;
}
template <typename C, int E, int STG>
__device__ __forceinline__ EpiIn<C> staged_inputs(const PassArgs<float>& a, const C* stg, int e) {
    EpiIn<C> in;
    const unsigned n = blockDim.x, i = threadIdx.x;
    in.V[0] = stg[(0 * E + e) * n + i];
    in.psi[0] = stg[(1 * E + e) * n + i];
    if constexpr (STG > 1) {
        in.k[0] = stg[(2 * E + e) * n + i];
        in.p0[0] = stg[(3 * E + e) * n + i];
    }
    if constexpr (STG == 4)
        if (a.lo[0] != nullptr) in.xo[0] = stg[(4 * E + e) * n + i];
    return in;
}

// v: the NF inverse-transformed fields at global index gi (kinetic part per
// psi component, dipolar potential field last); in: the loaded inputs.
// For EPI_RK, nv receives the new state of each component (the value stored
// in buf[1] for stages 1-3, in buf[0] for stage 4).
template <typename R, int NF, int EPI, bool MAYRED, int STG, class H = BuiltinHam>
__device__ __forceinline__ void epilogue_point(const PassArgs<R>& a, const typename H::template Coef<R>& hc,
                                               const PsiScale<R>& ps,
                                               const typename Cx<R>::T* v, const EpiIn<typename Cx<R>::T>& in,
                                               long long gi, int cur, DD* acc, typename Cx<R>::T* nv) {
    typedef typename Cx<R>::T C;
    constexpr int MC = maxc_of<NF>();
    const int nc = ncomp_of<NF>(a);
    if constexpr (EPI == EPI_STORE) {
#pragma unroll
        for (int f = 0; f < NF; ++f) a.w[f][gi] = v[f];
        return;
    } else {
        C T[2], psi[2], V[2], hmu[2], hen[2];
        const R phi = (NF > 1 && a.dens) ? v[NF - 1].x : (R)0;
#pragma unroll
        for (int c = 0; c < MC; ++c) {
            if (c < nc) {
                T[c] = v[c];
                V[c] = in.V[c];
            }
        }
        if constexpr (EPI == EPI_RK) {
            const int stage = STG ? STG : a.stage;
            const bool want_en = MAYRED && (stage == 4) && a.want_obs;
#pragma unroll
            for (int c = 0; c < MC; ++c)
                if (c < nc) psi[c] = in.psi[c];
            H::template point<R, C, MC>(a, nc, hc, psi, T, V, phi, want_en, hmu, hen);
            const R cr = (R)a.c_re, ci = (R)a.c_im;
#pragma unroll
            for (int c = 0; c < MC; ++c) {
                if (c >= nc) continue;
                const C hm = hmu[c];
                if (stage == 1) {
                    a.kacc[c][gi] = hm;
                    nv[c] = rk_axpy_r(psi[c], cr, ci, hm);
                    a.buf[1][c][gi] = nv[c];
                } else if (stage < 4) {
                    a.kacc[c][gi] = rk_kacc_r(in.k[c], hm);
                    nv[c] = rk_axpy_r(in.p0[c], cr, ci, hm);
                    a.buf[1][c][gi] = nv[c];
                } else {
                    if constexpr (sizeof(R) == 4) {
                        if (a.lo[0] != nullptr) {
                            C lo;
                            nv[c] = rk_final_comp(in.p0[c], in.xo[c], cr, ci, in.k[c], hm, lo);
                            a.lo[c][gi] = lo;
                        } else {
                            nv[c] = rk_final_r(in.p0[c], cr, ci, in.k[c], hm);
                        }
                    } else {
                        nv[c] = rk_final_r(in.p0[c], cr, ci, in.k[c], hm);
                    }
                    a.buf[0][c][gi] = nv[c];
                    if (MAYRED && a.want_obs) {
                        const double2 h = to_d(hm);
                        const double2 n = to_d(nv[c]);
                        const double2 he = to_d(hen[c]);
                        acc[3 * c + 0] = dd_add(acc[3 * c + 0], n.x * n.x + n.y * n.y);
                        acc[3 * c + 1] = dd_add(acc[3 * c + 1], n.x * h.x + n.y * h.y);
                        acc[3 * c + 2] = dd_add(acc[3 * c + 2], n.x * he.x + n.y * he.y);
                    }
                }
            }
            return;
        } else if constexpr (EPI == EPI_HB) {
            // BECUpdatePsi (src/parallel.cu:294-302) on psi = s_cur*X_cur and
            // psi_old = s_old*X_old; psi~ is written over X_old.
#pragma unroll
            for (int c = 0; c < MC; ++c)
                if (c < nc) psi[c] = in.psi[c];
            H::template point<R, C, MC>(a, nc, hc, psi, T, V, phi, true, hmu, hen);
#pragma unroll
            for (int c = 0; c < MC; ++c) {
                if (c >= nc) continue;
                const double so = ps.old[c];
                const C xo = in.xo[c];
                const double ox = (double)xo.x * so, oy = (double)xo.y * so;
                const double mu = (nc == 1) ? 0 * ps.mu[0] : ps.mu[c];
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
        } else if constexpr (EPI == EPI_RKI) {
            const int stage = STG ? STG : a.stage;
            double2 p0[2];
#pragma unroll
            for (int c = 0; c < MC; ++c) {
                if (c >= nc) continue;
                const double s = ps.cur[c];
                const C x = in.p0[c];
                p0[c] = make_double2((double)x.x * s, (double)x.y * s);
                psi[c] = (stage == 1) ? from_d<C>(p0[c]) : in.psi[c];
            }
            H::template point<R, C, MC>(a, nc, hc, psi, T, V, phi, stage == 1, hmu, hen);
#pragma unroll
            for (int c = 0; c < MC; ++c) {
                if (c >= nc) continue;
                const double2 h = to_d(hmu[c]);
                if (stage == 1) {
                    const double2 p = to_d(psi[c]);
                    const double2 he = to_d(hen[c]);
                    acc[3 * c + 0] = dd_add(acc[3 * c + 0], p.x * p.x + p.y * p.y);
                    acc[3 * c + 1] = dd_add(acc[3 * c + 1], p.x * h.x + p.y * h.y);
                    acc[3 * c + 2] = dd_add(acc[3 * c + 2], p.x * he.x + p.y * he.y);
                    a.kacc[c][gi] = hmu[c];
                    nv[c] = from_d<C>(rk_axpy(p0[c], a.c_re, a.c_im, h));
                    a.buf[1][c][gi] = nv[c];
                } else if (stage < 4) {
                    const double2 k = to_d(in.k[c]);
                    a.kacc[c][gi] = from_d<C>(make_double2(k.x + 2.0 * h.x, k.y + 2.0 * h.y));
                    nv[c] = from_d<C>(rk_axpy(p0[c], a.c_re, a.c_im, h));
                    a.buf[1][c][gi] = nv[c];
                } else {
                    nv[c] = from_d<C>(rk_final(p0[c], a.c_re, a.c_im, to_d(in.k[c]), h));
                    a.buf[0][c][gi] = nv[c];
                    const double2 n = to_d(nv[c]);
                    acc[3 * c + 0] = dd_add(acc[3 * c + 0], n.x * n.x + n.y * n.y);
                }
            }
            return;
        } else if constexpr (EPI == EPI_ADJ) {
            // Reverse of one stage of the real-time RK4 step with
            // f(psi) = -i h(psi), h = T + W + g|psi|^2 + Phi[|psi|^2] (one
            // component; Phi = 0 without a k-space interaction):
            //   jt = J^T mu = i (T mu + (W.re + 2 g |psi_s|^2 + Phi[|psi_s|^2]) mu - i W.im mu)
            //                 - i g psi_s^2 conj(mu) + 2 Phi[Im(conj(mu) psi_s)] psi_s
            //   q  += Im(conj(mu) psi_s)           (control-gradient density)
            //   stage 4: acc = lambda + jt; 3, 2: acc += jt; 1: lambda <- acc + jt
            //   next mu = c_re * lambda + c_im * jt   (stages 4, 3, 2)
            const C mu = in.psi[0], ps = in.p0[0], lam = in.k[0];
            const C Tm = T[0];
            const R g = hc.g_mu;
            const R n2 = ps.x * ps.x + ps.y * ps.y;
            R aw = V[0].x + 2 * g * n2;
            // k-space interaction (dipolar, soft core): phi = Phi[|psi_s|^2]
            // acts like the potential; its Jacobian psi_s Phi[2 Re(conj(psi_s) d)]
            // transposes to 2 Phi[Im(conj(mu) psi_s)] psi_s (Phi symmetric)
            if (NF > 1 && a.dens) aw += phi;
            const R Ar = Tm.x + aw * mu.x + V[0].y * mu.y;
            const R Ai = Tm.y + aw * mu.y - V[0].y * mu.x;
            const R s2r = ps.x * ps.x - ps.y * ps.y, s2i = 2 * ps.x * ps.y;
            const R Br = s2r * mu.x + s2i * mu.y;
            const R Bi = s2i * mu.x - s2r * mu.y;
            C jt = mk(-Ai + g * Bi, Ar - g * Br);
            if (NF > 1 && a.dens) {
                const R pr = 2 * v[NF - 1].y;
                jt.x += pr * ps.x;
                jt.y += pr * ps.y;
            }
            R q = mu.x * ps.y - mu.y * ps.x;
            R* qf = reinterpret_cast<R*>(a.out[1]);
            const int stage = a.stage;
            C acc2;
            if (stage == 4) {
                acc2 = mk(lam.x + jt.x, lam.y + jt.y);
            } else {
                acc2 = mk(in.xo[0].x + jt.x, in.xo[0].y + jt.y);
                q += in.aux.x;
            }
            qf[gi] = q;
            if (stage == 1) {
                a.out[0][gi] = acc2;
            } else {
                a.kacc[0][gi] = acc2;
                const R cl = (R)a.c_re, cj = (R)a.c_im;
                a.buf[1][0][gi] = mk(cl * lam.x + cj * jt.x, cl * lam.y + cj * jt.y);
            }
            (void)nv;
            return;
        } else {
            // EPI_APPLYH / EPI_OBS
#pragma unroll
            for (int c = 0; c < 2; ++c)
                if (c < nc) psi[c] = in.psi[c];
            H::template point<R, C, MC>(a, nc, hc, psi, T, V, phi, true, hmu, hen);
            if constexpr (EPI == EPI_APPLYH) {
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    if (c >= nc) continue;
                    if (a.out[2 * c]) a.out[2 * c][gi] = hmu[c];
                    if (a.out[2 * c + 1]) a.out[2 * c + 1][gi] = hen[c];
                }
                return;
            } else {
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    if (c >= nc) continue;
                    const double2 p = to_d(psi[c]), h = to_d(hmu[c]), he = to_d(hen[c]);
                    acc[3 * c + 0] = dd_add(acc[3 * c + 0], p.x * p.x + p.y * p.y);
                    acc[3 * c + 1] = dd_add(acc[3 * c + 1], p.x * h.x + p.y * h.y);
                    acc[3 * c + 2] = dd_add(acc[3 * c + 2], p.x * he.x + p.y * he.y);
                }
            }
        }
    }
}

// Epilogue of E points (register e at line position pos(e)): inputs of a
// chunk of EC points are loaded first, then the chunk is computed and stored.
// One-field passes take chunks of 4 points (2 for the adjoint and for the
// complex64 RK stage 4, which also reads the low part of the state: their
// inputs would spill), two-field passes 1: as many loads in flight as the
// register budget of the launch bounds holds without spilling.
// FUSE: v[f][e] is replaced by the new RK state of component f (and, for the
// dipolar density field, its |psi|^2), ready for the forward x transform.
template <typename R, int NF, int EPI, bool MAYRED, int L, int E, int T, int Rr, bool FUSE = false, int STG = 0,
          class H = BuiltinHam, bool STAGED = false>
__device__ __forceinline__ void epilogue_line(const PassArgs<R>& a, const typename H::template Coef<R>& hc,
                                              const PsiScale<R>& ps,
                                              typename Cx<R>::T (&v)[NF][E], long long g0, int cur, DD* acc,
                                              const typename Cx<R>::T* stg = nullptr) {
    typedef typename Cx<R>::T C;
    constexpr bool LO = EPI == EPI_RK && sizeof(R) == 4 && (STG == 4 || STG == 0);  // may read the low part
    constexpr int EC0 = (NF > 1) ? 1 : ((EPI == EPI_ADJ || LO) ? 2 : 4);
    constexpr int EC = (E % EC0 == 0) ? EC0 : ((E % 4 == 0) ? 4 : ((E % 2 == 0) ? 2 : 1));
#pragma unroll
    for (int e0 = 0; e0 < E; e0 += EC) {
        EpiIn<C> in[EC];
#pragma unroll
        for (int j = 0; j < EC; ++j) {
            if constexpr (STAGED) {
                static_assert(sizeof(R) == 4 && NF == 1 && EPI == EPI_RK && STG != 0, "staged inputs: XK_RKS only");
                in[j] = staged_inputs<C, E, STG>(a, stg, e0 + j);
            } else {
                in[j] = load_inputs<R, EPI, NF, STG>(a, ps, g0 + reg_off<L, E, T, Rr>(e0 + j), cur);
            }
        }
#pragma unroll
        for (int j = 0; j < EC; ++j) {
            C tmp[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) tmp[f] = v[f][e0 + j];
            C nv[2];
            epilogue_point<R, NF, EPI, MAYRED, STG, H>(a, hc, ps, tmp, in[j], g0 + reg_off<L, E, T, Rr>(e0 + j), cur,
                                                    acc, nv);
            if constexpr (FUSE) {
                const int npsi = npsi_of<NF>(a);
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    if (f < npsi) v[f][e0 + j] = nv[f < 2 ? f : 1];
                    else v[f][e0 + j] = mk(nv[0].x * nv[0].x + nv[0].y * nv[0].y, (R)0);
                }
            }
        }
    }
}

// Epilogue of a line with the op of the kernel role.
template <typename R, int NF, int KIND, int L, int E, int T, int Rr, class H = BuiltinHam>
__device__ __forceinline__ void epilogue_dispatch(const PassArgs<R>& a, const typename H::template Coef<R>& hc,
                                                  const PsiScale<R>& ps,
                                                  typename Cx<R>::T (&v)[NF][E], long long g0, int cur, DD* acc,
                                                  const typename Cx<R>::T* stg = nullptr) {
#define GPE_EPI(OP, RED) epilogue_line<R, NF, OP, RED, L, E, T, Rr, false, 0, H>(a, hc, ps, v, g0, cur, acc)
    if constexpr (KIND == XK_STORE) GPE_EPI(EPI_STORE, false);
    else if constexpr (KIND == XK_RK) GPE_EPI(EPI_RK, false);
    else if constexpr (KIND == XK_RKF) {
        // the hot real-time kernel: one copy of the epilogue per stage class
        if (a.stage == 1) epilogue_line<R, NF, EPI_RK, false, L, E, T, Rr, true, 1, H>(a, hc, ps, v, g0, cur, acc);
        else if (a.stage < 4) epilogue_line<R, NF, EPI_RK, false, L, E, T, Rr, true, 2, H>(a, hc, ps, v, g0, cur, acc);
        else epilogue_line<R, NF, EPI_RK, false, L, E, T, Rr, true, 4, H>(a, hc, ps, v, g0, cur, acc);
    } else if constexpr (KIND == XK_RKS) {
        if (a.stage == 1)
            epilogue_line<R, NF, EPI_RK, false, L, E, T, Rr, true, 1, H, true>(a, hc, ps, v, g0, cur, acc, stg);
        else if (a.stage < 4)
            epilogue_line<R, NF, EPI_RK, false, L, E, T, Rr, true, 2, H, true>(a, hc, ps, v, g0, cur, acc, stg);
        else
            epilogue_line<R, NF, EPI_RK, false, L, E, T, Rr, true, 4, H, true>(a, hc, ps, v, g0, cur, acc, stg);
    } else if constexpr (KIND == XK_RKO) {  // launched for stage 4 only
        epilogue_line<R, NF, EPI_RK, true, L, E, T, Rr, false, 4, H>(a, hc, ps, v, g0, cur, acc);
    }
    else if constexpr (KIND == XK_HB) GPE_EPI(EPI_HB, true);
    else if constexpr (KIND == XK_RKI) GPE_EPI(EPI_RKI, true);
    else if constexpr (KIND == XK_RKIF)  // stages 1-3, the new stage state then x-forward transformed
        epilogue_line<R, NF, EPI_RKI, true, L, E, T, Rr, true, 0, H>(a, hc, ps, v, g0, cur, acc);
    else if constexpr (KIND == XK_ADJ) GPE_EPI(EPI_ADJ, false);
    else if constexpr (KIND == XK_AH) {
        // the apply-H kernel serves both EPI_APPLYH and EPI_OBS
        if (a.epi == EPI_OBS) GPE_EPI(EPI_OBS, true);
        else GPE_EPI(EPI_APPLYH, true);
    } else {  // XK_FULL: run-time op
        switch (a.epi) {
            case EPI_STORE: GPE_EPI(EPI_STORE, false); break;
            case EPI_RK: GPE_EPI(EPI_RK, true); break;
            case EPI_HB: GPE_EPI(EPI_HB, true); break;
            case EPI_RKI: GPE_EPI(EPI_RKI, true); break;
            case EPI_APPLYH: GPE_EPI(EPI_APPLYH, true); break;
            default: GPE_EPI(EPI_OBS, true); break;
        }
    }
#undef GPE_EPI
}

template <typename R>
__device__ __forceinline__ bool epi_reduces(const PassArgs<R>& a) {
    return a.epi == EPI_HB || a.epi == EPI_OBS || (a.epi == EPI_RK && a.stage == 4 && a.want_obs) ||
           (a.epi == EPI_RKI && (a.stage == 1 || a.stage == 4));
}

// Kernel roles that may reduce (the others never touch the partials).
template <int KIND>
__host__ __device__ constexpr bool kind_reduces() {
    return KIND == XK_RKO || KIND == XK_HB || KIND == XK_RKI || KIND == XK_RKIF || KIND == XK_AH || KIND == XK_FULL;
}

// Resident CTAs per SM the launch bounds ask for: complex64 lines of up to 8
// values per thread fit three 256-thread CTAs; complex128 or longer register
// arrays, two; two fields and long arrays, one.
template <typename R, int L, int NF>
__host__ __device__ constexpr int pass_min_blocks() {
    constexpr int E = Plan<L>::E;
    constexpr int w = (int)sizeof(R) / 4 * E * NF;  // 32-bit words of line values per thread / 2
    return w <= 8 ? 3 : (w <= 16 ? 2 : 1);
}

// ---- X pass -----------------------------------------------------------------------
// One CTA = `rows` consecutive rows of the x axis, T threads per row.  Shared
// memory: one padded exchange row per line (rows * xpad(L) elements).
// Roles with the FP64 reductions hold more live values: one CTA fewer.  The
// one-field real-time RK roles fit 64 registers: one CTA more.
// The one-field heavy-ball and apply-H roles (both precisions) and the
// complex64 observables role carry three reduced sums and fit the
// non-reducing budget without spills for lines of 8 values (-Xptxas -v:
// 80 registers complex64, 128 complex128), so they keep the CTA.
template <typename R, int L, int NF, int KIND>
__host__ __device__ constexpr bool xpass_light_reduce() {
    return NF == 1 && Plan<L>::E == 8 &&
           (KIND == XK_HB || KIND == XK_AH || (KIND == XK_RKO && sizeof(R) == 4));
}
template <typename R, int L, int NF, int KIND>
__host__ __device__ constexpr int xpass_min_blocks() {
    return (NF == 1 && (KIND == XK_RKF || KIND == XK_RK || KIND == XK_RKS) && pass_min_blocks<R, L, NF>() == 3)
               ? 4
               : (kind_reduces<KIND>() && pass_min_blocks<R, L, NF>() > 1 && !xpass_light_reduce<R, L, NF, KIND>()
                      ? pass_min_blocks<R, L, NF>() - 1
                      : pass_min_blocks<R, L, NF>());
}

// Warms L2 with a tile's real-time RK epilogue inputs (V, the stage state
// and, after stage 1, the accumulator and psi0, at stage 4 the low part of
// psi0: nr consecutive rows of L points from global index t0) while the
// inverse transform runs.  On the first stage of a step they come from HBM;
// later stages find them in L2.
template <typename R, int NF>
__device__ __forceinline__ void prefetch_rk_inputs(const PassArgs<R>& a, long long t0, int nr, int L) {
    typedef typename Cx<R>::T C;
    const unsigned lines = ((unsigned)nr * (unsigned)L * (unsigned)sizeof(C) + 127u) / 128u;
    const unsigned nf = a.stage > 1 ? ((a.stage == 4 && a.lo[0] != nullptr) ? 5u : 4u) : 2u;
    const unsigned total = (unsigned)ncomp_of<NF>(a) * nf * lines;
    for (unsigned i = threadIdx.x; i < total; i += blockDim.x) {
        const unsigned l = i % lines, fc = i / lines, f = fc % nf, c = fc / nf;
        const C* base = f == 0 ? a.vext[c]
                               : (f == 1 ? a.pin[c] : (f == 2 ? a.kacc[c] : (f == 3 ? a.buf[0][c] : a.lo[c])));
        const char* p = reinterpret_cast<const char*>(base + t0) + (size_t)l * 128u;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
    }
}

// One tile of an x pass: `rows` rows from row tile*rows of instance inst
// (ntiles tiles per instance), after the kernel's wait on the previous grid.
// k_xpass runs one tile per CTA; the persistent batch kernel loops over tiles.
template <typename R, int L, int NF, int KIND, class H = BuiltinHam>
__device__ __forceinline__ void xpass_tile(const PassArgs<R>& a, int rows, unsigned tile, unsigned inst,
                                           unsigned ntiles, unsigned char* smem_raw) {
    typedef typename Cx<R>::T C;
    constexpr int E = Plan<L>::E;
    constexpr int T = Plan<L>::T;
    constexpr int RinF = Plan<L>::in_radix(false);
    constexpr int RoutF = Plan<L>::out_radix(false);
    const InstPtr ip = select_instance_at(a, inst);
    const long long boff = ip.boff;
    if (a.check_done && ip.sc->done) return;

    C* X = reinterpret_cast<C*>(smem_raw);
    const unsigned b = threadIdx.x / T, t = threadIdx.x % T;
    const int row = (int)tile * rows + (int)b;
    const bool valid = row < a.nrows;
    // g0 + reg_off(e): global index of register e of this thread's line
    const long long g0 = boff + (long long)(valid ? row : 0) * L + t;
    const RowAddr<C, L> addr{X + b * xpad(L)};
    const int cur = ip.sc->cur_slot;
    const PsiScale<R> ps = load_scales<R>(ip.sc, cur);
    // reduced quantities: three per component (norm, <h_mu>, <h_en> or the
    // role's equivalents); a one-field pass serves one component
    constexpr int NQ = NF == 1 ? 3 : MAXQ;
    DD acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[q] = DD{0.0, 0.0};
    C v[NF][E];

    if constexpr (KIND == XK_FWD || KIND == XK_FULL) {
        const int npsi = npsi_of<NF>(a);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long long gi = g0 + reg_off<L, E, T, RinF>(e);
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                if (f < npsi) {
                    v[f][e] = valid ? load_psi<R>(a, ps, f, gi, cur) : mk((R)0, (R)0);
                } else if (a.epi == EPI_ADJ) {
                    // adjoint chain: the stage argument's density |psi_s|^2 and
                    // Im(conj(mu) psi_s), the two real inputs of the k-space
                    // interaction's Jacobian, as one complex field (the table
                    // is real and even in k, so the parts stay apart)
                    const C p = v[0][e];
                    const C q = valid ? a.buf[0][0][gi] : mk((R)0, (R)0);
                    v[f][e] = mk(q.x * q.x + q.y * q.y, p.x * q.y - p.y * q.x);
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
                    const long long gi = g0 + reg_off<L, E, T, RoutF>(e);
#pragma unroll
                    for (int f = 0; f < NF; ++f) a.w[f][gi] = v[f][e];
                }
            }
            return;
        } else {
            // x is the only transformed axis: k-space multiply here.
            const int iy = row % a.ny, iz = row / a.ny;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int pos = reg_pos<L, E, T, RoutF>((int)t, e);
                C tmp[NF];
#pragma unroll
                for (int f = 0; f < NF; ++f) tmp[f] = v[f][e];
                if (valid) spec_point<R, NF>(a, tmp, pos, iy, iz, g0 + reg_off<L, E, T, RoutF>(e));
#pragma unroll
                for (int f = 0; f < NF; ++f) v[f][e] = tmp[f];
            }
        }
    } else {
        // inverse input pattern straight from the transformed fields
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long long gi = g0 + reg_off<L, E, T, RoutF>(e);
#pragma unroll
            for (int f = 0; f < NF; ++f) v[f][e] = valid ? a.w[f][gi] : mk((R)0, (R)0);
        }
    }
    if constexpr (KIND != XK_FWD) {
        const typename H::template Coef<R> hc = H::template coef<R>(a, ip.prms);
#pragma unroll
        for (int f = 0; f < NF; ++f) line_fft_inv<L>(v[f], addr, a.tw, t);
        if constexpr (KIND == XK_RKS) {
            // this thread's staged inputs (issued at kernel start) have landed
            asm volatile("cp.async.wait_all;" ::: "memory");
            const C* stg = reinterpret_cast<const C*>(smem_raw + xstage_offset<C>(rows, L));
            if (valid) epilogue_dispatch<R, NF, KIND, L, E, T, RinF, H>(a, hc, ps, v, g0, cur, acc, stg);
        } else {
            if (valid) epilogue_dispatch<R, NF, KIND, L, E, T, RinF, H>(a, hc, ps, v, g0, cur, acc);
        }
        if constexpr (KIND == XK_RKF || KIND == XK_RKS || KIND == XK_RKIF) {
            // next stage's x-forward pass on the state just written (in place on w)
#pragma unroll
            for (int f = 0; f < NF; ++f) line_fft_fwd<L>(v[f], addr, a.tw, t);
            if (valid) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const long long gi = g0 + reg_off<L, E, T, RoutF>(e);
#pragma unroll
                    for (int f = 0; f < NF; ++f) a.w[f][gi] = v[f][e];
                }
            }
        }
        if constexpr (kind_reduces<KIND>()) {
            if (epi_reduces(a)) {
                reduce_and_finalize<R, NQ>(a, ip, acc, reduce_scratch(), tile, ntiles);
            }
        }
    }
}

// XK_RKS: each thread copies the epilogue inputs of its E points (V and the
// stage state; from stage 2 the accumulator and psi0; at stage 4 the low
// part) from global memory into its own shared-memory slots with 8-byte
// asynchronous copies (one group), in the order staged_inputs reads them.
// Each thread reads back only what it copied itself, so the wait for its own
// group is all the synchronisation needed.
template <typename R, int L>
__device__ __forceinline__ void stage_rk_inputs(const PassArgs<R>& a, int rows, unsigned char* smem_raw) {
    typedef typename Cx<R>::T C;
    static_assert(sizeof(C) == 8, "staged inputs: complex64 only");
    constexpr int E = Plan<L>::E;
    constexpr int T = Plan<L>::T;
    constexpr int RinF = Plan<L>::in_radix(false);
    const long long boff = select_instance(a).boff;
    const unsigned b = threadIdx.x / T, t = threadIdx.x % T;
    const int row = (int)blockIdx.x * rows + (int)b;
    if (row < a.nrows) {
        const long long g0 = boff + (long long)row * L + t;
        C* stg = reinterpret_cast<C*>(smem_raw + xstage_offset<C>(rows, L));
        const int nfs = a.stage == 1 ? 2 : ((a.stage == 4 && a.lo[0] != nullptr) ? 5 : 4);
        const unsigned n = blockDim.x, i = threadIdx.x;
        for (int f = 0; f < nfs; ++f) {
            const C* src = f == 0 ? a.vext[0] : (f == 1 ? a.pin[0] : (f == 2 ? a.kacc[0] : (f == 3 ? a.buf[0][0] : a.lo[0])));
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const C* gp = src + g0 + reg_off<L, E, T, RinF>(e);
                const unsigned sa = (unsigned)__cvta_generic_to_shared(stg + (f * E + e) * n + i);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gp) : "memory");
            }
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

template <typename R, int L, int NF, int KIND, class H = BuiltinHam>
__global__ void __launch_bounds__(256, (xpass_min_blocks<R, L, NF, KIND>())) k_xpass(PassArgs<R> a, int rows) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if constexpr (KIND == XK_RKS) {
        // the inputs were written two or more launches earlier (see below)
        stage_rk_inputs<R, L>(a, rows, smem_raw);
    } else if constexpr (KIND == XK_RKF || KIND == XK_RK || KIND == XK_RKO) {
        // The epilogue inputs were written two or more launches earlier, so
        // the L2 prefetch may run before the wait for the preceding grid
        // (with programmatic launch this CTA can start during its tail);
        // a prefetch is only a cache hint either way.
        const long long boff = select_instance(a).boff;
        const int nr = min(rows, a.nrows - (int)blockIdx.x * rows);
        if (nr > 0) prefetch_rk_inputs<R, NF>(a, boff + (long long)blockIdx.x * rows * L, nr, L);
    }
    pass_prologue_sync();
    xpass_tile<R, L, NF, KIND, H>(a, rows, blockIdx.x, a.nbatch > 1 ? blockIdx.y : 0u, gridDim.x, smem_raw);
}

// ---- strided pass -----------------------------------------------------------------
// One CTA = tx consecutive x values x the whole line along y or z, for one
// outer index (blockIdx.x = outer * ntx + x block).  Thread (b, t) = (line
// b of the tile, thread t of the line); b is the fast index so that a warp
// loads tx consecutive x values per line position.  Shared memory: the
// exchange buffer S[pos * tx + b].
// Strided passes hold no epilogue state: two CTAs more than pass_min_blocks
// for the short (complex64, E <= 8) lines (48 registers, no spills).
template <typename R, int L, int NF>
__host__ __device__ constexpr int spass_min_blocks() {
    return pass_min_blocks<R, L, NF>() == 3 ? 5 : pass_min_blocks<R, L, NF>();
}

// TX: x values per CTA (tile width); MB: resident CTAs per SM the launch
// bounds ask for.  The defaults are spass_tx and spass_min_blocks; other
// (TX, MB) pairs are autotuner variants (gpe_tune.cu).
// One tile of a strided pass (tile = outer * ntx + x block) of instance inst,
// after the kernel's wait on the previous grid; k_spass runs one tile per
// CTA, the persistent batch kernel loops over tiles.
template <typename R, int L, int NF, int TX>
__device__ __forceinline__ void spass_tile(const PassArgs<R>& a, int ntx, unsigned tile, unsigned inst,
                                           unsigned char* smem_raw) {
    typedef typename Cx<R>::T C;
    constexpr int E = Plan<L>::E;
    constexpr int T = Plan<L>::T;
    constexpr int RinF = Plan<L>::in_radix(false);
    constexpr int RoutF = Plan<L>::out_radix(false);
    const InstPtr ip = select_instance_at(a, inst);
    const long long boff = ip.boff;
    if (a.check_done && ip.sc->done) return;

    C* X = reinterpret_cast<C*>(smem_raw);
    constexpr int tx = TX;
    const int xb = (int)tile % ntx, outer = (int)tile / ntx;
    const int x0 = xb * tx;
    const unsigned b = threadIdx.x % tx, t = threadIdx.x / tx;
    const bool valid = x0 + (int)b < a.nx;
    const long long ss = a.sstride;
    // g0 + reg_off(e) * ss: global index of register e of this thread's line
    const long long g0 = boff + (long long)outer * a.ostride + x0 + (valid ? b : 0) + (long long)t * ss;
    const ColAddr<C, tx> addr{X + b};
    const int mode = a.mode;
    C v[NF][E];

    if (mode == SM_INV) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long long gi = g0 + (long long)reg_off<L, E, T, RoutF>(e) * ss;
#pragma unroll
            for (int f = 0; f < NF; ++f) v[f][e] = valid ? a.w[f][gi] : mk((R)0, (R)0);
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) line_fft_inv<L>(v[f], addr, a.tw, t);
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long long gi = g0 + (long long)reg_off<L, E, T, RinF>(e) * ss;
#pragma unroll
            for (int f = 0; f < NF; ++f) v[f][e] = valid ? a.w[f][gi] : mk((R)0, (R)0);
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) line_fft_fwd<L>(v[f], addr, a.tw, t);
        if (mode == SM_FWD) {
            if (valid) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const long long gi = g0 + (long long)reg_off<L, E, T, RoutF>(e) * ss;
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
                const int pos = reg_pos<L, E, T, RoutF>((int)t, e);
                C tmp[NF];
#pragma unroll
                for (int f = 0; f < NF; ++f) tmp[f] = v[f][e];
                if (valid) {
                    const int iy = (a.sax == 2) ? outer : pos;
                    const int iz = (a.sax == 2) ? pos : outer;
                    spec_point<R, NF>(a, tmp, x0 + (int)b, iy, iz, g0 + (long long)reg_off<L, E, T, RoutF>(e) * ss);
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
            const long long gi = g0 + (long long)reg_off<L, E, T, RinF>(e) * ss;
#pragma unroll
            for (int f = 0; f < NF; ++f) a.w[f][gi] = v[f][e];
        }
    }
}

template <typename R, int L, int NF, int TX, int MB>
__global__ void __launch_bounds__(TX * Plan<L>::T, MB) k_spass(PassArgs<R> a, int ntx) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pass_prologue_sync();
    spass_tile<R, L, NF, TX>(a, ntx, blockIdx.x, a.nbatch > 1 ? blockIdx.y : 0u, smem_raw);
}

// ---- paired complex64 strided pass ------------------------------------------------
// k_spass for complex64 fields with an even nx, two lines per thread
// (gpe_pair.cuh): one CTA = 2*TXP consecutive x values x the whole line for
// one outer index; thread (b, t) = (pair b of the tile, thread t of the line),
// b fast, so a quarter warp loads 8 pairs = 128 contiguous bytes of a line
// position.  Shared memory: S[pos * TXP + b], 16-byte pair slots.
// Default resident CTAs of a paired pass: spass2_mb_default (gpe_kernels.cuh).
template <int L, int NF, int TXP>
__host__ __device__ constexpr int spass2_min_blocks() {
    return spass2_mb_default(L, NF, TXP);
}

template <int NF>
__device__ __forceinline__ void spec_point2(const PassArgs<float>& a, cpair (&v)[NF], int ix, int iy, int iz,
                                            long long gi) {
    const int npsi = npsi_of<NF>(a);
    if (a.spec == SPEC_PX) {  // v * kx per lane, in FP64 as the scalar pass
        const double k0 = a.kx[ix], k1 = a.kx[ix + 1];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            v[f].x.v = make_float2((float)(v[f].x.v.x * k0), (float)(v[f].x.v.y * k1));
            v[f].y.v = make_float2((float)(v[f].y.v.x * k0), (float)(v[f].y.v.y * k1));
        }
        return;
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        if (f < npsi) {
            const double rl = a.rot[f < 2 ? f : 0];
            f2x fac;
            if (rl == 0.0) {
                // (k2x + k2y) + k2z in float, lane by lane as the scalar pass
                const f2x kxx{*reinterpret_cast<const float2*>(a.k2s[0] + ix)};
                const float ky2 = a.k2s[1][iy], kz2 = a.k2s[2][iz];
                fac = (kxx + f2x{make_float2(ky2, ky2)}) + f2x{make_float2(kz2, kz2)};
            } else {
                const double kyz = a.ky[iy] * a.ky[iy] + a.kz[iz] * a.kz[iz];
                const double k0 = a.kx[ix], k1 = a.kx[ix + 1];
                fac.v = make_float2((float)(a.lap_scale * (k0 * k0 + kyz) - k0 * rl),
                                    (float)(a.lap_scale * (k1 * k1 + kyz) - k1 * rl));
            }
            v[f].x = v[f].x * fac;
            v[f].y = v[f].y * fac;
        } else {
            const f2x d{*reinterpret_cast<const float2*>(a.vdd + gi)};
            v[f].x = v[f].x * d;
            v[f].y = v[f].y * d;
        }
    }
}

// One tile of a paired strided pass (tile = outer * ntx + x block) of
// instance inst, after the wait on the previous grid; k_spass2 runs one tile
// per CTA, the persistent RK4 step kernel (gpe_flow.cuh) runs many.
template <int L, int NF, int TXP, int PV>
__device__ __forceinline__ void spass2_tile(const PassArgs<float>& a, int ntx, unsigned tile, unsigned inst,
                                            unsigned char* smem_raw) {
    typedef Plan<L, PV> PL;
    constexpr int E = PL::E;
    constexpr int T = PL::T;
    constexpr int RinF = PL::in_radix(false);
    constexpr int RoutF = PL::out_radix(false);
    const InstPtr ip = select_instance_at(a, inst);
    const long long boff = ip.boff;
    if (a.check_done && ip.sc->done) return;

    cpair* X = reinterpret_cast<cpair*>(smem_raw);
    const int xb = (int)tile % ntx, outer = (int)tile / ntx;
    const int x0 = xb * (2 * TXP);
    const unsigned b = threadIdx.x % TXP, t = threadIdx.x / TXP;
    const int xa = x0 + 2 * (int)b;
    const bool valid = xa < a.nx;  // nx is even: a pair is whole or absent
    const long long ss = a.sstride;
    // g0 + reg_off(e) * ss: global index of the first value of register e's pair
    const long long g0 = boff + (long long)outer * a.ostride + (valid ? xa : x0) + (long long)t * ss;
    const ColAddr<cpair, TXP> addr{X + b};
    const float4* tw = a.tw2;
    const int mode = a.mode;
    cpair v[NF][E];
    const cpair zero{f2x{make_float2(0.f, 0.f)}, f2x{make_float2(0.f, 0.f)}};

    if (mode == SM_INV) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long long gi = g0 + (long long)reg_off<L, E, T, RoutF>(e) * ss;
#pragma unroll
            for (int f = 0; f < NF; ++f)
                v[f][e] = valid ? pair_from(*reinterpret_cast<const float4*>(a.w[f] + gi)) : zero;
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) line_fft_inv<L, PV>(v[f], addr, tw, t);
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long long gi = g0 + (long long)reg_off<L, E, T, RinF>(e) * ss;
#pragma unroll
            for (int f = 0; f < NF; ++f)
                v[f][e] = valid ? pair_from(*reinterpret_cast<const float4*>(a.w[f] + gi)) : zero;
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) line_fft_fwd<L, PV>(v[f], addr, tw, t);
        if (mode == SM_FWD) {
            if (valid) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const long long gi = g0 + (long long)reg_off<L, E, T, RoutF>(e) * ss;
#pragma unroll
                    for (int f = 0; f < NF; ++f) *reinterpret_cast<float4*>(a.w[f] + gi) = pair_to(v[f][e]);
                }
            }
            return;
        }
        if (a.spec != SPEC_NONE) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int pos = reg_pos<L, E, T, RoutF>((int)t, e);
                cpair tmp[NF];
#pragma unroll
                for (int f = 0; f < NF; ++f) tmp[f] = v[f][e];
                if (valid) {
                    const int iy = (a.sax == 2) ? outer : pos;
                    const int iz = (a.sax == 2) ? pos : outer;
                    spec_point2<NF>(a, tmp, xa, iy, iz, g0 + (long long)reg_off<L, E, T, RoutF>(e) * ss);
                }
#pragma unroll
                for (int f = 0; f < NF; ++f) v[f][e] = tmp[f];
            }
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) line_fft_inv<L, PV>(v[f], addr, tw, t);
    }
    if (valid) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const long long gi = g0 + (long long)reg_off<L, E, T, RinF>(e) * ss;
#pragma unroll
            for (int f = 0; f < NF; ++f) *reinterpret_cast<float4*>(a.w[f] + gi) = pair_to(v[f][e]);
        }
    }
}

template <int L, int NF, int TXP, int MB, int PV>
__global__ void __launch_bounds__(TXP * Plan<L, PV>::T, MB) k_spass2(PassArgs<float> a, int ntx) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pass_prologue_sync();
    spass2_tile<L, NF, TXP, PV>(a, ntx, blockIdx.x, a.nbatch > 1 ? blockIdx.y : 0u, smem_raw);
}

// ---- launchers ----------------------------------------------------------------------
// rows: rows per CTA (x pass); smem: exchange buffer bytes; both chosen by the host.
// Launch with programmatic stream serialization (see pass_prologue_sync).
template <typename K, typename... Args>
cudaError_t launch_pass(K kernel, unsigned grid, unsigned nbatch, unsigned threads, size_t smem, cudaStream_t st,
                        Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid, nbatch);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Exchange buffers above the default 48 KB (short lines with E = 12..24
// values per thread and 256 rows, complex128) need the opt-in attribute.  The
// attribute belongs to one device, so it is recorded per device (bit d of
// done_mask, devices 0..63; others set it on every launch), and the mask is
// atomic because distinct handles may launch from different host threads.
// The opt-in is needed once dynamic + static shared memory passes 48 KB; the
// pass kernels' static arrays are a few KB, so it is made from 32 KB of
// dynamic memory on.
template <typename K>
cudaError_t allow_smem(K kernel, size_t smem, std::atomic<unsigned long long>& done_mask) {
    if (smem <= 32 * 1024) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
    if (bit && (done_mask.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    if (e == cudaSuccess && bit) done_mask.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

template <typename R, int L, int NF, int KIND, class H = BuiltinHam>
cudaError_t launch_xpass_kind(const PassArgs<R>& a, int rows, size_t smem, cudaStream_t st) {
    static std::atomic<unsigned long long> attr{0};
    cudaError_t e = allow_smem(k_xpass<R, L, NF, KIND, H>, smem, attr);
    if (e != cudaSuccess) return e;
    const int threads = rows * Plan<L>::T;
    const int grid = (a.nrows + rows - 1) / rows;
    return launch_pass(k_xpass<R, L, NF, KIND, H>, (unsigned)grid, (unsigned)a.nbatch, (unsigned)threads, smem, st, a,
                       rows);
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
        case EPI_ADJ: return XK_ADJ;
        default: return XK_AH;
    }
}

// H: the Hamiltonian policy (BuiltinHam for the library's plugins; a user
// plugin instantiates UserHam<U>, which has no adjoint role).
template <typename R, int L, int NF, class H = BuiltinHam>
cudaError_t launch_xpass(const PassArgs<R>& a, int rows, size_t smem, cudaStream_t st) {
    int kind = xkind_of(a.mode, a.epi);
    if (kind == XK_RK && a.want_obs && a.stage == 4) kind = XK_RKO;
    else if (kind == XK_RK && a.fuse_fwd) kind = XK_RKF;
    else if (kind == XK_RKI && a.fuse_fwd) kind = XK_RKIF;
    if constexpr (NF == 1 && sizeof(R) == 4 && H::builtin) {
        if (kind == XK_RKF && a.xstage) {  // staged epilogue inputs: exchange rows + the staging slots
            const int threads = rows * Plan<L>::T;
            const int nfs = a.stage == 1 ? 2 : ((a.stage == 4 && a.lo[0] != nullptr) ? 5 : 4);
            const size_t sm = xstage_offset<float2>(rows, L) + (size_t)nfs * Plan<L>::E * threads * sizeof(float2);
            return launch_xpass_kind<R, L, NF, XK_RKS, H>(a, rows, sm, st);
        }
    }
    if (kind == XK_ADJ) {
        if constexpr (NF <= 2 && H::builtin) return launch_xpass_kind<R, L, NF, XK_ADJ, H>(a, rows, smem, st);
        return cudaErrorNotSupported;
    }
    switch (kind) {
        case XK_FWD: return launch_xpass_kind<R, L, NF, XK_FWD, H>(a, rows, smem, st);
        case XK_STORE: return launch_xpass_kind<R, L, NF, XK_STORE, H>(a, rows, smem, st);
        case XK_RK: return launch_xpass_kind<R, L, NF, XK_RK, H>(a, rows, smem, st);
        case XK_RKO: return launch_xpass_kind<R, L, NF, XK_RKO, H>(a, rows, smem, st);
        case XK_RKF: return launch_xpass_kind<R, L, NF, XK_RKF, H>(a, rows, smem, st);
        case XK_HB: return launch_xpass_kind<R, L, NF, XK_HB, H>(a, rows, smem, st);
        case XK_RKI: return launch_xpass_kind<R, L, NF, XK_RKI, H>(a, rows, smem, st);
        case XK_RKIF: return launch_xpass_kind<R, L, NF, XK_RKIF, H>(a, rows, smem, st);
        case XK_AH: return launch_xpass_kind<R, L, NF, XK_AH, H>(a, rows, smem, st);
        default: return launch_xpass_kind<R, L, NF, XK_FULL, H>(a, rows, smem, st);
    }
}

// smem is recomputed here from the tile (the host passes the default's size).
template <typename R, int L, int NF, int TX = spass_tx(L, (int)sizeof(typename Cx<R>::T)),
          int MB = spass_min_blocks<R, L, NF>()>
cudaError_t launch_spass(const PassArgs<R>& a, int nouter, size_t /*smem*/, cudaStream_t st) {
    static std::atomic<unsigned long long> attr{0};
    const size_t smem = (size_t)L * TX * sizeof(typename Cx<R>::T);
    cudaError_t e = allow_smem(k_spass<R, L, NF, TX, MB>, smem, attr);
    if (e != cudaSuccess) return e;
    const int threads = TX * Plan<L>::T;
    const int ntx = (a.nx + TX - 1) / TX;
    return launch_pass(k_spass<R, L, NF, TX, MB>, (unsigned)(ntx * nouter), (unsigned)a.nbatch, (unsigned)threads,
                       smem, st, a, ntx);
}

template <int L, int NF, int TXP = spass2_txp(L), int MB = spass2_min_blocks<L, NF, TXP>(), int PV = 0>
cudaError_t launch_spass2(const PassArgs<float>& a, int nouter, size_t /*smem*/, cudaStream_t st) {
    static std::atomic<unsigned long long> attr{0};
    const size_t smem = (size_t)L * TXP * sizeof(float4);
    cudaError_t e = allow_smem(k_spass2<L, NF, TXP, MB, PV>, smem, attr);
    if (e != cudaSuccess) return e;
    const int threads = TXP * Plan<L, PV>::T;
    const int ntx = (a.nx + 2 * TXP - 1) / (2 * TXP);
    return launch_pass(k_spass2<L, NF, TXP, MB, PV>, (unsigned)(ntx * nouter), (unsigned)a.nbatch,
                       (unsigned)threads, smem, st, a, ntx);
}

// Strided-pass variant V of length L, one field (svar in gpe_kernels.cuh).
// *found is false when the variant does not exist for this length/precision.
template <typename R, int L, int V>
cudaError_t launch_svar_v(const PassArgs<R>& a, int nouter, cudaStream_t st, bool* found) {
    constexpr SVar s = svar((int)sizeof(typename Cx<R>::T), L, V);
    if constexpr (!s.ok) {
        *found = false;
        return cudaSuccess;
    } else if constexpr (s.paired) {
        if constexpr (sizeof(R) == 4) {
            return launch_spass2<L, 1, s.tile, s.mb, s.pv>(a, nouter, 0, st);
        } else {
            *found = false;
            return cudaSuccess;
        }
    } else {
        return launch_spass<R, L, 1, s.tile, s.mb>(a, nouter, 0, st);
    }
}
template <typename R, int L>
cudaError_t launch_svar(int v, const PassArgs<R>& a, int nouter, cudaStream_t st, bool* found) {
    *found = true;
    switch (v) {
        case 0: return launch_svar_v<R, L, 0>(a, nouter, st, found);
        case 1: return launch_svar_v<R, L, 1>(a, nouter, st, found);
        case 2: return launch_svar_v<R, L, 2>(a, nouter, st, found);
        case 3: return launch_svar_v<R, L, 3>(a, nouter, st, found);
        case 4: return launch_svar_v<R, L, 4>(a, nouter, st, found);
        case 5: return launch_svar_v<R, L, 5>(a, nouter, st, found);
        case 6: return launch_svar_v<R, L, 6>(a, nouter, st, found);
        case 7: return launch_svar_v<R, L, 7>(a, nouter, st, found);
        case 8: return launch_svar_v<R, L, 8>(a, nouter, st, found);
        case 9: return launch_svar_v<R, L, 9>(a, nouter, st, found);
        case 10: return launch_svar_v<R, L, 10>(a, nouter, st, found);
        case 11: return launch_svar_v<R, L, 11>(a, nouter, st, found);
        default: *found = false; return cudaSuccess;
    }
}
static_assert(NSVAR == 12, "launch_svar lists every variant");

// Threads per line for a length (host side).
inline int plan_threads(int L) { return L / make_plan(L).E; }

}  // namespace gpe
