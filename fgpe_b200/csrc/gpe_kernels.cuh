// gpe_kernels.cuh -- fused axis-pass kernels of the GPE step.
//
// One stage of the reference's RK4 step is cuFFT-forward -> Laplace ->
// cuFFT-inverse -> plugin pointwise kernel -> 1..2 stage kernels
// (src/oneComponentGPSolver.cu:170-187, src/baseHamiltonian.cu:86-96).  Here a
// stage is a chain of axis passes over the 3D field (x fastest):
//
//   X_FWD  rows along x: prologue (stage state, lazy renormalisation,
//          dipolar density) + forward x-FFT                      -> W
//   S_FWD  strided lines (y) forward                               W -> W
//   S_FKI  last strided axis: forward FFT, k-space multiply (kinetic
//          2 pi^2 k^2/N, dipolar V(k)/N), inverse FFT              W -> W
//   S_INV  strided lines inverse                                   W -> W
//   X_INV  rows along x: inverse x-FFT + epilogue (Hamiltonian plugin
//          term, RK4 / heavy-ball stage arithmetic, FP64 compensated
//          reductions with a last-block device finalize)
//
// and X_FULL does all of it in one kernel when x is the only axis.
#pragma once

#include "gpe_common.cuh"
#include "gpe_fft.cuh"
#include "gpe_pair.cuh"
#include "../../include/gpe.h"

namespace gpe {

enum PassMode { XM_FWD = 0, XM_INV = 1, XM_FULL = 2, SM_FWD = 3, SM_INV = 4, SM_FKI = 5 };
// Prologue / epilogue psi source.
enum ProOp {
    PRO_PIN = 0,      // psi = pin[c]
    PRO_CUR = 1,      // psi = scale[cur][c] * buf[cur][c]        (heavy ball)
    PRO_A_SCALED = 2  // psi = scale[cur][c] * buf[0][c]          (RK4 imaginary, stage 1)
};
enum EpiOp {
    EPI_STORE = 0,   // W <- inverse transform (gpe_fft, gpe_laplace)
    EPI_RK = 1,      // real-time RK4 stage
    EPI_HB = 2,      // heavy-ball imaginary step + renormalisation reductions
    EPI_APPLYH = 3,  // out <- h_mu, h_en
    EPI_OBS = 4,     // reductions of |psi|^2, Re(psi* h_mu), Re(psi* h_en)
    EPI_RKI = 5,     // imaginary-time RK4 stage
    EPI_ADJ = 6      // adjoint of one real-time RK4 stage (control gradient)
};
enum SpecOp { SPEC_NONE = 0, SPEC_KIN = 1, SPEC_PX = 2 };
// Compile-time role of an x-pass kernel: forward only, inverse + one epilogue
// family, or the x-only full pass (run-time epilogue).  Specialising keeps the
// register count and code size of each kernel to what its role needs.
// XK_RK runs the real-time stages without reductions (the hot path); XK_RKO
// is the same stage with the logging reductions of the last step of a chunk;
// XK_RKF is XK_RK followed by the forward x transform of the state it just
// wrote, which is the x-forward pass of the next stage.
// XK_ADJ is the adjoint stage epilogue of the control gradient.
// XK_RKS is XK_RKF with the epilogue inputs staged: every thread copies the
// values its epilogue will read (V, the stage state, the accumulator, psi0,
// the low part) into its own shared-memory slots with asynchronous copies at
// kernel start, before the wait on the previous pass, so that they are in
// flight during the inverse transform (complex64, one field).
// XK_RKIF is XK_RKI (imaginary-time RK4 stage) followed by the forward x
// transform of the stage state it wrote (stages 1-3: the next stage's
// x-forward pass, as XK_RKF does in real time).
enum XKind { XK_FWD = 0, XK_STORE = 1, XK_RK = 2, XK_HB = 3, XK_RKI = 4, XK_AH = 5, XK_FULL = 6, XK_RKO = 7,
             XK_RKF = 8, XK_ADJ = 9, XK_RKS = 10, XK_RKIF = 11 };
constexpr int NXKIND = 12;  // SPEC_PX: BECVPx, src/parallel.cu:283-292

constexpr int MAXQ = 6;       // reduced quantities per launch (3 per component)
template <typename R>
struct PassArgs {
    typedef typename Cx<R>::T C;
    int nx, ny, nz;
    int nrows;               // X pass: rows = ny*nz
    int ncomp;               // 1 or 2
    int dens;                // 1: field index ncomp is the dipolar density
    int tx;                  // strided pass: lines (x values) per CTA, spass_tx(L, sizeof(C))
    int mode, pro, epi, spec, stage, ham, sax;
    int check_done;          // exit when sc->done is set (stepping chunks)
    int want_obs;            // RK stage 4: logging reductions
    int fuse_fwd;            // RK epilogue: also x-forward transform the new state into w
    int xstage;              // complex64 fused RK epilogue: stage its inputs (XK_RKS)
    // Batched instances (gpe_batch): blockIdx.y selects the instance; its
    // fields sit bstride elements apart, its d_h_params, scalars and partial
    // sums at prms + 32*inst, sc + inst, partials + pstride*inst.
    int nbatch;              // 1 for a single handle
    long long bstride;
    long long pstride;
    C* w[3];                 // transformed fields (work buffers)
    C* buf[2][2];            // [slot][comp] state buffers (A = slot 0, B = slot 1)
    C* kacc[2];              // RK accumulators
    C* lo[2];                // complex64 real-time RK4: low part of the step state (buf[0] = high part) or null
    const C* pin[2];         // PRO_PIN source
    const C* vext[2];
    C* out[4];               // EPI_APPLYH: h_mu c0, h_en c0, h_mu c1, h_en c1
    const C* tw;             // roots of unity for this pass's length
    const float4* tw2;       // complex64: the same roots as (cos, cos, sin, sin) for the paired passes
    const C* twz;            // fused y-z kernel: roots of unity of the z length (tw holds y's)
    const double* kx;
    const double* ky;
    const double* kz;
    const float* k2s[3];     // complex64: lap_scale * k^2 per axis, rounded to float (null for complex128)
    const R* vdd;            // dipolar kernel / N (spectral order) or null
    const double* prms;      // d_h_params
    DevScalars* sc;
    double* partials;        // [CTA][MAXQ][2] (at least ny*nz CTAs)
    long long sstride;       // strided pass: element stride along the line
    long long ostride;       // strided pass: stride of the outer index
    double t;                // Hamiltonian time (BEC quench)
    double dt, beta, lap_scale, DV, eps;
    double npart[2];
    double c_re, c_im;       // RK stage coefficient (stage 1..3 axpy; final uses c/6)
    double rot[2];           // moving-frame term: lambda/N per component, 0 = off
};

// Strided pass tile width: x values per CTA, the largest power of two up to
// 128 bytes of a row (16 complex64 / 8 complex128 values) whose CTA of
// tx * T threads stays within 256 threads.  A compile-time constant of the
// kernel, so that the shared-memory column addressing folds into offsets.
__host__ __device__ constexpr int spass_tx(int L, int esz) {
    const int T = L / make_plan(L).E;
    int tx = 128 / esz;
    while (tx > 1 && tx * T > 256) tx /= 2;
    return tx;
}

// Paired complex64 strided pass (k_spass2) tile, in pairs of x values.
// Default tile: up to 16 pairs (32 x values, 256 bytes of a row) in a CTA of
// at most 128 threads (8 pairs = 128 bytes for lines of 16 threads, 4 pairs
// for 32).
__host__ __device__ constexpr int spass2_txp(int L) {
    const int T = L / make_plan(L).E;
    int txp = 16;
    while (txp > 1 && txp * T > 128) txp /= 2;
    return txp;
}

// ---- strided-pass variants (the autotuner's search space) --------------------
// A variant fixes the implementation of a one-field strided pass (scalar
// lines, k_spass, or paired complex64 lines, k_spass2), its tile width (x
// values, or pairs of x values, per CTA) and the resident CTAs per SM its
// launch bounds ask for (which sets the register budget).  Variant 0 is the
// default of each precision; the others exist for the tuned lengths
// (GPE_TUNED_*) only and are picked per (grid, axis, pass mode) by
// gpe_tune.  The CTA count of a pass against the SM's resident slots decides
// how full its last wave is, so tile and occupancy are searched together.
struct SVar {
    int ok;      // 1 when the variant exists for this length and precision
    int paired;  // 1: k_spass2 (complex64 only)
    int tile;    // TX (scalar) or TXP (paired)
    int mb;      // __launch_bounds__ min blocks
    int pv;      // radix-order variant of the line FFT (make_plan), paired passes
};
constexpr int NSVAR = 12;

// Default resident CTAs of the scalar strided pass (as pass_min_blocks /
// spass_min_blocks in gpe_kernels_impl.cuh): words of line values per thread.
__host__ __device__ constexpr int spass_mb_default(int esz, int L, int NF) {
    const int w = esz / 8 * make_plan(L).E * NF;  // esz 8 (complex64) or 16 (complex128)
    const int pm = w <= 8 ? 3 : (w <= 16 ? 2 : 1);
    return pm == 3 ? 5 : pm;
}
// Default resident CTAs of the paired pass (register budget: the pair values
// plus 48, or 64 for plans with 12 or more values per thread).
__host__ __device__ constexpr int spass2_mb_default(int L, int NF, int txp, int pv = 0) {
    const int E = make_plan(L, pv).E;
    const int regs0 = E * 4 * NF + (E > 8 ? 64 : 48);
    const int regs = regs0 < 64 ? 64 : regs0;
    const int threads = (txp * (L / E) + 31) / 32 * 32;
    const int b = 65536 / (threads * regs);
    const int bw = 2048 / threads;
    return b < 1 ? 1 : (b > bw ? bw : (b > 32 ? 32 : b));
}
__host__ __device__ constexpr SVar svar_make(int esz, int L, int paired, int tile, int mb, int pv = 0) {
    const PlanSpec ps = make_plan(L, pv);
    const int T = ps.ok ? L / ps.E : 0;
    const int threads = tile * T;
    const int wthreads = (threads + 31) / 32 * 32;
    const bool ok = ps.ok && tile >= 1 && mb >= 1 && mb <= 32 && threads >= 1 &&
                    threads <= (paired ? 512 : 256) && wthreads * mb <= 2048 && (!paired || esz == 8) &&
                    (pv == 0 || paired) && 65536 / (wthreads * mb) >= 32;
    return SVar{ok ? 1 : 0, paired, tile, mb, pv};
}
// esz: bytes per complex value (8: complex64, 16: complex128); NF = 1.
__host__ __device__ constexpr SVar svar(int esz, int L, int v) {
    const int tx = spass_tx(L, esz);
    const int mb0 = spass_mb_default(esz, L, 1);
    if (v == 0) return SVar{make_plan(L).ok ? 1 : 0, 0, tx, mb0, 0};
    if (esz == 8) {
        const int tp = spass2_txp(L);
        switch (v) {
            case 1: return svar_make(8, L, 1, tp, spass2_mb_default(L, 1, tp));
            case 2: return svar_make(8, L, 1, tp, spass2_mb_default(L, 1, tp) + 1);
            case 3: return svar_make(8, L, 1, tp, spass2_mb_default(L, 1, tp) + 2);
            case 4: return svar_make(8, L, 1, tp / 2, spass2_mb_default(L, 1, tp / 2));
            case 5: return svar_make(8, L, 1, tp / 2, spass2_mb_default(L, 1, tp / 2) + 2);
            case 6: return svar_make(8, L, 1, tp * 2, spass2_mb_default(L, 1, tp * 2));
            case 7: return svar_make(8, L, 1, tp * 2, spass2_mb_default(L, 1, tp * 2) + 1);
            case 8: return svar_make(8, L, 0, tx / 2, mb0 * 2);
            case 9: return svar_make(8, L, 0, tx, mb0 + 1);
            case 10: return svar_make(8, L, 1, tp, spass2_mb_default(L, 1, tp, 1), 1);
            case 11: return svar_make(8, L, 1, tp, spass2_mb_default(L, 1, tp, 2), 2);
            default: return SVar{0, 0, 0, 0, 0};
        }
    }
    switch (v) {
        case 1: return svar_make(16, L, 0, tx, mb0 + 1);
        case 2: return svar_make(16, L, 0, tx, mb0 + 2);
        case 3: return svar_make(16, L, 0, tx / 2, mb0 * 2);
        case 4: return svar_make(16, L, 0, tx / 2, mb0 * 2 + 2);
        case 5: return svar_make(16, L, 0, tx * 2, mb0 > 1 ? mb0 / 2 : 1);
        default: return SVar{0, 0, 0, 0, 0};
    }
}

// ---- shared-memory line addressing -----------------------------------------
// X pass exchange rows: line position pos of row b at S[b*xpad(L) + xmap(L, pos)].
// A half warp (16 lanes of 8-byte values) is one 128-byte wavefront when its
// lanes fall on distinct bank pairs.  The Stockham exchanges of a row store
// and load with strides 1, 2, 8, 16 ... (the radix-8 stores of the forward
// plan, the radix-2 stores that start the reversed inverse plan), so the map
// is chosen per length by counting the wavefronts of every exchange of both
// plans: an XOR of the low four bits with a higher bit field for the long
// powers of two and for 192/384 (no padding), a double padding for 64 and
// 96, one slot every 8 otherwise.  The map only places values; the
// arithmetic and its results do not depend on it.
__host__ __device__ constexpr int xmap(int L, int pos) {
    return (L == 128 || L == 256 || L == 512 || L == 1024) ? (pos ^ ((pos >> 3) & 15))
           : (L == 192 || L == 384)                       ? (pos ^ ((pos >> 2) & 15))
           : (L == 64)                                    ? (pos + (pos >> 3) + (pos >> 5))
           : (L == 96)                                    ? (pos + 2 * (pos >> 3) + (pos >> 5))
                                                          : (pos + (pos >> 3));
}
// Row stride: one past the largest mapped position.
__host__ __device__ constexpr int xpad(int L) {
    return (L == 128 || L == 256 || L == 512 || L == 1024 || L == 192 || L == 384) ? L
           : (L == 64 || L == 96)                                                 ? xmap(L, L - 1) + 1
                                                                                  : L + (L >> 3);
}
template <typename C, int L> struct RowAddr {  // X pass: S[b*xpad(L) + xmap(L, pos)]
    C* base;
    __device__ __forceinline__ C* operator()(unsigned pos) const { return base + xmap(L, (int)pos); }
};
template <typename C, int TX> struct ColAddr {  // strided pass: S[pos*TX + b]
    C* base;
    __device__ __forceinline__ C* operator()(unsigned pos) const { return base + pos * (unsigned)TX; }
};

// ---- compensated FP64 reductions --------------------------------------------
struct DD {
    double s, c;
};
__device__ __forceinline__ DD dd_add(DD a, double v) {
    double t = a.s + v;
    double e = (fabs(a.s) >= fabs(v)) ? (a.s - t) + v : (v - t) + a.s;
    return DD{t, a.c + e};
}
__device__ __forceinline__ DD dd_merge(DD a, DD b) {
    DD r = dd_add(a, b.s);
    r.c += b.c;
    return r;
}

// Block-wide deterministic reduction of NQ compensated sums; result valid in
// thread 0.  red: shared scratch of 32*NQ DD.
// The last warp may be partial (line lengths with T = 3, 9, ... threads per
// line): shuffles use the mask of the lanes that exist.
template <int NQ>
__device__ __forceinline__ void block_reduce(DD (&acc)[NQ], DD* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    const int wl = min(32, (int)blockDim.x - warp * 32);
    const unsigned mask = (wl == 32) ? 0xffffffffu : ((1u << wl) - 1u);
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            DD o;
            o.s = __shfl_down_sync(mask, acc[q].s, off);
            o.c = __shfl_down_sync(mask, acc[q].c, off);
            if (lane + off < wl) acc[q] = dd_merge(acc[q], o);
        }
    }
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NQ; ++q) red[warp * NQ + q] = acc[q];
    __syncthreads();
    if (warp == 0) {
        const int wl0 = min(32, (int)blockDim.x);
        const unsigned mask0 = (wl0 == 32) ? 0xffffffffu : ((1u << wl0) - 1u);
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            DD v = (lane < nwarps) ? red[lane * NQ + q] : DD{0.0, 0.0};
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                DD o;
                o.s = __shfl_down_sync(mask0, v.s, off);
                o.c = __shfl_down_sync(mask0, v.c, off);
                if (lane + off < wl0) v = dd_merge(v, o);
            }
            acc[q] = v;
        }
    }
    __syncthreads();
}

// d_quench_as, hamiltonians/BEC_oneComponent.cu:167-178.
__device__ __forceinline__ double quench_as(double time, const double* prms) {
    double a0 = prms[0], a1 = prms[1], a2 = prms[2];
    double t1 = prms[3], t2 = prms[4], t3 = prms[5];
    if (0 < time && time <= t1) return a0 + (a1 - a0) / (t1)*time;
    if (t1 < time && time <= t2) return a1;
    if (t2 < time && time <= t3) return a1 + (a2 - a1) / (t3 - t2) * (time - t2);
    return a2;
}

// hpp/header.hpp:27 pi literal.
#define GPE_PI_REF 3.141592653589793

// Pointwise Hamiltonian term.  T = kinetic part (the reference's d_hpsi after
// alg_Laplace), psi, V, phi (dipolar mean field).  Writes h_mu and, when
// want_en, h_en.  Formulas and evaluation order follow
//  BEC     hamiltonians/BEC_oneComponent.cu:128-165
//  BEC2    hamiltonians/BEC_twoComponent.cu:168-244 (en variant keeps the
//          vext1[ix].y read of line 208 for component 2)
//  TEMPLATE hamiltonians/single_template.cu:333-373.
template <typename R>
struct HamCoef {
    R g_en, g_mu;                  // BEC: 2 pi a, 4 pi a
    R g11e, g12e, g22e, g11m, g12m, g22m;
};

// MC: largest component count the caller can have (1 when its pass carries one field).
template <typename R, typename C, int MC = 2>
__device__ __forceinline__ void ham_point(int ham, int ncomp, const HamCoef<R>& hc, const C* psi, const C* T,
                                          const C* V, R phi, bool want_en, C* hmu, C* hen) {
    if (ham == GPE_HAM_BEC || ham == GPE_HAM_DIPOLAR || ham == GPE_HAM_SOFT) {  // SOFT: g = 0
        const R px = psi[0].x, py = psi[0].y;
        const R n = px * px + py * py;
        R rX, rY;
        if (want_en) {
            rX = (V[0].x + hc.g_en * n) + (R)0.5 * phi;
            rY = V[0].y;
            hen[0] = mk(T[0].x + rX * px - rY * py, T[0].y + rX * py + rY * px);
        }
        rX = (V[0].x + hc.g_mu * n) + phi;
        rY = V[0].y;
        hmu[0] = mk(T[0].x + rX * px - rY * py, T[0].y + rX * py + rY * px);
    } else if (MC > 1 && ham == GPE_HAM_BEC2) {
        const R x1 = psi[0].x, y1 = psi[0].y, x2 = psi[1].x, y2 = psi[1].y;
        const R n1 = x1 * x1 + y1 * y1, n2 = x2 * x2 + y2 * y2;
        R aX, aY;
        if (want_en) {
            aX = (V[0].x + hc.g11e * n1 + hc.g12e * n2);
            aY = V[0].y;
            hen[0] = mk(T[0].x + aX * x1 - aY * y1, T[0].y + aX * y1 + aY * x1);
        }
        aX = (V[0].x + hc.g11m * n1 + hc.g12m * n2);
        aY = V[0].y;
        hmu[0] = mk(T[0].x + (aX * x1 - aY * y1), T[0].y + (aX * y1 + aY * x1));
        if (want_en) {
            aX = (V[1].x + hc.g22e * n2 + hc.g12e * n1);
            aY = V[1].y;
            hen[1] = mk(T[1].x + aX * x2 - aY * y2, T[1].y + aX * y2 + aY * x2);
            aX = (V[1].x + hc.g22m * n2 + hc.g12m * n1);
            aY = V[0].y;  // hamiltonians/BEC_twoComponent.cu:208
        } else {
            aX = (V[1].x + hc.g22m * n2 + hc.g12m * n1);
            aY = V[1].y;
        }
        hmu[1] = mk(T[1].x + (aX * x2 - aY * y2), T[1].y + (aX * y2 + aY * x2));
    } else {
#pragma unroll
        for (int c = 0; c < MC; ++c) {
            if (c >= ncomp) continue;
            hmu[c] = T[c];
            if (want_en) hen[c] = T[c];
        }
    }
}

template <typename R>
__device__ __forceinline__ HamCoef<R> make_coef(const PassArgs<R>& a, const double* prms) {
    HamCoef<R> hc;
    double q = (a.ham == GPE_HAM_BEC || a.ham == GPE_HAM_DIPOLAR) ? quench_as(a.t, prms) : 0.0;
    hc.g_en = (R)(2 * GPE_PI_REF * q);
    hc.g_mu = (R)(4 * GPE_PI_REF * q);
    const double a11 = prms[0], a22 = prms[1], a12 = prms[2];
    hc.g11e = (R)(2 * GPE_PI_REF * a11);
    hc.g12e = (R)(2 * GPE_PI_REF * a12);
    hc.g22e = (R)(2 * GPE_PI_REF * a22);
    hc.g11m = (R)(4 * GPE_PI_REF * a11);
    hc.g12m = (R)(4 * GPE_PI_REF * a12);
    hc.g22m = (R)(4 * GPE_PI_REF * a22);
    return hc;
}

// Exact-form helpers in FP64 for the stage arithmetic.
__device__ __forceinline__ double2 to_d(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ double2 to_d(double2 v) { return v; }
template <typename C> __device__ __forceinline__ C from_d(double2 v);
template <> __device__ __forceinline__ float2 from_d<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <> __device__ __forceinline__ double2 from_d<double2>(double2 v) { return v; }

// UpdateRKStep, complex overload (src/parallel.cu:238-244).
__device__ __forceinline__ double2 rk_axpy(double2 old, double cr, double ci, double2 h) {
    return make_double2(old.x + (cr * h.x - ci * h.y), old.y + (cr * h.y + ci * h.x));
}
// FinalRKStep (src/parallel.cu:261-271).
__device__ __forceinline__ double2 rk_final(double2 old, double cr, double ci, double2 k, double2 h) {
    double aX = k.x + h.x, aY = k.y + h.y;
    return make_double2(old.x + (cr * aX - ci * aY) / 6.0, old.y + (cr * aY + ci * aX) / 6.0);
}

// The same three stage updates in the field's own precision: the real-time
// RK4 stages of the complex64 form run in FP32 (the complex128 form is the
// FP64 arithmetic above, operation for operation).
template <typename C, typename R>
__device__ __forceinline__ C rk_axpy_r(C old, R cr, R ci, C h) {
    return mk(old.x + (cr * h.x - ci * h.y), old.y + (cr * h.y + ci * h.x));
}
// (complex64 multiplies by the rounded 1/6 instead of dividing by 6.)
template <typename C, typename R>
__device__ __forceinline__ C rk_final_r(C old, R cr, R ci, C k, C h) {
    const R aX = k.x + h.x, aY = k.y + h.y;
    if constexpr (sizeof(R) == 8) {
        return mk(old.x + (cr * aX - ci * aY) / (R)6, old.y + (cr * aY + ci * aX) / (R)6);
    } else {
        const R s = (R)(1.0 / 6.0);
        return mk(old.x + (cr * aX - ci * aY) * s, old.y + (cr * aY + ci * aX) * s);
    }
}
template <typename C>
__device__ __forceinline__ C rk_kacc_r(C k, C h) {
    return mk(k.x + 2 * h.x, k.y + 2 * h.y);
}

// Error-free sum (Knuth's TwoSum): s + e == a + b exactly, s = fl(a + b).
__device__ __forceinline__ float two_sum(float a, float b, float& e) {
    const float s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    return s;
}
// Compensated final stage of the complex64 form: the step state is carried as
// hi + lo (two float32 values per real component), and the new state
// hi + (d + lo) is split again by TwoSum.  The rounding of the stored state
// then does not accumulate over steps: rounding the state to float32 each
// step is a random walk in the norm (about 1e-7 after 10^4 steps at 128^3);
// carried this way the drift stays at the float64 RK4 level.
__device__ __forceinline__ float2 rk_final_comp(float2 hi, float2 lo, float cr, float ci, float2 k, float2 h,
                                                float2& lo_out) {
    const float aX = k.x + h.x, aY = k.y + h.y;
    const float s = (float)(1.0 / 6.0);
    const float dX = (cr * aX - ci * aY) * s, dY = (cr * aY + ci * aX) * s;
    float ex, ey;
    const float nx = two_sum(hi.x, __fadd_rn(dX, lo.x), ex);
    const float ny = two_sum(hi.y, __fadd_rn(dY, lo.y), ey);
    lo_out = make_float2(ex, ey);
    return make_float2(nx, ny);
}

// ---- last-block finalize ------------------------------------------------------
// Called by every block after its own reduction (thread 0 holds acc).

// ---- kernels ----------------------------------------------------------------

// k_xpass<R, L, NF, KIND>(PassArgs<R> a, int rows) and
// k_spass<R, L, NF>(PassArgs<R> a, int ntx): see gpe_kernels_impl.cuh.

}  // namespace gpe
