// gpe_fft.cuh -- register/shared-memory Stockham FFT for one grid line.
//
// Replaces the cuFFT Z2Z transforms of the reference (src/parallel.cu:77-110,
// src/baseHamiltonian.cu:89,95).  A line of length L is split over T = L/E
// threads that each hold E values in registers.  Pass p with radix R does E/R
// radix-R butterflies per thread (Stockham autosort: read stride L/R, twiddle
// exp(-+2 pi i r k/(Ns R)), write to (j/Ns)*Ns*R + j%Ns + r*Ns), exchanging
// through shared memory between passes only.  The first pass reads its
// inputs straight from global memory and the last pass leaves its outputs in
// registers, so a fused forward -> k-space multiply -> inverse needs no shared
// memory round trip in the middle (the inverse runs the radices reversed).
//
// Register position convention: after a pass of radix Rr, register e = q*Rr + r
// holds the value at line position t + q*T + r*(L/Rr).
#pragma once

#include "gpe_common.cuh"

namespace gpe {

struct PlanSpec {
    int M;       // number of passes
    int R[12];   // radices in forward order
    int E;       // values per thread
    int ok;      // 1 when the length has a plan
};

__host__ __device__ constexpr int gcd_c(int a, int b) { return b == 0 ? a : gcd_c(b, a % b); }
__host__ __device__ constexpr int lcm_c(int a, int b) { return a / gcd_c(a, b) * b; }

// Plan: powers of two use radix 8 with one trailing 4 or 2 (E = 8); lengths
// with factors 3 or 5 use radix 4 (and one 2) for the power-of-two part so that
// E = lcm(radices) stays <= 24.  pv selects an alternative radix order for the
// autotuner (same radices or smaller ones, other placement):
//   powers of two: 1 = the 4 or 2 first, then the 8s; 2 = radix 4s (and one
//                  trailing 2: E = 4);
//   mixed:         1 = the 3s and 5s first; 2 = the 2 first, then 4s, 3s, 5s.
// A variant that gives no plan (or the default's order) has ok = 0.
__host__ __device__ constexpr PlanSpec make_plan(int L, int pv = 0) {
    PlanSpec p{0, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}, 1, 0};
    if (L < 1 || pv < 0 || pv > 2) return p;
    if (L == 1) {
        p.ok = pv == 0 ? 1 : 0;
        p.E = 1;
        return p;
    }
    int m = L, p2 = 0, n3 = 0, n5 = 0;
    while (m % 2 == 0) { m /= 2; ++p2; }
    while (m % 3 == 0) { m /= 3; ++n3; }
    while (m % 5 == 0) { m /= 5; ++n5; }
    if (m != 1) return p;
    if (n3 == 0 && n5 == 0) {
        if (pv == 2) {
            if (p2 < 3) return p;
            while (p2 >= 2) { p.R[p.M++] = 4; p2 -= 2; }
            if (p2 == 1) p.R[p.M++] = 2;
        } else {
            const int lead = p2 % 3;  // the 4 or 2
            if (pv == 1) {
                if (lead == 0 || p2 < 3) return p;
                p.R[p.M++] = lead == 2 ? 4 : 2;
            }
            while (p2 >= 3) { p.R[p.M++] = 8; p2 -= 3; }
            if (pv == 0) {
                if (p2 == 2) p.R[p.M++] = 4;
                if (p2 == 1) p.R[p.M++] = 2;
            }
        }
    } else {
        const bool two = p2 % 2 == 1;
        if (pv == 1) {
            if (p2 == 0) return p;
            for (int i = 0; i < n3; ++i) p.R[p.M++] = 3;
            for (int i = 0; i < n5; ++i) p.R[p.M++] = 5;
        }
        if (pv == 2) {
            if (!two || p2 < 3) return p;
            p.R[p.M++] = 2;
        }
        while (p2 >= 2) { p.R[p.M++] = 4; p2 -= 2; }
        if (pv != 2 && p2 == 1) p.R[p.M++] = 2;
        if (pv != 1) {
            for (int i = 0; i < n3; ++i) p.R[p.M++] = 3;
            for (int i = 0; i < n5; ++i) p.R[p.M++] = 5;
        }
    }
    if (p.M > 12) return p;
    int e = 1;
    for (int i = 0; i < p.M; ++i) e = lcm_c(e, p.R[i]);
    if (e > 24 || L % e != 0) return p;
    p.E = e;
    p.ok = 1;
    return p;
}

template <int L, int PV = 0>
struct Plan {
    static constexpr PlanSpec spec = make_plan(L, PV);
    static_assert(spec.ok, "FFT length has no plan");
    static constexpr int M = spec.M;
    static constexpr int E = spec.E;
    static constexpr int T = L / spec.E;
    __host__ __device__ static constexpr int radix(int p, bool rev) { return rev ? spec.R[M - 1 - p] : spec.R[p]; }
    __host__ __device__ static constexpr int ns(int p, bool rev) {
        int s = 1;
        for (int i = 0; i < p; ++i) s *= radix(i, rev);
        return s;
    }
    // Radix whose position pattern the registers follow before pass 0 / after the last pass.
    __host__ __device__ static constexpr int in_radix(bool rev) { return M == 0 ? 1 : radix(0, rev); }
    __host__ __device__ static constexpr int out_radix(bool rev) { return M == 0 ? 1 : radix(M - 1, rev); }
};

// Line position of register e for a pattern of radix Rr: t + reg_off(e).
template <int L, int E, int T, int Rr>
__host__ __device__ constexpr int reg_off(int e) {
    return (e / Rr) * T + (e % Rr) * (L / Rr);
}
template <int L, int E, int T, int Rr>
__device__ __forceinline__ int reg_pos(int t, int e) {
    return t + reg_off<L, E, T, Rr>(e);
}

// Real component type of a complex type C (float / double; the paired
// complex64 type of gpe_pair.cuh specialises it to float), and the type its
// twiddle table holds (C itself here; a broadcast pair for the paired type).
template <typename C> struct RealOf { typedef decltype(C().x) T; };
template <typename C> struct TwOf { typedef C T; };

// ---- small DFTs, X_q = sum_r x_r exp(SIGN 2 pi i r q / R) ------------------
// i*SIGN*b
template <int SIGN, typename C> __device__ __forceinline__ C rot_i(C b) {
    return (SIGN < 0) ? mk(b.y, -b.x) : mk(-b.y, b.x);
}

template <int R, int SIGN, typename C> struct Butterfly;

template <int SIGN, typename C> struct Butterfly<2, SIGN, C> {
    __device__ __forceinline__ static void run(C* v) {
        C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <int SIGN, typename C> struct Butterfly<4, SIGN, C> {
    __device__ __forceinline__ static void run(C* v) {
        C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        C b0 = cadd(v[1], v[3]), b1 = rot_i<SIGN>(csub(v[1], v[3]));
        v[0] = cadd(a0, b0);
        v[2] = csub(a0, b0);
        v[1] = cadd(a1, b1);
        v[3] = csub(a1, b1);
    }
};

template <int SIGN, typename C> struct Butterfly<8, SIGN, C> {
    __device__ __forceinline__ static void run(C* v) {
        typedef typename RealOf<C>::T R;
        const R h = (R)0.70710678118654752440084436210484903928;  // 1/sqrt(2)
        C e[4] = {v[0], v[2], v[4], v[6]};
        C o[4] = {v[1], v[3], v[5], v[7]};
        Butterfly<4, SIGN, C>::run(e);
        Butterfly<4, SIGN, C>::run(o);
        // w8^q o[q], w8 = exp(SIGN i pi/4)
        C o1 = (SIGN < 0) ? mk(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x))
                          : mk(h * (o[1].x - o[1].y), h * (o[1].y + o[1].x));
        C o2 = rot_i<SIGN>(o[2]);
        C o3 = (SIGN < 0) ? mk(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y))
                          : mk(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y));
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);
        v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);
        v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);
        v[7] = csub(e[3], o3);
    }
};

template <int SIGN, typename C> struct Butterfly<3, SIGN, C> {
    __device__ __forceinline__ static void run(C* v) {
        typedef typename RealOf<C>::T R;
        const R s3 = (R)0.86602540378443864676372317075293618;  // sin(2 pi/3)
        C t1 = cadd(v[1], v[2]);
        C t2 = mk(v[0].x - (R)0.5 * t1.x, v[0].y - (R)0.5 * t1.y);
        C d = csub(v[1], v[2]);
        C it = rot_i<SIGN>(mk(s3 * d.x, s3 * d.y));
        v[0] = cadd(v[0], t1);
        v[1] = cadd(t2, it);
        v[2] = csub(t2, it);
    }
};

template <int SIGN, typename C> struct Butterfly<5, SIGN, C> {
    __device__ __forceinline__ static void run(C* v) {
        typedef typename RealOf<C>::T R;
        const R c1 = (R)0.30901699437494742410229341718281906;   // cos(2 pi/5)
        const R c2 = (R)-0.80901699437494742410229341718281906;  // cos(4 pi/5)
        const R s1 = (R)0.95105651629515357211643933337938214;   // sin(2 pi/5)
        const R s2 = (R)0.58778525229247312916870595463907277;   // sin(4 pi/5)
        C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        C t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        C a1 = mk(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
        C a2 = mk(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
        C b1 = rot_i<SIGN>(mk(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
        C b2 = rot_i<SIGN>(mk(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
        v[0] = mk(v[0].x + t1.x + t2.x, v[0].y + t1.y + t2.y);
        v[1] = cadd(a1, b1);
        v[4] = csub(a1, b1);
        v[2] = cadd(a2, b2);
        v[3] = csub(a2, b2);
    }
};

// ---- Stockham passes ---------------------------------------------------------
// Addr: functor, C* operator()(int pos) -> shared-memory slot of line position pos.
// tw: forward roots of unity exp(-2 pi i m/L), m in [0, L).
// Index arithmetic is unsigned so that (t + q*T) / Ns and % Ns split into a
// per-thread part and a compile-time part whenever T is a multiple of Ns.
template <int L, int P, int SIGN, bool REV, int PV, typename C, typename Addr>
__device__ __forceinline__ void fft_passes(C (&v)[Plan<L, PV>::E], const Addr& addr,
                                           const typename TwOf<C>::T* __restrict__ tw, unsigned t) {
    typedef Plan<L, PV> PL;
    constexpr int M = PL::M;
    if constexpr (P < M) {
        constexpr int R = PL::radix(P, REV);
        constexpr int Ns = PL::ns(P, REV);
        constexpr int E = PL::E;
        constexpr int T = PL::T;
        constexpr int G = E / R;
        if constexpr (P > 0) {
#pragma unroll
            for (int q = 0; q < G; ++q)
#pragma unroll
                for (int r = 0; r < R; ++r) v[q * R + r] = *addr(t + (unsigned)(q * T + r * (L / R)));
        }
#pragma unroll
        for (int q = 0; q < G; ++q) {
            if constexpr (Ns > 1) {
                const unsigned j = t + (unsigned)(q * T);
                const unsigned k = j % (unsigned)Ns;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    const typename TwOf<C>::T w = __ldg(tw + (unsigned)r * k * (unsigned)(L / (Ns * R)));
                    v[q * R + r] = (SIGN < 0) ? cmul(v[q * R + r], w) : cmulc(v[q * R + r], w);
                }
            }
            Butterfly<R, SIGN, C>::run(&v[q * R]);
        }
        if constexpr (P < M - 1) {
            __syncthreads();
#pragma unroll
            for (int q = 0; q < G; ++q) {
                const unsigned j = t + (unsigned)(q * T);
                const unsigned k = j % (unsigned)Ns;
                const unsigned idxD = (j / (unsigned)Ns) * (unsigned)(Ns * R) + k;
#pragma unroll
                for (int r = 0; r < R; ++r) *addr(idxD + (unsigned)(r * Ns)) = v[q * R + r];
            }
            __syncthreads();
            fft_passes<L, P + 1, SIGN, REV, PV>(v, addr, tw, t);
        }
    }
}

// Forward transform: registers in in_radix(false) pattern -> out_radix(false) pattern.
template <int L, int PV = 0, typename C, typename Addr>
__device__ __forceinline__ void line_fft_fwd(C (&v)[Plan<L, PV>::E], const Addr& addr,
                                             const typename TwOf<C>::T* __restrict__ tw, unsigned t) {
    fft_passes<L, 0, -1, false, PV>(v, addr, tw, t);
}
// Inverse (unnormalised) transform with the radices reversed:
// registers in in_radix(true) == out_radix(false) pattern -> out_radix(true) == in_radix(false).
template <int L, int PV = 0, typename C, typename Addr>
__device__ __forceinline__ void line_fft_inv(C (&v)[Plan<L, PV>::E], const Addr& addr,
                                             const typename TwOf<C>::T* __restrict__ tw, unsigned t) {
    fft_passes<L, 0, +1, true, PV>(v, addr, tw, t);
}

}  // namespace gpe
