// gpe_pair.cuh -- two complex64 lines per thread, packed FP32x2 arithmetic.
//
// Blackwell (sm_100) issues FP32 add, subtract, multiply and fused
// multiply-add on a pair of floats as one instruction (add/sub/mul/fma
// .rn.f32x2).  The strided complex64 passes are bound by instruction issue
// and memory latency, not by bytes, so each thread there transforms the lines
// of two neighbouring x values at once: the two values of one line position
// arrive in one 16-byte load (x is the fastest axis), are held as a structure
// of arrays -- x = (re_a, re_b), y = (im_a, im_b) -- and every butterfly,
// twiddle multiply and k-space multiply runs once for both lines.  Per line
// that halves the floating-point, load/store, shared-memory and twiddle
// instructions of the scalar path (gpe_fft.cuh with float2), with the same
// Stockham plans and the same register/line-position conventions.
#pragma once

#include "gpe_fft.cuh"

namespace gpe {

// Two floats operated on as one packed FP32x2 value.
struct f2x {
    float2 v;
};

__device__ __forceinline__ f2x operator+(f2x a, f2x b) { return f2x{__fadd2_rn(a.v, b.v)}; }
// (the runtime header has no packed subtract; the PTX instruction exists)
__device__ __forceinline__ f2x operator-(f2x a, f2x b) {
    f2x r;
    asm("{\n\t.reg .b64 pa, pb, pd;\n\t"
        "mov.b64 pa, {%2, %3};\n\t"
        "mov.b64 pb, {%4, %5};\n\t"
        "sub.rn.f32x2 pd, pa, pb;\n\t"
        "mov.b64 {%0, %1}, pd;\n\t}"
        : "=f"(r.v.x), "=f"(r.v.y)
        : "f"(a.v.x), "f"(a.v.y), "f"(b.v.x), "f"(b.v.y));
    return r;
}
__device__ __forceinline__ f2x operator-(f2x a) { return f2x{__fmul2_rn(make_float2(-1.0f, -1.0f), a.v)}; }
__device__ __forceinline__ f2x operator*(float s, f2x a) { return f2x{__fmul2_rn(make_float2(s, s), a.v)}; }
__device__ __forceinline__ f2x operator*(f2x a, f2x b) { return f2x{__fmul2_rn(a.v, b.v)}; }
// a * b + c
__device__ __forceinline__ f2x fma2(f2x a, f2x b, f2x c) { return f2x{__ffma2_rn(a.v, b.v, c.v)}; }

// Complex values of two lines: x = real parts, y = imaginary parts.
struct __align__(16) cpair {
    f2x x, y;
};
__device__ __forceinline__ cpair mk(f2x x, f2x y) { return cpair{x, y}; }

template <> struct RealOf<cpair> { typedef float T; };
// Twiddle table entry of the paired path: (cos, cos, sin, sin), one 16-byte
// load that yields the broadcast pairs the packed multiply needs.
template <> struct TwOf<cpair> { typedef float4 T; };

// a * w and a * conj(w) for w = (c, s) given as (c, c, s, s).
__device__ __forceinline__ cpair cmul(cpair a, float4 w) {
    const f2x c{make_float2(w.x, w.y)}, s{make_float2(w.z, w.w)};
    return cpair{a.x * c - a.y * s, fma2(a.x, s, a.y * c)};
}
__device__ __forceinline__ cpair cmulc(cpair a, float4 w) {
    const f2x c{make_float2(w.x, w.y)}, s{make_float2(w.z, w.w)};
    return cpair{fma2(a.x, c, a.y * s), a.y * c - a.x * s};
}

// 16-byte global value (re_a, im_a, re_b, im_b) <-> pair.
__device__ __forceinline__ cpair pair_from(float4 q) {
    return cpair{f2x{make_float2(q.x, q.z)}, f2x{make_float2(q.y, q.w)}};
}
__device__ __forceinline__ float4 pair_to(cpair p) { return make_float4(p.x.v.x, p.y.v.x, p.x.v.y, p.y.v.y); }

}  // namespace gpe
