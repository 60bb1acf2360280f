// gpe_dispatch.cuh -- run-time dispatch from a grid length to the pass-kernel
// instantiation compiled for it (one translation unit per length family and
// precision, gpe_inst_*.cu).
#pragma once

#include "gpe_batch_args.cuh"
#include "gpe_kernels.cuh"

namespace gpe {

#define GPE_FAMILIES(X) X(p2) X(p2b) X(p3) X(p3b) X(p5) X(p5b) X(p9) X(p9b)

#define GPE_DECL_ONE(F, P, R, NF)                                                                      \
    bool dispatch_x_##F##_##P##_##NF(int L, const PassArgs<R>& a, int rows, size_t smem, cudaStream_t st, cudaError_t* err);    \
    bool dispatch_s_##F##_##P##_##NF(int L, const PassArgs<R>& a, int nouter, size_t smem, cudaStream_t st, cudaError_t* err);
#define GPE_DECL_FAMILY(F) GPE_DECL_ONE(F, f, float, 1) GPE_DECL_ONE(F, f, float, 2) \
                           GPE_DECL_ONE(F, d, double, 1) GPE_DECL_ONE(F, d, double, 2)
GPE_FAMILIES(GPE_DECL_FAMILY)
#undef GPE_DECL_FAMILY
#undef GPE_DECL_ONE

#define GPE_DISPATCH_FN(R, P)                                                                        \
    inline bool dispatch_x(int L, int NF, const PassArgs<R>& a, int rows, size_t smem, cudaStream_t st, cudaError_t* err) { \
        GPE_FAMILIES(GPE_TRYX_##P)                                                                   \
        return false;                                                                                \
    }                                                                                                \
    inline bool dispatch_s(int L, int NF, const PassArgs<R>& a, int nouter, size_t smem, cudaStream_t st, \
                           cudaError_t* err) {                                                       \
        GPE_FAMILIES(GPE_TRYS_##P)                                                                   \
        return false;                                                                                \
    }
#define GPE_TRYX_f(F) if (NF == 1 ? dispatch_x_##F##_f_1(L, a, rows, smem, st, err) : dispatch_x_##F##_f_2(L, a, rows, smem, st, err)) return true;
#define GPE_TRYX_d(F) if (NF == 1 ? dispatch_x_##F##_d_1(L, a, rows, smem, st, err) : dispatch_x_##F##_d_2(L, a, rows, smem, st, err)) return true;
#define GPE_TRYS_f(F) if (NF == 1 ? dispatch_s_##F##_f_1(L, a, nouter, smem, st, err) : dispatch_s_##F##_f_2(L, a, nouter, smem, st, err)) return true;
#define GPE_TRYS_d(F) if (NF == 1 ? dispatch_s_##F##_d_1(L, a, nouter, smem, st, err) : dispatch_s_##F##_d_2(L, a, nouter, smem, st, err)) return true;
GPE_DISPATCH_FN(float, f)
GPE_DISPATCH_FN(double, d)

#define GPE_DECL_S2(F)                                                                                        \
    bool dispatch_s2_##F##_f_1(int L, const PassArgs<float>& a, int nouter, size_t smem, cudaStream_t st,   \
                               cudaError_t* err);                                                           \
    bool dispatch_s2_##F##_f_2(int L, const PassArgs<float>& a, int nouter, size_t smem, cudaStream_t st,   \
                               cudaError_t* err);
GPE_FAMILIES(GPE_DECL_S2)
#undef GPE_DECL_S2
#define GPE_DECL_SV(F)                                                                                        \
    bool dispatch_sv_##F##_f_1(int L, int v, const PassArgs<float>& a, int nouter, cudaStream_t st,             \
                               cudaError_t* err);                                                            \
    bool dispatch_sv_##F##_d_1(int L, int v, const PassArgs<double>& a, int nouter, cudaStream_t st,            \
                               cudaError_t* err);
GPE_FAMILIES(GPE_DECL_SV)
#undef GPE_DECL_SV
// Autotuner variant v of the one-field strided pass at a tuned length.
inline bool dispatch_sv(int L, int v, const PassArgs<float>& a, int nouter, cudaStream_t st, cudaError_t* err) {
#define GPE_TRYSV(F) \
    if (dispatch_sv_##F##_f_1(L, v, a, nouter, st, err)) return true;
    GPE_FAMILIES(GPE_TRYSV)
#undef GPE_TRYSV
    return false;
}
inline bool dispatch_sv(int L, int v, const PassArgs<double>& a, int nouter, cudaStream_t st, cudaError_t* err) {
#define GPE_TRYSV(F) \
    if (dispatch_sv_##F##_d_1(L, v, a, nouter, st, err)) return true;
    GPE_FAMILIES(GPE_TRYSV)
#undef GPE_TRYSV
    return false;
}

// Fused y-z cluster kernel of a 3D complex64 stage (gpe_yz.cu).
bool yz_shape_supported(int ly, int lz);
bool dispatch_yz(int ly, int lz, const PassArgs<float>& a, cudaStream_t st, cudaError_t* err);

// Paired complex64 strided pass (needs an even nx; see k_spass2).
inline bool dispatch_s2(int L, int NF, const PassArgs<float>& a, int nouter, size_t smem, cudaStream_t st,
                        cudaError_t* err) {
#define GPE_TRYS2(F)                                                                                        \
    if (NF == 1 ? dispatch_s2_##F##_f_1(L, a, nouter, smem, st, err) : dispatch_s2_##F##_f_2(L, a, nouter, smem, st, err)) \
        return true;
    GPE_FAMILIES(GPE_TRYS2)
#undef GPE_TRYS2
    return false;
}

}  // namespace gpe
