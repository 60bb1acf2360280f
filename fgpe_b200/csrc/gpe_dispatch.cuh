// gpe_dispatch.cuh -- run-time dispatch from a grid length to the pass-kernel
// instantiation compiled for it (one translation unit per length family and
// precision, gpe_inst_*.cu).
#pragma once

#include "gpe_kernels.cuh"

namespace gpe {

#define GPE_FAMILIES(X) X(p2) X(p3) X(p5) X(p9)

#define GPE_DECL_FAMILY(F)                                                                                       \
    bool dispatch_x_##F##_f(int L, int NF, const PassArgs<float>& a, cudaStream_t st, cudaError_t* err);        \
    bool dispatch_s_##F##_f(int L, int NF, const PassArgs<float>& a, int nouter, cudaStream_t st,               \
                            cudaError_t* err);                                                                   \
    bool dispatch_x_##F##_d(int L, int NF, const PassArgs<double>& a, cudaStream_t st, cudaError_t* err);       \
    bool dispatch_s_##F##_d(int L, int NF, const PassArgs<double>& a, int nouter, cudaStream_t st,              \
                            cudaError_t* err);
GPE_FAMILIES(GPE_DECL_FAMILY)
#undef GPE_DECL_FAMILY

inline bool dispatch_x(int L, int NF, const PassArgs<float>& a, cudaStream_t st, cudaError_t* err) {
#define GPE_TRY(F) if (dispatch_x_##F##_f(L, NF, a, st, err)) return true;
    GPE_FAMILIES(GPE_TRY)
#undef GPE_TRY
    return false;
}
inline bool dispatch_x(int L, int NF, const PassArgs<double>& a, cudaStream_t st, cudaError_t* err) {
#define GPE_TRY(F) if (dispatch_x_##F##_d(L, NF, a, st, err)) return true;
    GPE_FAMILIES(GPE_TRY)
#undef GPE_TRY
    return false;
}
inline bool dispatch_s(int L, int NF, const PassArgs<float>& a, int nouter, cudaStream_t st, cudaError_t* err) {
#define GPE_TRY(F) if (dispatch_s_##F##_f(L, NF, a, nouter, st, err)) return true;
    GPE_FAMILIES(GPE_TRY)
#undef GPE_TRY
    return false;
}
inline bool dispatch_s(int L, int NF, const PassArgs<double>& a, int nouter, cudaStream_t st, cudaError_t* err) {
#define GPE_TRY(F) if (dispatch_s_##F##_d(L, NF, a, nouter, st, err)) return true;
    GPE_FAMILIES(GPE_TRY)
#undef GPE_TRY
    return false;
}

}  // namespace gpe
