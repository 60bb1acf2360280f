// gpe_inst_body.cuh -- included by gpe_inst_*.cu after defining GPE_R (float
// or double), GPE_SFX (f or d), GPE_FAM (length family), GPE_NF (fields per
// pass, 1 or 2) and GPE_SIZES(X).
#include "gpe_kernels_impl.cuh"

#define GPE_CAT2(a, b) a##b
#define GPE_CAT(a, b) GPE_CAT2(a, b)
#define GPE_NAME(kind) GPE_CAT(GPE_CAT(GPE_CAT(kind, GPE_FAM), GPE_CAT(_, GPE_SFX)), GPE_CAT(_, GPE_NF))

namespace gpe {

#define GPE_XCASE(L)                                     \
    case L:                                              \
        *err = launch_xpass<GPE_R, L, GPE_NF>(a, rows, smem, st);    \
        return true;
#define GPE_SCASE(L)                                             \
    case L:                                                      \
        *err = launch_spass<GPE_R, L, GPE_NF>(a, nouter, smem, st);    \
        return true;

bool GPE_NAME(dispatch_x_)(int L, const PassArgs<GPE_R>& a, int rows, size_t smem, cudaStream_t st, cudaError_t* err) {
    switch (L) {
        GPE_SIZES(GPE_XCASE)
        default:
            return false;
    }
}

bool GPE_NAME(dispatch_s_)(int L, const PassArgs<GPE_R>& a, int nouter, size_t smem, cudaStream_t st, cudaError_t* err) {
    switch (L) {
        GPE_SIZES(GPE_SCASE)
        default:
            return false;
    }
}

}  // namespace gpe
