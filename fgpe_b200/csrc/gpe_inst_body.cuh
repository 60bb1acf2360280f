// gpe_inst_body.cuh -- included by gpe_inst_*.cu after defining GPE_R (float
// or double), GPE_SFX (f or d), GPE_FAM (family name) and GPE_SIZES(X).
#include "gpe_kernels_impl.cuh"

#define GPE_CAT2(a, b) a##b
#define GPE_CAT(a, b) GPE_CAT2(a, b)
#define GPE_CAT4(a, b, c, d) GPE_CAT(GPE_CAT(a, b), GPE_CAT(c, d))

namespace gpe {

#define GPE_XCASE(L)                                                                        \
    case L:                                                                                 \
        *err = (NF == 1) ? launch_xpass<GPE_R, L, 1>(a, st) : launch_xpass<GPE_R, L, 2>(a, st); \
        return true;
#define GPE_SCASE(L)                                                                                          \
    case L:                                                                                                   \
        *err = (NF == 1) ? launch_spass<GPE_R, L, 1>(a, nouter, st) : launch_spass<GPE_R, L, 2>(a, nouter, st); \
        return true;

bool GPE_CAT4(dispatch_x_, GPE_FAM, _, GPE_SFX)(int L, int NF, const PassArgs<GPE_R>& a, cudaStream_t st,
                                                cudaError_t* err) {
    switch (L) {
        GPE_SIZES(GPE_XCASE)
        default:
            return false;
    }
}

bool GPE_CAT4(dispatch_s_, GPE_FAM, _, GPE_SFX)(int L, int NF, const PassArgs<GPE_R>& a, int nouter, cudaStream_t st,
                                                cudaError_t* err) {
    switch (L) {
        GPE_SIZES(GPE_SCASE)
        default:
            return false;
    }
}

}  // namespace gpe
