// gpe_inst_body.cuh -- included by gpe_inst_*.cu after defining GPE_R (float
// or double), GPE_SFX (f or d), GPE_FAM (length family), GPE_NF (fields per
// pass, 1 or 2), GPE_SIZES(X) and GPE_TUNED(X) (the family's lengths with
// autotuner variants); GPE_PAIRED (complex64 units) adds the paired strided
// passes.
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

#if GPE_NF == 1
#define GPE_SVCASE(L)                                                   \
    case L: {                                                           \
        bool found = false;                                             \
        *err = launch_svar<GPE_R, L>(v, a, nouter, st, &found);         \
        return found;                                                   \
    }
// Autotuner variants of the one-field strided pass at the tuned lengths.
bool GPE_NAME(dispatch_sv_)(int L, int v, const PassArgs<GPE_R>& a, int nouter, cudaStream_t st, cudaError_t* err) {
    switch (L) {
        GPE_TUNED(GPE_SVCASE)
        default:
            return false;
    }
}
#endif

#ifdef GPE_PAIRED
#define GPE_S2CASE(L)                                            \
    case L:                                                      \
        *err = launch_spass2<L, GPE_NF>(a, nouter, smem, st);    \
        return true;
// Paired complex64 strided passes (two lines per thread, nx even).
bool GPE_NAME(dispatch_s2_)(int L, const PassArgs<float>& a, int nouter, size_t smem, cudaStream_t st,
                            cudaError_t* err) {
    switch (L) {
        GPE_SIZES(GPE_S2CASE)
        default:
            return false;
    }
}
#endif

}  // namespace gpe
