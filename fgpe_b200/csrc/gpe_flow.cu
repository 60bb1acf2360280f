// gpe_flow.cu -- instantiations of the persistent RK4 step kernel
// (gpe_flow.cuh) for the cubic complex64 grids it serves.
#include "gpe_flow.cuh"

namespace gpe {

#define GPE_FLOW_LENGTHS(X) X(128) X(256)

bool flow_shape_supported(int nx, int ny, int nz) {
    if (nx != ny || ny != nz) return false;
#define GPE_FLOW_IS(L) \
    if (nx == L) return FlowGeom<L>::ok;
    GPE_FLOW_LENGTHS(GPE_FLOW_IS)
#undef GPE_FLOW_IS
    return false;
}

int flow_rows(int L) {
#define GPE_FLOW_ROWS(N) \
    if (L == N) return FlowGeom<N>::ROWS;
    GPE_FLOW_LENGTHS(GPE_FLOW_ROWS)
#undef GPE_FLOW_ROWS
    return 0;
}

int flow_ntx(int L) {
#define GPE_FLOW_NTX(N) \
    if (L == N) return FlowGeom<N>::NTX;
    GPE_FLOW_LENGTHS(GPE_FLOW_NTX)
#undef GPE_FLOW_NTX
    return 0;
}

int flow_ctas_per_sm(int L) {
#define GPE_FLOW_OCC(N) \
    if (L == N) return flow_occupancy<N>();
    GPE_FLOW_LENGTHS(GPE_FLOW_OCC)
#undef GPE_FLOW_OCC
    return 0;
}

int flow_strided_ctas_per_sm(int L) {
#define GPE_FLOW_SOCC(N) \
    if (L == N) return flow_strided_occupancy<N>();
    GPE_FLOW_LENGTHS(GPE_FLOW_SOCC)
#undef GPE_FLOW_SOCC
    return 0;
}

bool dispatch_flow_strided(int L, const FlowArgs& fa, int grid, cudaStream_t st, cudaError_t* err) {
#define GPE_FLOW_SCASE(N)                            \
    if (L == N) {                                    \
        *err = launch_flow_strided<N>(fa, grid, st); \
        return true;                                 \
    }
    GPE_FLOW_LENGTHS(GPE_FLOW_SCASE)
#undef GPE_FLOW_SCASE
    return false;
}

bool dispatch_flow(int L, bool obs, const FlowArgs& fa, int grid, cudaStream_t st, cudaError_t* err) {
#define GPE_FLOW_CASE(N)                                                                       \
    if (L == N) {                                                                              \
        *err = obs ? launch_flow<N, true>(fa, grid, st) : launch_flow<N, false>(fa, grid, st); \
        return true;                                                                           \
    }
    GPE_FLOW_LENGTHS(GPE_FLOW_CASE)
#undef GPE_FLOW_CASE
    return false;
}

}  // namespace gpe
