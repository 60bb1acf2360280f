// gpe_yz.cu -- instantiations of the fused y-z cluster kernel (gpe_yz.cuh)
// for the complex64 grids it serves: y and z lengths 64 and 128.
#include "gpe_yz.cuh"

namespace gpe {

#define GPE_YZ_SHAPES(X) X(128, 128) X(128, 64) X(64, 128) X(64, 64)

bool yz_shape_supported(int ly, int lz) {
#define GPE_YZ_IS(Y, Z) \
    if (ly == Y && lz == Z) return YZGeom<Y, Z>::ok;
    GPE_YZ_SHAPES(GPE_YZ_IS)
#undef GPE_YZ_IS
    return false;
}

bool dispatch_yz(int ly, int lz, const PassArgs<float>& a, cudaStream_t st, cudaError_t* err) {
#define GPE_YZ_CASE(Y, Z)                  \
    if (ly == Y && lz == Z) {              \
        *err = launch_yz<Y, Z>(a, st);     \
        return true;                       \
    }
    GPE_YZ_SHAPES(GPE_YZ_CASE)
#undef GPE_YZ_CASE
    return false;
}

}  // namespace gpe
