// gpe_common.cuh -- shared device types for libgpe (complex helpers, device
// scalar block, error plumbing).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gpe {

// Complex storage type per real type: float2 (complex64) / double2 (complex128).
template <typename R> struct Cx;
template <> struct Cx<float> { typedef float2 T; };
template <> struct Cx<double> { typedef double2 T; };

__host__ __device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }
__host__ __device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
    return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// Device-resident solver scalars: the reference keeps these in the host PARS
// array (hpp/oneComponentGPSolver.hpp:20-39) and pays a host round trip per
// reduction; here they live on the device so a chunk of steps runs with no
// host synchronisation.
struct DevScalars {
    double scale[2][2];     // [slot][comp] lazy renormalisation factor of buf[slot]
    double mu[2];           // PARS[MU] / MU1, MU2
    double en[2];           // PARS[EN]
    double en_prev[2];      // PARS[EN_PREV]
    double norm[2];         // PARS[NORM]
    double mu_prev[2];      // RK4-imag: mu of the previous step
    double obs[8];          // last raw reductions (observables / logging)
    int cur_slot;           // which of buf[0]/buf[1] holds the current psi
    int done;               // convergence or error: later kernels of a chunk exit
    int converged;
    int iters_done;         // iterations applied since the last reset of the counter
    int status;             // 0 ok, GPE_ERR_DIVERGED when a reduction is not finite
    int have_mu_prev;
    unsigned int counter;   // last-block-done ticket for fused reductions
    int pad;
};

}  // namespace gpe
