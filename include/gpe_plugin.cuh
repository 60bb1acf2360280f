/*
 * gpe_plugin.cuh -- writing a user Hamiltonian plugin for libgpe (CUDA C++).
 *
 * The reference lets a plugin author write the Hamiltonian kernels
 * themselves (hamiltonians/BEC_oneComponent.hpp:8-22: a __global__ kernel
 * (t, psi, KEpsi, vext, h_en, h_mu, N, prms) launched from alg_calcHpsi;
 * hamiltonians/single_template.cu:333-373 is the empty slot).  Here the
 * Hamiltonian is evaluated inside the fused x-inverse pass of every stage,
 * so a plugin supplies the pointwise term as a functor and this header
 * instantiates the pass kernels with it in the plugin's own translation unit:
 *
 *   #include "gpe_plugin.cuh"
 *   struct MyHam {
 *       template <typename R> struct Coef { R g; };             // per-CTA constants
 *       template <typename R>
 *       __device__ static Coef<R> coef(const double* prms, double t) {   // d_h_params, time
 *           return Coef<R>{(R)(4 * 3.141592653589793 * prms[0])};
 *       }
 *       template <typename R, typename C>                      // C = float2 / double2
 *       __device__ static void point(const Coef<R>& k, C psi, C T, C V, bool want_en, C& hmu, C& hen) {
 *           const R n = psi.x * psi.x + psi.y * psi.y;
 *           const R ur = V.x + k.g * n, ui = V.y;
 *           hmu = {T.x + ur * psi.x - ui * psi.y, T.y + ur * psi.y + ui * psi.x};   // h_mu
 *           if (want_en) hen = ...;                                               // h_en
 *       }
 *   };
 *   GPE_DEFINE_USER_HAMILTONIAN(MyHam, my_ham_plugin)
 *
 * T is the kinetic part at the point (the reference's KEpsi), V the complex
 * external potential, psi the wavefunction; hmu is the term the time
 * stepping uses (alg_calcHpsiMU), hen the energy density's (alg_calcHpsi).
 * Compile with nvcc -gencode arch=compute_100a,code=sm_100a -std=c++17
 * -Xcompiler -fPIC -shared, with -I to this directory and to the library's
 * fgpe_b200/csrc; the lengths compiled are GPE_USER_SIZES (define it before
 * including this header, e.g. #define GPE_USER_SIZES(X) X(64) X(128)).  The
 * host creates a handle with hamiltonian = GPE_HAM_USER and calls
 * gpe_set_user_hamiltonian(h, my_ham_plugin()).
 */
#pragma once

#include "gpe.h"
#include "gpe_kernels_impl.cuh"

#ifndef GPE_USER_SIZES
#define GPE_USER_SIZES(X) X(64) X(96) X(128) X(192) X(256) X(384) X(512)
#endif

namespace gpe {

template <class U, typename R>
int user_launch_x(int L, const void* pass_args, int rows, size_t smem, void* stream, int* cuda_err) {
    const PassArgs<R>& a = *static_cast<const PassArgs<R>*>(pass_args);
    cudaError_t e = cudaSuccess;
    bool found = false;
    switch (L) {
#define GPE_USER_CASE(N)                                                                      \
    case N:                                                                                   \
        e = launch_xpass<R, N, 1, UserHam<U>>(a, rows, smem, static_cast<cudaStream_t>(stream)); \
        found = true;                                                                         \
        break;
        GPE_USER_SIZES(GPE_USER_CASE)
#undef GPE_USER_CASE
        default:
            break;
    }
    *cuda_err = (int)e;
    return found ? 1 : 0;
}

}  // namespace gpe

#define GPE_DEFINE_USER_HAMILTONIAN(U, NAME)                                                     \
    extern "C" const gpe_user_hamiltonian* NAME(void) {                                         \
        static const gpe_user_hamiltonian ops = {GPE_ABI_VERSION, &gpe::user_launch_x<U, float>, \
                                                 &gpe::user_launch_x<U, double>};               \
        return &ops;                                                                            \
    }
