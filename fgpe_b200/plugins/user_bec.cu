// user_bec.cu -- a user Hamiltonian plugin written against include/gpe_plugin.cuh:
// the one-component BEC term of hamiltonians/BEC_oneComponent.cu:128-178
// (h_mu = T + (V + 4 pi a(t) |psi|^2) psi, h_en with 2 pi a(t), a(t) the
// quench profile d_quench_as of prms[0..5]) as a user functor.  It is the
// example for plugin authors and the test of the plug-point: a handle with
// GPE_HAM_USER and this plugin must reproduce GPE_HAM_BEC to the rounding of
// the precision.
#define GPE_USER_SIZES(X) X(16) X(32) X(64) X(128)
#include "gpe_plugin.cuh"

struct UserBEC {
    template <typename R>
    struct Coef {
        R g_en, g_mu;  // 2 pi a(t), 4 pi a(t)
    };
    template <typename R>
    __device__ static Coef<R> coef(const double* prms, double t) {
        // hamiltonians/BEC_oneComponent.cu:167-178
        const double a0 = prms[0], a1 = prms[1], a2 = prms[2], t1 = prms[3], t2 = prms[4], t3 = prms[5];
        double a = a2;
        if (0 < t && t <= t1) a = a0 + (a1 - a0) / (t1)*t;
        else if (t1 < t && t <= t2) a = a1;
        else if (t2 < t && t <= t3) a = a1 + (a2 - a1) / (t3 - t2) * (t - t2);
        const double pi = 3.141592653589793;
        return Coef<R>{(R)(2 * pi * a), (R)(4 * pi * a)};
    }
    template <typename R, typename C>
    __device__ static void point(const Coef<R>& k, C psi, C T, C V, bool want_en, C& hmu, C& hen) {
        // hamiltonians/BEC_oneComponent.cu:128-165
        const R px = psi.x, py = psi.y;
        const R n = px * px + py * py;
        const R phi = (R)0;  // no mean-field term of its own
        if (want_en) {
            const R rX = (V.x + k.g_en * n) + (R)0.5 * phi, rY = V.y;
            hen = C{T.x + rX * px - rY * py, T.y + rX * py + rY * px};
        }
        const R rX = (V.x + k.g_mu * n) + phi, rY = V.y;
        hmu = C{T.x + rX * px - rY * py, T.y + rX * py + rY * px};
    }
};

GPE_DEFINE_USER_HAMILTONIAN(UserBEC, gpe_user_bec)
