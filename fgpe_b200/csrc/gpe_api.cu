// gpe_api.cu -- C ABI of libgpe: handle lifecycle, device buffers, and the
// host-side orchestration of the fused pass chains (see include/gpe.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gpe.h"
#include "gpe_dispatch.cuh"
#include "gpe_flow_args.cuh"
#include "gpe_init.cuh"
#include "gpe_sizes.h"

using namespace gpe;

namespace {

thread_local std::string g_err;

gpe_status fail(gpe_status s, const std::string& msg) {
    g_err = msg;
    return s;
}

#define GPE_CUDA(call)                                                                                      \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess)                                                                              \
            return fail(e_ == cudaErrorMemoryAllocation ? GPE_ERR_OUT_OF_MEMORY : GPE_ERR_CUDA,              \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                                \
    } while (0)

#define GPE_TRY(expr)                      \
    do {                                   \
        gpe_status s_ = (expr);            \
        if (s_ != GPE_OK) return s_;       \
    } while (0)

bool length_compiled(int L) {
#define GPE_IS(n) if (L == n) return true;
    GPE_SIZES_p2(GPE_IS) GPE_SIZES_p2b(GPE_IS) GPE_SIZES_p3(GPE_IS) GPE_SIZES_p3b(GPE_IS)
    GPE_SIZES_p5(GPE_IS) GPE_SIZES_p5b(GPE_IS) GPE_SIZES_p9(GPE_IS) GPE_SIZES_p9b(GPE_IS)
#undef GPE_IS
    return false;
}

int plan_T(int L) { return L / make_plan(L).E; }

enum StateMode { ST_CANON = 0, ST_HB = 1, ST_RKI = 2 };

constexpr int YZ_XB_HOST = 4;  // x values per slab of the fused y-z kernel (YZ_XB, gpe_yz.cuh)

}  // namespace

// Lets other translation units of the library (gpe_noalloc.cu) record the
// message that gpe_last_error_string() returns.
namespace gpe {
void set_last_error(const char* msg) { g_err = msg; }
}  // namespace gpe

struct gpe_handle {
    gpe_config cfg;
    int prec = GPE_C128;
    int nx = 1, ny = 1, nz = 1;
    long long N = 1;
    int ncomp = 1, dens = 0, nf = 1;
    int nb = 1;  // instances held (gpe_batch groups); fields of instance i start at i*N
    size_t esz = 16;
    cudaStream_t st = 0;
    void* A[2] = {nullptr, nullptr};
    void* B[2] = {nullptr, nullptr};
    void* K[2] = {nullptr, nullptr};
    void* V[2] = {nullptr, nullptr};
    void* W[3] = {nullptr, nullptr, nullptr};
    void* O[4] = {nullptr, nullptr, nullptr, nullptr};
    void* tw[3] = {nullptr, nullptr, nullptr};
    float4* tw2[3] = {nullptr, nullptr, nullptr};  // complex64: (cos, cos, sin, sin) per axis
    // pass variants (gpe_tune): svar[axis][mode] for the strided passes
    // (mode 0 forward, 1 forward*k*inverse, 2 inverse; 0 = default variant),
    // xrows = rows per CTA of the x passes (0 = default)
    int svar[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    int xrows = 0;
    // user Hamiltonian plugin (GPE_HAM_USER, gpe_set_user_hamiltonian)
    const gpe_user_hamiltonian* user = nullptr;
    // 1: the strided part of a 3D complex64 stage runs as the fused y-z
    // cluster kernel (k_yz, gpe_yz.cuh) where the grid allows it
    int yz = 0;
    // 1: real-time RK4 steps of a complex64 one-component cubic grid run as
    // one persistent launch per step (k_flow_step, gpe_flow.cuh); its
    // dependency counters, the launch parity and the wait bound
    int flow = 0;
    // 1: the fused real-time RK x pass of a complex64 one-field chain stages
    // its epilogue inputs in shared memory (XK_RKS)
    int xstage = 0;
    FlowSync* flow_sync = nullptr;
    long long flow_launches = 0;
    unsigned flow_bound = 1u << 22;
    double* kax[3] = {nullptr, nullptr, nullptr};
    float* k2s[3] = {nullptr, nullptr, nullptr};  // complex64: lap_scale * k^2 per axis
    double* obs_part = nullptr;                    // OBS_BLOCKS partial sums + the result
    void* vdd = nullptr;
    double* prms = nullptr;
    DevScalars* sc = nullptr;
    double* partials = nullptr;
    void* stage128 = nullptr;  // complex128 staging (complex64 handles)
    // complex64 single handles: low part of the real-time step state (A holds
    // the high part), valid while only real-time steps have written A
    void* Lo[2] = {nullptr, nullptr};
    bool lo_valid = false;
    long long launches = 0;
    int mode = ST_CANON;
    bool hb_old_valid = true;
    // W[0..nf-1] hold the x-forward transform of the state in A (left by the
    // last real-time stage); any other operation clears it.
    bool w_fwd_A = false;
    // control gradient (gpe_control_*): basis G[k] (real, field precision),
    // saved base potential, work fields, checkpoints
    int nctrl = 0;
    void* ctrlG = nullptr;
    void* V0 = nullptr;
    void* adj[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    void* qf = nullptr;
    double* d_u = nullptr;
    double* d_part = nullptr;
    double* d_grad = nullptr;
    std::vector<void*> cps;
    std::vector<void*> cps_lo;  // complex64: low parts of the checkpoints
    // imaginary-time chunks: pinned copies of the device's done flag and the
    // events that mark when each copy has landed
    int* flag_host = nullptr;
    cudaEvent_t flag_ev[2] = {nullptr, nullptr};
    // per-pass event timing (gpe_profile_enable)
    bool prof = false;
    std::vector<cudaEvent_t> ev_free;
    struct Rec {
        int kind;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
};

// ---- small element-wise kernels ------------------------------------------------------
namespace {

template <typename C>
__global__ void k_from_c128(C* dst, const double2* src, long long n) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = from_d<C>(src[i]);
}
template <typename C>
__global__ void k_to_c128(double2* dst, const C* src, long long n) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = to_d(src[i]);
}
// low part of a complex128 state stored as complex64: src - hi, rounded
__global__ void k_lo_residual(float2* lo, const float2* hi, const double2* src, long long n) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) lo[i] = make_float2((float)(src[i].x - (double)hi[i].x), (float)(src[i].y - (double)hi[i].y));
}
// A complex128 state into a complex64 handle in one pass: the high part
// (rounded) into both state slots, the rounding residual into the low part
// (k_from_c128, the copy of A into B and k_lo_residual, fused).
__global__ void k_set_state_c64(float2* a, float2* b, float2* lo, const double2* src, long long n) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) {
        const double2 v = src[i];
        const float2 hi = make_float2((float)v.x, (float)v.y);
        a[i] = hi;
        b[i] = hi;
        lo[i] = make_float2((float)(v.x - (double)hi.x), (float)(v.y - (double)hi.y));
    }
}
// high + low parts of a compensated complex64 state
__global__ void k_to_c128_hilo(double2* dst, const float2* hi, const float2* lo, long long n) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = make_double2((double)hi[i].x + (double)lo[i].x, (double)hi[i].y + (double)lo[i].y);
}
template <typename C>
__global__ void k_copy(C* dst, const C* src, long long n) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}
// Materialise psi and psi_old of a lazily renormalised state (ScalarMultiply,
// hpp/parallel.hpp:205-212): heavy ball: A <- s_cur*buf[cur], B <- s_old*buf[1-cur];
// RK4-imaginary: A <- s_cur*A.
template <typename C>
__global__ void k_canon(C* A, C* B, const DevScalars* sc, int comp, int hb, long long n) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int cur = sc->cur_slot;
    const double sc0 = sc->scale[cur][comp], sc1 = sc->scale[1 - cur][comp];
    if (hb) {
        const C a = A[i], b = B[i];
        const C p = (cur == 0) ? a : b;
        const C o = (cur == 0) ? b : a;
        A[i] = from_d<C>(make_double2((double)p.x * sc0, (double)p.y * sc0));
        B[i] = from_d<C>(make_double2((double)o.x * sc1, (double)o.y * sc1));
    } else {
        const C a = A[i];
        A[i] = from_d<C>(make_double2((double)a.x * sc0, (double)a.y * sc0));
    }
}
__global__ void k_reset_iters(DevScalars* sc, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        sc[i].iters_done = 0;
        sc[i].counter = 0;  // 0 after every complete launch; a launch cut short leaves it stale
    }
}
__global__ void k_reset_scales(DevScalars* sc) {
    sc->scale[0][0] = sc->scale[0][1] = sc->scale[1][0] = sc->scale[1][1] = 1.0;
    sc->cur_slot = 0;
}

inline unsigned blocks_for(long long n, int thr) { return (unsigned)((n + thr - 1) / thr); }

// ---- control-gradient helpers ------------------------------------------------------------
// V = V0 + sum_k u[k] G_k (real part), the potential of one controlled step.
template <typename C, typename R>
__global__ void k_form_control_v(C* V, const C* V0, const R* G, const double* u, int nctrl, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    C v = V0[i];
    double w = (double)v.x;
    for (int k = 0; k < nctrl; ++k) w += u[k] * (double)G[(long long)k * n + i];
    v.x = (decltype(v.x))w;
    V[i] = v;
}
// dst = (cr + i ci) * src
template <typename C>
__global__ void k_cscale(C* dst, const C* src, double cr, double ci, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const C a = src[i];
    dst[i] = from_d<C>(make_double2(cr * a.x - ci * a.y, cr * a.y + ci * a.x));
}
// Per-block FP64 partial sums, fixed order: mode 0: sum conj(a) b (2 values);
// mode 1: sum_x G_k(x) q(x) for k < nq (q real, G real).
constexpr int CTRL_BLOCKS = 128;
template <typename C, typename R>
__global__ void k_ctrl_partials(int mode, const C* a, const C* b, const R* q, const R* G, int nq, long long n,
                                double* part) {
    __shared__ double sh[256];
    double acc[2 * 64];
    const int nv = mode == 0 ? 2 : nq;
    for (int k = 0; k < nv; ++k) acc[k] = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (mode == 0) {
            const C x = a[i], y = b[i];
            acc[0] += (double)x.x * y.x + (double)x.y * y.y;
            acc[1] += (double)x.x * y.y - (double)x.y * y.x;
        } else {
            const double qq = (double)q[i];
            for (int k = 0; k < nq; ++k) acc[k] += (double)G[(long long)k * n + i] * qq;
        }
    }
    for (int k = 0; k < nv; ++k) {
        sh[threadIdx.x] = acc[k];
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(long long)blockIdx.x * nv + k] = sh[0];
        __syncthreads();
    }
}
// ---- logging-cadence observables ----------------------------------------------------
// Per-block FP64 (Neumaier) sums of a pointwise quantity of one or two fields:
//  OBS_COS   cos(2 pi x/L) |a|^2               CalcAverageCos, src/parallel.cu:535-561
//  OBS_COS2  cos(2 pi x/L) |a + sign b|^2      CalcAverageCos, src/parallel.cu:739-771
//  OBS_PHASE atan2(a) - atan2(b)               CalculateRelativePhase, src/parallel.cu:774-802
//  OBS_DSZ   sqrt(|a|^2 |b|^2) sin(phase)      CalculateDszDt, src/parallel.cu:805-839
// x[ix] = -XMAX + (ix + 1/2) DX (src/baseHamiltonian.cu:25-51), ix = i % nx.
enum { OBS_COS = 0, OBS_COS2 = 1, OBS_PHASE = 2, OBS_DSZ = 3 };
constexpr int OBS_BLOCKS = 128;
template <typename C>
__global__ void k_obs_partials(int kind, const C* a, const C* b, double sign, double xmax, double dx, double L,
                               int nx, long long n, double* part) {
    __shared__ double sh_s[256], sh_c[256];
    double s = 0.0, comp = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double ax = a[i].x, ay = a[i].y;
        double v;
        if (kind == OBS_COS || kind == OBS_COS2) {
            const double x = -xmax + (double)(i % nx) * dx + 0.5 * dx;
            double px = ax, py = ay;
            if (kind == OBS_COS2) {
                px += sign * (double)b[i].x;
                py += sign * (double)b[i].y;
            }
            v = cos(2.0 * 3.141592653589793 * x / L) * (px * px + py * py);
        } else {
            const double bx = b[i].x, by = b[i].y;
            const double ph = atan2(ay, ax) - atan2(by, bx);
            v = (kind == OBS_PHASE) ? ph : sqrt((ax * ax + ay * ay) * (bx * bx + by * by)) * sin(ph);
        }
        const double t = s + v;  // Neumaier
        comp += (fabs(s) >= fabs(v)) ? (s - t) + v : (v - t) + s;
        s = t;
    }
    sh_s[threadIdx.x] = s;
    sh_c[threadIdx.x] = comp;
    __syncthreads();
    if (threadIdx.x == 0) {
        double ts = 0.0, tc = 0.0;
        for (int k = 0; k < (int)blockDim.x; ++k) {
            const double v = sh_s[k];
            const double t = ts + v;
            tc += ((fabs(ts) >= fabs(v)) ? (ts - t) + v : (v - t) + ts) + sh_c[k];
            ts = t;
        }
        part[blockIdx.x] = ts + tc;
    }
}

// out[k] = sum over blocks of part[b][k], block order.
__global__ void k_ctrl_final(const double* part, int nblocks, int nv, double* out) {
    const int k = threadIdx.x;
    if (k >= nv) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += part[(long long)b * nv + k];
    out[k] = s;
}

// Spherical real-space cut-off factor of the dipolar kernel,
// c(q) = 1 + 3cos(q)/q^2 - 3sin(q)/q^3 = 3 int_0^q j2(x)/x dx.  Below q = 0.5
// the closed form cancels (relative error about 1e-16 * 30/q^4), so there the
// power series c(q) = 3 sum_n (-1)^n q^(2n+2) / ((2n+2) 2^n n! (2n+5)!!) is
// summed instead (eight terms: the first omitted one is below 1e-22 of c).
inline double dipolar_cutoff_factor(double q) {
    if (q >= 0.5) return 1.0 + 3.0 * std::cos(q) / (q * q) - 3.0 * std::sin(q) / (q * q * q);
    double sum = 0.0, pw = q * q, fact2n = 1.0, nfact = 1.0, dfact = 15.0;  // 2^n, n!, (2n+5)!!
    for (int n = 0; n < 8; ++n) {
        if (n > 0) {
            fact2n *= 2.0;
            nfact *= n;
            dfact *= (2.0 * n + 5.0);
            pw *= -q * q;
        }
        sum += pw / ((2.0 * n + 2.0) * fact2n * nfact * dfact);
    }
    return 3.0 * sum;
}

// Host copy of the dipolar kernel (see gpe_config docs / GPE_HAM_DIPOLAR),
// the unused DipoleDipoleInteraction of src/parallel.cu:326-352 with a
// spherical cut-off, divided by N for the unnormalised inverse FFT unless
// per_n is false (gpe_kspace_kernel returns the kernel itself).
void host_vdd(const gpe_config& c, const std::vector<double>* k, std::vector<double>& out, bool per_n = true) {
    const long long N = (long long)c.nx * c.ny * c.nz;
    out.assign(N, 0.0);
    if (c.hamiltonian == GPE_HAM_SOFT) {
        // SoftCoreInteraction_1D/2D/3D, src/parallel.cu:360-477 (a = prms[0],
        // U = prms[1], k = 2 pi |k|, small-k forms below 1e-6), / N
        const double a = c.prms[0], U = c.prms[1], pi = 3.141592653589793;
        for (int iz = 0; iz < c.nz; ++iz)
            for (int iy = 0; iy < c.ny; ++iy)
                for (int ix = 0; ix < c.nx; ++ix) {
                    const long long idx = ((long long)iz * c.ny + iy) * c.nx + ix;
                    const double kx = k[0][ix], ky = k[1][iy], kz = k[2][iz];
                    const double kk = 2 * pi * std::sqrt(kx * kx + ky * ky + kz * kz);
                    double v;
                    if (c.dim == 1)
                        v = kk < 1e-6 ? U * 2 * a * (1 - (a * kk) * (a * kk) / 6.0) : U * 2 * std::sin(a * kk) / kk;
                    else if (c.dim == 2)
                        v = kk < 1e-6 ? U * pi * a * a : 2 * pi * a * U * std::cyl_bessel_j(1.0, kk * a) / kk;
                    else
                        v = kk < 1e-6 ? U * (4. / 3.) * pi * std::pow(a, 3)
                                      : 4 * pi * U * std::pow(a, 3) * (std::sin(kk * a) - kk * a * std::cos(kk * a)) /
                                            std::pow(kk * a, 3);
                    out[idx] = per_n ? v / (double)N : v;
                }
        return;
    }
    const double add = c.prms[6];
    double d[3] = {c.prms[7], c.prms[8], c.prms[9]};
    const double dn = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (dn > 0)
        for (double& v : d) v /= dn;
    const double R = c.prms[10];
    const double pi = 3.141592653589793;
    for (int iz = 0; iz < c.nz; ++iz)
        for (int iy = 0; iy < c.ny; ++iy)
            for (int ix = 0; ix < c.nx; ++ix) {
                const long long idx = ((long long)iz * c.ny + iy) * c.nx + ix;
                const double kx = k[0][ix], ky = k[1][iy], kz = k[2][iz];
                const double num = kx * d[0] + ky * d[1] + kz * d[2];
                const double den = std::sqrt(kx * kx + ky * ky + kz * kz);
                double v = 0.0;
                if (den >= 1e-6) {
                    v = 12.0 * pi * add * ((num / den) * (num / den) - 1.0 / 3.0);
                    if (R > 0) {
                        const double q = 2.0 * pi * den * R;
                        v *= dipolar_cutoff_factor(q);
                    }
                }
                out[idx] = per_n ? v / (double)N : v;
            }
}

// x/k axes: BaseHamiltonian::InitializeKspace, src/baseHamiltonian.cu:53-82,
// with DKX, KXMAX of src/params.cu:206-211 (odd-N formula kept).
void host_kaxes(const gpe_config& c, std::vector<double>* k) {
    const int NX[3] = {c.nx, c.ny, c.nz};
    for (int d = 0; d < 3; ++d) {
        const int n = NX[d];
        const double DX = c.dx[d];
        const double DKX = 1.0 / (n * DX);
        const double KXMAX = 1.0 / (2.0 * DX);
        k[d].assign(n, 0.0);
        for (int ik = 0; ik <= n / 2 && ik < n; ++ik) k[d][ik] = (ik)*DKX;
        for (int ik = n / 2 + 1; ik < n; ++ik) k[d][ik] = -KXMAX + (ik - (n / 2)) * DKX;
        const bool zero = (c.dim == 1 && d > 0) || (c.dim == 2 && d == 2);
        if (zero)
            for (int i = 0; i < n; ++i) k[d][i] = 0.0;
    }
}

template <typename C>
void host_twiddles(int L, std::vector<C>& tw) {
    tw.resize(L);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int m = 0; m < L; ++m) {
        const long double a = -two_pi * (long double)m / (long double)L;
        tw[m].x = (decltype(tw[m].x))cosl(a);
        tw[m].y = (decltype(tw[m].y))sinl(a);
    }
}

// ---- pass chains -------------------------------------------------------------------------
template <typename R>
struct Ctx {
    typedef typename Cx<R>::T C;
    gpe_handle* h;
    C* A(int c) const { return (C*)h->A[c]; }
    C* B(int c) const { return (C*)h->B[c]; }
};

// Moving-frame term of the plugins' alg_calcHpsi (trotate): lambda = prms[11 + c],
// applied as - (lambda/N) kx in the kinetic multiplier where the reference
// adds alg_addVPx: heavy-ball imaginary steps, stage 4 of a one-component
// real-time step, apply-H and the observables.
template <typename R>
void set_rotation(gpe_handle* h, PassArgs<R>& a, bool on) {
    const bool plugin = h->cfg.hamiltonian != GPE_HAM_TEMPLATE;
    for (int c = 0; c < 2; ++c)
        a.rot[c] = (on && plugin && c < h->ncomp) ? h->cfg.prms[11 + c] / (double)h->N : 0.0;
}

template <typename R>
PassArgs<R> base_args(gpe_handle* h) {
    typedef typename Cx<R>::T C;
    PassArgs<R> a;
    std::memset(&a, 0, sizeof(a));
    a.nx = h->nx;
    a.ny = h->ny;
    a.nz = h->nz;
    a.nrows = h->ny * h->nz;
    a.ncomp = h->ncomp;
    a.dens = h->dens;
    for (int f = 0; f < 3; ++f) a.w[f] = (C*)h->W[f];
    for (int c = 0; c < 2; ++c) {
        a.buf[0][c] = (C*)h->A[c];
        a.buf[1][c] = (C*)h->B[c];
        a.kacc[c] = (C*)h->K[c];
        a.vext[c] = (const C*)h->V[c];
        a.pin[c] = (const C*)h->A[c];
    }
    a.twz = nullptr;
    a.kx = h->kax[0];
    a.ky = h->kax[1];
    a.kz = h->kax[2];
    for (int d = 0; d < 3; ++d) a.k2s[d] = h->k2s[d];
    a.vdd = (const R*)h->vdd;
    a.prms = h->prms;
    a.sc = h->sc;
    a.partials = h->partials;
    a.ham = h->cfg.hamiltonian;
    a.spec = SPEC_KIN;
    a.dt = h->cfg.dt;
    a.beta = h->cfg.beta;
    a.lap_scale = 19.739208802 / (double)h->N;  // src/parallel.cu:199
    a.DV = h->cfg.dx[0] * h->cfg.dx[1] * h->cfg.dx[2];
    a.eps = h->cfg.epsilon_e;
    a.npart[0] = h->cfg.npart[0];
    a.npart[1] = h->cfg.npart[1];
    a.nbatch = h->nb;
    a.bstride = h->nb > 1 ? h->N : 0;
    a.pstride = (long long)h->ny * h->nz * MAXQ * 2;
    a.xstage = h->xstage;
    return a;
}

cudaEvent_t take_event(gpe_handle* h) {
    if (!h->ev_free.empty()) {
        cudaEvent_t e = h->ev_free.back();
        h->ev_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Brackets one launch with events when profiling is on.
struct ProfScope {
    gpe_handle* h;
    int kind;
    cudaEvent_t a = nullptr;
    ProfScope(gpe_handle* h_, int kind_) : h(h_), kind(kind_) {
        if (h->prof) {
            a = take_event(h);
            cudaEventRecord(a, h->st);
        }
    }
    ~ProfScope() {
        if (a) {
            cudaEvent_t b = take_event(h);
            cudaEventRecord(b, h->st);
            h->recs.push_back(gpe_handle::Rec{kind, a, b});
        }
    }
};

int prof_kind(int mode) {
    switch (mode) {
        case XM_FWD: return 0;
        case XM_INV: return 1;
        case XM_FULL: return 2;
        case SM_FWD: return 3;
        case SM_INV: return 4;
        default: return 5;
    }
}

// x pass: `rows` lines of T threads per CTA (256 threads when the line allows),
// one padded shared-memory exchange row per line.
template <typename R>
gpe_status launch_x(gpe_handle* h, PassArgs<R> a, int nf, int mode) {
    typedef typename Cx<R>::T C;
    ProfScope ps(h, prof_kind(mode));
    a.mode = mode;
    a.tw = (const C*)h->tw[0];
    const int L = h->nx;
    const int T = plan_T(L);
    int rows = (256 / T) > 0 ? 256 / T : 1;
    if (h->xrows > 0 && h->xrows < rows) rows = h->xrows;
    const size_t smem = (size_t)rows * xpad(L) * sizeof(C);
    cudaError_t err = cudaSuccess;
    if (a.ham == GPE_HAM_USER && mode != XM_FWD && a.epi != EPI_STORE) {
        // the passes that evaluate the Hamiltonian run the user plugin's kernels
        if (!h->user) return fail(GPE_ERR_INVALID_ARG, "GPE_HAM_USER handle without gpe_set_user_hamiltonian");
        int e = 0;
        const int found = sizeof(R) == 4 ? h->user->launch_x_c64(L, &a, rows, smem, (void*)h->st, &e)
                                         : h->user->launch_x_c128(L, &a, rows, smem, (void*)h->st, &e);
        if (!found)
            return fail(GPE_ERR_UNSUPPORTED, "the user Hamiltonian plugin has no kernel for length " + std::to_string(L));
        err = (cudaError_t)e;
    } else if (!dispatch_x(L, nf, a, rows, smem, h->st, &err)) {
        return fail(GPE_ERR_UNSUPPORTED, "no x-pass kernel for length " + std::to_string(L));
    }
    if (err != cudaSuccess) return fail(GPE_ERR_CUDA, std::string("x pass launch: ") + cudaGetErrorString(err));
    h->launches++;
    return GPE_OK;
}

// Strided pass along y (axis 1) or z (axis 2): tx consecutive x values per
// CTA (spass_tx: 128-byte rows, 16 complex64 / 8 complex128 values, at most
// 256 threads); x blocks past nx are masked.
template <typename R>
gpe_status launch_s(gpe_handle* h, PassArgs<R> a, int nf, int axis, int mode) {
    typedef typename Cx<R>::T C;
    ProfScope ps(h, prof_kind(mode));
    const int L = axis == 1 ? h->ny : h->nz;
    const int tx = spass_tx(L, (int)sizeof(C));
    a.mode = mode;
    a.sax = axis;
    a.tx = tx;
    a.tw = (const C*)h->tw[axis];
    a.tw2 = h->tw2[axis];
    int nouter;
    if (axis == 1) {
        a.sstride = h->nx;
        a.ostride = (long long)h->nx * h->ny;
        nouter = h->nz;
    } else {
        a.sstride = (long long)h->nx * h->ny;
        a.ostride = h->nx;
        nouter = h->ny;
    }
    cudaError_t err = cudaSuccess;
    bool found = false;
    // pass variant (gpe_tune): 1 = paired complex64 lines at the default tile
    // (any length; two-field passes only where both fields' pairs fit the
    // register budget: 8 values per thread, lines of 64 or more); 2.. = the
    // tuned lengths' one-field variants; paired variants need an even nx
    const int mi = mode == SM_FWD ? 0 : (mode == SM_FKI ? 1 : 2);
    const int v = h->svar[axis][mi];
    if (v == 1 && sizeof(R) == 4 && h->nx % 2 == 0 && (nf == 1 || (make_plan(L).E <= 8 && L >= 64))) {
        if constexpr (sizeof(R) == 4)
            found = dispatch_s2(L, nf, a, nouter, (size_t)L * spass2_txp(L) * sizeof(float4), h->st, &err);
    } else if (v >= 2 && nf == 1 && (!svar((int)sizeof(C), L, v).paired || h->nx % 2 == 0)) {
        found = dispatch_sv(L, v, a, nouter, h->st, &err);
    }
    if (!found) found = dispatch_s(L, nf, a, nouter, (size_t)L * tx * sizeof(C), h->st, &err);
    if (!found) return fail(GPE_ERR_UNSUPPORTED, "no strided-pass kernel for length " + std::to_string(L));
    if (err != cudaSuccess) return fail(GPE_ERR_CUDA, std::string("strided pass launch: ") + cudaGetErrorString(err));
    h->launches++;
    return GPE_OK;
}

// Full kinetic chain: x-forward with prologue, strided forward passes, the
// last strided axis forward * k-space * inverse, strided inverse passes,
// x-inverse with epilogue.  a.pro / a.epi / a.stage ... are set by the caller.
// skip_fwd: W already holds the x-forward transform of the stage input.
// Whether the fused y-z cluster kernel can serve a chain of nf fields.
bool yz_usable(const gpe_handle* h, int nf) {
    return h->prec == GPE_C64 && nf == 1 && h->ny > 1 && h->nz > 1 && h->nx % YZ_XB_HOST == 0 &&
           yz_shape_supported(h->ny, h->nz);
}

// The fused y-z kernel in place of the three strided passes (profiled as
// pass kind 5).
template <typename R>
gpe_status launch_yz_chain(gpe_handle* h, PassArgs<R> a) {
    if constexpr (sizeof(R) == 4) {
        ProfScope ps(h, 5);
        a.tw = (const float2*)h->tw[1];
        a.twz = (const float2*)h->tw[2];
        cudaError_t err = cudaSuccess;
        if (!dispatch_yz(h->ny, h->nz, a, h->st, &err))
            return fail(GPE_ERR_UNSUPPORTED, "no fused y-z kernel for this grid");
        if (err != cudaSuccess) return fail(GPE_ERR_CUDA, std::string("y-z kernel launch: ") + cudaGetErrorString(err));
        h->launches++;
        return GPE_OK;
    } else {
        (void)a;
        return fail(GPE_ERR_UNSUPPORTED, "the fused y-z kernel is complex64 only");
    }
}

bool flow_strided_usable(const gpe_handle* h, int nf);
gpe_status launch_flow_strided(gpe_handle* h, const PassArgs<float>& a);

template <typename R>
gpe_status run_chain(gpe_handle* h, const PassArgs<R>& a, int nf, bool skip_fwd = false) {
    int axes[2], na = 0;
    if (h->ny > 1) axes[na++] = 1;
    if (h->nz > 1) axes[na++] = 2;
    if (na == 0) return launch_x<R>(h, a, nf, XM_FULL);
    if (!skip_fwd) GPE_TRY(launch_x<R>(h, a, nf, XM_FWD));
    if (h->yz && yz_usable(h, nf)) {
        GPE_TRY(launch_yz_chain<R>(h, a));
        return launch_x<R>(h, a, nf, XM_INV);
    }
    if constexpr (sizeof(R) == 4) {
        if (na == 2 && flow_strided_usable(h, nf)) {
            GPE_TRY(launch_flow_strided(h, a));
            return launch_x<R>(h, a, nf, XM_INV);
        }
    }
    for (int i = 0; i < na - 1; ++i) GPE_TRY(launch_s<R>(h, a, nf, axes[i], SM_FWD));
    GPE_TRY(launch_s<R>(h, a, nf, axes[na - 1], SM_FKI));
    for (int i = na - 2; i >= 0; --i) GPE_TRY(launch_s<R>(h, a, nf, axes[i], SM_INV));
    return launch_x<R>(h, a, nf, XM_INV);
}

gpe_status sync_read_scalars(gpe_handle* h, DevScalars* out) {
    GPE_CUDA(cudaMemcpyAsync(out, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->st));
    GPE_CUDA(cudaStreamSynchronize(h->st));
    return GPE_OK;
}

// Synchronise and report a device-side error recorded by a kernel (bounded
// wait expired, non-finite reduction).
gpe_status check_device_status(gpe_handle* h) {
    DevScalars s;
    GPE_TRY(sync_read_scalars(h, &s));
    if (s.status == GPE_ERR_TIMEOUT) return fail(GPE_ERR_TIMEOUT, "a bounded device wait expired");
    if (s.status == GPE_ERR_DIVERGED) return fail(GPE_ERR_DIVERGED, "non-finite norm, energy or chemical potential");
    return GPE_OK;
}

template <typename R>
gpe_status canonicalize_t(gpe_handle* h) {
    typedef typename Cx<R>::T C;
    if (h->mode == ST_CANON) return GPE_OK;
    h->w_fwd_A = false;
    h->lo_valid = false;
    const int thr = 256;
    for (int i = 0; i < h->nb; ++i) {
        for (int c = 0; c < h->ncomp; ++c) {
            k_canon<C><<<blocks_for(h->N, thr), thr, 0, h->st>>>((C*)h->A[c] + i * h->N, (C*)h->B[c] + i * h->N,
                                                                 h->sc + i, c, h->mode == ST_HB, h->N);
            h->launches++;
        }
        k_reset_scales<<<1, 1, 0, h->st>>>(h->sc + i);
        h->launches++;
    }
    GPE_CUDA(cudaGetLastError());
    if (h->mode == ST_RKI) h->hb_old_valid = false;
    h->mode = ST_CANON;
    return GPE_OK;
}

gpe_status canonicalize(gpe_handle* h) {
    return h->prec == GPE_C64 ? canonicalize_t<float>(h) : canonicalize_t<double>(h);
}

template <typename R>
gpe_status copy_field(gpe_handle* h, void* dst, const void* src) {
    typedef typename Cx<R>::T C;
    k_copy<C><<<blocks_for(h->N * h->nb, 256), 256, 0, h->st>>>((C*)dst, (const C*)src, h->N * h->nb);
    h->launches++;
    GPE_CUDA(cudaGetLastError());
    return GPE_OK;
}

// Whether real-time steps of this handle run as one persistent launch per
// step (k_flow_step, gpe_flow.cuh): complex64, one component and one
// transformed field, a built-in pointwise Hamiltonian, a cubic grid the
// kernel is compiled for, and the option on (gpe_set_flow or the tuner).
bool flow_eligible(const gpe_handle* h) {
    return h->prec == GPE_C64 && h->ncomp == 1 && h->nf == 1 && h->nb == 1 &&
           (h->cfg.hamiltonian == GPE_HAM_BEC || h->cfg.hamiltonian == GPE_HAM_TEMPLATE) && h->nx % 2 == 0 &&
           flow_shape_supported(h->nx, h->ny, h->nz);
}
bool flow_usable(const gpe_handle* h) { return h->flow == 1 && h->flow_sync && flow_eligible(h); }
// Mode 2: the strided passes of a one-field complex64 chain on a cubic grid
// the kernel is compiled for (any epilogue: the x passes keep their launches).
bool flow_strided_usable(const gpe_handle* h, int nf) {
    return h->flow == 2 && h->flow_sync && h->prec == GPE_C64 && nf == 1 && h->nb == 1 && h->nx % 2 == 0 &&
           flow_shape_supported(h->nx, h->ny, h->nz);
}

// Switches the persistent step on (allocating and zeroing its counters) or
// off; bound = 0 keeps the current wait bound.
gpe_status flow_enable(gpe_handle* h, int on, unsigned bound) {
    if (bound) h->flow_bound = bound;
    h->flow = on;
    if (!on) return GPE_OK;
    if (!h->flow_sync) GPE_CUDA(cudaMalloc((void**)&h->flow_sync, sizeof(FlowSync)));
    GPE_CUDA(cudaMemsetAsync(h->flow_sync, 0, sizeof(FlowSync), h->st));
    h->flow_launches = 0;
    return GPE_OK;
}

// The arguments launch_s would give the y forward, z forward * k-space *
// inverse and y inverse passes of a chain with arguments a.
void flow_strided_args(const gpe_handle* h, const PassArgs<float>& a0, FlowArgs& fa) {
    const int modes[3] = {SM_FWD, SM_FKI, SM_INV};
    for (int m = 0; m < 3; ++m) {
        PassArgs<float> a = a0;
        const int axis = m == 1 ? 2 : 1;
        a.mode = modes[m];
        a.sax = axis;
        a.tx = spass_tx(axis == 1 ? h->ny : h->nz, (int)sizeof(float2));
        a.tw = (const float2*)h->tw[axis];
        a.tw2 = h->tw2[axis];
        a.sstride = axis == 1 ? (long long)h->nx : (long long)h->nx * h->ny;
        a.ostride = axis == 1 ? (long long)h->nx * h->ny : (long long)h->nx;
        fa.s[m] = a;
    }
}

// The three strided passes of a one-field complex64 chain as one launch.
gpe_status launch_flow_strided(gpe_handle* h, const PassArgs<float>& a) {
    ProfScope ps(h, GPE_PROF_SFLOW);
    FlowArgs fa;
    std::memset(&fa, 0, sizeof(fa));
    flow_strided_args(h, a, fa);
    fa.sync = h->flow_sync;
    fa.set = (int)(h->flow_launches & 1);
    fa.ntx = flow_ntx(h->nx);
    fa.wait_bound = h->flow_bound;
    int dev = 0, sms = 0;
    GPE_CUDA(cudaGetDevice(&dev));
    GPE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int per_sm = flow_strided_ctas_per_sm(h->nx);
    if (per_sm < 1) return fail(GPE_ERR_CUDA, "persistent strided stage: no resident CTA");
    cudaError_t err = cudaSuccess;
    if (!dispatch_flow_strided(h->nx, fa, sms * per_sm, h->st, &err))
        return fail(GPE_ERR_UNSUPPORTED, "no persistent strided-stage kernel for this grid");
    if (err != cudaSuccess)
        return fail(GPE_ERR_CUDA, std::string("persistent strided-stage launch: ") + cudaGetErrorString(err));
    h->flow_launches++;
    h->launches++;
    return GPE_OK;
}

// One real-time RK4 step as one launch: the strided passes take the
// arguments launch_s would give them, the x tiles those of launch_x with the
// fused stage epilogue (sa[s-1]: the arguments of stage s).
template <typename R>
gpe_status launch_flow_step(gpe_handle* h, const PassArgs<R> (&sa)[4], bool obs) {
    if constexpr (sizeof(R) == 4) {
        ProfScope ps(h, GPE_PROF_FLOW);
        FlowArgs fa;
        std::memset(&fa, 0, sizeof(fa));
        flow_strided_args(h, sa[0], fa);
        for (int s = 0; s < 4; ++s) {
            fa.x[s] = sa[s];
            fa.x[s].mode = XM_INV;
            fa.x[s].tw = (const float2*)h->tw[0];
        }
        fa.sync = h->flow_sync;
        fa.set = (int)(h->flow_launches & 1);
        fa.ntx = flow_ntx(h->nx);
        fa.rows = flow_rows(h->nx);
        fa.wait_bound = h->flow_bound;
        int dev = 0, sms = 0;
        GPE_CUDA(cudaGetDevice(&dev));
        GPE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const int per_sm = flow_ctas_per_sm(h->nx);
        if (per_sm < 1) return fail(GPE_ERR_CUDA, "persistent step kernel: no resident CTA");
        cudaError_t err = cudaSuccess;
        if (!dispatch_flow(h->nx, obs, fa, sms * per_sm, h->st, &err))
            return fail(GPE_ERR_UNSUPPORTED, "no persistent step kernel for this grid");
        if (err != cudaSuccess) return fail(GPE_ERR_CUDA, std::string("persistent step launch: ") + cudaGetErrorString(err));
        h->flow_launches++;
        h->launches++;
        return GPE_OK;
    } else {
        (void)h;
        (void)sa;
        (void)obs;
        return fail(GPE_ERR_UNSUPPORTED, "the persistent step kernel is complex64 only");
    }
}

// ---- stepping ----------------------------------------------------------------------------
// compensate: complex64 handles carry the step state as high (A) + low (Lo)
// parts across steps and calls (rk_final_comp); off for the control
// gradient, whose checkpoints hold A alone.
template <typename R>
gpe_status step_real_t(gpe_handle* h, int first, int nsteps, double* obs_out, bool compensate = true) {
    typedef typename Cx<R>::T C;
    GPE_TRY(canonicalize_t<R>(h));
    h->hb_old_valid = false;
    const double dt = h->cfg.dt;
    PassArgs<R> a = base_args<R>(h);
    a.epi = EPI_RK;
    a.pro = PRO_PIN;
    if (sizeof(R) == 4 && h->Lo[0] != nullptr) {
        if (compensate) {
            if (!h->lo_valid)
                for (int c = 0; c < h->ncomp; ++c) GPE_CUDA(cudaMemsetAsync(h->Lo[c], 0, h->esz * h->N, h->st));
            h->lo_valid = true;
            for (int c = 0; c < h->ncomp; ++c) a.lo[c] = (C*)h->Lo[c];
        } else {
            h->lo_valid = false;
        }
    }
    // Each stage's x-inverse epilogue also x-forward transforms the state it
    // writes (the next stage's input) unless it runs the logging reductions;
    // the next stage then starts at the strided passes.
    const bool can_fuse = h->ny > 1 || h->nz > 1;
    bool w_ready = can_fuse && h->w_fwd_A;
    h->w_fwd_A = false;
    // the arguments of stage s of step `it` (the chain's and the persistent
    // step kernel's alike)
    auto stage_args = [&](PassArgs<R>& sa, int s, int it, bool want_obs) {
        sa.stage = s;
        for (int c = 0; c < 2; ++c) sa.pin[c] = (s == 1) ? (const C*)h->A[c] : (const C*)h->B[c];
        // src/oneComponentGPSolver.cu:137-138,155,175,184: m05Idt, mIdt and PARS[T]
        sa.c_re = 0.0;
        sa.c_im = (s <= 2) ? -0.5 * dt : -1.0 * dt;
        sa.t = (s == 1) ? (double)it * dt : (s < 4) ? (it + 0.5) * dt : (double)(it + 1) * dt;
        sa.want_obs = (want_obs && s == 4) ? 1 : 0;
        sa.fuse_fwd = (can_fuse && !sa.want_obs) ? 1 : 0;
        // stages 1-3 use alg_calcHpsiMU, stage 4 alg_calcHpsi
        // (src/oneComponentGPSolver.cu:170-190)
        set_rotation<R>(h, sa, s == 4 && h->ncomp == 1);
    };
    const bool flow = flow_usable(h);
    for (int j = 0; j < nsteps; ++j) {
        const int it = first + j;
        const bool obs_step = obs_out != nullptr && j == nsteps - 1;
        if (flow) {
            PassArgs<R> sa[4] = {a, a, a, a};
            for (int s = 1; s <= 4; ++s) stage_args(sa[s - 1], s, it, obs_step);
            if (sa[3].rot[0] == 0.0) {  // the moving-frame term runs on the chain
                if (!w_ready) GPE_TRY(launch_x<R>(h, sa[0], h->nf, XM_FWD));
                GPE_TRY(launch_flow_step<R>(h, sa, obs_step));
                w_ready = !obs_step;
                continue;
            }
        }
        for (int s = 1; s <= 4; ++s) {
            stage_args(a, s, it, obs_step);
            GPE_TRY(run_chain<R>(h, a, h->nf, w_ready));
            w_ready = a.fuse_fwd != 0;
        }
    }
    h->w_fwd_A = w_ready;
    if (obs_out && nsteps > 0) {
        DevScalars s;
        GPE_TRY(sync_read_scalars(h, &s));
        for (int q = 0; q < 3 * h->ncomp; ++q) obs_out[q] = s.obs[q];
        if (s.status == GPE_ERR_TIMEOUT) return fail(GPE_ERR_TIMEOUT, "a bounded device wait expired");
        if (s.status == GPE_ERR_DIVERGED) return fail(GPE_ERR_DIVERGED, "non-finite observable");
    }
    return GPE_OK;
}

// State-mode switch before imaginary-time iterations: RK4 keeps psi in A with
// a lazy scale; heavy ball needs psi_old in B.
template <typename R>
gpe_status imag_prepare(gpe_handle* h) {
    h->w_fwd_A = false;
    h->lo_valid = false;
    const bool rk = h->cfg.imag_scheme == GPE_IMAG_RK4;
    if (rk) {
        if (h->mode == ST_HB) GPE_TRY(canonicalize_t<R>(h));
        h->mode = ST_RKI;
    } else {
        if (h->mode == ST_RKI) GPE_TRY(canonicalize_t<R>(h));
        if (!h->hb_old_valid) {
            GPE_TRY(canonicalize_t<R>(h));
            for (int c = 0; c < h->ncomp; ++c) GPE_TRY(copy_field<R>(h, h->B[c], h->A[c]));
            h->hb_old_valid = true;
        }
        h->mode = ST_HB;
    }
    // Reset the per-call iteration counters.
    k_reset_iters<<<blocks_for(h->nb, 128), 128, 0, h->st>>>(h->sc, h->nb);
    h->launches++;
    GPE_CUDA(cudaGetLastError());
    return GPE_OK;
}

// Launches nsteps imaginary-time iterations (no synchronisation).
template <typename R>
gpe_status imag_issue(gpe_handle* h, int first, int nsteps) {
    typedef typename Cx<R>::T C;
    const double dt = h->cfg.dt;
    const bool rk = h->cfg.imag_scheme == GPE_IMAG_RK4;
    PassArgs<R> a = base_args<R>(h);
    a.check_done = 1;
    for (int j = 0; j < nsteps; ++j) {
        const int it = first + j;
        a.t = (double)it * dt;  // src/oneComponentGPSolver.cu:52 PARS[T] = iteration*dt
        if (!rk) {
            a.pro = PRO_CUR;
            a.epi = EPI_HB;
            a.stage = 0;
            set_rotation<R>(h, a, true);  // src/oneComponentGPSolver.cu:62 alg_calcHpsi
            GPE_TRY(run_chain<R>(h, a, h->nf));
        } else {
            // Stages 1-3 x-forward transform the stage state they write (the
            // next stage's input, XK_RKIF); stage 1 keeps its own x-forward
            // pass, whose prologue applies the renormalisation scale that
            // stage 4's reduction sets.
            const bool can_fuse = h->ny > 1 || h->nz > 1;
            bool w_ready = false;
            for (int s = 1; s <= 4; ++s) {
                a.epi = EPI_RKI;
                a.stage = s;
                a.pro = (s == 1) ? PRO_A_SCALED : PRO_PIN;
                for (int c = 0; c < 2; ++c) a.pin[c] = (const C*)h->B[c];
                a.c_re = (s <= 2) ? -0.5 * dt : -1.0 * dt;
                a.c_im = 0.0;
                a.fuse_fwd = (can_fuse && s < 4) ? 1 : 0;
                GPE_TRY(run_chain<R>(h, a, h->nf, w_ready));
                w_ready = a.fuse_fwd != 0;
            }
            a.fuse_fwd = 0;
        }
    }
    return GPE_OK;
}

// Imaginary-time iterations are issued in chunks of IMAG_CHUNK.  After each
// chunk an asynchronous copy of the device's done flag (convergence or error)
// lands in pinned host memory; the host reads the flag of a chunk while the
// next chunk is already queued, and stops issuing once it is set.  So the
// device never idles between chunks, and a call that converges early issues
// at most one chunk past the converging iteration (whose kernels exit at
// once on the flag) instead of every requested iteration.
constexpr int IMAG_CHUNK = 64;

template <typename R>
gpe_status step_imag_t(gpe_handle* h, int first, int nsteps, int* iters_done, int* converged) {
    GPE_TRY(imag_prepare<R>(h));
    int issued = 0, slot = 0, prev = -1;
    while (issued < nsteps) {
        const int n = std::min(IMAG_CHUNK, nsteps - issued);
        GPE_TRY(imag_issue<R>(h, first + issued, n));
        issued += n;
        if (issued >= nsteps) break;
        GPE_CUDA(cudaMemcpyAsync(h->flag_host + slot, &h->sc->done, sizeof(int), cudaMemcpyDeviceToHost, h->st));
        GPE_CUDA(cudaEventRecord(h->flag_ev[slot], h->st));
        if (prev >= 0) {
            GPE_CUDA(cudaEventSynchronize(h->flag_ev[prev]));
            if (h->flag_host[prev]) break;
        }
        prev = slot;
        slot ^= 1;
    }
    DevScalars s;
    GPE_TRY(sync_read_scalars(h, &s));
    if (iters_done) *iters_done = s.iters_done;
    if (converged) *converged = s.converged;
    if (s.status == GPE_ERR_DIVERGED) return fail(GPE_ERR_DIVERGED, "non-finite norm, energy or chemical potential");
    if (s.status == GPE_ERR_TIMEOUT) return fail(GPE_ERR_TIMEOUT, "a bounded device wait expired");
    return GPE_OK;
}

template <typename R>
gpe_status apply_chain_t(gpe_handle* h, int epi, double t, int comp_only, int spec = SPEC_KIN) {
    h->w_fwd_A = false;
    GPE_TRY(canonicalize_t<R>(h));
    PassArgs<R> a = base_args<R>(h);
    a.pro = PRO_PIN;
    a.epi = epi;
    a.t = t;
    a.spec = spec;
    if (spec == SPEC_PX) a.ham = GPE_HAM_TEMPLATE;
    int nf = h->nf;
    if (comp_only >= 0) {  // single component, kinetic only (Laplace / FFT tools)
        a.ncomp = 1;
        a.dens = 0;
        a.pin[0] = (const typename Cx<R>::T*)h->A[comp_only];
        nf = 1;
    }
    for (int q = 0; q < 4; ++q) a.out[q] = (typename Cx<R>::T*)h->O[q];
    // alg_calcHpsi (both outputs) carries the moving-frame term, alg_Laplace
    // and alg_calcPx do not
    set_rotation<R>(h, a, comp_only < 0 && spec == SPEC_KIN && (epi == EPI_APPLYH || epi == EPI_OBS));
    return run_chain<R>(h, a, nf);
}

template <typename R>
gpe_status fft_t(gpe_handle* h, int comp, int sign) {
    h->w_fwd_A = false;
    h->lo_valid = false;
    typedef typename Cx<R>::T C;
    GPE_TRY(canonicalize_t<R>(h));
    PassArgs<R> a = base_args<R>(h);
    a.ncomp = 1;
    a.dens = 0;
    a.pin[0] = (const C*)h->A[comp];
    a.w[0] = (C*)h->A[comp];
    a.pro = PRO_PIN;
    a.epi = EPI_STORE;
    int axes[2], na = 0;
    if (h->ny > 1) axes[na++] = 1;
    if (h->nz > 1) axes[na++] = 2;
    if (sign < 0) {
        GPE_TRY(launch_x<R>(h, a, 1, XM_FWD));
        for (int i = 0; i < na; ++i) GPE_TRY(launch_s<R>(h, a, 1, axes[i], SM_FWD));
    } else {
        for (int i = na - 1; i >= 0; --i) GPE_TRY(launch_s<R>(h, a, 1, axes[i], SM_INV));
        GPE_TRY(launch_x<R>(h, a, 1, XM_INV));
    }
    h->hb_old_valid = false;
    return GPE_OK;
}

gpe_status check_handle(gpe_handle* h) {
    if (!h) return fail(GPE_ERR_INVALID_ARG, "null handle");
    return GPE_OK;
}
gpe_status check_comp(gpe_handle* h, int comp) {
    if (comp < 0 || comp >= h->ncomp) return fail(GPE_ERR_INVALID_ARG, "component index out of range");
    return GPE_OK;
}

// Device c128 pointer -> state buffer of comp (conversion for complex64).
gpe_status upload_c128_device(gpe_handle* h, int comp, const void* dev_c128, void* dst) {
    if (h->prec == GPE_C128) {
        GPE_CUDA(cudaMemcpyAsync(dst, dev_c128, 16 * h->N, cudaMemcpyDeviceToDevice, h->st));
    } else {
        k_from_c128<float2><<<blocks_for(h->N, 256), 256, 0, h->st>>>((float2*)dst, (const double2*)dev_c128, h->N);
        h->launches++;
        GPE_CUDA(cudaGetLastError());
    }
    (void)comp;
    return GPE_OK;
}

gpe_status upload_c128_host(gpe_handle* h, const double* host, void* dst) {
    if (h->prec == GPE_C128) {
        GPE_CUDA(cudaMemcpyAsync(dst, host, 16 * h->N, cudaMemcpyHostToDevice, h->st));
        GPE_CUDA(cudaStreamSynchronize(h->st));
        return GPE_OK;
    }
    GPE_CUDA(cudaMemcpyAsync(h->stage128, host, 16 * h->N, cudaMemcpyHostToDevice, h->st));
    GPE_TRY(upload_c128_device(h, 0, h->stage128, dst));
    GPE_CUDA(cudaStreamSynchronize(h->st));
    return GPE_OK;
}

// lo: low part added to a complex64 source (the compensated state), or null.
gpe_status download_c128_host(gpe_handle* h, const void* src, double* host, const void* lo = nullptr) {
    if (h->prec == GPE_C128) {
        GPE_CUDA(cudaMemcpyAsync(host, src, 16 * h->N, cudaMemcpyDeviceToHost, h->st));
    } else {
        if (lo)
            k_to_c128_hilo<<<blocks_for(h->N, 256), 256, 0, h->st>>>((double2*)h->stage128, (const float2*)src,
                                                                     (const float2*)lo, h->N);
        else
            k_to_c128<float2><<<blocks_for(h->N, 256), 256, 0, h->st>>>((double2*)h->stage128, (const float2*)src,
                                                                        h->N);
        h->launches++;
        GPE_CUDA(cudaGetLastError());
        GPE_CUDA(cudaMemcpyAsync(host, h->stage128, 16 * h->N, cudaMemcpyDeviceToHost, h->st));
    }
    GPE_CUDA(cudaStreamSynchronize(h->st));
    return GPE_OK;
}

// After psi of component comp was stored as complex64 from the complex128
// array src (device): its rounding residual becomes the low part, so the
// compensated state equals the input; the other components' low parts are
// zeroed if they were not valid.
gpe_status set_low_part(gpe_handle* h, int comp, const void* src_c128) {
    if (!h->Lo[comp]) return GPE_OK;
    if (!h->lo_valid)
        for (int c = 0; c < h->ncomp; ++c) GPE_CUDA(cudaMemsetAsync(h->Lo[c], 0, h->esz * h->N, h->st));
    k_lo_residual<<<blocks_for(h->N, 256), 256, 0, h->st>>>((float2*)h->Lo[comp], (const float2*)h->A[comp],
                                                             (const double2*)src_c128, h->N);
    h->launches++;
    GPE_CUDA(cudaGetLastError());
    h->lo_valid = true;
    return GPE_OK;
}

gpe_status ensure_out_buffers(gpe_handle* h) {
    for (int q = 0; q < 2 * h->ncomp; ++q)
        if (!h->O[q]) GPE_CUDA(cudaMalloc(&h->O[q], h->esz * h->N));
    return GPE_OK;
}

void free_all(gpe_handle* h) {
    void* ptrs[] = {h->A[0], h->A[1], h->B[0], h->B[1], h->K[0], h->K[1], h->V[0], h->V[1], h->W[0], h->W[1],
                    h->W[2], h->O[0], h->O[1], h->O[2], h->O[3], h->tw[0], h->tw[1], h->tw[2], h->tw2[0],
                    h->tw2[1], h->tw2[2], h->kax[0],
                    h->kax[1], h->kax[2], h->vdd, h->prms, h->sc, h->partials, h->stage128, h->Lo[0], h->Lo[1],
                    h->k2s[0], h->k2s[1], h->k2s[2], h->obs_part};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    void* cptrs[] = {h->ctrlG, h->V0, h->adj[0], h->adj[1], h->adj[2], h->adj[3], h->adj[4], h->adj[5], h->adj[6],
                     h->qf, h->d_u, h->d_part, h->d_grad, h->flow_sync};
    for (void* p : cptrs)
        if (p) cudaFree(p);
    for (void* p : h->cps)
        if (p) cudaFree(p);
    for (void* p : h->cps_lo)
        if (p) cudaFree(p);
    if (h->flag_host) cudaFreeHost(h->flag_host);
    for (cudaEvent_t e : h->flag_ev)
        if (e) cudaEventDestroy(e);
    for (auto& r : h->recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : h->ev_free) cudaEventDestroy(e);
}

}  // namespace

// ==========================================================================================
extern "C" {

int gpe_abi_version(void) { return GPE_ABI_VERSION; }

const char* gpe_last_error_string(void) { return g_err.c_str(); }

const char* gpe_status_string(gpe_status s) {
    switch (s) {
        case GPE_OK: return "ok";
        case GPE_ERR_INVALID_ARG: return "invalid argument";
        case GPE_ERR_UNSUPPORTED: return "unsupported";
        case GPE_ERR_CUDA: return "CUDA error";
        case GPE_ERR_OUT_OF_MEMORY: return "out of memory";
        case GPE_ERR_DIVERGED: return "diverged";
        case GPE_ERR_TIMEOUT: return "timeout";
        case GPE_ERR_IO: return "I/O error";
    }
    return "unknown status";
}

gpe_status gpe_config_init(gpe_config* cfg) {
    if (!cfg) return fail(GPE_ERR_INVALID_ARG, "null config");
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->abi_version = GPE_ABI_VERSION;
    cfg->nx = cfg->ny = cfg->nz = 1;
    cfg->dim = 1;
    cfg->dx[0] = cfg->dx[1] = cfg->dx[2] = 1.0;
    cfg->ncomp = 1;
    cfg->precision = GPE_C128;
    cfg->hamiltonian = GPE_HAM_BEC;
    cfg->imag_scheme = GPE_IMAG_HEAVYBALL;
    cfg->npart[0] = cfg->npart[1] = 1.0;
    return GPE_OK;
}

int gpe_fft_length_supported(int n) { return (n >= 1 && make_plan(n).ok && length_compiled(n)) ? 1 : 0; }

gpe_status gpe_kspace_kernel(const gpe_config* cfg, double* out) {
    if (!cfg || !out) return fail(GPE_ERR_INVALID_ARG, "null argument");
    if (cfg->abi_version != GPE_ABI_VERSION) return fail(GPE_ERR_INVALID_ARG, "abi_version mismatch");
    if (cfg->hamiltonian != GPE_HAM_DIPOLAR && cfg->hamiltonian != GPE_HAM_SOFT)
        return fail(GPE_ERR_INVALID_ARG, "the k-space kernel exists for GPE_HAM_DIPOLAR and GPE_HAM_SOFT only");
    if (cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1) return fail(GPE_ERR_INVALID_ARG, "grid sizes must be >= 1");
    std::vector<double> kax[3], v;
    host_kaxes(*cfg, kax);
    host_vdd(*cfg, kax, v, false);
    std::memcpy(out, v.data(), sizeof(double) * v.size());
    return GPE_OK;
}

}  // extern "C"

namespace {

// ---- control gradient (the adjoint of the controlled real-time RK4 step) -----------------
// One controlled step n: V <- V0 + sum_k u[n,k] G_k, then the real-time RK4
// step of gpe_step_real.
template <typename R>
gpe_status ctrl_form_v(gpe_handle* h, int n) {
    typedef typename Cx<R>::T C;
    k_form_control_v<C, R><<<blocks_for(h->N, 256), 256, 0, h->st>>>((C*)h->V[0], (const C*)h->V0,
                                                                      (const R*)h->ctrlG, h->d_u + (size_t)n * h->nctrl,
                                                                      h->nctrl, h->N);
    h->launches++;
    GPE_CUDA(cudaGetLastError());
    return GPE_OK;
}

// Stage arguments of step n from psi_n = S: Pa, Pb, Pc (RK stages 1-3 with
// their states written to separate fields).
template <typename R>
gpe_status ctrl_stage_args(gpe_handle* h, void* S, void* Pa, void* Pb, void* Pc, int n) {
    typedef typename Cx<R>::T C;
    const double dt = h->cfg.dt;
    PassArgs<R> a = base_args<R>(h);
    a.epi = EPI_RK;
    a.pro = PRO_PIN;
    a.buf[0][0] = (C*)S;
    void* outs[3] = {Pa, Pb, Pc};
    const bool can_fuse = h->ny > 1 || h->nz > 1;
    bool w_ready = false;
    for (int s = 1; s <= 3; ++s) {
        a.stage = s;
        a.pin[0] = (const C*)(s == 1 ? S : outs[s - 2]);
        a.buf[1][0] = (C*)outs[s - 1];
        a.c_re = 0.0;
        a.c_im = (s <= 2) ? -0.5 * dt : -1.0 * dt;
        a.t = (s == 1) ? (double)n * dt : (n + 0.5) * dt;
        a.want_obs = 0;
        a.fuse_fwd = (can_fuse && s < 3) ? 1 : 0;
        GPE_TRY(run_chain<R>(h, a, h->nf, w_ready));
        w_ready = a.fuse_fwd != 0;
    }
    h->w_fwd_A = false;
    return GPE_OK;
}

// Reverse of step n: lambda (adj[0]) <- lambda_n, q (qf) <- gradient density.
template <typename R>
gpe_status ctrl_adjoint_step(gpe_handle* h, void* S, void* Pa, void* Pb, void* Pc, int n) {
    typedef typename Cx<R>::T C;
    const double dt = h->cfg.dt;
    C* lam = (C*)h->adj[0];
    C* acc = (C*)h->adj[1];
    C* mu = (C*)h->adj[2];
    k_cscale<C><<<blocks_for(h->N, 256), 256, 0, h->st>>>(mu, lam, dt / 6.0, 0.0, h->N);
    h->launches++;
    PassArgs<R> a = base_args<R>(h);
    a.epi = EPI_ADJ;
    a.pro = PRO_PIN;
    a.pin[0] = mu;
    a.buf[1][0] = mu;
    a.kacc[0] = acc;
    a.out[0] = lam;
    a.out[1] = (C*)h->qf;
    void* args[5] = {nullptr, S, Pa, Pb, Pc};  // psi_s of stage s
    const double cl[5] = {0.0, 0.0, dt / 6.0, dt / 3.0, dt / 3.0};   // lambda coefficient of the next mu
    const double cj[5] = {0.0, 0.0, 0.5 * dt, 0.5 * dt, dt};         // jt coefficient of the next mu
    for (int s = 4; s >= 1; --s) {
        a.stage = s;
        a.buf[0][0] = (C*)args[s];
        a.c_re = cl[s];
        a.c_im = cj[s];
        a.t = (s == 1) ? (double)n * dt : (s < 4) ? (n + 0.5) * dt : (double)(n + 1) * dt;
        GPE_TRY(run_chain<R>(h, a, h->nf));
    }
    h->w_fwd_A = false;
    GPE_CUDA(cudaGetLastError());
    return GPE_OK;
}

// grad[n*nctrl + k] = sum_x G_k(x) q(x), FP64, on the device.
template <typename R>
gpe_status ctrl_reduce_grad(gpe_handle* h, int n) {
    typedef typename Cx<R>::T C;
    k_ctrl_partials<C, R><<<CTRL_BLOCKS, 256, 0, h->st>>>(1, nullptr, nullptr, (const R*)h->qf, (const R*)h->ctrlG,
                                                         h->nctrl, h->N, h->d_part);
    k_ctrl_final<<<1, 64, 0, h->st>>>(h->d_part, CTRL_BLOCKS, h->nctrl, h->d_grad + (size_t)n * h->nctrl);
    h->launches += 2;
    GPE_CUDA(cudaGetLastError());
    return GPE_OK;
}

// complex64: the forward steps carry the compensated state (high part in A,
// low part in Lo, as gpe_step_real does), and the checkpoints keep both
// parts; the stage arguments of the adjoint are the high parts, as in the
// forward step.
template <typename R>
gpe_status control_gradient_t(gpe_handle* h, const double* host_u, int nsteps, const double* host_target, int K,
                              double* loss_out, double* host_grad) {
    typedef typename Cx<R>::T C;
    GPE_TRY(canonicalize_t<R>(h));
    h->w_fwd_A = false;
    h->hb_old_valid = false;
    const bool comp = sizeof(R) == 4 && h->Lo[0] != nullptr;
    if (comp && !h->lo_valid) {
        GPE_CUDA(cudaMemsetAsync(h->Lo[0], 0, h->esz * h->N, h->st));
        h->lo_valid = true;
    }
    const size_t fb = h->esz * h->N;
    const int ncp = (nsteps + K - 1) / K + 1;
    // buffers: u, grad, partials, work fields, checkpoints (kept for reuse)
    cudaFree(h->d_u);
    cudaFree(h->d_grad);
    h->d_u = h->d_grad = nullptr;
    GPE_CUDA(cudaMalloc((void**)&h->d_u, sizeof(double) * (size_t)nsteps * h->nctrl + 8));
    GPE_CUDA(cudaMalloc((void**)&h->d_grad, sizeof(double) * (size_t)nsteps * h->nctrl + 8));
    if (!h->d_part) GPE_CUDA(cudaMalloc((void**)&h->d_part, sizeof(double) * CTRL_BLOCKS * 64));
    if (!h->qf) GPE_CUDA(cudaMalloc(&h->qf, sizeof(R) * h->N));
    for (int i = 0; i < 7; ++i)
        if (!h->adj[i]) GPE_CUDA(cudaMalloc(&h->adj[i], fb));
    const int nstore = ncp + K + 1;
    while ((int)h->cps.size() < nstore) {
        void* p = nullptr;
        GPE_CUDA(cudaMalloc(&p, fb));
        h->cps.push_back(p);
    }
    while (comp && (int)h->cps_lo.size() < ncp) {
        void* p = nullptr;
        GPE_CUDA(cudaMalloc(&p, fb));
        h->cps_lo.push_back(p);
    }
    GPE_CUDA(cudaMemcpyAsync(h->d_u, host_u, sizeof(double) * (size_t)nsteps * h->nctrl, cudaMemcpyHostToDevice, h->st));
    GPE_CUDA(cudaMemcpyAsync(h->V0, h->V[0], fb, cudaMemcpyDeviceToDevice, h->st));
    void* target = h->adj[6];
    GPE_TRY(upload_c128_host(h, host_target, target));
    // forward with checkpoints cps[0..ncp-1] (cps[j] = psi at step j*K)
    auto save_cp = [&](int j) -> gpe_status {
        GPE_CUDA(cudaMemcpyAsync(h->cps[j], h->A[0], fb, cudaMemcpyDeviceToDevice, h->st));
        if (comp) GPE_CUDA(cudaMemcpyAsync(h->cps_lo[j], h->Lo[0], fb, cudaMemcpyDeviceToDevice, h->st));
        return GPE_OK;
    };
    auto load_cp = [&](int j) -> gpe_status {
        GPE_CUDA(cudaMemcpyAsync(h->A[0], h->cps[j], fb, cudaMemcpyDeviceToDevice, h->st));
        if (comp) {
            GPE_CUDA(cudaMemcpyAsync(h->Lo[0], h->cps_lo[j], fb, cudaMemcpyDeviceToDevice, h->st));
            h->lo_valid = true;
        }
        h->w_fwd_A = false;  // A was replaced: W no longer holds its transform
        return GPE_OK;
    };
    GPE_TRY(save_cp(0));
    for (int n = 0; n < nsteps; ++n) {
        GPE_TRY(ctrl_form_v<R>(h, n));
        GPE_TRY(step_real_t<R>(h, n, 1, nullptr, comp));
        if ((n + 1) % K == 0 && n + 1 < nsteps) GPE_TRY(save_cp((n + 1) / K));
    }
    // loss = 1 - |o|^2, o = sum conj(target) psi_T DV (psi_T = high + low part)
    double o[2] = {0.0, 0.0};
    for (int part = 0; part < (comp ? 2 : 1); ++part) {
        k_ctrl_partials<C, R><<<CTRL_BLOCKS, 256, 0, h->st>>>(0, (const C*)target,
                                                             (const C*)(part ? h->Lo[0] : h->A[0]), nullptr,
                                                             nullptr, 0, h->N, h->d_part);
        k_ctrl_final<<<1, 64, 0, h->st>>>(h->d_part, CTRL_BLOCKS, 2, h->d_grad);
        h->launches += 2;
        double op[2];
        GPE_CUDA(cudaMemcpyAsync(op, h->d_grad, sizeof(op), cudaMemcpyDeviceToHost, h->st));
        GPE_CUDA(cudaStreamSynchronize(h->st));
        o[0] += op[0];
        o[1] += op[1];
    }
    const double DV = h->cfg.dx[0] * h->cfg.dx[1] * h->cfg.dx[2];
    o[0] *= DV;
    o[1] *= DV;
    if (loss_out) *loss_out = 1.0 - (o[0] * o[0] + o[1] * o[1]);
    if (host_grad) {
        // lambda_T = -2 o target DV
        k_cscale<C><<<blocks_for(h->N, 256), 256, 0, h->st>>>((C*)h->adj[0], (const C*)target, -2.0 * o[0] * DV,
                                                            -2.0 * o[1] * DV, h->N);
        h->launches++;
        void** seg = h->cps.data() + ncp;  // K + 1 states of one segment
        for (int j = (nsteps - 1) / K; j >= 0; --j) {
            const int n0 = j * K, n1 = std::min(nsteps, n0 + K);
            GPE_TRY(load_cp(j));
            for (int n = n0; n < n1; ++n) {
                GPE_CUDA(cudaMemcpyAsync(seg[n - n0], h->A[0], fb, cudaMemcpyDeviceToDevice, h->st));
                if (n + 1 < n1) {
                    GPE_TRY(ctrl_form_v<R>(h, n));
                    GPE_TRY(step_real_t<R>(h, n, 1, nullptr, comp));
                }
            }
            for (int n = n1 - 1; n >= n0; --n) {
                GPE_TRY(ctrl_form_v<R>(h, n));
                GPE_TRY(ctrl_stage_args<R>(h, seg[n - n0], h->adj[3], h->adj[4], h->adj[5], n));
                GPE_TRY(ctrl_adjoint_step<R>(h, seg[n - n0], h->adj[3], h->adj[4], h->adj[5], n));
                GPE_TRY(ctrl_reduce_grad<R>(h, n));
            }
        }
        GPE_CUDA(cudaMemcpyAsync(host_grad, h->d_grad, sizeof(double) * (size_t)nsteps * h->nctrl,
                                 cudaMemcpyDeviceToHost, h->st));
    }
    // leave psi and V as they were
    GPE_TRY(load_cp(0));
    GPE_CUDA(cudaMemcpyAsync(h->V[0], h->V0, fb, cudaMemcpyDeviceToDevice, h->st));
    GPE_CUDA(cudaStreamSynchronize(h->st));
    h->w_fwd_A = false;
    return check_device_status(h);
}

void tune_apply_cache(gpe_handle* h);  // autotuner section below

// A handle holding nb instances of one configuration (nb > 1: a gpe_batch
// group; instance i's fields start at element i*N, its parameters, scalars
// and partial sums at prms + 32*i, sc + i, partials + ny*nz*MAXQ*2*i).
gpe_status create_handle(const gpe_config* cfg, int nb, gpe_handle** out) {
    if (!cfg || !out) return fail(GPE_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (cfg->abi_version != GPE_ABI_VERSION) return fail(GPE_ERR_INVALID_ARG, "abi_version mismatch");
    if (cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1) return fail(GPE_ERR_INVALID_ARG, "grid sizes must be >= 1");
    if (cfg->ncomp < 1 || cfg->ncomp > 2) return fail(GPE_ERR_INVALID_ARG, "ncomp must be 1 or 2");
    if (cfg->precision != GPE_C128 && cfg->precision != GPE_C64) return fail(GPE_ERR_INVALID_ARG, "bad precision");
    if (cfg->hamiltonian < GPE_HAM_BEC || cfg->hamiltonian > GPE_HAM_USER)
        return fail(GPE_ERR_INVALID_ARG, "bad hamiltonian");
    if (cfg->ncomp == 2 && cfg->hamiltonian != GPE_HAM_BEC2 && cfg->hamiltonian != GPE_HAM_TEMPLATE)
        return fail(GPE_ERR_UNSUPPORTED, "two components need GPE_HAM_BEC2 or GPE_HAM_TEMPLATE");
    if (cfg->ncomp == 1 && cfg->hamiltonian == GPE_HAM_BEC2)
        return fail(GPE_ERR_INVALID_ARG, "GPE_HAM_BEC2 needs two components");
    if (cfg->imag_scheme != GPE_IMAG_HEAVYBALL && cfg->imag_scheme != GPE_IMAG_RK4)
        return fail(GPE_ERR_INVALID_ARG, "bad imag_scheme");
    const int L3[3] = {cfg->nx, cfg->ny, cfg->nz};
    for (int d = 0; d < 3; ++d)
        if (!gpe_fft_length_supported(L3[d]))
            return fail(GPE_ERR_UNSUPPORTED, "grid length " + std::to_string(L3[d]) + " has no compiled FFT plan");
    if ((long long)cfg->nx * cfg->ny * cfg->nz > (1LL << 31))
        return fail(GPE_ERR_UNSUPPORTED, "grid larger than 2^31 points");

    gpe_handle* h = new gpe_handle();
    h->cfg = *cfg;
    h->prec = cfg->precision;
    h->nx = cfg->nx;
    h->ny = cfg->ny;
    h->nz = cfg->nz;
    h->N = (long long)cfg->nx * cfg->ny * cfg->nz;
    h->ncomp = cfg->ncomp;
    h->dens = (cfg->hamiltonian == GPE_HAM_DIPOLAR || cfg->hamiltonian == GPE_HAM_SOFT) ? 1 : 0;
    h->nf = h->ncomp + h->dens;
    h->esz = h->prec == GPE_C128 ? 16 : 8;
    h->nb = nb;

    auto bail = [&](gpe_status s) {
        free_all(h);
        delete h;
        return s;
    };
    auto dmalloc = [&](void** p, size_t bytes) -> bool {
        cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) {
            g_err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
            return false;
        }
        return true;
    };
    const size_t fb = h->esz * h->N * nb;
    for (int c = 0; c < h->ncomp; ++c) {
        if (!dmalloc(&h->A[c], fb) || !dmalloc(&h->B[c], fb) || !dmalloc(&h->K[c], fb) || !dmalloc(&h->V[c], fb))
            return bail(GPE_ERR_OUT_OF_MEMORY);
        cudaMemsetAsync(h->A[c], 0, fb, h->st);
        cudaMemsetAsync(h->B[c], 0, fb, h->st);
        cudaMemsetAsync(h->K[c], 0, fb, h->st);
        cudaMemsetAsync(h->V[c], 0, fb, h->st);
    }
    for (int f = 0; f < h->nf; ++f)
        if (!dmalloc(&h->W[f], fb)) return bail(GPE_ERR_OUT_OF_MEMORY);
    if (h->prec == GPE_C64 && !dmalloc(&h->stage128, 16 * h->N)) return bail(GPE_ERR_OUT_OF_MEMORY);
    if (h->prec == GPE_C64 && nb == 1)
        for (int c = 0; c < h->ncomp; ++c)
            if (!dmalloc(&h->Lo[c], h->esz * h->N)) return bail(GPE_ERR_OUT_OF_MEMORY);

    // Twiddles, k axes, dipolar kernel, parameters, scalars, partial sums.
    std::vector<double> kax[3];
    host_kaxes(*cfg, kax);
    for (int d = 0; d < 3; ++d) {
        if (!dmalloc((void**)&h->kax[d], sizeof(double) * L3[d])) return bail(GPE_ERR_OUT_OF_MEMORY);
        cudaMemcpy(h->kax[d], kax[d].data(), sizeof(double) * L3[d], cudaMemcpyHostToDevice);
        if (h->prec == GPE_C64) {
            std::vector<float> k2s(L3[d]);
            const double lap_scale = 19.739208802 / (double)h->N;  // src/parallel.cu:199
            for (int i = 0; i < L3[d]; ++i) k2s[i] = (float)(lap_scale * kax[d][i] * kax[d][i]);
            if (!dmalloc((void**)&h->k2s[d], sizeof(float) * L3[d])) return bail(GPE_ERR_OUT_OF_MEMORY);
            cudaMemcpy(h->k2s[d], k2s.data(), sizeof(float) * L3[d], cudaMemcpyHostToDevice);
        }
        if (h->prec == GPE_C128) {
            std::vector<double2> tw;
            host_twiddles(L3[d], tw);
            if (!dmalloc(&h->tw[d], sizeof(double2) * L3[d])) return bail(GPE_ERR_OUT_OF_MEMORY);
            cudaMemcpy(h->tw[d], tw.data(), sizeof(double2) * L3[d], cudaMemcpyHostToDevice);
        } else {
            std::vector<float2> tw;
            host_twiddles(L3[d], tw);
            if (!dmalloc(&h->tw[d], sizeof(float2) * L3[d])) return bail(GPE_ERR_OUT_OF_MEMORY);
            cudaMemcpy(h->tw[d], tw.data(), sizeof(float2) * L3[d], cudaMemcpyHostToDevice);
            std::vector<float4> tw2(L3[d]);
            for (int m = 0; m < L3[d]; ++m) tw2[m] = make_float4(tw[m].x, tw[m].x, tw[m].y, tw[m].y);
            if (!dmalloc((void**)&h->tw2[d], sizeof(float4) * L3[d])) return bail(GPE_ERR_OUT_OF_MEMORY);
            cudaMemcpy(h->tw2[d], tw2.data(), sizeof(float4) * L3[d], cudaMemcpyHostToDevice);
        }
    }
    if (h->dens) {
        std::vector<double> v;
        host_vdd(*cfg, kax, v);
        if (h->prec == GPE_C128) {
            if (!dmalloc(&h->vdd, sizeof(double) * h->N)) return bail(GPE_ERR_OUT_OF_MEMORY);
            cudaMemcpy(h->vdd, v.data(), sizeof(double) * h->N, cudaMemcpyHostToDevice);
        } else {
            std::vector<float> vf(v.begin(), v.end());
            if (!dmalloc(&h->vdd, sizeof(float) * h->N)) return bail(GPE_ERR_OUT_OF_MEMORY);
            cudaMemcpy(h->vdd, vf.data(), sizeof(float) * h->N, cudaMemcpyHostToDevice);
        }
    }
    if (!dmalloc((void**)&h->prms, sizeof(double) * GPE_NO_HAMIL_PARAMS * nb)) return bail(GPE_ERR_OUT_OF_MEMORY);
    if (!dmalloc((void**)&h->sc, sizeof(DevScalars) * nb)) return bail(GPE_ERR_OUT_OF_MEMORY);
    {
        DevScalars s;
        std::memset(&s, 0, sizeof(s));
        s.scale[0][0] = s.scale[0][1] = s.scale[1][0] = s.scale[1][1] = 1.0;
        s.norm[0] = cfg->npart[0];
        s.norm[1] = cfg->npart[1];
        std::vector<DevScalars> sv(nb, s);
        std::vector<double> pv((size_t)GPE_NO_HAMIL_PARAMS * nb);
        for (int i = 0; i < nb; ++i)
            std::memcpy(pv.data() + (size_t)i * GPE_NO_HAMIL_PARAMS, cfg->prms, sizeof(double) * GPE_NO_HAMIL_PARAMS);
        cudaMemcpy(h->sc, sv.data(), sizeof(DevScalars) * nb, cudaMemcpyHostToDevice);
        cudaMemcpy(h->prms, pv.data(), sizeof(double) * pv.size(), cudaMemcpyHostToDevice);
    }
    if (cudaHostAlloc((void**)&h->flag_host, 2 * sizeof(int), cudaHostAllocDefault) != cudaSuccess)
        return bail(GPE_ERR_OUT_OF_MEMORY);
    for (cudaEvent_t& ev : h->flag_ev)
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return bail(GPE_ERR_CUDA);
    const size_t nblk = (size_t)h->ny * h->nz;  // x-pass CTAs hold >= 1 row each
    if (!dmalloc((void**)&h->partials, nblk * MAXQ * 2 * sizeof(double) * nb)) return bail(GPE_ERR_OUT_OF_MEMORY);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        g_err = std::string("gpe_create: ") + cudaGetErrorString(e);
        return bail(GPE_ERR_CUDA);
    }
    tune_apply_cache(h);
    *out = h;
    return GPE_OK;
}

}  // namespace

extern "C" {

gpe_status gpe_create(const gpe_config* cfg, gpe_handle** out) { return create_handle(cfg, 1, out); }

gpe_status gpe_destroy(gpe_handle* h) {
    if (!h) return GPE_OK;
    cudaStreamSynchronize(h->st);
    free_all(h);
    delete h;
    return GPE_OK;
}

gpe_status gpe_set_stream(gpe_handle* h, void* stream) {
    GPE_TRY(check_handle(h));
    h->st = (cudaStream_t)stream;
    return GPE_OK;
}

gpe_status gpe_set_params(gpe_handle* h, const double prms[GPE_NO_HAMIL_PARAMS]) {
    GPE_TRY(check_handle(h));
    if (!prms) return fail(GPE_ERR_INVALID_ARG, "null prms");
    std::memcpy(h->cfg.prms, prms, sizeof(double) * GPE_NO_HAMIL_PARAMS);
    GPE_CUDA(cudaMemcpyAsync(h->prms, h->cfg.prms, sizeof(double) * GPE_NO_HAMIL_PARAMS, cudaMemcpyHostToDevice, h->st));
    if (h->dens) {
        std::vector<double> kax[3], v;
        host_kaxes(h->cfg, kax);
        host_vdd(h->cfg, kax, v);
        GPE_CUDA(cudaStreamSynchronize(h->st));
        if (h->prec == GPE_C128) {
            GPE_CUDA(cudaMemcpy(h->vdd, v.data(), sizeof(double) * h->N, cudaMemcpyHostToDevice));
        } else {
            std::vector<float> vf(v.begin(), v.end());
            GPE_CUDA(cudaMemcpy(h->vdd, vf.data(), sizeof(float) * h->N, cudaMemcpyHostToDevice));
        }
    }
    GPE_CUDA(cudaStreamSynchronize(h->st));
    return GPE_OK;
}

// complex64 handles with a low part: the state of component comp from the
// complex128 array src (device) in one kernel, no synchronisation.
gpe_status set_state_c64(gpe_handle* h, int comp, const void* src) {
    if (!h->lo_valid)
        for (int c = 0; c < h->ncomp; ++c)
            if (c != comp) GPE_CUDA(cudaMemsetAsync(h->Lo[c], 0, h->esz * h->N, h->st));
    k_set_state_c64<<<blocks_for(h->N, 256), 256, 0, h->st>>>((float2*)h->A[comp], (float2*)h->B[comp],
                                                               (float2*)h->Lo[comp], (const double2*)src, h->N);
    h->launches++;
    GPE_CUDA(cudaGetLastError());
    h->lo_valid = true;
    h->hb_old_valid = true;
    return GPE_OK;
}

gpe_status gpe_set_psi(gpe_handle* h, int comp, const double* host_c128) {
    if (h) h->w_fwd_A = false;
    GPE_TRY(check_handle(h));
    GPE_TRY(check_comp(h, comp));
    if (!host_c128) return fail(GPE_ERR_INVALID_ARG, "null psi");
    GPE_TRY(canonicalize(h));
    if (h->prec == GPE_C64 && h->Lo[comp]) {  // one copy, one kernel, one synchronisation
        GPE_CUDA(cudaMemcpyAsync(h->stage128, host_c128, 16 * h->N, cudaMemcpyHostToDevice, h->st));
        GPE_TRY(set_state_c64(h, comp, h->stage128));
        GPE_CUDA(cudaStreamSynchronize(h->st));
        return GPE_OK;
    }
    GPE_TRY(upload_c128_host(h, host_c128, h->A[comp]));
    GPE_TRY(set_low_part(h, comp, h->stage128));
    GPE_CUDA(cudaMemcpyAsync(h->B[comp], h->A[comp], h->esz * h->N, cudaMemcpyDeviceToDevice, h->st));
    GPE_CUDA(cudaStreamSynchronize(h->st));
    h->hb_old_valid = true;
    return GPE_OK;
}

gpe_status gpe_set_psi_device(gpe_handle* h, int comp, const void* dev_c128) {
    if (h) h->w_fwd_A = false;
    GPE_TRY(check_handle(h));
    GPE_TRY(check_comp(h, comp));
    if (!dev_c128) return fail(GPE_ERR_INVALID_ARG, "null psi");
    GPE_TRY(canonicalize(h));
    if (h->prec == GPE_C64 && h->Lo[comp]) return set_state_c64(h, comp, dev_c128);
    GPE_TRY(upload_c128_device(h, comp, dev_c128, h->A[comp]));
    GPE_TRY(set_low_part(h, comp, dev_c128));
    GPE_CUDA(cudaMemcpyAsync(h->B[comp], h->A[comp], h->esz * h->N, cudaMemcpyDeviceToDevice, h->st));
    h->hb_old_valid = true;
    return GPE_OK;
}

gpe_status gpe_get_psi(gpe_handle* h, int comp, double* host_c128) {
    GPE_TRY(check_handle(h));
    GPE_TRY(check_comp(h, comp));
    if (!host_c128) return fail(GPE_ERR_INVALID_ARG, "null output");
    GPE_TRY(canonicalize(h));
    return download_c128_host(h, h->A[comp], host_c128, h->lo_valid ? h->Lo[comp] : nullptr);
}

gpe_status gpe_get_psi_device(gpe_handle* h, int comp, void* dev_c128) {
    GPE_TRY(check_handle(h));
    GPE_TRY(check_comp(h, comp));
    if (!dev_c128) return fail(GPE_ERR_INVALID_ARG, "null output");
    GPE_TRY(canonicalize(h));
    if (h->prec == GPE_C128) {
        GPE_CUDA(cudaMemcpyAsync(dev_c128, h->A[comp], 16 * h->N, cudaMemcpyDeviceToDevice, h->st));
    } else {
        if (h->lo_valid)
            k_to_c128_hilo<<<blocks_for(h->N, 256), 256, 0, h->st>>>((double2*)dev_c128, (const float2*)h->A[comp],
                                                                     (const float2*)h->Lo[comp], h->N);
        else
            k_to_c128<float2><<<blocks_for(h->N, 256), 256, 0, h->st>>>((double2*)dev_c128,
                                                                        (const float2*)h->A[comp], h->N);
        h->launches++;
        GPE_CUDA(cudaGetLastError());
    }
    return GPE_OK;
}

}  // extern "C"

namespace {

// Runs f on a complex128 device copy of component comp's psi, then sets psi
// from it (the precision's rounding and low part as gpe_set_psi_device).
template <class F>
gpe_status on_c128_psi(gpe_handle* h, int comp, F f) {
    GPE_TRY(check_handle(h));
    GPE_TRY(check_comp(h, comp));
    void* buf = nullptr;
    double* part = nullptr;
    gpe_status s = GPE_OK;
    if (cudaMalloc(&buf, 16 * h->N) != cudaSuccess || cudaMalloc((void**)&part, seed_partials_bytes()) != cudaSuccess)
        s = fail(GPE_ERR_OUT_OF_MEMORY, "seed work buffers");
    if (s == GPE_OK) s = gpe_get_psi_device(h, comp, buf);
    if (s == GPE_OK) {
        SeedGrid g;
        const int n[3] = {h->nx, h->ny, h->nz};
        for (int d = 0; d < 3; ++d) {
            g.n[d] = n[d];
            g.xmax[d] = h->cfg.xmax[d];
            g.dx[d] = h->cfg.dx[d];
        }
        const cudaError_t e = f((double2*)buf, g, part);
        if (e != cudaSuccess) s = fail(GPE_ERR_CUDA, std::string("seed kernels: ") + cudaGetErrorString(e));
    }
    if (s == GPE_OK) s = gpe_set_psi_device(h, comp, buf);
    cudaStreamSynchronize(h->st);
    if (buf) cudaFree(buf);
    if (part) cudaFree(part);
    return s;
}

}  // namespace

extern "C" {

gpe_status gpe_imprint_vortex_tube(gpe_handle* h, int comp, double ncirc) {
    return on_c128_psi(h, comp, [&](double2* p, const SeedGrid& g, double*) {
        return imprint_vortex_tube_c128(p, g, ncirc, h->st);
    });
}

gpe_status gpe_seed_lattice(gpe_handle* h, int comp, int lattice, double amp, double k, const double* off,
                            double seed_npart, double norm_npart) {
    if (lattice < GPE_LATTICE_1D || lattice > GPE_LATTICE_3D_SC) return fail(GPE_ERR_INVALID_ARG, "unknown lattice");
    if (!off) return fail(GPE_ERR_INVALID_ARG, "null offsets");
    if (!(seed_npart > 0) || !(norm_npart > 0)) return fail(GPE_ERR_INVALID_ARG, "particle numbers must be > 0");
    return on_c128_psi(h, comp, [&](double2* p, const SeedGrid& g, double* part) {
        return seed_lattice_c128(p, g, lattice, amp, k, off, seed_npart, norm_npart, part, h->st);
    });
}

gpe_status gpe_set_vext(gpe_handle* h, int comp, const double* host_c128) {
    GPE_TRY(check_handle(h));
    GPE_TRY(check_comp(h, comp));
    if (!host_c128) return fail(GPE_ERR_INVALID_ARG, "null vext");
    return upload_c128_host(h, host_c128, h->V[comp]);
}

gpe_status gpe_step_real(gpe_handle* h, int first_iteration, int nsteps, double* obs_out) {
    GPE_TRY(check_handle(h));
    if (nsteps < 0) return fail(GPE_ERR_INVALID_ARG, "nsteps < 0");
    return h->prec == GPE_C64 ? step_real_t<float>(h, first_iteration, nsteps, obs_out)
                              : step_real_t<double>(h, first_iteration, nsteps, obs_out);
}

gpe_status gpe_step_imag(gpe_handle* h, int first_iteration, int nsteps, int* iters_done, int* converged) {
    GPE_TRY(check_handle(h));
    if (nsteps < 0) return fail(GPE_ERR_INVALID_ARG, "nsteps < 0");
    return h->prec == GPE_C64 ? step_imag_t<float>(h, first_iteration, nsteps, iters_done, converged)
                              : step_imag_t<double>(h, first_iteration, nsteps, iters_done, converged);
}

gpe_status gpe_imag_state(gpe_handle* h, double* out) {
    GPE_TRY(check_handle(h));
    if (!out) return fail(GPE_ERR_INVALID_ARG, "null output");
    DevScalars s;
    GPE_TRY(sync_read_scalars(h, &s));
    for (int c = 0; c < h->ncomp; ++c) {
        out[4 * c + 0] = s.norm[c];
        out[4 * c + 1] = s.mu[c];
        out[4 * c + 2] = s.en[c];
        out[4 * c + 3] = s.en_prev[c];
    }
    return GPE_OK;
}

gpe_status gpe_reset_imag_state(gpe_handle* h) {
    GPE_TRY(check_handle(h));
    DevScalars s;
    GPE_TRY(sync_read_scalars(h, &s));
    for (int c = 0; c < 2; ++c) {
        s.mu[c] = s.en[c] = s.en_prev[c] = s.mu_prev[c] = 0.0;
        s.norm[c] = h->cfg.npart[c];
    }
    s.done = s.converged = s.iters_done = s.status = s.have_mu_prev = 0;
    s.counter = 0;
    GPE_CUDA(cudaMemcpyAsync(h->sc, &s, sizeof(s), cudaMemcpyHostToDevice, h->st));
    GPE_CUDA(cudaStreamSynchronize(h->st));
    return GPE_OK;
}

gpe_status gpe_laplace(gpe_handle* h, int comp, double* host_out_c128) {
    GPE_TRY(check_handle(h));
    GPE_TRY(check_comp(h, comp));
    if (!host_out_c128) return fail(GPE_ERR_INVALID_ARG, "null output");
    GPE_TRY(h->prec == GPE_C64 ? apply_chain_t<float>(h, EPI_STORE, 0.0, comp)
                               : apply_chain_t<double>(h, EPI_STORE, 0.0, comp));
    GPE_TRY(check_device_status(h));
    return download_c128_host(h, h->W[0], host_out_c128);
}

gpe_status gpe_apply_h(gpe_handle* h, double t, int comp, double* hmu, double* hen) {
    GPE_TRY(check_handle(h));
    GPE_TRY(check_comp(h, comp));
    GPE_TRY(ensure_out_buffers(h));
    GPE_TRY(h->prec == GPE_C64 ? apply_chain_t<float>(h, EPI_APPLYH, t, -1)
                               : apply_chain_t<double>(h, EPI_APPLYH, t, -1));
    GPE_TRY(check_device_status(h));
    if (hmu) GPE_TRY(download_c128_host(h, h->O[2 * comp], hmu));
    if (hen) GPE_TRY(download_c128_host(h, h->O[2 * comp + 1], hen));
    return GPE_OK;
}

gpe_status gpe_observables(gpe_handle* h, double t, double* out) {
    GPE_TRY(check_handle(h));
    if (!out) return fail(GPE_ERR_INVALID_ARG, "null output");
    GPE_TRY(h->prec == GPE_C64 ? apply_chain_t<float>(h, EPI_OBS, t, -1) : apply_chain_t<double>(h, EPI_OBS, t, -1));
    DevScalars s;
    GPE_TRY(sync_read_scalars(h, &s));
    for (int q = 0; q < 3 * h->ncomp; ++q) out[q] = s.obs[q];
    if (s.status == GPE_ERR_DIVERGED) return fail(GPE_ERR_DIVERGED, "non-finite observable");
    return GPE_OK;
}

gpe_status gpe_momentum_x(gpe_handle* h, int comp, double* px) {
    GPE_TRY(check_handle(h));
    GPE_TRY(check_comp(h, comp));
    if (!px) return fail(GPE_ERR_INVALID_ARG, "null output");
    GPE_TRY(h->prec == GPE_C64 ? apply_chain_t<float>(h, EPI_OBS, 0.0, comp, SPEC_PX)
                               : apply_chain_t<double>(h, EPI_OBS, 0.0, comp, SPEC_PX));
    DevScalars s;
    GPE_TRY(sync_read_scalars(h, &s));
    *px = s.obs[1];
    return GPE_OK;
}

}  // extern "C"

// kind: OBS_*; c2 < 0 for the one-field kinds.  Returns the sum times DV,
// as the reference's reduction (src/baseHamiltonian.cu:112-150) does.
template <typename R>
gpe_status observable_t(gpe_handle* h, int kind, int c1, int c2, double sign, double* out) {
    typedef typename Cx<R>::T C;
    GPE_TRY(canonicalize_t<R>(h));
    if (!h->obs_part) GPE_CUDA(cudaMalloc(&h->obs_part, sizeof(double) * (OBS_BLOCKS + 1)));
    k_obs_partials<C><<<OBS_BLOCKS, 256, 0, h->st>>>(kind, (const C*)h->A[c1], c2 >= 0 ? (const C*)h->A[c2] : nullptr,
                                                     sign, h->cfg.xmax[0], h->cfg.dx[0], 2.0 * h->cfg.xmax[0], h->nx,
                                                     h->N, h->obs_part);
    k_ctrl_final<<<1, 64, 0, h->st>>>(h->obs_part, OBS_BLOCKS, 1, h->obs_part + OBS_BLOCKS);
    h->launches += 2;
    GPE_CUDA(cudaGetLastError());
    double r = 0.0;
    GPE_CUDA(cudaMemcpyAsync(&r, h->obs_part + OBS_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    GPE_CUDA(cudaStreamSynchronize(h->st));
    *out = r * h->cfg.dx[0] * h->cfg.dx[1] * h->cfg.dx[2];
    return GPE_OK;
}

gpe_status observable(gpe_handle* h, int kind, int c1, int c2, double sign, double* out) {
    GPE_TRY(check_handle(h));
    if (!out) return fail(GPE_ERR_INVALID_ARG, "null output");
    if (h->nb != 1) return fail(GPE_ERR_INVALID_ARG, "observables of batched instances are not supported");
    return h->prec == GPE_C64 ? observable_t<float>(h, kind, c1, c2, sign, out)
                              : observable_t<double>(h, kind, c1, c2, sign, out);
}

extern "C" {

gpe_status gpe_average_cos(gpe_handle* h, int comp, double* out) {
    GPE_TRY(check_handle(h));
    GPE_TRY(check_comp(h, comp));
    return observable(h, OBS_COS, comp, -1, 0.0, out);
}

gpe_status gpe_average_cos2(gpe_handle* h, int sign, double* out) {
    GPE_TRY(check_handle(h));
    if (h->ncomp != 2) return fail(GPE_ERR_INVALID_ARG, "needs two components");
    if (sign != 1 && sign != -1) return fail(GPE_ERR_INVALID_ARG, "sign must be +1 or -1");
    return observable(h, OBS_COS2, 0, 1, (double)sign, out);
}

gpe_status gpe_relative_phase(gpe_handle* h, double* out) {
    GPE_TRY(check_handle(h));
    if (h->ncomp != 2) return fail(GPE_ERR_INVALID_ARG, "needs two components");
    return observable(h, OBS_PHASE, 0, 1, 0.0, out);
}

gpe_status gpe_dsz_dt(gpe_handle* h, double* out) {
    GPE_TRY(check_handle(h));
    if (h->ncomp != 2) return fail(GPE_ERR_INVALID_ARG, "needs two components");
    return observable(h, OBS_DSZ, 0, 1, 0.0, out);
}

gpe_status gpe_fft(gpe_handle* h, int comp, int sign) {
    GPE_TRY(check_handle(h));
    GPE_TRY(check_comp(h, comp));
    if (sign != -1 && sign != 1) return fail(GPE_ERR_INVALID_ARG, "sign must be -1 or +1");
    GPE_TRY(h->prec == GPE_C64 ? fft_t<float>(h, comp, sign) : fft_t<double>(h, comp, sign));
    return check_device_status(h);
}

gpe_status gpe_set_user_hamiltonian(gpe_handle* h, const gpe_user_hamiltonian* ops) {
    GPE_TRY(check_handle(h));
    if (h->cfg.hamiltonian != GPE_HAM_USER) return fail(GPE_ERR_INVALID_ARG, "the handle's hamiltonian is not GPE_HAM_USER");
    if (!ops || ops->abi_version != GPE_ABI_VERSION || !ops->launch_x_c64 || !ops->launch_x_c128)
        return fail(GPE_ERR_INVALID_ARG, "null plugin table or abi_version mismatch");
    h->user = ops;
    return GPE_OK;
}

gpe_status gpe_sync(gpe_handle* h) {
    GPE_TRY(check_handle(h));
    GPE_CUDA(cudaStreamSynchronize(h->st));
    GPE_CUDA(cudaGetLastError());
    return check_device_status(h);
}

long long gpe_kernel_launches(const gpe_handle* h) { return h ? h->launches : 0; }

gpe_status gpe_profile_enable(gpe_handle* h, int enable) {
    GPE_TRY(check_handle(h));
    h->prof = enable != 0;
    return GPE_OK;
}

gpe_status gpe_profile_read(gpe_handle* h, double* ms_out, long long* count_out) {
    GPE_TRY(check_handle(h));
    GPE_CUDA(cudaStreamSynchronize(h->st));
    double ms[GPE_PROF_KINDS] = {0};
    long long cnt[GPE_PROF_KINDS] = {0};
    for (auto& r : h->recs) {
        float t = 0.f;
        GPE_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
        ms[r.kind] += t;
        cnt[r.kind] += 1;
        h->ev_free.push_back(r.a);
        h->ev_free.push_back(r.b);
    }
    h->recs.clear();
    for (int k = 0; k < GPE_PROF_KINDS; ++k) {
        if (ms_out) ms_out[k] = ms[k];
        if (count_out) count_out[k] = cnt[k];
    }
    return GPE_OK;
}

gpe_status gpe_control_set_basis(gpe_handle* h, int nctrl, const double* host_G) {
    GPE_TRY(check_handle(h));
    const int ham = h->cfg.hamiltonian;
    if (h->ncomp != 1 || (ham != GPE_HAM_BEC && ham != GPE_HAM_DIPOLAR && ham != GPE_HAM_SOFT) || h->nb != 1 ||
        h->cfg.prms[11] != 0)
        return fail(GPE_ERR_UNSUPPORTED,
                    "the control gradient needs one component, GPE_HAM_BEC, GPE_HAM_DIPOLAR or GPE_HAM_SOFT, "
                    "and no moving-frame term");
    if (nctrl < 1 || nctrl > 64 || !host_G) return fail(GPE_ERR_INVALID_ARG, "nctrl must be 1..64 with a basis");
    const size_t rs = h->prec == GPE_C64 ? 4 : 8;
    if (h->ctrlG) cudaFree(h->ctrlG);
    h->ctrlG = nullptr;
    GPE_CUDA(cudaMalloc(&h->ctrlG, rs * (size_t)nctrl * h->N));
    if (!h->V0) GPE_CUDA(cudaMalloc(&h->V0, h->esz * h->N));
    if (rs == 8) {
        GPE_CUDA(cudaMemcpy(h->ctrlG, host_G, 8 * (size_t)nctrl * h->N, cudaMemcpyHostToDevice));
    } else {
        std::vector<float> g((size_t)nctrl * h->N);
        for (size_t i = 0; i < g.size(); ++i) g[i] = (float)host_G[i];
        GPE_CUDA(cudaMemcpy(h->ctrlG, g.data(), 4 * g.size(), cudaMemcpyHostToDevice));
    }
    h->nctrl = nctrl;
    return GPE_OK;
}

gpe_status gpe_control_gradient(gpe_handle* h, const double* host_u, int nsteps, const double* host_target_c128,
                                int checkpoint_every, double* loss_out, double* host_grad) {
    GPE_TRY(check_handle(h));
    if (!h->nctrl) return fail(GPE_ERR_INVALID_ARG, "no control basis (gpe_control_set_basis)");
    if (!host_u || !host_target_c128 || nsteps < 1 || checkpoint_every < 1)
        return fail(GPE_ERR_INVALID_ARG, "null u/target, nsteps < 1 or checkpoint_every < 1");
    return h->prec == GPE_C64
               ? control_gradient_t<float>(h, host_u, nsteps, host_target_c128, checkpoint_every, loss_out, host_grad)
               : control_gradient_t<double>(h, host_u, nsteps, host_target_c128, checkpoint_every, loss_out,
                                            host_grad);
}

// ---- batched independent instances -------------------------------------------------------
}  // extern "C"

struct gpe_batch {
    int n = 0;
    int prec = GPE_C128;
    std::vector<gpe_handle*> groups;     // one per distinct grid geometry
    std::vector<int> gidx, ginst;        // instance -> group, index within the group
    cudaStream_t st = 0;
    cudaGraphExec_t exec = nullptr;      // one iteration of every group
    cudaGraph_t graph = nullptr;
    bool use_graph = true;
    long long graph_launches = 0;        // kernels per replay of the graph
    long long replayed = 0;              // kernels run by graph replays
    // persistent stage launches (gpe_batch_set_persistent): one cooperative
    // launch per RK4 stage for every group
    int mode = GPE_BATCH_PER_GROUP;      // gpe_batch_set_launch_mode
    unsigned wait_bound = 0;             // iterations a grid-barrier wait may spin
    void* stage_args = nullptr;          // device PassArgs [4 stages][3 phases][BATCH_MAX_GROUPS]
    GridBar* bar = nullptr;
    int stage_grid = 0;                  // CTAs of the last stage launch
    long long stage_launches = 0;        // stage kernels launched directly
    // early stop: per chunk of iterations, whether any instance still runs
    int* d_running = nullptr;            // device [2], one per chunk slot
    int* flag_host = nullptr;            // pinned [2]
    cudaEvent_t flag_ev[2] = {nullptr, nullptr};
};

namespace {

bool same_geometry(const gpe_config& a, const gpe_config& b) {
    if (a.nx != b.nx || a.ny != b.ny || a.nz != b.nz || a.dim != b.dim) return false;
    for (int d = 0; d < 3; ++d)
        if (a.xmax[d] != b.xmax[d] || a.dx[d] != b.dx[d]) return false;
    return true;
}

gpe_status batch_inst(gpe_batch* b, int inst, gpe_handle** h, size_t* off) {
    if (!b) return fail(GPE_ERR_INVALID_ARG, "null batch");
    if (inst < 0 || inst >= b->n) return fail(GPE_ERR_INVALID_ARG, "instance index out of range");
    *h = b->groups[b->gidx[inst]];
    *off = (size_t)b->ginst[inst] * (size_t)(*h)->N * (*h)->esz;
    return GPE_OK;
}

void batch_drop_graph(gpe_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// Bound of a grid-barrier wait when the caller gives none: 2^24 sleeps of
// 64 ns or more (over a second), far beyond any phase of a stage.
constexpr unsigned BATCH_WAIT_DEFAULT = 1u << 24;

// Why the groups cannot run in the persistent stage kernel ("" when they can).
std::string batch_persistent_reason(const gpe_batch* b) {
    if (b->groups.size() > (size_t)BATCH_MAX_GROUPS) return "more than 8 grid geometries";
    for (const gpe_handle* h : b->groups) {
        if (h->cfg.imag_scheme != GPE_IMAG_RK4) return "imag_scheme is not GPE_IMAG_RK4";
        if (h->nz != 1 || h->ny < 2) return "an instance grid is not two-dimensional (ny > 1, nz = 1)";
        if (!batch_length_supported(h->nx) || !batch_length_supported(h->ny))
            return "a grid length outside 64, 96, 128, 192, 256, 384, 512";
        if (h->nf != 1 || h->ncomp != 1) return "an instance transforms more than one field";
    }
    return "";
}

// The pass arguments of every stage, phase and group, as imag_issue builds
// them for run_chain (RK4 imaginary time; the batch's couplings are time
// independent, so t = 0 as in the per-group iteration), uploaded once.
template <typename R>
gpe_status batch_build_stages(gpe_batch* b) {
    typedef typename Cx<R>::T C;
    const int ng = (int)b->groups.size();
    std::vector<PassArgs<R>> host((size_t)4 * 3 * BATCH_MAX_GROUPS);
    std::memset((void*)host.data(), 0, sizeof(PassArgs<R>) * host.size());
    for (int s = 1; s <= 4; ++s) {
        for (int g = 0; g < ng; ++g) {
            gpe_handle* h = b->groups[g];
            PassArgs<R> a = base_args<R>(h);
            a.check_done = 1;
            a.t = 0.0;
            a.epi = EPI_RKI;
            a.stage = s;
            a.pro = (s == 1) ? PRO_A_SCALED : PRO_PIN;
            for (int c = 0; c < 2; ++c) a.pin[c] = (const C*)h->B[c];
            a.c_re = (s <= 2) ? -0.5 * h->cfg.dt : -1.0 * h->cfg.dt;
            a.c_im = 0.0;
            PassArgs<R>* ph = &host[(size_t)(s - 1) * 3 * BATCH_MAX_GROUPS + g];
            // phase A: launch_x(XM_FWD)
            ph[0] = a;
            ph[0].mode = XM_FWD;
            ph[0].tw = (const C*)h->tw[0];
            // phase B: launch_s(axis 1, SM_FKI) with batch_rows(ny) x values per tile
            PassArgs<R>& y = ph[BATCH_MAX_GROUPS];
            y = a;
            y.mode = SM_FKI;
            y.sax = 1;
            y.tx = batch_rows(h->ny);
            y.tw = (const C*)h->tw[1];
            y.tw2 = h->tw2[1];
            y.sstride = h->nx;
            y.ostride = (long long)h->nx * h->ny;
            // phase C: launch_x(XM_INV), the EPI_RKI epilogue
            ph[2 * BATCH_MAX_GROUPS] = a;
            ph[2 * BATCH_MAX_GROUPS].mode = XM_INV;
            ph[2 * BATCH_MAX_GROUPS].tw = (const C*)h->tw[0];
        }
    }
    if (!b->stage_args) GPE_CUDA(cudaMalloc(&b->stage_args, sizeof(PassArgs<R>) * host.size()));
    GPE_CUDA(cudaMemcpy(b->stage_args, host.data(), sizeof(PassArgs<R>) * host.size(), cudaMemcpyHostToDevice));
    if (!b->bar) GPE_CUDA(cudaMalloc((void**)&b->bar, sizeof(GridBar)));
    GPE_CUDA(cudaMemset(b->bar, 0, sizeof(GridBar)));
    return GPE_OK;
}

// The tile lists of stage s: per group, its instances' x tiles (batch_rows(nx)
// rows each) and strided tiles (batch_rows(ny) x values each), group-major.
template <typename R>
BatchStage<R> batch_stage_desc(const gpe_batch* b, int s, unsigned* max_tiles) {
    BatchStage<R> d;
    std::memset((void*)&d, 0, sizeof(d));
    d.args = (const PassArgs<R>*)b->stage_args + (size_t)(s - 1) * 3 * BATCH_MAX_GROUPS;
    d.ngroups = (int)b->groups.size();
    unsigned xs = 0, ss = 0;
    for (int g = 0; g < d.ngroups; ++g) {
        const gpe_handle* h = b->groups[g];
        const int rx = batch_rows(h->nx), ty = batch_rows(h->ny);
        d.lx[g] = h->nx;
        d.ly[g] = h->ny;
        d.ntx[g] = (h->nx + ty - 1) / ty;
        d.xt[g] = (unsigned)((h->ny * h->nz + rx - 1) / rx);
        d.st[g] = (unsigned)(d.ntx[g] * h->nz);
        d.xstart[g] = xs;
        d.sstart[g] = ss;
        xs += d.xt[g] * (unsigned)h->nb;
        ss += d.st[g] * (unsigned)h->nb;
    }
    d.xstart[d.ngroups] = xs;
    d.sstart[d.ngroups] = ss;
    d.bar = b->bar;
    d.wait_bound = b->wait_bound ? b->wait_bound : BATCH_WAIT_DEFAULT;
    *max_tiles = std::max(xs, ss);
    return d;
}

template <typename R>
gpe_status batch_issue_stages(gpe_batch* b) {
    for (int s = 1; s <= 4; ++s) {
        unsigned max_tiles = 0;
        const BatchStage<R> d = batch_stage_desc<R>(b, s, &max_tiles);
        BatchLaunchInfo li{0, 0, 0, 0};
        const cudaError_t e = launch_batch_stage(d, max_tiles, b->st, &li);
        b->stage_grid = li.grid;
        if (e != cudaSuccess)
            return fail(GPE_ERR_CUDA, std::string("batch stage launch: ") + cudaGetErrorString(e) + " (CTAs per SM " +
                                          std::to_string(li.per_sm) + ", SMs " + std::to_string(li.nsm) + ", grid " +
                                          std::to_string(li.grid) + ", dynamic shared memory " +
                                          std::to_string(li.smem) + " B)");
        b->stage_launches++;
    }
    return GPE_OK;
}

// GPE_BATCH_GROUPED: per stage three launches (x forward, strided, x
// inverse), each over the tiles of every instance of every group.
template <typename R>
gpe_status batch_issue_phases(gpe_batch* b) {
    for (int s = 1; s <= 4; ++s) {
        unsigned max_tiles = 0;
        const BatchStage<R> d = batch_stage_desc<R>(b, s, &max_tiles);
        for (int ph = 0; ph < 3; ++ph) {
            const cudaError_t e = launch_batch_phase(d, ph, b->st);
            if (e != cudaSuccess) return fail(GPE_ERR_CUDA, std::string("batch phase launch: ") + cudaGetErrorString(e));
            b->stage_launches++;
        }
    }
    return GPE_OK;
}

template <typename R>
gpe_status batch_issue_iteration(gpe_batch* b) {
    if (b->mode == GPE_BATCH_PERSISTENT) return batch_issue_stages<R>(b);
    if (b->mode == GPE_BATCH_GROUPED) return batch_issue_phases<R>(b);
    for (gpe_handle* h : b->groups) GPE_TRY(imag_issue<R>(h, 0, 1));
    return GPE_OK;
}

// Captures one imaginary-time iteration of every group into a CUDA graph.
template <typename R>
gpe_status batch_capture(gpe_batch* b) {
    if (b->exec || !b->use_graph) return GPE_OK;
    if (b->st == 0) {
        b->use_graph = false;  // the legacy default stream cannot be captured
        return GPE_OK;
    }
    long long before = b->stage_launches, after = 0;
    for (gpe_handle* h : b->groups) before += h->launches;
    GPE_CUDA(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
    gpe_status s = batch_issue_iteration<R>(b);
    after = b->stage_launches;
    for (gpe_handle* h : b->groups) after += h->launches;
    // captured launches have not run: count them per replay instead
    b->graph_launches = after - before;
    b->replayed -= after - before;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->st, &g);
    if (s != GPE_OK || e != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        b->replayed += b->graph_launches;
        b->graph_launches = 0;
        b->use_graph = false;  // fall back to direct launches
        return GPE_OK;
    }
    b->graph = g;
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        batch_drop_graph(b);
        b->replayed += b->graph_launches;
        b->graph_launches = 0;
        b->use_graph = false;
    }
    return GPE_OK;
}

// Sets *running when any of the n instances has not converged (or failed).
__global__ void k_any_running(const DevScalars* sc, int n, int* running) {
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (!sc[i].done) *running = 1;
}

gpe_status batch_flags(gpe_batch* b) {
    if (b->flag_host) return GPE_OK;
    GPE_CUDA(cudaMalloc((void**)&b->d_running, 2 * sizeof(int)));
    GPE_CUDA(cudaHostAlloc((void**)&b->flag_host, 2 * sizeof(int), cudaHostAllocDefault));
    for (cudaEvent_t& ev : b->flag_ev) GPE_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    return GPE_OK;
}

// Iterations are issued in chunks of IMAG_CHUNK as for one handle: after
// each chunk a flag (any instance still running) lands in pinned memory, the
// host reads the previous chunk's flag while the next chunk is queued, and
// stops issuing once every instance has converged.
template <typename R>
gpe_status batch_step_imag_t(gpe_batch* b, int nsteps, int* iters_done, int* converged) {
    for (gpe_handle* h : b->groups) GPE_TRY(imag_prepare<R>(h));
    if (b->mode == GPE_BATCH_PERSISTENT) GPE_CUDA(cudaMemsetAsync(b->bar, 0, sizeof(GridBar), b->st));
    GPE_TRY(batch_capture<R>(b));
    GPE_TRY(batch_flags(b));
    int issued = 0, slot = 0, prev = -1;
    while (issued < nsteps) {
        const int n = std::min(IMAG_CHUNK, nsteps - issued);
        for (int j = 0; j < n; ++j) {
            if (b->exec) {
                GPE_CUDA(cudaGraphLaunch(b->exec, b->st));
                b->replayed += b->graph_launches;
            } else {
                GPE_TRY(batch_issue_iteration<R>(b));
            }
        }
        issued += n;
        if (issued >= nsteps) break;
        GPE_CUDA(cudaMemsetAsync(b->d_running + slot, 0, sizeof(int), b->st));
        for (gpe_handle* h : b->groups) {
            k_any_running<<<1, 256, 0, b->st>>>(h->sc, h->nb, b->d_running + slot);
            b->groups[0]->launches++;
        }
        GPE_CUDA(cudaMemcpyAsync(b->flag_host + slot, b->d_running + slot, sizeof(int), cudaMemcpyDeviceToHost, b->st));
        GPE_CUDA(cudaEventRecord(b->flag_ev[slot], b->st));
        if (prev >= 0) {
            GPE_CUDA(cudaEventSynchronize(b->flag_ev[prev]));
            if (!b->flag_host[prev]) break;
        }
        prev = slot;
        slot ^= 1;
    }
    GPE_CUDA(cudaStreamSynchronize(b->st));
    GPE_CUDA(cudaGetLastError());
    if (b->mode == GPE_BATCH_PERSISTENT) {
        GridBar bar;
        GPE_CUDA(cudaMemcpy(&bar, b->bar, sizeof(bar), cudaMemcpyDeviceToHost));
        if (bar.status == GPE_ERR_TIMEOUT)
            return fail(GPE_ERR_TIMEOUT, "a grid-barrier wait of the persistent batch kernel expired");
    }
    bool diverged = false;
    std::vector<DevScalars> sv;
    for (size_t g = 0; g < b->groups.size(); ++g) {
        gpe_handle* h = b->groups[g];
        sv.resize(h->nb);
        GPE_CUDA(cudaMemcpy(sv.data(), h->sc, sizeof(DevScalars) * h->nb, cudaMemcpyDeviceToHost));
        for (int i = 0; i < b->n; ++i) {
            if (b->gidx[i] != (int)g) continue;
            const DevScalars& d = sv[b->ginst[i]];
            if (iters_done) iters_done[i] = d.iters_done;
            if (converged) converged[i] = d.converged;
            diverged = diverged || d.status == GPE_ERR_DIVERGED;
        }
    }
    if (diverged) return fail(GPE_ERR_DIVERGED, "an instance has a non-finite norm, energy or chemical potential");
    return GPE_OK;
}

}  // namespace

extern "C" {

gpe_status gpe_batch_create(const gpe_config* cfgs, int n, gpe_batch** out) {
    if (!cfgs || !out || n < 1) return fail(GPE_ERR_INVALID_ARG, "null argument or n < 1");
    *out = nullptr;
    const gpe_config& c0 = cfgs[0];
    for (int i = 0; i < n; ++i) {
        const gpe_config& c = cfgs[i];
        if (c.abi_version != GPE_ABI_VERSION) return fail(GPE_ERR_INVALID_ARG, "abi_version mismatch");
        if (c.ncomp != 1) return fail(GPE_ERR_UNSUPPORTED, "batched instances have one component");
        if (c.hamiltonian != GPE_HAM_BEC && c.hamiltonian != GPE_HAM_TEMPLATE)
            return fail(GPE_ERR_UNSUPPORTED, "batched instances use GPE_HAM_BEC or GPE_HAM_TEMPLATE");
        if (c.precision != c0.precision || c.hamiltonian != c0.hamiltonian || c.imag_scheme != c0.imag_scheme ||
            c.dt != c0.dt || c.beta != c0.beta || c.epsilon_e != c0.epsilon_e || c.npart[0] != c0.npart[0])
            return fail(GPE_ERR_INVALID_ARG,
                        "batched instances share precision, hamiltonian, imag_scheme, dt, beta, epsilon_e, npart");
        if (c.prms[3] > 0 || c.prms[4] > 0 || c.prms[5] > 0)
            return fail(GPE_ERR_UNSUPPORTED, "batched instances have a time-independent coupling (prms[3..5] <= 0)");
        if (c.prms[11] != 0 || c.prms[12] != 0)
            return fail(GPE_ERR_UNSUPPORTED, "batched instances have no moving-frame term (prms[11..12] = 0)");
    }
    gpe_batch* b = new gpe_batch();
    b->n = n;
    b->prec = c0.precision;
    b->gidx.assign(n, -1);
    b->ginst.assign(n, 0);
    std::vector<std::vector<int>> members;
    for (int i = 0; i < n; ++i) {
        int g = -1;
        for (size_t k = 0; k < members.size(); ++k)
            if (same_geometry(cfgs[members[k][0]], cfgs[i])) g = (int)k;
        if (g < 0) {
            g = (int)members.size();
            members.emplace_back();
        }
        b->gidx[i] = g;
        b->ginst[i] = (int)members[g].size();
        members[g].push_back(i);
    }
    for (auto& m : members) {
        gpe_handle* h = nullptr;
        gpe_status s = create_handle(&cfgs[m[0]], (int)m.size(), &h);
        if (s != GPE_OK) {
            gpe_batch_destroy(b);
            return s;
        }
        b->groups.push_back(h);
        for (size_t k = 0; k < m.size(); ++k)
            cudaMemcpy(h->prms + k * GPE_NO_HAMIL_PARAMS, cfgs[m[k]].prms, sizeof(double) * GPE_NO_HAMIL_PARAMS,
                       cudaMemcpyHostToDevice);
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        gpe_batch_destroy(b);
        return fail(GPE_ERR_CUDA, std::string("gpe_batch_create: ") + cudaGetErrorString(e));
    }
    *out = b;
    return GPE_OK;
}

gpe_status gpe_batch_destroy(gpe_batch* b) {
    if (!b) return GPE_OK;
    cudaStreamSynchronize(b->st);
    batch_drop_graph(b);
    if (b->stage_args) cudaFree(b->stage_args);
    if (b->bar) cudaFree(b->bar);
    if (b->d_running) cudaFree(b->d_running);
    if (b->flag_host) cudaFreeHost(b->flag_host);
    for (cudaEvent_t e : b->flag_ev)
        if (e) cudaEventDestroy(e);
    for (gpe_handle* h : b->groups) {
        free_all(h);
        delete h;
    }
    delete b;
    return GPE_OK;
}

gpe_status gpe_batch_set_stream(gpe_batch* b, void* cuda_stream) {
    if (!b) return fail(GPE_ERR_INVALID_ARG, "null batch");
    if ((cudaStream_t)cuda_stream != b->st) batch_drop_graph(b);
    b->st = (cudaStream_t)cuda_stream;
    b->use_graph = true;
    for (gpe_handle* h : b->groups) h->st = b->st;
    return GPE_OK;
}

gpe_status gpe_batch_set_psi(gpe_batch* b, int inst, const double* host_c128) {
    gpe_handle* h;
    size_t off;
    GPE_TRY(batch_inst(b, inst, &h, &off));
    if (!host_c128) return fail(GPE_ERR_INVALID_ARG, "null psi");
    GPE_TRY(canonicalize(h));
    char* A = (char*)h->A[0] + off;
    GPE_TRY(upload_c128_host(h, host_c128, A));
    GPE_CUDA(cudaMemcpyAsync((char*)h->B[0] + off, A, h->esz * h->N, cudaMemcpyDeviceToDevice, h->st));
    GPE_CUDA(cudaStreamSynchronize(h->st));
    h->hb_old_valid = true;
    return GPE_OK;
}

gpe_status gpe_batch_set_vext(gpe_batch* b, int inst, const double* host_c128) {
    gpe_handle* h;
    size_t off;
    GPE_TRY(batch_inst(b, inst, &h, &off));
    if (!host_c128) return fail(GPE_ERR_INVALID_ARG, "null vext");
    return upload_c128_host(h, host_c128, (char*)h->V[0] + off);
}

gpe_status gpe_batch_get_psi(gpe_batch* b, int inst, double* host_c128) {
    gpe_handle* h;
    size_t off;
    GPE_TRY(batch_inst(b, inst, &h, &off));
    if (!host_c128) return fail(GPE_ERR_INVALID_ARG, "null output");
    GPE_TRY(canonicalize(h));
    return download_c128_host(h, (char*)h->A[0] + off, host_c128);
}

gpe_status gpe_batch_step_imag(gpe_batch* b, int nsteps, int* iters_done, int* converged) {
    if (!b) return fail(GPE_ERR_INVALID_ARG, "null batch");
    if (nsteps < 0) return fail(GPE_ERR_INVALID_ARG, "nsteps < 0");
    return b->prec == GPE_C64 ? batch_step_imag_t<float>(b, nsteps, iters_done, converged)
                              : batch_step_imag_t<double>(b, nsteps, iters_done, converged);
}

gpe_status gpe_batch_imag_state(gpe_batch* b, int inst, double* out) {
    gpe_handle* h;
    size_t off;
    GPE_TRY(batch_inst(b, inst, &h, &off));
    if (!out) return fail(GPE_ERR_INVALID_ARG, "null output");
    DevScalars d;
    GPE_CUDA(cudaStreamSynchronize(h->st));
    GPE_CUDA(cudaMemcpy(&d, h->sc + b->ginst[inst], sizeof(d), cudaMemcpyDeviceToHost));
    out[0] = d.norm[0];
    out[1] = d.mu[0];
    out[2] = d.en[0];
    out[3] = d.en_prev[0];
    return GPE_OK;
}

gpe_status gpe_batch_set_launch_mode(gpe_batch* b, int mode, unsigned int wait_bound) {
    if (!b) return fail(GPE_ERR_INVALID_ARG, "null batch");
    if (mode != GPE_BATCH_PER_GROUP && mode != GPE_BATCH_PERSISTENT && mode != GPE_BATCH_GROUPED)
        return fail(GPE_ERR_INVALID_ARG, "unknown batch launch mode");
    if (mode != GPE_BATCH_PER_GROUP) {
        const std::string why = batch_persistent_reason(b);
        if (!why.empty()) return fail(GPE_ERR_UNSUPPORTED, "all-group batch launches: " + why);
        GPE_CUDA(cudaStreamSynchronize(b->st));
        GPE_TRY(b->prec == GPE_C64 ? batch_build_stages<float>(b) : batch_build_stages<double>(b));
    }
    batch_drop_graph(b);  // the captured launches carry the old choice and bound
    b->mode = mode;
    b->wait_bound = wait_bound;
    b->use_graph = true;
    return GPE_OK;
}

int gpe_batch_launch_mode(const gpe_batch* b) { return b ? b->mode : GPE_BATCH_PER_GROUP; }

gpe_status gpe_batch_set_persistent(gpe_batch* b, int enable, unsigned int wait_bound) {
    return gpe_batch_set_launch_mode(b, enable ? GPE_BATCH_PERSISTENT : GPE_BATCH_PER_GROUP, wait_bound);
}

int gpe_batch_persistent(const gpe_batch* b) { return (b && b->mode == GPE_BATCH_PERSISTENT) ? 1 : 0; }

gpe_status gpe_batch_persistent_info(const gpe_batch* b, long long* out) {
    if (!b || !out) return fail(GPE_ERR_INVALID_ARG, "null argument");
    const cudaError_t e = batch_stage_attributes(b->prec == GPE_C64 ? 8 : 16, out);
    if (e != cudaSuccess) return fail(GPE_ERR_CUDA, std::string("stage kernel attributes: ") + cudaGetErrorString(e));
    out[8] = b->stage_grid;
    return GPE_OK;
}

long long gpe_batch_kernel_launches(const gpe_batch* b) {
    if (!b) return 0;
    long long n = b->replayed + b->stage_launches;
    for (const gpe_handle* h : b->groups) n += h->launches;
    return n;
}

}  // extern "C"

// ==========================================================================================
// Autotuner: pass variants per grid (no counterpart in the reference, which
// leaves the transform plan to cuFFT's planner, src/parallel.cu:77-110).
//
// For a grid, precision and field count the tuner times, on a temporary
// handle, every strided-pass variant (svar: scalar or paired complex64 lines,
// tile width, resident CTAs per SM, radix order) of each strided axis and pass
// mode with CUDA events, keeps the fastest, then times whole steps of the
// workload (real-time RK4 steps or imaginary-time iterations) for each
// x-pass row count per CTA (which sets how full the x pass's last wave is),
// and keeps the fastest.  The result is one line of a JSON-lines cache,
// keyed by (nx, ny, nz, precision, fields, instances), which gpe_create and
// gpe_batch_create apply when a cache is set (gpe_set_tune_cache or
// $GPE_TUNE_CACHE).  Without a cache every handle uses the default variants.
// ==========================================================================================
#include <fstream>
#include <mutex>
#include <sstream>

namespace {

std::mutex g_tune_mu;
std::string g_tune_path;
bool g_tune_path_set = false;

std::string tune_cache_path() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_tune_path_set) return g_tune_path;
    const char* env = std::getenv("GPE_TUNE_CACHE");
    return env ? std::string(env) : std::string();
}

bool length_tuned(int L) {
#define GPE_IS(n) if (L == n) return true;
    GPE_TUNED_p2(GPE_IS) GPE_TUNED_p2b(GPE_IS) GPE_TUNED_p3(GPE_IS) GPE_TUNED_p3b(GPE_IS)
    GPE_TUNED_p5(GPE_IS) GPE_TUNED_p5b(GPE_IS) GPE_TUNED_p9(GPE_IS) GPE_TUNED_p9b(GPE_IS)
#undef GPE_IS
    return false;
}

// Whether strided-pass variant v can serve axis `axis` of handle h (see launch_s).
bool variant_usable(const gpe_handle* h, int axis, int v) {
    const int L = axis == 1 ? h->ny : h->nz;
    const int esz = (int)h->esz;
    if (v == 0) return true;
    if (v == 1)
        return esz == 8 && h->nx % 2 == 0 && (h->nf == 1 || (make_plan(L).E <= 8 && L >= 64));
    if (v < 0 || v >= NSVAR || h->nf != 1 || !length_tuned(L)) return false;
    const SVar s = svar(esz, L, v);
    return s.ok && (!s.paired || h->nx % 2 == 0);
}

struct TuneKey {
    int nx, ny, nz, prec, nf, nb;
};
TuneKey tune_key(const gpe_handle* h) { return TuneKey{h->nx, h->ny, h->nz, h->prec, h->nf, h->nb}; }

bool json_int(const std::string& line, const char* key, int* out) {
    const std::string k = std::string("\"") + key + "\":";
    const size_t p = line.find(k);
    if (p == std::string::npos) return false;
    char* end = nullptr;
    const long v = std::strtol(line.c_str() + p + k.size(), &end, 10);
    if (end == line.c_str() + p + k.size()) return false;
    *out = (int)v;
    return true;
}

bool line_key(const std::string& line, TuneKey* k) {
    return json_int(line, "nx", &k->nx) && json_int(line, "ny", &k->ny) && json_int(line, "nz", &k->nz) &&
           json_int(line, "prec", &k->prec) && json_int(line, "nf", &k->nf) && json_int(line, "nb", &k->nb);
}
bool same_key(const TuneKey& a, const TuneKey& b) {
    return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.prec == b.prec && a.nf == b.nf && a.nb == b.nb;
}

std::string tune_line(const gpe_handle* h, double def_us, double tuned_us) {
    std::ostringstream o;
    const TuneKey k = tune_key(h);
    o << "{\"nx\":" << k.nx << ",\"ny\":" << k.ny << ",\"nz\":" << k.nz << ",\"prec\":" << k.prec
      << ",\"nf\":" << k.nf << ",\"nb\":" << k.nb;
    for (int ax = 1; ax <= 2; ++ax)
        for (int m = 0; m < 3; ++m) o << ",\"s" << ax << m << "\":" << h->svar[ax][m];
    o << ",\"xrows\":" << h->xrows << ",\"yz\":" << h->yz << ",\"flow\":" << h->flow << ",\"xstage\":" << h->xstage;
    char buf[64];
    std::snprintf(buf, sizeof(buf), ",\"default_us\":%.3f,\"tuned_us\":%.3f}", def_us, tuned_us);
    o << buf;
    return o.str();
}

// Applies the cache line of h's key, if any (the last one in the file wins).
// Variants that do not exist for h are ignored.
void tune_apply_cache(gpe_handle* h) {
    const std::string path = tune_cache_path();
    if (path.empty()) return;
    std::ifstream f(path);
    if (!f) return;
    const TuneKey want = tune_key(h);
    std::string line, hit;
    while (std::getline(f, line)) {
        TuneKey k;
        if (line_key(line, &k) && same_key(k, want)) hit = line;
    }
    if (hit.empty()) return;
    for (int ax = 1; ax <= 2; ++ax)
        for (int m = 0; m < 3; ++m) {
            const std::string key = "s" + std::to_string(ax) + std::to_string(m);
            int v = 0;
            if (json_int(hit, key.c_str(), &v) && variant_usable(h, ax, v)) h->svar[ax][m] = v;
        }
    int r = 0;
    if (json_int(hit, "xrows", &r) && r >= 0 && r <= 256) h->xrows = r;
    int yz = 0;
    if (json_int(hit, "yz", &yz) && (yz == 0 || (yz == 1 && yz_usable(h, h->nf)))) h->yz = yz;
    int xs = 0;
    if (json_int(hit, "xstage", &xs) && (xs == 0 || xs == 1)) h->xstage = xs;
    int fl = 0;
    if (json_int(hit, "flow", &fl) && ((fl == 1 && flow_eligible(h)) || fl == 2)) flow_enable(h, fl, 0);
}

// Replaces the line of h's key in the cache file (or appends it).
gpe_status tune_store(const gpe_handle* h, const char* path, double def_us, double tuned_us) {
    if (!path || !path[0]) return GPE_OK;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::vector<std::string> keep;
    {
        std::ifstream f(path);
        std::string line;
        const TuneKey want = tune_key(h);
        while (f && std::getline(f, line)) {
            TuneKey k;
            if (line.empty() || (line_key(line, &k) && same_key(k, want))) continue;
            keep.push_back(line);
        }
    }
    keep.push_back(tune_line(h, def_us, tuned_us));
    const std::string tmp = std::string(path) + ".tmp";
    {
        std::ofstream o(tmp, std::ios::trunc);
        if (!o) return fail(GPE_ERR_IO, std::string("cannot write ") + tmp);
        for (const auto& l : keep) o << l << "\n";
        if (!o) return fail(GPE_ERR_IO, std::string("cannot write ") + tmp);
    }
    if (std::rename(tmp.c_str(), path) != 0) return fail(GPE_ERR_IO, std::string("cannot replace ") + path);
    return GPE_OK;
}

// A normalised uniform state in every instance and component: the tuning
// handle's steps then run their full arithmetic (no zero norms).
template <typename C>
__global__ void k_fill_const(C* dst, double v, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = from_d<C>(make_double2(v, 0.0));
}

// Microseconds per launch of one strided pass (3 untimed launches, then 20).
template <typename R>
gpe_status time_pass(gpe_handle* h, int axis, int mode, double* us) {
    PassArgs<R> a = base_args<R>(h);
    a.pro = PRO_PIN;
    a.epi = EPI_STORE;
    for (int i = 0; i < 3; ++i) GPE_TRY(launch_s<R>(h, a, h->nf, axis, mode));
    cudaEvent_t e0, e1;
    GPE_CUDA(cudaEventCreate(&e0));
    GPE_CUDA(cudaEventCreate(&e1));
    cudaEventRecord(e0, h->st);
    gpe_status s = GPE_OK;
    for (int i = 0; i < 20 && s == GPE_OK; ++i) s = launch_s<R>(h, a, h->nf, axis, mode);
    cudaEventRecord(e1, h->st);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s != GPE_OK) return s;
    if (e != cudaSuccess) return fail(GPE_ERR_CUDA, std::string("tuner timing: ") + cudaGetErrorString(e));
    *us = 1e3 * ms / 20.0;
    return GPE_OK;
}

// Microseconds per step of the workload: 0 real-time RK4 steps, 1 imaginary-
// time iterations of the handle's scheme (the tuning config never converges).
// Median of three groups of 10 steps after 3 untimed ones.
template <typename R>
gpe_status time_steps(gpe_handle* h, int workload, double* us) {
    auto issue = [&](int n) -> gpe_status {
        if (workload == 0) return step_real_t<R>(h, 0, n, nullptr);
        GPE_TRY(imag_prepare<R>(h));
        return imag_issue<R>(h, 0, n);
    };
    GPE_TRY(issue(3));
    double t[3];
    for (int r = 0; r < 3; ++r) {
        cudaEvent_t e0, e1;
        GPE_CUDA(cudaEventCreate(&e0));
        GPE_CUDA(cudaEventCreate(&e1));
        cudaEventRecord(e0, h->st);
        gpe_status s = issue(10);
        cudaEventRecord(e1, h->st);
        cudaError_t e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (s != GPE_OK) return s;
        if (e != cudaSuccess) return fail(GPE_ERR_CUDA, std::string("tuner timing: ") + cudaGetErrorString(e));
        t[r] = 1e3 * ms / 10.0;
    }
    std::sort(t, t + 3);
    *us = t[1];
    return GPE_OK;
}

// Tunes handle h (a temporary of the config to tune) in place.
template <typename R>
gpe_status tune_handle_t(gpe_handle* h, int workload, double* report) {
    typedef typename Cx<R>::T C;
    const double DV = h->cfg.dx[0] * h->cfg.dx[1] * h->cfg.dx[2];
    const double amp = std::sqrt(h->cfg.npart[0] / ((double)h->N * DV));
    for (int c = 0; c < h->ncomp; ++c) {
        k_fill_const<C><<<blocks_for(h->N * h->nb, 256), 256, 0, h->st>>>((C*)h->A[c], amp, h->N * h->nb);
        k_fill_const<C><<<blocks_for(h->N * h->nb, 256), 256, 0, h->st>>>((C*)h->B[c], amp, h->N * h->nb);
    }
    GPE_CUDA(cudaGetLastError());
    GPE_CUDA(cudaStreamSynchronize(h->st));
    h->hb_old_valid = true;
    double def_us = 0.0;
    GPE_TRY(time_steps<R>(h, workload, &def_us));
    int timed = 0;
    int axes[2], na = 0;
    if (h->ny > 1) axes[na++] = 1;
    if (h->nz > 1) axes[na++] = 2;
    for (int i = 0; i < na; ++i) {
        const int ax = axes[i];
        const int modes[2] = {SM_FWD, SM_INV};
        const int nm = (i == na - 1) ? 1 : 2;
        for (int j = 0; j < nm; ++j) {
            const int mode = (i == na - 1) ? SM_FKI : modes[j];
            const int mi = mode == SM_FWD ? 0 : (mode == SM_FKI ? 1 : 2);
            int best = 0;
            double best_us = 1e30;
            for (int v = 0; v < NSVAR; ++v) {
                if (!variant_usable(h, ax, v)) continue;
                h->svar[ax][mi] = v;
                double us = 0.0;
                if (time_pass<R>(h, ax, mode, &us) != GPE_OK) {
                    cudaGetLastError();
                    continue;
                }
                ++timed;
                if (us < best_us * 0.99) {
                    best_us = us;
                    best = v;
                }
            }
            h->svar[ax][mi] = best;
        }
    }
    // x-pass rows per CTA: whole steps with the chosen strided variants
    const int T = plan_T(h->nx);
    const int rmax = (256 / T) > 0 ? 256 / T : 1;
    int best_r = 0;
    double best_us = 1e30;
    // from a quarter of the longest tile up: at 128 (16 threads a row) four
    // rows make 64-thread CTAs, sixteen of which fill an SM's 64 warps; a
    // larger tile is kept only when it is 1 % faster, so near-ties go to the
    // fuller occupancy (whose lead grows when the step starts from a cold L2)
    for (int r = rmax / 4 > 1 ? rmax / 4 : 1; r <= rmax; ++r) {
        h->xrows = (r == rmax) ? 0 : r;
        double us = 0.0;
        GPE_TRY(time_steps<R>(h, workload, &us));
        ++timed;
        if (us < best_us * 0.99) {
            best_us = us;
            best_r = h->xrows;
        }
    }
    h->xrows = best_r;
    // the fused y-z cluster kernel against the chosen strided passes
    if (yz_usable(h, h->nf)) {
        h->yz = 1;
        double us = 0.0;
        gpe_status s = time_steps<R>(h, workload, &us);
        ++timed;
        if (s != GPE_OK || !(us < best_us * 0.99)) {
            cudaGetLastError();
            h->yz = 0;
        }
        GPE_CUDA(cudaStreamSynchronize(h->st));
    }
    double tuned_us = 0.0;
    GPE_TRY(time_steps<R>(h, workload, &tuned_us));
    // real-time complex64 one-field chains: the fused x pass with staged
    // epilogue inputs, at the chosen rows and at half and a quarter of the
    // longest tile (staging takes shared memory, so fewer rows may pay)
    if (workload == 0 && h->prec == GPE_C64 && h->nf == 1 && h->nb == 1 && (h->ny > 1 || h->nz > 1)) {
        const int rows0 = h->xrows;
        const int rtry[3] = {rows0, rmax / 2, rmax / 4};
        int best_rows = rows0;
        bool keep = false;
        for (int k = 0; k < 3; ++k) {
            if (rtry[k] < 0 || (k > 0 && (rtry[k] < 1 || rtry[k] == rows0))) continue;
            h->xstage = 1;
            h->xrows = rtry[k];
            double us = 0.0;
            const gpe_status s = time_steps<R>(h, workload, &us);
            ++timed;
            if (s == GPE_OK && us < tuned_us * 0.99) {
                tuned_us = us;
                best_rows = rtry[k];
                keep = true;
            } else {
                cudaGetLastError();
            }
        }
        h->xstage = keep ? 1 : 0;
        h->xrows = keep ? best_rows : rows0;
        GPE_CUDA(cudaStreamSynchronize(h->st));
    }
    // real-time steps as one persistent launch each (same arithmetic)
    if (workload == 0 && flow_eligible(h)) {
        double us = 0.0;
        gpe_status s = flow_enable(h, 1, 0);
        if (s == GPE_OK) s = time_steps<R>(h, workload, &us);
        ++timed;
        int st = 0;
        if (h->flow_sync) {
            cudaStreamSynchronize(h->st);
            cudaMemcpy(&st, &h->flow_sync->status, sizeof(int), cudaMemcpyDeviceToHost);
        }
        if (s != GPE_OK || st != 0 || !(us < tuned_us * 0.99)) {
            cudaGetLastError();
            h->flow = 0;
        } else {
            tuned_us = us;
        }
        GPE_CUDA(cudaStreamSynchronize(h->st));
    }
    // the three strided passes of each stage as one persistent launch
    if (h->flow == 0 && h->prec == GPE_C64 && h->nf == 1 && h->nb == 1 && h->nx % 2 == 0 &&
        flow_shape_supported(h->nx, h->ny, h->nz)) {
        double us = 0.0;
        gpe_status s = flow_enable(h, 2, 0);
        if (s == GPE_OK) s = time_steps<R>(h, workload, &us);
        ++timed;
        int st = 0;
        if (h->flow_sync) {
            cudaStreamSynchronize(h->st);
            cudaMemcpy(&st, &h->flow_sync->status, sizeof(int), cudaMemcpyDeviceToHost);
        }
        if (s != GPE_OK || st != 0 || !(us < tuned_us * 0.99)) {
            cudaGetLastError();
            h->flow = 0;
        } else {
            tuned_us = us;
        }
        GPE_CUDA(cudaStreamSynchronize(h->st));
    }
    // the choices were made pass by pass and step by step; keep them only if
    // together they beat the default variants (small grids are noisy)
    if (!(tuned_us < def_us)) {
        for (int ax = 0; ax < 3; ++ax)
            for (int m = 0; m < 3; ++m) h->svar[ax][m] = 0;
        h->xrows = 0;
        h->yz = 0;
        h->flow = 0;
        h->xstage = 0;
        tuned_us = def_us;
    }
    if (report) {
        report[0] = def_us;
        report[1] = tuned_us;
        report[2] = timed;
    }
    return GPE_OK;
}

// Tunes a temporary handle of cfg with nb instances; variants out in *h_out
// (the caller destroys it).
gpe_status tune_config(const gpe_config* cfg, int nb, int workload, double* report, gpe_handle** h_out) {
    gpe_config c = *cfg;
    c.epsilon_e = -1.0;  // never converges: every timed iteration does its work
    gpe_handle* h = nullptr;
    GPE_TRY(create_handle(&c, nb, &h));
    for (int ax = 0; ax < 3; ++ax)
        for (int m = 0; m < 3; ++m) h->svar[ax][m] = 0;
    h->xrows = 0;
    h->yz = 0;
    h->flow = 0;
    h->xstage = 0;
    gpe_status s = h->prec == GPE_C64 ? tune_handle_t<float>(h, workload, report)
                                      : tune_handle_t<double>(h, workload, report);
    if (s != GPE_OK) {
        cudaStreamSynchronize(h->st);
        free_all(h);
        delete h;
        return s;
    }
    *h_out = h;
    return GPE_OK;
}

}  // namespace

extern "C" {

gpe_status gpe_set_tune_cache(const char* path) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_path_set = path != nullptr;
    g_tune_path = path ? path : "";
    return GPE_OK;
}

gpe_status gpe_tune(const gpe_config* cfg, int workload, const char* cache_path, double* report) {
    if (!cfg) return fail(GPE_ERR_INVALID_ARG, "null config");
    if (workload != 0 && workload != 1) return fail(GPE_ERR_INVALID_ARG, "workload must be 0 (real) or 1 (imaginary)");
    gpe_handle* h = nullptr;
    double rep[3] = {0, 0, 0};
    GPE_TRY(tune_config(cfg, 1, workload, rep, &h));
    gpe_status s = tune_store(h, cache_path, rep[0], rep[1]);
    if (report) {
        report[0] = rep[0];
        report[1] = rep[1];
        report[2] = rep[2];
        for (int ax = 1; ax <= 2; ++ax)
            for (int m = 0; m < 3; ++m) report[3 + (ax - 1) * 3 + m] = h->svar[ax][m];
        report[9] = h->xrows;
        report[10] = h->yz;
        report[11] = h->flow;
        report[12] = h->xstage;
    }
    cudaStreamSynchronize(h->st);
    free_all(h);
    delete h;
    return s;
}

gpe_status gpe_set_flow(gpe_handle* h, int on, unsigned wait_bound) {
    GPE_TRY(check_handle(h));
    if (on < 0 || on > 2) return fail(GPE_ERR_INVALID_ARG, "mode must be 0, 1 or 2");
    GPE_TRY(flow_enable(h, on, wait_bound));
    GPE_CUDA(cudaStreamSynchronize(h->st));
    return GPE_OK;
}

gpe_status gpe_set_x_staging(gpe_handle* h, int on) {
    GPE_TRY(check_handle(h));
    if (on != 0 && on != 1) return fail(GPE_ERR_INVALID_ARG, "on must be 0 or 1");
    h->xstage = on;
    return GPE_OK;
}

int gpe_x_staging(const gpe_handle* h) { return h ? h->xstage : 0; }

int gpe_flow_active(const gpe_handle* h) {
    if (!h) return 0;
    if (flow_usable(h)) return 1;
    return flow_strided_usable(h, h->nf) && h->ny > 1 && h->nz > 1 ? 2 : 0;
}

gpe_status gpe_flow_status(gpe_handle* h, int* status_out) {
    GPE_TRY(check_handle(h));
    if (!status_out) return fail(GPE_ERR_INVALID_ARG, "null status");
    *status_out = 0;
    GPE_CUDA(cudaStreamSynchronize(h->st));
    if (!h->flow_sync) return GPE_OK;
    int st = 0;
    GPE_CUDA(cudaMemcpy(&st, &h->flow_sync->status, sizeof(int), cudaMemcpyDeviceToHost));
    *status_out = st;
    if (st != 0) {  // re-arm: counters, tickets and both status words
        GPE_CUDA(cudaMemset(h->flow_sync, 0, sizeof(FlowSync)));
        int hs = 0;
        GPE_CUDA(cudaMemcpy(&hs, &h->sc->status, sizeof(int), cudaMemcpyDeviceToHost));
        if (hs == GPE_ERR_TIMEOUT) GPE_CUDA(cudaMemset(&h->sc->status, 0, sizeof(int)));
        h->flow_launches = 0;
    }
    return GPE_OK;
}

gpe_status gpe_get_pass_variants(const gpe_handle* h, int* out) {
    if (!h || !out) return fail(GPE_ERR_INVALID_ARG, "null argument");
    for (int ax = 1; ax <= 2; ++ax)
        for (int m = 0; m < 3; ++m) out[(ax - 1) * 3 + m] = h->svar[ax][m];
    out[6] = h->xrows;
    out[7] = h->yz;
    return GPE_OK;
}

gpe_status gpe_set_pass_variants(gpe_handle* h, const int* in) {
    if (!h || !in) return fail(GPE_ERR_INVALID_ARG, "null argument");
    for (int ax = 1; ax <= 2; ++ax)
        for (int m = 0; m < 3; ++m)
            if (!variant_usable(h, ax, in[(ax - 1) * 3 + m]))
                return fail(GPE_ERR_UNSUPPORTED, "pass variant " + std::to_string(in[(ax - 1) * 3 + m]) +
                                                     " does not exist for axis " + std::to_string(ax));
    if (in[6] < 0 || in[6] > 256) return fail(GPE_ERR_INVALID_ARG, "xrows must be 0..256");
    if (in[7] != 0 && !(in[7] == 1 && yz_usable(h, h->nf)))
        return fail(GPE_ERR_UNSUPPORTED, "the fused y-z kernel does not serve this grid");
    for (int ax = 1; ax <= 2; ++ax)
        for (int m = 0; m < 3; ++m) h->svar[ax][m] = in[(ax - 1) * 3 + m];
    h->xrows = in[6];
    h->yz = in[7];
    return GPE_OK;
}

int gpe_pass_variant_exists(const gpe_config* cfg, int axis, int v) {
    if (!cfg || axis < 1 || axis > 2) return 0;
    gpe_handle tmp;
    tmp.nx = cfg->nx;
    tmp.ny = cfg->ny;
    tmp.nz = cfg->nz;
    tmp.esz = cfg->precision == GPE_C64 ? 8 : 16;
    tmp.nf = cfg->ncomp + ((cfg->hamiltonian == GPE_HAM_DIPOLAR || cfg->hamiltonian == GPE_HAM_SOFT) ? 1 : 0);
    const int L = axis == 1 ? cfg->ny : cfg->nz;
    if (L <= 1) return v == 0 ? 1 : 0;
    return variant_usable(&tmp, axis, v) ? 1 : 0;
}

gpe_status gpe_batch_tune(gpe_batch* b, const char* cache_path, double* report) {
    if (!b) return fail(GPE_ERR_INVALID_ARG, "null batch");
    for (size_t g = 0; g < b->groups.size(); ++g) {
        gpe_handle* hg = b->groups[g];
        gpe_handle* t = nullptr;
        double rep[3] = {0, 0, 0};
        GPE_TRY(tune_config(&hg->cfg, hg->nb, 1, rep, &t));
        for (int ax = 0; ax < 3; ++ax)
            for (int m = 0; m < 3; ++m) hg->svar[ax][m] = t->svar[ax][m];
        hg->xrows = t->xrows;
        hg->yz = t->yz;
        gpe_status s = tune_store(t, cache_path, rep[0], rep[1]);
        cudaStreamSynchronize(t->st);
        free_all(t);
        delete t;
        GPE_TRY(s);
        if (report) {
            report[2 * g] = rep[0];
            report[2 * g + 1] = rep[1];
        }
    }
    batch_drop_graph(b);  // the captured iteration holds the old kernels
    b->use_graph = true;
    return GPE_OK;
}

int gpe_batch_groups(const gpe_batch* b) { return b ? (int)b->groups.size() : 0; }

}  // extern "C"
