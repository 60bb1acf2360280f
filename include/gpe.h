/*
 * gpe.h -- C ABI of the B200-native Gross-Pitaevskii solver (libgpe.so).
 *
 * The reference (fGPE v0.3) exposes its hot path as a C++ class hierarchy,
 * not an FFI:  Cuda <- BaseHamiltonian <- OneComponentGPSolver /
 * TwoComponentGPSolver <- BEConeComponent / BECtwoComponent / SingleTemplate.
 * Every entry point below replaces one member (or one member sequence) of that
 * hierarchy; the replaced reference interface is cited beside each one as
 * path:line inside the reference project.  The C++ plugin classes in
 * fgpe_b200/host/ call these functions the way the reference's plugins call
 * their base-class members.
 *
 * Conventions
 *  - Every call returns gpe_status; GPE_OK is 0.  On failure
 *    gpe_last_error_string() returns a one-line message (thread-local).
 *    Nothing here calls exit(); the reference exits on a missing key
 *    (src/input_variables.cu:171-209) and prints-and-continues on CUDA errors
 *    (src/parallel.cu:7-11, CCE).
 *  - Host wavefunction / potential buffers are interleaved complex128
 *    (re, im pairs of double), index z*NX*NY + y*NX + x (hpp/header.hpp:20,
 *    ID macro), i.e. exactly the bytes of a .wdat file
 *    (src/output.cu:262-277).  The complex64 form converts on the device.
 *  - A handle owns its device buffers; it is not thread-shared, distinct
 *    handles are independent.  All GPU work of a handle is issued on the
 *    stream set by gpe_set_stream (default: the legacy default stream).
 *  - Units are the reference's code units: lengths in a_ho, time in 1/omega_ho,
 *    energies in hbar*omega_ho (src/params.cu:223-279).
 */
#ifndef GPE_B200_GPE_H
#define GPE_B200_GPE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPE_ABI_VERSION 2
/* hpp/header.hpp:23  NO_HAMIL_PARAMS: size of d_h_params */
#define GPE_NO_HAMIL_PARAMS 32

typedef enum gpe_status {
    GPE_OK = 0,
    GPE_ERR_INVALID_ARG = 1,   /* null pointer, bad component, bad enum   */
    GPE_ERR_UNSUPPORTED = 2,   /* grid length with no FFT plan, option off */
    GPE_ERR_CUDA = 3,          /* a CUDA runtime call failed               */
    GPE_ERR_OUT_OF_MEMORY = 4, /* device or pinned allocation failed       */
    GPE_ERR_DIVERGED = 5,      /* NaN/Inf seen by the device watchdog      */
    GPE_ERR_TIMEOUT = 6,       /* a bounded device wait gave up            */
    GPE_ERR_IO = 7             /* file could not be opened / short read    */
} gpe_status;

/* Storage / arithmetic form of the fields.
 *  GPE_C128: complex128 everywhere (the drop-in; cuFFT Z2Z in the reference,
 *            src/parallel.cu:97-102).
 *  GPE_C64 : complex64 fields, FFT butterflies and real-time RK4 stage
 *            updates in FP32; norm, energy, chemical potential, the
 *            imaginary-time update, renormalisation and the convergence
 *            test stay FP64 (compensated sums).  Between real-time steps
 *            the state is carried as float32 high + low parts (error-free
 *            sum at the last stage), so its rounding does not accumulate;
 *            gpe_set_psi stores the complex128 input's rounding residual as
 *            the low part and gpe_get_psi returns the sum.  Imaginary-time
 *            steps and gpe_fft use the high part alone and drop the low
 *            part; the control gradient carries both parts through its
 *            forward steps and checkpoints. */
typedef enum gpe_precision { GPE_C128 = 0, GPE_C64 = 1 } gpe_precision;

/* Which Hamiltonian plugin supplies the pointwise term.
 *  GPE_HAM_BEC      hamiltonians/BEC_oneComponent.cu:128-178 (prms[0..5] = quench a0,a1,a2,t1,t2,t3)
 *  GPE_HAM_BEC2     hamiltonians/BEC_twoComponent.cu:168-244 (prms[0..2] = a11,a22,a12)
 *  GPE_HAM_TEMPLATE hamiltonians/single_template.cu:333-373  (h = T only)
 *  GPE_HAM_DIPOLAR  GPE_HAM_BEC plus a k-space dipolar term; prms[6] = a_dd,
 *                   prms[7..9] = dipole direction, prms[10] = spherical
 *                   real-space cut-off radius R (0 = no cut-off).  The kernel
 *                   is 12*pi*a_dd*((k.d)^2/k^2 - 1/3) as in
 *                   src/parallel.cu:326-352 (never called there), times
 *                   1 + 3cos(kR)/(kR)^2 - 3sin(kR)/(kR)^3 with k in rad/length
 *                   (summed as its power series below kR = 0.5, where the
 *                   closed form cancels; 0 at k = 0, the limit).
 *  GPE_HAM_SOFT     one component, h = T + (V + Phi) psi with the mean field
 *                   Phi = IFFT(V~(k) FFT|psi|^2) / N of a soft-core
 *                   interaction, V~ of SoftCoreInteraction_1D/2D/3D
 *                   (src/parallel.cu:360-477, never called there) by
 *                   gpe_config.dim: prms[0] = a (radius), prms[1] = U,
 *                   k = 2 pi |k| in rad/length; 1D 2U sin(ak)/k, 2D
 *                   2 pi a U J1(ka)/k, 3D 4 pi U a^3 (sin ka - ka cos ka)/(ka)^3,
 *                   with the reference's small-k forms below k = 1e-6.  No
 *                   contact term; the energy density takes Phi/2.
 *  Moving-frame term (the plugins' trotate option, BaseHamiltonian::alg_addVPx,
 *  src/baseHamiltonian.cu:198-211): for every Hamiltonian but the template,
 *  prms[11 + c] = lambda_c (2 pi omega / (omho aho) in the reference,
 *  hamiltonians/BEC_oneComponent.cu:98-101) adds -lambda_c P_x psi_c, with
 *  P_x psi = IFFT(kx FFT psi)/N and kx in cycles/length, exactly where the
 *  reference's alg_calcHpsi adds it: heavy-ball imaginary steps, stage 4 of a
 *  one-component real-time step, gpe_apply_h and gpe_observables. */
typedef enum gpe_hamiltonian {
    GPE_HAM_BEC = 0,
    GPE_HAM_BEC2 = 1,
    GPE_HAM_TEMPLATE = 2,
    GPE_HAM_DIPOLAR = 3,
    GPE_HAM_SOFT = 4,
    /* One component, the pointwise term supplied by a user plugin
     * (gpe_set_user_hamiltonian, include/gpe_plugin.cuh): the counterpart of
     * the reference's user-written Hamiltonian kernels
     * (hamiltonians/BEC_oneComponent.hpp:8-22, the empty slot
     * hamiltonians/single_template.cu:333-373). */
    GPE_HAM_USER = 5
} gpe_hamiltonian;

/* Imaginary-time scheme.
 *  GPE_IMAG_HEAVYBALL  the reference's scheme, src/parallel.cu:294-302 with the
 *                      loop of src/oneComponentGPSolver.cu:46-95 (1 component)
 *                      and src/twoComponentGPSolver.cu:35-105 (2 components).
 *  GPE_IMAG_RK4        classic RK4 on d(psi)/d(tau) = -H psi, renormalised to
 *                      npart after every step; mu and E of the normalised
 *                      state; converged when |mu_n - mu_{n-1}| < epsilon_e.
 *                      Not in the reference (its imaginary time is not RK4). */
typedef enum gpe_imag_scheme { GPE_IMAG_HEAVYBALL = 0, GPE_IMAG_RK4 = 1 } gpe_imag_scheme;

typedef struct gpe_config {
    int    abi_version;          /* must be GPE_ABI_VERSION                     */
    int    nx, ny, nz;           /* Params::NX[3]   hpp/params.hpp:23          */
    int    dim;                  /* Params::DIM     src/params.cu:145-154      */
    double xmax[3];              /* Params::XMAX, code units                   */
    double dx[3];                /* Params::DX, code units                     */
    int    ncomp;                /* 1 or 2                                      */
    int    precision;            /* gpe_precision                              */
    int    hamiltonian;          /* gpe_hamiltonian                            */
    int    imag_scheme;          /* gpe_imag_scheme                            */
    double prms[GPE_NO_HAMIL_PARAMS]; /* d_h_params, hpp/parallel.hpp:39      */
    double dt;                   /* code units: p.dt*p.omho/1000               */
    double beta;                 /* heavy-ball momentum, input key "beta"      */
    double npart[2];             /* norm targets, Params::npart / npart1,2     */
    double epsilon_e;            /* convergence threshold, input "epsilon_e"   */
    int    reserved[8];          /* must be zero                                */
} gpe_config;

typedef struct gpe_handle gpe_handle;

/* ---- library ---------------------------------------------------------- */
int         gpe_abi_version(void);
const char* gpe_last_error_string(void);
const char* gpe_status_string(gpe_status s);
/* Fill cfg with defaults (abi_version set, 1 component, C128, BEC, heavy-ball). */
gpe_status  gpe_config_init(gpe_config* cfg);
/* 1 when a grid length has a device FFT plan (products of 2, 3 and 5 up to
 * 1024 whose plan needs at most 24 values per thread), else 0. */
int         gpe_fft_length_supported(int n);
/* The k-space interaction kernel V~(k) that gpe_create uploads for
 * GPE_HAM_DIPOLAR or GPE_HAM_SOFT (documented with gpe_hamiltonian), before
 * the division by the number of points that the unnormalised inverse
 * transform needs: out[iz*NY*NX + iy*NX + ix] at the k axes of
 * BaseHamiltonian::InitializeKspace (src/baseHamiltonian.cu:53-82), FP64,
 * NX*NY*NZ values.  Host arithmetic only (no device is touched).  The dipolar
 * form is the reference's DipoleDipoleInteraction (src/parallel.cu:326-352)
 * times the spherical cut-off factor; the soft-core forms are
 * SoftCoreInteraction_1D/2D/3D (src/parallel.cu:360-477). */
gpe_status  gpe_kspace_kernel(const gpe_config* cfg, double* out);

/* ---- lifecycle: replaces Cuda::Cuda / ~Cuda (src/parallel.cu:14-113,
 * hpp/parallel.hpp:80-126) and BaseHamiltonian::InitializeKspace/Space
 * (src/baseHamiltonian.cu:25-82). ---------------------------------------- */
gpe_status gpe_create(const gpe_config* cfg, gpe_handle** out);
gpe_status gpe_destroy(gpe_handle* h);
/* cudaStream_t passed as void*; NULL = legacy default stream. */
gpe_status gpe_set_stream(gpe_handle* h, void* cuda_stream);
/* Replaces the H2D copy of d_h_params (hamiltonians/BEC_oneComponent.cu:15). */
gpe_status gpe_set_params(gpe_handle* h, const double prms[GPE_NO_HAMIL_PARAMS]);

/* ---- data in / out: replaces the cudaMemcpyAsync calls of
 * src/oneComponentGPSolver.cu:32-34,127-129,98,211 and
 * src/twoComponentGPSolver.cu:23-28,107-108. comp is 0 or 1. ------------- */
/* Sets psi (and the heavy-ball previous state psi_old, as the reference does). */
gpe_status gpe_set_psi(gpe_handle* h, int comp, const double* host_c128);
gpe_status gpe_get_psi(gpe_handle* h, int comp, double* host_c128);
gpe_status gpe_set_vext(gpe_handle* h, int comp, const double* host_c128);
/* Device-resident variants: interleaved complex128 device pointers. */
gpe_status gpe_set_psi_device(gpe_handle* h, int comp, const void* dev_c128);
gpe_status gpe_get_psi_device(gpe_handle* h, int comp, void* dev_c128);

/* ---- stepping ---------------------------------------------------------- */
/* Real-time RK4, OneComponentGPSolver::runRealTimeEvol body
 * (src/oneComponentGPSolver.cu:150-208) / TwoComponentGPSolver::runRealTimeEvol
 * (src/twoComponentGPSolver.cu:142-202).  Runs nsteps steps; step j uses the
 * reference's iteration number first_iteration+j for its stage times
 * (iteration*dt, (iteration+0.5)*dt, (iteration+1)*dt).  If obs_out is not
 * NULL, the last step also reduces, per component c, obs_out[3c+0] = sum |psi|^2 DV,
 * obs_out[3c+1] = sum Re(conj(psi) h_mu) DV and obs_out[3c+2] = sum Re(conj(psi) h_en) DV
 * pairing the new psi with H of the stage-4 argument, which is what the
 * reference's status hook reads (hamiltonians/BEC_oneComponent.cu:347-348). */
gpe_status gpe_step_real(gpe_handle* h, int first_iteration, int nsteps, double* obs_out);

/* Imaginary time (scheme per config).  Heavy-ball: one call runs up to
 * nsteps iterations of src/oneComponentGPSolver.cu:46-95 (or the 2-component
 * loop), first_iteration being the reference's `iteration` of the first one.
 * Stops early at the reference's convergence test; *iters_done counts the
 * iterations applied (the converging one included), *converged is 1 if the
 * test fired.  Per-iteration state (E, E_prev, mu, norm) persists across calls. */
gpe_status gpe_step_imag(gpe_handle* h, int first_iteration, int nsteps,
                         int* iters_done, int* converged);
/* PARS after the last imaginary iteration, per component c:
 * out[4c+0] = NORM, out[4c+1] = MU, out[4c+2] = EN, out[4c+3] = EN_PREV,
 * with the reference's definitions (1 comp: NORM = npart; 2 comp: NORM is the
 * pre-renormalisation norm, src/twoComponentGPSolver.cu:64-83). */
gpe_status gpe_imag_state(gpe_handle* h, double* out);
/* Resets E, E_prev, mu and the convergence flag (a fresh PARS array). */
gpe_status gpe_reset_imag_state(gpe_handle* h);

/* ---- primitives -------------------------------------------------------- */
/* BaseHamiltonian::alg_Laplace (src/baseHamiltonian.cu:86-96): out = IFFT(2pi^2 k^2/N FFT psi_comp). */
gpe_status gpe_laplace(gpe_handle* h, int comp, double* host_out_c128);
/* Plugin alg_calcHpsi (both h_mu and h_en) at time t, e.g.
 * hamiltonians/BEC_oneComponent.cu:92-111; either output may be NULL. */
gpe_status gpe_apply_h(gpe_handle* h, double t, int comp,
                       double* host_hmu_c128, double* host_hen_c128);
/* Raw reductions of the current psi with H(psi) at time t, per component c:
 * out[3c+0] = sum |psi|^2 DV, out[3c+1] = sum Re(conj(psi) h_mu) DV,
 * out[3c+2] = sum Re(conj(psi) h_en) DV.  BaseHamiltonian::alg_calcNorm and
 * alg_calc2Observables (src/baseHamiltonian.cu:173-179,230-236) divide these
 * by the caller's norm. */
gpe_status gpe_observables(gpe_handle* h, double t, double* out);
/* BaseHamiltonian::alg_calcPx (src/baseHamiltonian.cu:184-195) before the
 * plugin's division: sum Re(conj(psi) IFFT(kx FFT psi)) DV with the
 * unnormalised inverse transform of the reference (kx in cycles/length). */
gpe_status gpe_momentum_x(gpe_handle* h, int comp, double* px);

/* Logging-cadence observables of the plugins' status lines, reduced on the
 * device (FP64, compensated) and returned as the reference's reduction
 * returns them: the grid sum times DV (src/baseHamiltonian.cu:112-150).
 * x[ix] = -xmax[0] + (ix + 1/2) dx[0], L = 2 xmax[0].
 * gpe_average_cos: sum cos(2 pi x/L) |psi_comp|^2 DV — alg_calcCos
 *   (hamiltonians/BEC_oneComponent.cu:115-121, BEC_twoComponent.cu:147-152)
 *   with CalcAverageCos (src/parallel.cu:535-561); the plugins divide it by
 *   the norm (BEC_oneComponent.cu:349-350).
 * gpe_average_cos2: the same for psi_0 + sign psi_1, sign = +1 or -1
 *   (src/parallel.cu:739-771; the reference's two-field alg_calcCos,
 *   BEC_twoComponent.cu:154-160, launches it without its sign, i.e. +1).
 * gpe_relative_phase: sum (atan2 psi_0 - atan2 psi_1) DV
 *   (CalculateRelativePhase, src/parallel.cu:774-802).
 * gpe_dsz_dt: sum sqrt(|psi_0|^2 |psi_1|^2) sin(atan2 psi_0 - atan2 psi_1) DV
 *   (CalculateDszDt, src/parallel.cu:805-839).
 * The two-field forms need ncomp = 2.  A complex64 handle reduces the high
 * part of its state. */
gpe_status gpe_average_cos(gpe_handle* h, int comp, double* out);
gpe_status gpe_average_cos2(gpe_handle* h, int sign, double* out);
gpe_status gpe_relative_phase(gpe_handle* h, double* out);
gpe_status gpe_dsz_dt(gpe_handle* h, double* out);
/* Unnormalised 3D DFT of psi_comp in place, sign -1 (CUFFT_FORWARD) or +1
 * (CUFFT_INVERSE): the cufftExecZ2Z calls of src/baseHamiltonian.cu:89,95. */
gpe_status gpe_fft(gpe_handle* h, int comp, int sign);

/* ---- initial-state seeds on the device --------------------------------------
 * Psi::imprintVortexTube (src/psi.cu:155-164) and the Psi::force*Lattice
 * seeds (src/psi.cu:179-348) on component comp of the handle's psi, in FP64
 * whatever the precision (a complex64 handle keeps the seeded complex128
 * field as its compensated high + low parts).  The seeds add
 * amp * shape(x - off) * (seed_npart / DV)^(1/2) to psi and renormalise it to
 * norm_npart (Psi::add_lattice + Psi::normalize; the reference takes
 * seed_npart from the seed's component and norm_npart from component 1).
 * Grid points are cell centred: x_i = -xmax + i dx + dx/2. */
enum gpe_lattice {
    GPE_LATTICE_1D = 1,             /* amp (1 - cos k x) / 2            */
    GPE_LATTICE_2D_TRIANGULAR = 2,  /* three cosines at 120 degrees     */
    GPE_LATTICE_2D_SQUARE = 3,
    GPE_LATTICE_3D_HEX = 4,
    GPE_LATTICE_3D_FCC = 5,
    GPE_LATTICE_3D_BCC = 6,
    GPE_LATTICE_3D_SC = 7
};
/* psi *= exp(i Ncirc 2 pi x / (2 xmax_x)). */
gpe_status gpe_imprint_vortex_tube(gpe_handle* h, int comp, double ncirc);
/* off: 3 offsets (the unused ones of 1D/2D seeds are ignored). */
gpe_status gpe_seed_lattice(gpe_handle* h, int comp, int lattice, double amp, double k, const double* off,
                            double seed_npart, double norm_npart);

/* ---- optimal-control gradient (no counterpart in the reference) ------------
 * Real-time RK4 (the gpe_step_real scheme, one component, GPE_HAM_BEC,
 * GPE_HAM_DIPOLAR or GPE_HAM_SOFT) where step n uses the potential
 * W_n = V + sum_k u[n*nctrl + k] G_k, and the final-state infidelity
 * L = 1 - |o|^2, o = sum conj(target) psi(T) DV.
 * The gradient dL/du is the discrete adjoint of the RK4 step: each stage's
 * transpose Jacobian J^T mu = i (T + W + 2g|psi|^2 + Phi[|psi|^2]) mu
 * - i g psi^2 conj(mu) + 2 Phi[Im(conj(mu) psi)] psi (Phi: the k-space
 * interaction, 0 for GPE_HAM_BEC) runs through the same fused FFT passes,
 * both real densities of Phi in one transformed field; states are recomputed from
 * checkpoints every checkpoint_every steps (memory: about
 * nsteps/checkpoint_every + checkpoint_every + 8 fields). */
/* nctrl (1..64) real basis functions, host array nctrl x N (FP64). */
gpe_status gpe_control_set_basis(gpe_handle* h, int nctrl, const double* host_G);
/* From the handle's current psi (left unchanged, as is V): *loss_out and, if
 * host_grad is not NULL, host_grad[n*nctrl + k] = dL/du[n*nctrl + k]. */
gpe_status gpe_control_gradient(gpe_handle* h, const double* host_u, int nsteps, const double* host_target_c128,
                                int checkpoint_every, double* loss_out, double* host_grad);

/* ---- batched independent instances (no counterpart in the reference, whose
 * parameter sweeps are separate ./gpe runs) ----------------------------------
 * A batch holds n one-component instances that may differ in grid geometry
 * (nx, ny, nz, xmax, dx) and in d_h_params (e.g. the coupling); precision,
 * hamiltonian (GPE_HAM_BEC or GPE_HAM_TEMPLATE), imag_scheme, dt, beta,
 * epsilon_e and npart are shared, and the coupling is time-independent
 * (prms[3..5] <= 0).  Instances with the same geometry form a group whose
 * fields are contiguous; every pass kernel of a group advances all its
 * instances in one launch (blockIdx.y = instance), and one imaginary-time
 * iteration of every group is captured once into a CUDA graph that each
 * iteration replays (direct launches on the legacy default stream).
 * Instances that have converged skip their work on the device. */
typedef struct gpe_batch gpe_batch;
gpe_status gpe_batch_create(const gpe_config* cfgs, int n, gpe_batch** out);
gpe_status gpe_batch_destroy(gpe_batch* b);
gpe_status gpe_batch_set_stream(gpe_batch* b, void* cuda_stream);
gpe_status gpe_batch_set_psi(gpe_batch* b, int inst, const double* host_c128);
gpe_status gpe_batch_set_vext(gpe_batch* b, int inst, const double* host_c128);
gpe_status gpe_batch_get_psi(gpe_batch* b, int inst, double* host_c128);
/* Up to nsteps imaginary-time iterations of every unconverged instance (the
 * scheme of gpe_step_imag at time 0).  Per instance i: iters_done[i] counts the
 * iterations applied in this call, converged[i] is 1 once its test fired
 * (arrays of n; either may be NULL). */
gpe_status gpe_batch_step_imag(gpe_batch* b, int nsteps, int* iters_done, int* converged);
/* gpe_imag_state of one instance: out[0..3] = NORM, MU, EN, EN_PREV. */
gpe_status gpe_batch_imag_state(gpe_batch* b, int inst, double* out);
/* Kernels of this library run for the batch so far (graph replays included). */
long long  gpe_batch_kernel_launches(const gpe_batch* b);
/* Launch modes of a batch's imaginary-time iterations.
 *   GPE_BATCH_PER_GROUP  one launch per pass per geometry group (12 per group
 *                        an iteration), the tuned pass variants (default);
 *   GPE_BATCH_PERSISTENT one cooperative launch per RK4 stage (4 an iteration,
 *                        see gpe_batch_set_persistent);
 *   GPE_BATCH_GROUPED    one launch per pass over the tiles of every group
 *                        (12 an iteration), one tile per CTA.
 * The two all-group modes share the conditions of gpe_batch_set_persistent;
 * wait_bound applies to GPE_BATCH_PERSISTENT. */
enum gpe_batch_mode { GPE_BATCH_PER_GROUP = 0, GPE_BATCH_PERSISTENT = 1, GPE_BATCH_GROUPED = 2 };
gpe_status gpe_batch_set_launch_mode(gpe_batch* b, int mode, unsigned int wait_bound);
int        gpe_batch_launch_mode(const gpe_batch* b);
/* Persistent launches: one cooperative kernel per RK4 stage runs the stage's
 * three passes for every instance of every group, with a grid-wide barrier
 * between the passes (4 launches an iteration instead of 12 per group).
 * Needs GPE_IMAG_RK4, two-dimensional grids (ny > 1, nz = 1) of lengths 64,
 * 96, 128, 192, 256, 384 or 512, and at most 8 geometry groups; else
 * GPE_ERR_UNSUPPORTED.  wait_bound: iterations a barrier wait may spin
 * (0 = about a second); a wait that runs out ends the launch and
 * gpe_batch_step_imag returns GPE_ERR_TIMEOUT (the state of that call is
 * then undefined; the next call starts clean).  enable = 0 restores the
 * per-group launches.  No counterpart in the reference (one instance per
 * process). */
gpe_status gpe_batch_set_persistent(gpe_batch* b, int enable, unsigned int wait_bound);
int        gpe_batch_persistent(const gpe_batch* b);
/* Resources of the batch's persistent stage kernel, out[0..8]: registers per
 * thread, static shared memory (B), threads per CTA allowed, local memory per
 * thread (B), resident CTAs per SM, SMs, cooperative launch supported (0/1),
 * dynamic shared memory (B), CTAs of the last stage launch. */
gpe_status gpe_batch_persistent_info(const gpe_batch* b, long long* out);

/* ---- user Hamiltonian plugins ------------------------------------------------
 * A plugin is a shared library compiled from the user's .cu file with
 * include/gpe_plugin.cuh: it instantiates this library's x-pass kernels with
 * the user's pointwise functor (GPE_DEFINE_USER_HAMILTONIAN) and exports a
 * function returning this table.  The launchers take the library's internal
 * pass-argument block (opaque here), return 1 when they have a kernel for
 * the line length L, and store the CUDA error code in *cuda_err. */
typedef struct gpe_user_hamiltonian {
    int abi_version; /* GPE_ABI_VERSION */
    int (*launch_x_c64)(int L, const void* pass_args, int rows, size_t smem, void* stream, int* cuda_err);
    int (*launch_x_c128)(int L, const void* pass_args, int rows, size_t smem, void* stream, int* cuda_err);
} gpe_user_hamiltonian;
/* Installs the plugin for a GPE_HAM_USER handle (the table must outlive the
 * handle).  Every pass that evaluates the Hamiltonian then runs the plugin's
 * kernels; a length the plugin was not built for fails with
 * GPE_ERR_UNSUPPORTED.  The control gradient does not take user plugins. */
gpe_status gpe_set_user_hamiltonian(gpe_handle* h, const gpe_user_hamiltonian* ops);

/* ---- allocation-free norm (no counterpart in the reference) -------------
 * dev_out[0] = DV * sum |psi[i]|^2 over n complex128 points of a caller-owned
 * device array (interleaved re, im; 16-byte aligned), issued on cuda_stream
 * (NULL = legacy default stream) and not synchronised.  It needs no handle and
 * allocates nothing: its block partials live in a fixed 128 KiB device array
 * inside the library, for callers whose device memory is already reserved by
 * their own allocator or that must avoid the synchronisation cudaFree
 * implies.  n above GPE_NORM_NOALLOC_MAX_POINTS is rejected with
 * GPE_ERR_UNSUPPORTED.  The first call on each device does a one-time set-up
 * (scratch address lookup, a synchronous zeroing of its completion counter):
 * make it before any stream capture starts on that device.  The scratch
 * address found there is kept for the life of the process: after
 * cudaDeviceReset on a device it would point into the destroyed context, so
 * do not call this entry point on that device again in the same process.
 * Calls that may overlap on one device share the scratch and race; order
 * them on one stream.  The result is the same bits on every call for the
 * same input. */
#define GPE_NORM_NOALLOC_MAX_POINTS 134217728LL /* 512^3 */
gpe_status gpe_norm_noalloc(const void* dev_psi_c128, long long n, double dv, double* dev_out,
                            void* cuda_stream);

/* ---- autotuner (no counterpart in the reference, which leaves the transform
 * plan to cuFFT's planner, cufftPlan1d/2d/3d at src/parallel.cu:77-110) -----
 * The pass kernels come in variants: per strided axis and pass mode
 * (forward, forward*k-space*inverse, inverse) the implementation (scalar
 * lines, or two complex64 lines per thread with packed FP32x2 arithmetic),
 * the tile width, the resident CTAs per SM and the radix order of the line
 * FFT; per grid the x pass's rows per CTA; for 3D complex64 grids with y and
 * z lengths 64 or 128 (and nx a multiple of 4), whether the three strided
 * passes of a stage run as one kernel over thread-block clusters (y-z slabs
 * held in distributed shared memory, one read and one write of the work
 * field).  Variant 0 / rows 0 / fused 0 are the defaults, which every handle
 * uses unless a tuning result applies.
 *
 * gpe_tune times every variant that exists for cfg's grid (CUDA events on a
 * temporary handle: each strided pass alone, the rows by whole steps of the
 * workload, 0 = real-time RK4 steps, 1 = imaginary-time iterations), keeps
 * the fastest, and stores one line keyed by (nx, ny, nz, precision, fields,
 * instances = 1) in the JSON-lines file cache_path (replacing a line of the
 * same key; NULL = do not store).  report (may be NULL) receives 13 values:
 * default and tuned microseconds per step, variants timed, the chosen
 * variants s[axis 1][mode 0..2], s[axis 2][mode 0..2], the rows, the
 * fused y-z flag, the persistent mode (gpe_set_flow: 1 only for the
 * real-time workload, 2 for either) and the x-staging flag
 * (gpe_set_x_staging, real-time workload). */
gpe_status gpe_tune(const gpe_config* cfg, int workload, const char* cache_path, double* report);
/* Process-wide: gpe_create and gpe_batch_create apply the cache line that
 * matches a new handle (or batch group); NULL = read $GPE_TUNE_CACHE if set. */
gpe_status gpe_set_tune_cache(const char* path);
/* Tunes every geometry group of a batch in place (imaginary-time
 * iterations with the group's instance count), drops its captured graph, and
 * stores a line per group in cache_path (may be NULL).  report (may be NULL):
 * 2 values per group, default and tuned microseconds per iteration. */
gpe_status gpe_batch_tune(gpe_batch* b, const char* cache_path, double* report);
int        gpe_batch_groups(const gpe_batch* b);
/* The handle's variants as 8 ints: s[1][0..2], s[2][0..2], rows, fused y-z.
 * Setting checks that each variant exists (gpe_pass_variant_exists) for the
 * grid and that the fused kernel serves it. */
gpe_status gpe_get_pass_variants(const gpe_handle* h, int* out8);
gpe_status gpe_set_pass_variants(gpe_handle* h, const int* in8);
/* 1 when strided-pass variant v (0 .. 11) exists for axis 1 (y) or 2 (z) of
 * cfg's grid, precision and fields; variant 0 always does.  Host only. */
int        gpe_pass_variant_exists(const gpe_config* cfg, int axis, int v);

/* ---- persistent RK4 step (no counterpart in the reference, whose step is
 * eight cuFFT calls and a dozen element-wise kernels,
 * src/oneComponentGPSolver.cu:166-190) -------------------------------------
 * on = 1: each real-time RK4 step of gpe_step_real runs as ONE launch whose
 * CTAs take the tiles of the step's sixteen axis passes from one ordered list,
 * every tile waiting only for the tiles whose output it reads (per x block
 * or z plane), so the passes overlap instead of draining between launches.
 * The tiles are the pass kernels' own, so the results equal the per-pass
 * chain's bit for bit.  It serves complex64 one-component handles on cubic
 * grids of length 128 or 256 with GPE_HAM_BEC or GPE_HAM_TEMPLATE and no
 * moving-frame term; for every other handle, and for the step of a call that
 * returns the logging observables, the per-pass chain runs (the option is
 * kept).  wait_bound: 32 ns sleeps a tile's wait may take before the launch
 * gives up (0 keeps the current bound, default 2^22); a launch that gives
 * up records GPE_ERR_TIMEOUT in the handle's status word (reported by the
 * next call that reads the device scalars, e.g. gpe_step_real with
 * observables) and in the step's own status word, after which later
 * persistent steps do nothing until gpe_flow_status re-arms them. */
gpe_status gpe_set_flow(gpe_handle* h, int on, unsigned wait_bound);
/* on = 2 (persistent strided stage): the three strided passes of every
 * one-field complex64 pass chain of a cubic 128 or 256 grid (real- and
 * imaginary-time steps, apply-H, observables) run as one launch per stage
 * whose CTAs stream the y-forward, z forward*k-space*inverse and y-inverse
 * tiles of each x block, every tile waiting only for the tiles of its x
 * block that it reads (the x passes keep their own launches); results equal
 * the chain with the default radix order bit for bit.  The same wait bound,
 * timeout status and re-arm apply. */
/* 1 when the handle's real-time steps run as the persistent step, 2 when its
 * strided stages run as one launch each, 0 otherwise. */
int        gpe_flow_active(const gpe_handle* h);
/* Synchronises; *status_out = 0 or GPE_ERR_TIMEOUT (a persistent step gave
 * up since the last call).  After a timeout the counters and both status
 * words are reset; the fields hold the partial step and must be set again. */
gpe_status gpe_flow_status(gpe_handle* h, int* status_out);

/* on = 1: the fused x-inverse pass of a complex64 one-field real-time RK4
 * stage copies its epilogue inputs (V, the stage state, the accumulator,
 * psi0, the low part) into shared memory with asynchronous copies at kernel
 * start, before its wait on the previous pass, so that they are in flight
 * during the inverse transform instead of being loaded after it; results
 * are unchanged bit for bit.  Other handles ignore it.  A tuner variant
 * (cache key xstage), off by default. */
gpe_status gpe_set_x_staging(gpe_handle* h, int on);
int        gpe_x_staging(const gpe_handle* h);

/* Synchronise the handle's stream and report any asynchronous error. */
gpe_status gpe_sync(gpe_handle* h);
/* Number of this library's kernels launched by the handle so far. */
long long  gpe_kernel_launches(const gpe_handle* h);

/* ---- measurement (no counterpart in the reference, whose only timing is
 * unsynchronised host chrono, src/oneComponentGPSolver.cu:153,197-200) ----- */
#define GPE_PROF_KINDS 8
#define GPE_PROF_FLOW 6
#define GPE_PROF_SFLOW 7
/* Pass kinds: 0 x-forward (+prologue), 1 x-inverse (+epilogue), 2 x-full,
 * 3 strided forward, 4 strided inverse, 5 strided forward*k-space*inverse
 * (with the fused y-z kernel: that kernel, and no kinds 3 and 4), 6 the
 * persistent RK4 step (gpe_set_flow mode 1: one launch for the whole step),
 * 7 the persistent strided stage (mode 2: the three strided passes). */
/* When enabled, every pass launch is bracketed by CUDA events on the
 * handle's stream. */
gpe_status gpe_profile_enable(gpe_handle* h, int enable);
/* Synchronises the stream and returns, per pass kind, the summed event time
 * in ms and the launch count since the previous read (arrays of
 * GPE_PROF_KINDS; either may be NULL). */
gpe_status gpe_profile_read(gpe_handle* h, double* ms_out, long long* count_out);

#ifdef __cplusplus
}
#endif
#endif /* GPE_B200_GPE_H */
