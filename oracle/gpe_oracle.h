/*
 * gpe_oracle.h -- FP64 host oracle for the GPE hot path.  TEST INFRASTRUCTURE:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker / the timed CPU baseline.  The
 * product (libgpe.so) never calls it.
 *
 * It is a CPU restatement of the reference's algorithm (fGPE v0.3, a CUDA-only
 * program with no CPU path): grids and units, the pseudo-spectral kinetic
 * operator, the Hamiltonian plugins, the heavy-ball imaginary-time loop and the
 * RK4 real-time loop, with the reference's quirks kept (each function cites
 * the reference file:line it follows).  Its FFT is its own mixed-radix
 * Stockham transform (radix 2/3/4/5 plus a direct DFT for other primes) with
 * twiddles rounded from long double; sums are Neumaier-compensated; loops over
 * grid lines run under OpenMP.
 *
 * Parity pinning: checked against numpy.fft for the transform and against
 * golden outputs of the reference's own CUDA build (tests/golden/).
 *
 * The entry points mirror include/gpe.h one for one (orc_ prefix) and take the
 * same gpe_config.
 */
#ifndef GPE_B200_ORACLE_H
#define GPE_B200_ORACLE_H
#include "../include/gpe.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_solver orc_solver;

void        orc_set_threads(int n);
int         orc_get_threads(void);
orc_solver* orc_create(const gpe_config* cfg);
void        orc_destroy(orc_solver* s);
int         orc_set_params(orc_solver* s, const double* prms);
int         orc_set_psi(orc_solver* s, int comp, const double* c128);
int         orc_get_psi(orc_solver* s, int comp, double* c128);
int         orc_set_vext(orc_solver* s, int comp, const double* c128);
int         orc_step_real(orc_solver* s, int first_iteration, int nsteps, double* obs_out);
int         orc_step_imag(orc_solver* s, int first_iteration, int nsteps, int* iters_done, int* converged);
int         orc_imag_state(orc_solver* s, double* out);
int         orc_reset_imag_state(orc_solver* s);
int         orc_laplace(orc_solver* s, int comp, double* out_c128);
int         orc_apply_h(orc_solver* s, double t, int comp, double* hmu_c128, double* hen_c128);
int         orc_observables(orc_solver* s, double t, double* out);
int         orc_fft(orc_solver* s, int comp, int sign);

/* Stand-alone unnormalised 3D DFT (x fastest), sign -1 forward / +1 inverse. */
void        orc_fft3d(int nx, int ny, int nz, double* c128, int sign);
/* x, y, z and kx, ky, kz axes of BaseHamiltonian::InitializeSpace/Kspace. */
void        orc_axes(const gpe_config* cfg, double* x, double* y, double* z,
                     double* kx, double* ky, double* kz);

#ifdef __cplusplus
}
#endif
#endif
