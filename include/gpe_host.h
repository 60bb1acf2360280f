/*
 * gpe_host.h -- C entry points of the host-side mirror of the reference's
 * interface (input.txt / rinput.txt format, units, initial states, output file
 * layout, and the `gpe` driver itself).  Implemented in libgpe.so
 * (fgpe_b200/host/); pure host code except gpeh_run, which runs a simulation.
 */
#ifndef GPE_B200_GPE_HOST_H
#define GPE_B200_GPE_HOST_H

#ifdef __cplusplus
extern "C" {
#endif

/* Length of the parameter dump of gpeh_params (47 doubles). */
int         gpeh_dump_len(void);
/* Parse an input file with InputVariables + Params (t2component false) or
 * Params2 (true), replacing main.cu:30-56 and src/params.cu:134-279 /
 * src/params2.cu:28-186.  out layout: [0..2] NX, [3] DIM, [4] Npoints,
 * [5..7] XMAX, [8..10] DX, [11] DV, [12..14] KXMAX, [15..17] DKX, [18] V,
 * [19] dt, [20] epsilon_e, [21] time0, [22] niter, [23] itmod, [24] aho,
 * [25] omho, [26..28] ax, [29..31] omega, [32] mass, [33] npart, [34] a (a11),
 * [35] add (a22), [36] edd (a12), [37] aho2, [38] omho2, [39..41] ax2,
 * [42..44] omega2, [45] mass2, [46] npart2.  Returns the number of
 * components, or -1 with gpeh_last_error() set. */
int         gpeh_params(const char* input_file, double* out);
/* Initial psi of the BEC plugins (hamiltonians/BEC_oneComponent.cu:36-58,
 * hamiltonians/BEC_twoComponent.cu:41-73), component type 0 (one component)
 * or 1/2, as interleaved complex128.  0 on success, -1 on error. */
int         gpeh_init_psi(const char* input_file, int type, double* out_c128);
/* Initial Vext of the BEC plugins (hamiltonians/BEC_oneComponent.cu:63-83,
 * hamiltonians/BEC_twoComponent.cu:80-110). */
int         gpeh_init_vext(const char* input_file, int type, double* out_c128);
/* The one-component initial psi of gpeh_init_psi with a lattice seed added
 * (Psi::force*Lattice, src/psi.cu:179-348, used to start soft-core droplet
 * crystals): lattice 1 = 1D (offset offx), 2 = 2D triangular, 3 = 2D square,
 * 4 = 3D HEX, 5 = 3D FCC, 6 = 3D BCC, 7 = 3D simple cubic; amp, wave number k
 * and offsets in code units; type selects the particle number of the seed
 * (1 or 2).  Returns 0 or -1 (gpeh_last_error). */
int         gpeh_init_psi_lattice(const char* input_file, int lattice, double amp, double k, double offx,
                                  double offy, double offz, int type, double* out_c128);
/* Output::WriteWtxt / WriteWtxt_2c + WriteVariable2WTXT lines under the input
 * file's outprefix (src/output.cu:26-191). */
int         gpeh_write_info(const char* input_file, int ncycles, int nvars, const char** names,
                            const double* values, const char** units);
/* Run an input file exactly as `gpe <file>` does (main.cu:20-82).  Returns
 * the process exit code (0 ok). */
int         gpeh_run(const char* input_file);
const char* gpeh_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
