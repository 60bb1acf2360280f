// gpe_init.cuh -- device initial-state seeds (gpe_init.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/gpe.h"

namespace gpe {

// Cell-centred grid of a field: n points per axis, x_i = -xmax + i dx + dx/2.
struct SeedGrid {
    int n[3];
    double xmax[3], dx[3];
};

// Adds the lattice seed `kind` (GPE_LATTICE_*) with amplitude amp * (seed_npart
// / DV)^(1/2) to psi and renormalises psi to norm_npart; part: device scratch
// of seed_partials_bytes().
cudaError_t seed_lattice_c128(double2* psi, const SeedGrid& g, int kind, double amp, double k, const double off[3],
                              double seed_npart, double norm_npart, double* part, cudaStream_t st);
cudaError_t imprint_vortex_tube_c128(double2* psi, const SeedGrid& g, double ncirc, cudaStream_t st);
size_t seed_partials_bytes();

}  // namespace gpe
