// gpe_init.cu -- initial-state seeds on the device: the vortex-tube phase
// imprint (Psi::imprintVortexTube, src/psi.cu:155-164) and the lattice seeds
// with their renormalisation (Psi::force*Lattice + Psi::normalize,
// src/psi.cu:179-374), on a complex128 field in HBM.
//
// The arithmetic keeps the reference's expression order with every product
// and sum rounded on its own (no fused multiply-add), as the host compiler
// evaluates it, so the field differs from the host classes' only by the
// device cosine/sine (a few ulp) and the order of the norm's sum.
#include <cuda_runtime.h>

#include "gpe_init.cuh"

namespace gpe {

namespace {

__device__ __forceinline__ double M(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double A(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double S(double a, double b) { return __dsub_rn(a, b); }

// Cell-centred coordinate of index i along an axis (gridX/Y/Z).
__device__ __forceinline__ double coord(const SeedGrid& g, int d, int i) {
    return A(A(-g.xmax[d], M((double)i, g.dx[d])), M(0.5, g.dx[d]));
}

// The seed amplitude at (x, y, z), relative to the offsets (src/psi.cu:179-348).
__device__ double lattice_shape(int kind, double amp, double k, double x, double y, double z) {
    switch (kind) {
        case GPE_LATTICE_1D:
            return M(amp, S(1.0, cos(M(k, x)))) / 2.;
        case GPE_LATTICE_2D_TRIANGULAR: {
            const double h = sqrt(3.0) / 2;
            const double s = A(A(cos(M(k, x)), cos(M(k, A(M(-0.5, x), M(h, y))))), cos(M(k, S(M(-0.5, x), M(h, y)))));
            return M(amp, s) / 3;
        }
        case GPE_LATTICE_2D_SQUARE:
            return M(amp, A(cos(M(k, y)), cos(M(k, x)))) / 2;
        case GPE_LATTICE_3D_HEX: {
            const double r3 = sqrt(3.);
            const double u = A(-x, M(r3, y)) / 2., w = S(-x, M(r3, y)) / 2.;
            const double s = A(A(A(cos(M(k, u)), cos(M(k, x))), cos(M(k, z))), cos(M(k, w)));
            return M(amp, s) / 4.0;
        }
        case GPE_LATTICE_3D_FCC: {
            const double r3 = sqrt(3.);
            const double q[9] = {S(A(x, y), z) / r3, S(A(y, z), x) / r3, S(A(z, x), y) / r3,
                                 S(S(x, y), z) / r3, S(S(y, z), x) / r3, S(S(z, x), y) / r3,
                                 A(A(x, y), z) / r3, A(A(y, z), x) / r3, A(A(z, x), y) / r3};
            double s = cos(M(k, q[0]));
            for (int j = 1; j < 9; ++j) s = A(s, cos(M(k, q[j])));
            return M(amp, s) / 9.0;
        }
        case GPE_LATTICE_3D_BCC: {
            const double r2 = sqrt(2.0);
            const double q[6] = {A(x, y) / r2, A(z, y) / r2, A(z, x) / r2, S(x, y) / r2, S(z, y) / r2, S(z, x) / r2};
            double s = cos(M(k, q[0]));
            for (int j = 1; j < 6; ++j) s = A(s, cos(M(k, q[j])));
            return M(amp, s) / 6;
        }
        default:  // GPE_LATTICE_3D_SC
            return M(amp, A(A(cos(M(k, z)), cos(M(k, y))), cos(M(k, x)))) / 3;
    }
}

// psi <- shape * avg + psi  (Psi::add_lattice)
__global__ void k_seed(double2* psi, SeedGrid g, int kind, double amp, double k, double ox, double oy, double oz,
                       double avg) {
    const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i % g.n[0]), iy = (int)((i / g.n[0]) % g.n[1]), iz = (int)(i / ((long long)g.n[0] * g.n[1]));
        const double x = S(coord(g, 0, ix), ox), y = S(coord(g, 1, iy), oy), z = S(coord(g, 2, iz), oz);
        double2 p = psi[i];
        p.x = A(M(lattice_shape(kind, amp, k, x, y, z), avg), p.x);
        psi[i] = p;
    }
}

// psi <- (cos(c x), sin(c x)) * psi, c = Ncirc * 2 pi / (2 XMAX_x)
__global__ void k_vortex_tube(double2* psi, SeedGrid g, double ncirc) {
    const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
    const double pi = 3.141592653589793;
    const double xlen = M(2.0, g.xmax[0]);
    const double c = M(ncirc, 2.0);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double x = coord(g, 0, (int)(i % g.n[0]));
        const double arg = M(M(c, pi) / xlen, x);
        const double cr = cos(arg), ci = sin(arg);
        const double2 p = psi[i];
        psi[i] = make_double2(S(M(cr, p.x), M(ci, p.y)), A(M(cr, p.y), M(ci, p.x)));
    }
}

constexpr int SUM_BLOCKS = 592;  // 4 per SM of a 148-SM part; the sum's order is fixed by it

__global__ void k_abs2_partials(const double2* psi, long long n, double* part) {
    __shared__ double red[256];
    double s = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double2 p = psi[i];
        s = A(s, A(M(p.x, p.x), M(p.y, p.y)));
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = A(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// psi *= (npart / (sum |psi|^2 DX DY DZ))^(1/2)   (Psi::normalize)
__global__ void k_normalize(double2* psi, long long n, const double* part, int nparts, double npart, SeedGrid g) {
    __shared__ double fac;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nparts; ++b) s = A(s, part[b]);
        fac = sqrt(npart / M(M(M(s, g.dx[0]), g.dx[1]), g.dx[2]));
    }
    __syncthreads();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double2 p = psi[i];
        psi[i] = make_double2(M(p.x, fac), M(p.y, fac));
    }
}

unsigned grid_for(long long n) {
    const long long b = (n + 255) / 256;
    return (unsigned)(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

}  // namespace

cudaError_t seed_lattice_c128(double2* psi, const SeedGrid& g, int kind, double amp, double k, const double off[3],
                              double seed_npart, double norm_npart, double* part, cudaStream_t st) {
    const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
    const double avg = sqrt(seed_npart / ((g.dx[0] * g.dx[1]) * g.dx[2]));  // pow(npart / DV, 0.5)
    k_seed<<<grid_for(n), 256, 0, st>>>(psi, g, kind, amp, k, off[0], off[1], off[2], avg);
    k_abs2_partials<<<SUM_BLOCKS, 256, 0, st>>>(psi, n, part);
    k_normalize<<<grid_for(n), 256, 0, st>>>(psi, n, part, SUM_BLOCKS, norm_npart, g);
    return cudaGetLastError();
}

cudaError_t imprint_vortex_tube_c128(double2* psi, const SeedGrid& g, double ncirc, cudaStream_t st) {
    const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
    k_vortex_tube<<<grid_for(n), 256, 0, st>>>(psi, g, ncirc);
    return cudaGetLastError();
}

size_t seed_partials_bytes() { return sizeof(double) * SUM_BLOCKS; }

}  // namespace gpe
