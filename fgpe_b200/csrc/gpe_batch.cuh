// gpe_batch.cuh -- one persistent launch per RK4 stage for a batch of 2D
// imaginary-time instances of uneven grid sizes.
//
// The per-group path (gpe_batch_step_imag without the persistent option)
// launches every pass once per geometry group: 3 passes x 4 stages x groups
// launches per iteration (84 for the 7 sizes of the sweep), the small groups
// filling a fraction of the GPU per launch.  Here one cooperative launch per
// stage runs the stage's three passes for every instance of every group:
//   phase A  the x-forward tiles (prologue + x transform) of all instances,
//   phase B  the y forward * k-space * inverse tiles,
//   phase C  the x-inverse tiles with the imaginary-time RK4 epilogue and the
//            per-instance reductions (the last tile of an instance finalises),
// with a grid barrier between the phases.  The CTAs (co-resident: the launch
// is cooperative) take tiles from one list per phase -- (group, instance,
// tile) in group-major order -- in strides of the grid, so a small instance's
// tiles share the GPU with the large ones'.  The tile bodies are the pass
// kernels' own (xpass_tile, spass_tile), with 256-thread tiles for every
// length.  Converged instances skip their tiles on the device, as in the
// per-group kernels.
//
// The grid barrier is a counter and a generation in device memory.  Every
// wait has an iteration bound: a CTA that gives up records GPE_ERR_TIMEOUT in
// the barrier's status word and leaves the kernel, and every CTA checks that
// word after each barrier, so the launch ends (with the error on record) in
// bounded time whatever happens; the host reads the word after the batch's
// iterations.
#pragma once

#include "gpe_batch_args.cuh"
#include "gpe_kernels_impl.cuh"

namespace gpe {

__device__ __forceinline__ unsigned ld_volatile_u(const unsigned* p) {
    return *reinterpret_cast<const volatile unsigned*>(p);
}
__device__ __forceinline__ int ld_volatile_i(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

// Every tile uses all the threads: rows x T = 256 for the x tiles, x values x
// T for the strided ones (T = the line's threads), so no thread of a CTA
// indexes past its tile.
#define GPE_BATCH_FULL(L) static_assert(batch_rows(L) * (L / make_plan(L).E) == BATCH_THREADS, "tile of " #L);
GPE_BATCH_LENGTHS(GPE_BATCH_FULL)
#undef GPE_BATCH_FULL

// Grid-wide barrier with a bounded wait; false when any CTA gave up (then the
// caller leaves the kernel).
__device__ __forceinline__ bool grid_sync_bounded(GridBar* bar, unsigned bound) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned g = ld_volatile_u(&bar->gen);
        __threadfence();
        if (atomicAdd(&bar->count, 1u) == gridDim.x - 1) {
            atomicExch(&bar->count, 0u);
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            unsigned it = 0;
            while (ld_volatile_u(&bar->gen) == g) {
                if (++it > bound) {
                    atomicExch(&bar->status, (int)GPE_ERR_TIMEOUT);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok = ld_volatile_i(&bar->status) == 0;
    }
    __syncthreads();
    return ok != 0;
}

// Group of a tile in a phase list with the given prefix sums.
__device__ __forceinline__ int batch_group_of(const unsigned* start, int ngroups, unsigned t) {
    int g = 0;
    while (g + 1 < ngroups && t >= start[g + 1]) ++g;
    return g;
}

// One RK4 stage (imaginary time) of every instance of every group.
// Resident CTAs per SM the launch bounds ask for: two for complex64 (128
// registers a thread), one for complex128, whose line registers would spill
// at two.
template <typename R>
__host__ __device__ constexpr int batch_min_blocks() {
    return sizeof(R) == 4 ? 2 : 1;
}

// Tile t of phase A (x forward: stage-state prologue + x transform).
template <typename R>
__device__ __forceinline__ void batch_tile_a(const BatchStage<R>& b, unsigned t, unsigned char* smem_raw) {
    const int ng = b.ngroups;
    const int g = batch_group_of(b.xstart, ng, t);
    const unsigned local = t - b.xstart[g], inst = local / b.xt[g], tile = local % b.xt[g];
    const PassArgs<R>& a = b.args[g];
    switch (b.lx[g]) {
#define GPE_BATCH_XF(L)                                                              \
    case L:                                                                          \
        xpass_tile<R, L, 1, XK_FWD>(a, batch_rows(L), tile, inst, b.xt[g], smem_raw); \
        break;
        GPE_BATCH_LENGTHS(GPE_BATCH_XF)
#undef GPE_BATCH_XF
        default:
            break;
    }
}

// Tile t of phase B (y forward * k-space * inverse).
template <typename R>
__device__ __forceinline__ void batch_tile_b(const BatchStage<R>& b, unsigned t, unsigned char* smem_raw) {
    const int ng = b.ngroups;
    const int g = batch_group_of(b.sstart, ng, t);
    const unsigned local = t - b.sstart[g], inst = local / b.st[g], tile = local % b.st[g];
    const PassArgs<R>& a = b.args[BATCH_MAX_GROUPS + g];
    switch (b.ly[g]) {
#define GPE_BATCH_S(L)                                                        \
    case L:                                                                   \
        spass_tile<R, L, 1, batch_rows(L)>(a, b.ntx[g], tile, inst, smem_raw); \
        break;
        GPE_BATCH_LENGTHS(GPE_BATCH_S)
#undef GPE_BATCH_S
        default:
            break;
    }
}

// Tile t of phase C (x inverse with the RK4 imaginary-time epilogue and the
// per-instance reductions).
template <typename R>
__device__ __forceinline__ void batch_tile_c(const BatchStage<R>& b, unsigned t, unsigned char* smem_raw) {
    const int ng = b.ngroups;
    const int g = batch_group_of(b.xstart, ng, t);
    const unsigned local = t - b.xstart[g], inst = local / b.xt[g], tile = local % b.xt[g];
    const PassArgs<R>& a = b.args[2 * BATCH_MAX_GROUPS + g];
    switch (b.lx[g]) {
#define GPE_BATCH_XI(L)                                                              \
    case L:                                                                          \
        xpass_tile<R, L, 1, XK_RKI>(a, batch_rows(L), tile, inst, b.xt[g], smem_raw); \
        break;
        GPE_BATCH_LENGTHS(GPE_BATCH_XI)
#undef GPE_BATCH_XI
        default:
            break;
    }
}

// One RK4 stage (imaginary time) of every instance of every group: the three
// phases in one cooperative launch, a bounded grid barrier between them.
template <typename R>
__global__ void __launch_bounds__(BATCH_THREADS, batch_min_blocks<R>()) k_batch_stage(BatchStage<R> b) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ng = b.ngroups;
    // a wait of an earlier stage gave up: the barrier counts are stale, so
    // no CTA takes part in this launch
    if (ld_volatile_i(&b.bar->status) != 0) return;
    for (unsigned t = blockIdx.x; t < b.xstart[ng]; t += gridDim.x) {
        batch_tile_a(b, t, smem_raw);
        __syncthreads();  // the next tile reuses the exchange storage
    }
    if (!grid_sync_bounded(b.bar, b.wait_bound)) return;
    for (unsigned t = blockIdx.x; t < b.sstart[ng]; t += gridDim.x) {
        batch_tile_b(b, t, smem_raw);
        __syncthreads();
    }
    if (!grid_sync_bounded(b.bar, b.wait_bound)) return;
    for (unsigned t = blockIdx.x; t < b.xstart[ng]; t += gridDim.x) {
        batch_tile_c(b, t, smem_raw);
        __syncthreads();
    }
}

// One phase of one stage for every instance of every group, one tile per
// CTA (grid = the phase's tile count): the grouped launch mode, three
// launches a stage with programmatic dependent launch between them.  The
// phase's own bodies only, so its registers are the phase's, not the whole
// stage's.
template <typename R, int PHASE>
__host__ __device__ constexpr int batch_phase_min_blocks() {
    return sizeof(R) == 4 ? (PHASE == 2 ? 2 : 3) : 2;
}

template <typename R, int PHASE>
__global__ void __launch_bounds__(BATCH_THREADS, (batch_phase_min_blocks<R, PHASE>())) k_batch_phase(BatchStage<R> b) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pass_prologue_sync();
    if constexpr (PHASE == 0) batch_tile_a(b, blockIdx.x, smem_raw);
    else if constexpr (PHASE == 1) batch_tile_b(b, blockIdx.x, smem_raw);
    else batch_tile_c(b, blockIdx.x, smem_raw);
}

}  // namespace gpe
