// gpe_batch_args.cuh -- host/device description of one persistent batch
// stage launch (the kernel is in gpe_batch.cuh, its launcher in gpe_batch.cu).
#pragma once

#include "gpe_kernels.cuh"

namespace gpe {

constexpr int BATCH_MAX_GROUPS = 8;
constexpr int BATCH_THREADS = 256;

struct GridBar {
    unsigned int count;  // CTAs arrived at the current barrier
    unsigned int gen;    // barriers completed
    int status;          // 0, or GPE_ERR_TIMEOUT when a wait gave up
    int pad;
};

// The lengths the persistent kernel is compiled for (x and y of each group).
#define GPE_BATCH_LENGTHS(X) X(64) X(96) X(128) X(192) X(256) X(384) X(512)

__host__ __device__ constexpr bool batch_length_ok(int L) {
    return L == 64 || L == 96 || L == 128 || L == 192 || L == 256 || L == 384 || L == 512;
}
// Rows per x tile and x values per strided tile: 256-thread tiles.
__host__ __device__ constexpr int batch_rows(int L) { return BATCH_THREADS / (L / make_plan(L).E); }
// Shared memory a tile of length L needs (the larger of its x and y roles).
__host__ __device__ constexpr size_t batch_smem(int L, int esz) {
    const size_t x = (size_t)batch_rows(L) * xpad(L) * esz;
    const size_t y = (size_t)L * batch_rows(L) * esz;
    return x > y ? x : y;
}

template <typename R>
struct BatchStage {
    const PassArgs<R>* args;  // device array [3][BATCH_MAX_GROUPS]: phases A, B, C of each group
    int ngroups;
    int lx[BATCH_MAX_GROUPS], ly[BATCH_MAX_GROUPS];
    int ntx[BATCH_MAX_GROUPS];                 // strided x blocks per instance
    unsigned xt[BATCH_MAX_GROUPS];             // x tiles per instance
    unsigned st[BATCH_MAX_GROUPS];             // strided tiles per instance
    unsigned xstart[BATCH_MAX_GROUPS + 1];     // first x tile of each group in the phase list
    unsigned sstart[BATCH_MAX_GROUPS + 1];     // first strided tile of each group
    GridBar* bar;
    unsigned wait_bound;                       // iterations a barrier wait may spin
};

// What a stage launch used: resident CTAs per SM, SMs, dynamic shared
// memory, grid (0 when nothing was launched).
struct BatchLaunchInfo {
    int per_sm, nsm, grid;
    size_t smem;
};

// Dynamic shared memory of the stage kernel and its launch (gpe_batch.cu):
// grid = co-resident CTAs, at most max_tiles.
size_t batch_stage_smem(int esz);
// Resources of the stage kernel for fields of esz bytes: registers, static
// shared memory, threads per CTA allowed, local memory per thread, resident
// CTAs per SM, SMs, cooperative launch support, dynamic shared memory.
cudaError_t batch_stage_attributes(int esz, long long* out);
bool batch_length_supported(int L);
// One phase (0 = x forward, 1 = strided, 2 = x inverse) of stage b for every
// instance, one tile per CTA, with programmatic dependent launch.
cudaError_t launch_batch_phase(const BatchStage<float>& b, int phase, cudaStream_t st);
cudaError_t launch_batch_phase(const BatchStage<double>& b, int phase, cudaStream_t st);
cudaError_t launch_batch_stage(const BatchStage<float>& b, unsigned max_tiles, cudaStream_t st, BatchLaunchInfo* info);
cudaError_t launch_batch_stage(const BatchStage<double>& b, unsigned max_tiles, cudaStream_t st,
                               BatchLaunchInfo* info);

}  // namespace gpe
