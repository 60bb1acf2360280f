// gpe_batch.cu -- launcher of the persistent batch stage kernel (gpe_batch.cuh).
#include <atomic>

#include "gpe_batch.cuh"

namespace gpe {

// Dynamic shared memory of the stage kernel: the largest tile of the lengths
// it serves.
size_t batch_stage_smem(int esz) {
    size_t m = 0;
#define GPE_BATCH_SM(L) m = m > batch_smem(L, esz) ? m : batch_smem(L, esz);
    GPE_BATCH_LENGTHS(GPE_BATCH_SM)
#undef GPE_BATCH_SM
    return m;
}

bool batch_length_supported(int L) { return batch_length_ok(L); }

template <typename R>
static cudaError_t launch_stage(const BatchStage<R>& b, unsigned max_tiles, cudaStream_t st, BatchLaunchInfo* info) {
    const size_t smem = batch_stage_smem((int)sizeof(typename Cx<R>::T));
    // CTAs per SM and SMs of each device, looked up once; the dynamic shared
    // memory is opted in whatever its size (the kernel's static arrays count
    // against the 48 KB default too)
    constexpr int MAXDEV = 64;
    static std::atomic<int> cached[MAXDEV];
    cudaError_t e;
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    int per_sm = 0, nsm = 0;
    const int c = (dev >= 0 && dev < MAXDEV) ? cached[dev].load() : 0;
    if (c > 0) {
        per_sm = c & 0xffff;
        nsm = c >> 16;
    } else {
        if ((e = cudaFuncSetAttribute(k_batch_stage<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
            cudaSuccess)
            return e;
        if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_stage<R>, BATCH_THREADS, smem)) !=
            cudaSuccess)
            return e;
        if (dev >= 0 && dev < MAXDEV && per_sm > 0 && per_sm < 0x10000 && nsm < 0x8000)
            cached[dev].store(per_sm | (nsm << 16));
    }
    if (info) {
        info->per_sm = per_sm;
        info->nsm = nsm;
        info->smem = smem;
        info->grid = 0;
    }
    if (per_sm < 1) return cudaErrorLaunchOutOfResources;
    // co-resident CTAs (the cooperative launch checks it), no more than the tiles
    unsigned grid = (unsigned)(per_sm * nsm);
    if (max_tiles < grid) grid = max_tiles > 0 ? max_tiles : 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(BATCH_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (info) info->grid = (int)grid;
    e = cudaLaunchKernelEx(&cfg, k_batch_stage<R>, b);
    if (e != cudaSuccess) cudaGetLastError();  // a refused launch leaves no error behind for later calls
    return e;
}

template <typename R, int PHASE>
static cudaError_t launch_phase_k(const BatchStage<R>& b, cudaStream_t st) {
    const size_t smem = batch_stage_smem((int)sizeof(typename Cx<R>::T));
    static std::atomic<unsigned long long> attr{0};
    cudaError_t e = allow_smem(k_batch_phase<R, PHASE>, smem, attr);
    if (e != cudaSuccess) return e;
    const unsigned tiles = PHASE == 1 ? b.sstart[b.ngroups] : b.xstart[b.ngroups];
    if (tiles == 0) return cudaSuccess;
    e = launch_pass(k_batch_phase<R, PHASE>, tiles, 1u, (unsigned)BATCH_THREADS, smem, st, b);
    if (e != cudaSuccess) cudaGetLastError();
    return e;
}

template <typename R>
static cudaError_t launch_phase(const BatchStage<R>& b, int phase, cudaStream_t st) {
    switch (phase) {
        case 0: return launch_phase_k<R, 0>(b, st);
        case 1: return launch_phase_k<R, 1>(b, st);
        default: return launch_phase_k<R, 2>(b, st);
    }
}

cudaError_t launch_batch_phase(const BatchStage<float>& b, int phase, cudaStream_t st) {
    return launch_phase<float>(b, phase, st);
}
cudaError_t launch_batch_phase(const BatchStage<double>& b, int phase, cudaStream_t st) {
    return launch_phase<double>(b, phase, st);
}

template <typename R>
static cudaError_t stage_attributes(long long* out) {
    const size_t smem = batch_stage_smem((int)sizeof(typename Cx<R>::T));
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k_batch_stage<R>);
    if (e != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_batch_stage<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
        cudaSuccess)
        return e;
    int dev = 0, nsm = 0, per_sm = 0, coop = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_stage<R>, BATCH_THREADS, smem)) !=
        cudaSuccess)
        return e;
    out[0] = fa.numRegs;
    out[1] = (long long)fa.sharedSizeBytes;
    out[2] = fa.maxThreadsPerBlock;
    out[3] = (long long)fa.localSizeBytes;
    out[4] = per_sm;
    out[5] = nsm;
    out[6] = coop;
    out[7] = (long long)smem;
    return cudaSuccess;
}

cudaError_t batch_stage_attributes(int esz, long long* out) {
    return esz == 8 ? stage_attributes<float>(out) : stage_attributes<double>(out);
}

cudaError_t launch_batch_stage(const BatchStage<float>& b, unsigned max_tiles, cudaStream_t st,
                               BatchLaunchInfo* info) {
    return launch_stage<float>(b, max_tiles, st, info);
}
cudaError_t launch_batch_stage(const BatchStage<double>& b, unsigned max_tiles, cudaStream_t st,
                               BatchLaunchInfo* info) {
    return launch_stage<double>(b, max_tiles, st, info);
}

}  // namespace gpe
