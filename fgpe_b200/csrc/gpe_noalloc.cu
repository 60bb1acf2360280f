// gpe_noalloc.cu -- gpe_norm_noalloc: the norm reduction sum |psi|^2 * DV of a
// caller-owned device complex128 array, written for callers that cannot have
// the library allocate device memory.
//
// The handle-based reductions (gpe_observables and the fused pass epilogues)
// keep their block partials in memory that gpe_create allocates.  This entry
// point keeps them in one fixed file-scope device array instead, so a call
// makes no cudaMalloc/cudaFree and needs no handle.  Callers that gain from
// that: an application whose own allocator has already reserved the device
// memory (a further cudaMalloc would fail), and a time-stepping loop that
// wants to check the norm between steps without the device-wide
// synchronisation that cudaFree implies.
//
// Limits and rules of use:
//  - At most GPE_NORM_NOALLOC_MAX_POINTS points (512^3) per call: the scratch
//    holds one 16-byte partial per block of 16384 points.  Larger n is
//    rejected with GPE_ERR_UNSUPPORTED before anything is launched.
//  - The first call on each device does a one-time set-up with that device
//    current: it looks up the scratch's device address (which may also load
//    this file's kernel onto the device) and zeroes the completion counter
//    with a synchronous cudaMemset.  Make that first call before any stream
//    capture begins on the device.  The address is cached per device for
//    the life of the process; cudaDeviceReset on a device leaves the cached
//    address pointing into the destroyed context, so the entry point must not
//    be called on that device again in the same process.
//  - What must start at zero: the completion counter in the first bytes of the
//    scratch.  It is zero when the module loads, the set-up zeroes it again,
//    and the last block of every call puts it back to zero.  The block
//    partials need no initial value: each block writes its own slot before
//    the last block reads it.
//  - Calls that may overlap on one device (different streams with no ordering
//    between them, or host threads issuing at once) share the scratch and
//    race: the result of either can be wrong.  Order them on one stream.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/gpe.h"

namespace gpe {
void set_last_error(const char* msg);
}

namespace {

constexpr int kThreads = 256;
constexpr int kItemsPerThread = 64;
constexpr long long kPointsPerBlock = (long long)kThreads * kItemsPerThread;  // 16384
constexpr int kMaxBlocks = (int)(GPE_NORM_NOALLOC_MAX_POINTS / kPointsPerBlock);  // 8192
constexpr size_t kHeaderBytes = 256;  // completion counter, padded to the alignment
constexpr size_t kScratchBytes = kHeaderBytes + (size_t)kMaxBlocks * sizeof(double2);  // 128 KiB + 256 B
constexpr int kMaxDevices = 64;

static_assert(GPE_NORM_NOALLOC_MAX_POINTS % kPointsPerBlock == 0, "limit must be whole blocks");

// Layout: [0, 4) unsigned completion counter; [256, 256 + 16 * kMaxBlocks)
// one (sum, compensation) pair per block.
static __device__ __align__(256) unsigned char g_norm_scratch[kScratchBytes];

std::mutex g_setup_mutex;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Neumaier-compensated accumulation: (s, c) holds s + c.
__device__ __forceinline__ void acc(double& s, double& c, double a) {
    double t = s + a;
    c += (fabs(s) >= fabs(a)) ? (s - t) + a : (a - t) + s;
    s = t;
}

// Merge two compensated pairs with an exact two-sum of the leading parts.
__device__ __forceinline__ void merge(double& s, double& c, double s2, double c2) {
    double t = s + s2;
    double bp = t - s;
    double err = (s - (t - bp)) + (s2 - bp);
    s = t;
    c = c + c2 + err;
}

// Fixed-shape block reduction (same tree on every call): warp shuffles, then
// the first warp over the warp results.  Result valid in thread 0.
__device__ void block_reduce(double& s, double& c) {
    __shared__ double ws[kThreads / 32], wc[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        double s2 = __shfl_down_sync(0xffffffffu, s, o);
        double c2 = __shfl_down_sync(0xffffffffu, c, o);
        merge(s, c, s2, c2);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        ws[w] = s;
        wc[w] = c;
    }
    __syncthreads();
    if (w == 0) {
        s = l < kThreads / 32 ? ws[l] : 0.0;
        c = l < kThreads / 32 ? wc[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            double s2 = __shfl_down_sync(0xffffffffu, s, o);
            double c2 = __shfl_down_sync(0xffffffffu, c, o);
            merge(s, c, s2, c2);
        }
    }
    __syncthreads();
}

// Block b sums points [b * 16384, (b + 1) * 16384) (a thread takes every
// 256th point, so the loads coalesce), stores its pair in the scratch, and
// the last block to finish sums the pairs in block order.  The grid depends
// only on n, so the result is the same bits on every call and every device.
__global__ void __launch_bounds__(kThreads) k_norm_noalloc(const double2* __restrict__ psi, long long n, double dv,
                                                           unsigned char* scratch, double* out) {
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch);
    double2* part = reinterpret_cast<double2*>(scratch + kHeaderBytes);
    __shared__ bool last;

    double s = 0.0, c = 0.0;
    const long long base = (long long)blockIdx.x * kPointsPerBlock + threadIdx.x;
#pragma unroll 8
    for (int k = 0; k < kItemsPerThread; ++k) {
        const long long i = base + (long long)k * kThreads;
        if (i < n) {
            const double2 v = __ldcs(psi + i);
            acc(s, c, v.x * v.x + v.y * v.y);
        }
    }
    block_reduce(s, c);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = make_double2(s, c);
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;

    __threadfence();
    s = 0.0;
    c = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kThreads) {
        const double2 p = __ldcg(part + b);
        merge(s, c, p.x, p.y);
    }
    block_reduce(s, c);
    if (threadIdx.x == 0) {
        out[0] = (s + c) * dv;
        *counter = 0u;  // ready for the next call
    }
}

gpe_status fail(gpe_status st, const char* msg) {
    gpe::set_last_error(msg);
    return st;
}

gpe_status cuda_fail(const char* what, cudaError_t e) {
    char buf[256];
    std::snprintf(buf, sizeof buf, "gpe_norm_noalloc: %s: %s", what, cudaGetErrorString(e));
    return fail(e == cudaErrorMemoryAllocation ? GPE_ERR_OUT_OF_MEMORY : GPE_ERR_CUDA, buf);
}

}  // namespace

extern "C" gpe_status gpe_norm_noalloc(const void* dev_psi_c128, long long n, double dv, double* dev_out,
                                       void* cuda_stream) {
    if (n < 0) return fail(GPE_ERR_INVALID_ARG, "gpe_norm_noalloc: negative point count");
    if (n > GPE_NORM_NOALLOC_MAX_POINTS) {
        char buf[200];
        std::snprintf(buf, sizeof buf,
                      "gpe_norm_noalloc: %lld points exceed the fixed scratch limit of %lld points (512^3)", n,
                      (long long)GPE_NORM_NOALLOC_MAX_POINTS);
        return fail(GPE_ERR_UNSUPPORTED, buf);
    }
    if (!dev_out) return fail(GPE_ERR_INVALID_ARG, "gpe_norm_noalloc: null output pointer");
    if (n > 0 && !dev_psi_c128) return fail(GPE_ERR_INVALID_ARG, "gpe_norm_noalloc: null psi pointer");
    if ((reinterpret_cast<uintptr_t>(dev_psi_c128) & 15u) != 0)
        return fail(GPE_ERR_INVALID_ARG, "gpe_norm_noalloc: psi must be 16-byte aligned (complex128)");
    if ((reinterpret_cast<uintptr_t>(dev_out) & 7u) != 0)
        return fail(GPE_ERR_INVALID_ARG, "gpe_norm_noalloc: output must be 8-byte aligned");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
    if (dev < 0 || dev >= kMaxDevices) return fail(GPE_ERR_UNSUPPORTED, "gpe_norm_noalloc: device ordinal above 63");

    unsigned char* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[dev]) {
            // One-time set-up for this device, which is current here.
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_norm_scratch);
            if (e != cudaSuccess) return cuda_fail("cudaGetSymbolAddress", e);
            if (!p) return fail(GPE_ERR_CUDA, "gpe_norm_noalloc: scratch address is null");
            e = cudaMemset(p, 0, kHeaderBytes);
            if (e != cudaSuccess) return cuda_fail("cudaMemset of the completion counter", e);
            g_scratch_addr[dev] = static_cast<unsigned char*>(p);
        }
        scratch = g_scratch_addr[dev];
    }

    const long long blocks = n == 0 ? 1 : (n + kPointsPerBlock - 1) / kPointsPerBlock;
    k_norm_noalloc<<<(unsigned)blocks, kThreads, 0, static_cast<cudaStream_t>(cuda_stream)>>>(
        static_cast<const double2*>(dev_psi_c128), n, dv, scratch, dev_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail("kernel launch", e);
    return GPE_OK;
}
