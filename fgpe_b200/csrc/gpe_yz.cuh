// gpe_yz.cuh -- the strided part of a 3D stage in one kernel: y forward,
// z forward * k-space * inverse, y inverse, over thread-block clusters.
//
// The separate strided passes (k_spass / k_spass2) each read and write the
// whole work field: 6 field transfers per stage, three kernel boundaries,
// and every pass waits on L2 latency for its lines.  Here a cluster of
// YZ_CS CTAs owns one slab of the field, YZ_XB consecutive x values by all y
// and all z (512 KB at 128^3 complex64), held in the CTAs' shared memory:
//   phase 1  CTA r loads its z planes [r*ZP, (r+1)*ZP) of the slab from the
//            work field and transforms their y lines in place (forward);
//   phase 2  CTA r takes the y rows [r*YR, (r+1)*YR): it reads its z lines
//            from the other CTAs' shared memory (distributed shared memory),
//            transforms them forward, multiplies by the k-space factor and
//            transforms back, holding the results in registers, and after a
//            cluster barrier writes them back where it read them;
//   phase 3  CTA r transforms its planes' y lines back (inverse) and stores
//            them to the work field.
// So a stage's strided work reads and writes the field once (2 transfers),
// with three cluster barriers and no global round trips in between.  The
// arithmetic is the line FFT of gpe_fft.cuh with the default plans and the
// k-space factor of spec_point, the same float operations per point as the
// three-pass chain with the scalar passes.
//
// Requirements (checked on the host, yz_supported): complex64, one field,
// nx a multiple of YZ_XB, y and z lengths with whole line batches (YZGeom::ok).
#pragma once

#include <cooperative_groups.h>

#include "gpe_kernels_impl.cuh"

namespace gpe {

constexpr int YZ_CS = 8;         // CTAs per cluster (portable cluster size)
constexpr int YZ_XB = 4;         // x values per slab: 32 bytes of a complex64 row
constexpr int YZ_THREADS = 256;

template <int LY, int LZ>
struct YZGeom {
    static constexpr int ZP = LZ / YZ_CS;            // z planes per CTA (phases 1, 3)
    static constexpr int YR = LY / YZ_CS;            // y rows per CTA (phase 2)
    // plane stride in elements: 32 bytes of padding put the four planes a half
    // warp touches in phases 1 and 3 on distinct shared-memory banks
    static constexpr int PS = LY * YZ_XB + 4;
    static constexpr int TY = Plan<LY>::T, TZ = Plan<LZ>::T;
    static constexpr int LPB_Y = YZ_THREADS / TY;    // y lines per batch (phases 1, 3)
    static constexpr int LPB_Z = YZ_THREADS / TZ;    // z lines per batch (phase 2)
    static constexpr int NB_Y = ZP * YZ_XB / (LPB_Y > 0 ? LPB_Y : 1);
    static constexpr int NB_Z = YR * YZ_XB / (LPB_Z > 0 ? LPB_Z : 1);
    static constexpr size_t smem_a = (size_t)ZP * PS * sizeof(float2);
    static constexpr size_t smem = smem_a + (size_t)(LPB_Z > 0 ? LPB_Z : 1) * LZ * sizeof(float2);
    static constexpr bool ok = LY % YZ_CS == 0 && LZ % YZ_CS == 0 && LPB_Y > 0 && LPB_Z > 0 &&
                               LPB_Y % YZ_XB == 0 && LPB_Z % YZ_XB == 0 && (ZP * YZ_XB) % LPB_Y == 0 &&
                               (YR * YZ_XB) % LPB_Z == 0 && smem <= 110 * 1024 && TY * LPB_Y == YZ_THREADS &&
                               TZ * LPB_Z == YZ_THREADS && NB_Z <= 4;
};

// Line storage of phases 1 and 3: position pos of line (zl, x) at A[zl*PS + pos*XB + x].
struct YLineAddr {
    float2* base;
    __device__ __forceinline__ float2* operator()(unsigned pos) const { return base + pos * (unsigned)YZ_XB; }
};
// Exchange storage of phase 2: position pos of batch line li at S[pos*LPB + li].
template <int LPB>
struct ZLineAddr {
    float2* base;
    __device__ __forceinline__ float2* operator()(unsigned pos) const { return base + pos * (unsigned)LPB; }
};

template <int LY, int LZ>
__global__ void __launch_bounds__(YZ_THREADS, 2) k_yz(PassArgs<float> a) {
    typedef YZGeom<LY, LZ> G;
    namespace cg = cooperative_groups;
    constexpr int EY = Plan<LY>::E, EZ = Plan<LZ>::E;
    constexpr int TY = G::TY, TZ = G::TZ;
    constexpr int RinY = Plan<LY>::in_radix(false), RoutY = Plan<LY>::out_radix(false);
    constexpr int RinZ = Plan<LZ>::in_radix(false), RoutZ = Plan<LZ>::out_radix(false);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* A = reinterpret_cast<float2*>(smem_raw);
    float2* S = reinterpret_cast<float2*>(smem_raw + G::smem_a);
    cg::cluster_group cluster = cg::this_cluster();

    pass_prologue_sync();
    const long long boff = select_instance(a).boff;
    // Uniform over the cluster: the flag is written by earlier launches only,
    // so either every CTA of the cluster leaves here or none does.
    if (a.check_done && (a.sc + (a.nbatch > 1 ? blockIdx.y : 0))->done) return;

    const int r = (int)cluster.block_rank();
    const int slab = (int)blockIdx.x / YZ_CS;
    const int xs = slab * YZ_XB;
    const long long NX = a.nx;
    const long long plane = NX * LY;  // elements per z plane of the field
    const unsigned tid = threadIdx.x;
    const float2* twy = a.tw;
    const float2* twz = a.twz;

    // ---- phase 1: load this CTA's planes, forward y transforms into A ----
    {
        const unsigned li = tid % G::LPB_Y, t = tid / G::LPB_Y;
#pragma unroll 1
        for (int b = 0; b < G::NB_Y; ++b) {
            const int line = b * G::LPB_Y + (int)li;
            const int zl = line / YZ_XB, x = line % YZ_XB;
            const long long g0 = boff + (long long)(r * G::ZP + zl) * plane + xs + x + (long long)t * NX;
            float2 v[EY];
#pragma unroll
            for (int e = 0; e < EY; ++e) v[e] = a.w[0][g0 + (long long)reg_off<LY, EY, TY, RinY>(e) * NX];
            const YLineAddr addr{A + zl * G::PS + x};
            line_fft_fwd<LY>(v, addr, twy, t);
            __syncthreads();  // the line's last exchange is read before its storage takes the output
#pragma unroll
            for (int e = 0; e < EY; ++e) *addr(t + (unsigned)reg_off<LY, EY, TY, RoutY>(e)) = v[e];
        }
    }
    cluster.sync();

    // ---- phase 2: z lines of this CTA's y rows, across the cluster ----------
    float2 res[G::NB_Z][EZ];
    {
        const unsigned li = tid % G::LPB_Z, t = tid / G::LPB_Z;
        const ZLineAddr<G::LPB_Z> addr{S + li};
#pragma unroll
        for (int b = 0; b < G::NB_Z; ++b) {
            const int line = b * G::LPB_Z + (int)li;
            const int y = r * G::YR + line / YZ_XB, x = line % YZ_XB;
            float2 v[EZ];
#pragma unroll
            for (int e = 0; e < EZ; ++e) {
                const int pos = (int)t + reg_off<LZ, EZ, TZ, RinZ>(e);
                const float2* rA = cluster.map_shared_rank(A, (unsigned)(pos / G::ZP));
                v[e] = rA[(pos % G::ZP) * G::PS + y * YZ_XB + x];
            }
            line_fft_fwd<LZ>(v, addr, twz, t);
            if (a.spec != SPEC_NONE) {
#pragma unroll
                for (int e = 0; e < EZ; ++e) {
                    float2 tmp[1] = {v[e]};
                    spec_point<float, 1>(a, tmp, xs + x, y, (int)t + reg_off<LZ, EZ, TZ, RoutZ>(e), 0);
                    v[e] = tmp[0];
                }
            }
            line_fft_inv<LZ>(v, addr, twz, t);
#pragma unroll
            for (int e = 0; e < EZ; ++e) res[b][e] = v[e];
            __syncthreads();  // the next batch reuses the exchange storage
        }
    }
    cluster.sync();  // every CTA has read its lines from the others
    {
        const unsigned li = tid % G::LPB_Z, t = tid / G::LPB_Z;
#pragma unroll
        for (int b = 0; b < G::NB_Z; ++b) {
            const int line = b * G::LPB_Z + (int)li;
            const int y = r * G::YR + line / YZ_XB, x = line % YZ_XB;
#pragma unroll
            for (int e = 0; e < EZ; ++e) {
                const int pos = (int)t + reg_off<LZ, EZ, TZ, RinZ>(e);
                float2* rA = cluster.map_shared_rank(A, (unsigned)(pos / G::ZP));
                rA[(pos % G::ZP) * G::PS + y * YZ_XB + x] = res[b][e];
            }
        }
    }
    cluster.sync();  // the results are in place in every CTA

    // ---- phase 3: inverse y transforms of this CTA's planes, store ---------
    {
        const unsigned li = tid % G::LPB_Y, t = tid / G::LPB_Y;
#pragma unroll 1
        for (int b = 0; b < G::NB_Y; ++b) {
            const int line = b * G::LPB_Y + (int)li;
            const int zl = line / YZ_XB, x = line % YZ_XB;
            const YLineAddr addr{A + zl * G::PS + x};
            float2 v[EY];
#pragma unroll
            for (int e = 0; e < EY; ++e) v[e] = *addr(t + (unsigned)reg_off<LY, EY, TY, RoutY>(e));
            __syncthreads();  // the line is read before its storage serves as the exchange buffer
            line_fft_inv<LY>(v, addr, twy, t);
            const long long g0 = boff + (long long)(r * G::ZP + zl) * plane + xs + x + (long long)t * NX;
#pragma unroll
            for (int e = 0; e < EY; ++e) a.w[0][g0 + (long long)reg_off<LY, EY, TY, RinY>(e) * NX] = v[e];
        }
    }
}

template <int LY, int LZ>
cudaError_t launch_yz(const PassArgs<float>& a, cudaStream_t st) {
    typedef YZGeom<LY, LZ> G;
    static_assert(G::ok, "no fused y-z kernel for this shape");
    static std::atomic<unsigned long long> attr{0};
    cudaError_t e = allow_smem(k_yz<LY, LZ>, G::smem, attr);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(a.nx / YZ_XB * YZ_CS), (unsigned)a.nbatch);
    cfg.blockDim = dim3(YZ_THREADS);
    cfg.dynamicSmemBytes = G::smem;
    cfg.stream = st;
    cudaLaunchAttribute attrs[2];
    attrs[0].id = cudaLaunchAttributeClusterDimension;
    attrs[0].val.clusterDim.x = YZ_CS;
    attrs[0].val.clusterDim.y = 1;
    attrs[0].val.clusterDim.z = 1;
    attrs[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attrs[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attrs;
    cfg.numAttrs = 2;
    return cudaLaunchKernelEx(&cfg, k_yz<LY, LZ>, a);
}

}  // namespace gpe
