// gpe_flow.cuh -- one persistent launch per real-time RK4 step.
//
// The per-pass chain (run_chain) launches the sixteen axis passes of a
// complex64 RK4 step one after another (per stage: y forward, z forward *
// k-space * inverse, y inverse, x inverse + stage epilogue + x forward of the
// new stage state).  Each launch is one wave of tiles at 128^3: every SM
// loads, then transforms, then stores, and the next pass starts only when the
// last tile of the previous one has finished.  Here the CTAs of one launch
// take the tiles of all sixteen passes from one ordered list (a ticket in
// device memory) and each tile waits only for the tiles whose output it
// reads, so the passes overlap: while some CTAs of an SM finish the tiles of
// one pass, others load the tiles of the next.
//
// Tile order and dependencies per stage (tiles are the pass kernels' own
// bodies: spass2_tile, xpass_tile<XK_RKF>; the arithmetic is theirs, bit for
// bit):
//   P1 y forward       (x block xb, plane z), xb-major   <- P4 of the previous
//                      stage in plane z (NY/rows tiles)
//   P2 z fwd*k*inv     (xb, row y), xb-major             <- P1 (xb, every z)
//   P3 y inverse       (xb, z), xb-major                 <- P2 (xb, every y)
//   P4 x inverse + RK4 stage + x forward (rows tile in plane z)
//                                                        <- P3 (every xb, z)
// Every dependency of a tile lies earlier in the list, and tiles are handed
// out in list order, so the smallest unfinished tile can always proceed: the
// launch cannot deadlock whatever the number of resident CTAs.  The write
// after read hazards of the in-place passes are covered by the same counters
// (a tile that overwrites a region waits for the tiles that read it).
//
// Synchronisation: a finished tile's threads meet at a barrier, then one
// thread fences and increments the tile's counter (release); a waiting
// thread polls the counter, fences (acquire) and releases its CTA with a
// barrier -- the pattern of a grid barrier, per tile.  Each wait is bounded
// (wait_bound sleeps of 32 ns): a CTA that gives up records GPE_ERR_TIMEOUT
// in the sticky status word and every CTA leaves at its next tile, so a
// launch always ends; later launches see the status and exit at once.
#pragma once

#include "gpe_flow_args.cuh"
#include "gpe_kernels_impl.cuh"

namespace gpe {

__device__ __forceinline__ unsigned flow_ld(const unsigned* p) { return *reinterpret_cast<const volatile unsigned*>(p); }
__device__ __forceinline__ int flow_ld_i(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

template <int L>
struct FlowGeom {
    static constexpr int TXP = spass2_txp(L);               // pairs per strided tile
    static constexpr int ST = TXP * Plan<L>::T;             // threads of a strided tile
    static constexpr int ROWS = FLOW_THREADS / Plan<L>::T;  // x rows per x tile
    static constexpr int NTX = L / (2 * TXP);               // strided tiles per x row
    static constexpr size_t SMEM_S = (size_t)L * TXP * sizeof(float4);
    static constexpr size_t SMEM_X = (size_t)ROWS * xpad(L) * sizeof(float2);
    static constexpr size_t SMEM = SMEM_S > SMEM_X ? SMEM_S : SMEM_X;
    static constexpr bool ok = ST == FLOW_THREADS && ROWS * Plan<L>::T == FLOW_THREADS && L % ROWS == 0 &&
                               L % (2 * TXP) == 0 && L <= FLOW_MAXC;
};

// Resident CTAs per SM the launch bounds ask for: 80 registers a thread,
// which the x tile's fused epilogue and the paired strided tile both fit
// without spills at length 128.
constexpr int FLOW_MIN_BLOCKS = 6;

// Which counter tile j of pass `pass` in stage s waits on and the count it
// needs (pointer null: no wait).
template <int L>
__device__ __forceinline__ void flow_deps(unsigned* cnt, unsigned s, unsigned pass, unsigned j, unsigned** wait,
                                          unsigned* need) {
    typedef FlowGeom<L> G;
    constexpr unsigned NT = G::NTX, ROWS = G::ROWS;
    unsigned* c0 = cnt;
    unsigned* c1 = cnt + FLOW_MAXC;
    unsigned* c2 = cnt + 2 * FLOW_MAXC;
    unsigned* c3 = cnt + 3 * FLOW_MAXC;
    *wait = nullptr;
    *need = 0;
    switch (pass) {
        case 0: {  // y forward (xb = j / L, z = j % L)
            const unsigned z = j % L;
            if (s > 0) {
                *wait = c3 + z;
                *need = (L / ROWS) * s;
            }
            break;
        }
        case 1:  // z forward * k * inverse (xb = j / L, y = j % L)
            *wait = c0 + j / L;
            *need = L * (s + 1);
            break;
        case 2:  // y inverse (xb = j / L, z = j % L)
            *wait = c1 + j / L;
            *need = L * (s + 1);
            break;
        default: {  // x rows tile j of plane z
            const unsigned z = (j * ROWS) / L;
            *wait = c2 + z;
            *need = NT * (s + 1);
            break;
        }
    }
}

// Launch prologue of the persistent kernels: waits for the previous grid
// (its memory is then visible), and CTA 0 zeroes the counter set of the
// next launch, which the previous launch used.  False when an earlier wait
// gave up (the launch then does nothing).
__device__ __forceinline__ bool flow_begin(FlowSync* sy, int set) {
    pass_prologue_sync();
    if (flow_ld_i(&sy->status) != 0) return false;
    if (blockIdx.x == 0) {
        unsigned* other = &sy->cnt[set ^ 1][0][0];
        for (int i = threadIdx.x; i < 4 * FLOW_MAXC; i += FLOW_THREADS) other[i] = 0u;
        if (threadIdx.x == 0) sy->ticket[set ^ 1] = 0u;
    }
    return true;
}

// Thread 0's part of taking a tile: `next` is the tile reserved earlier; the
// one after it is reserved now, then the wait for *w >= need (w null: no
// wait), bounded; an expired wait records GPE_ERR_TIMEOUT in the step's and
// the handle's status words.  Returns the tile, or `total` when the launch
// is over for this CTA.
__device__ __forceinline__ unsigned flow_take(FlowSync* sy, int set, unsigned& next, unsigned total, const unsigned* w,
                                              unsigned need, unsigned bound, int* hstatus) {
    const unsigned item = next;
    if (item >= total || flow_ld_i(&sy->status) != 0) return total;
    next = atomicAdd(&sy->ticket[set], 1u);
    if (w != nullptr && flow_ld(w) < need) {
        unsigned it = 0;
        while (flow_ld(w) < need) {
            if (++it > bound || flow_ld_i(&sy->status) != 0) {
                atomicExch(&sy->status, (int)GPE_ERR_TIMEOUT);
                atomicExch(hstatus, (int)GPE_ERR_TIMEOUT);
                return total;
            }
            __nanosleep(32);
        }
    }
    __threadfence();  // acquire: the tiles counted in *w are visible
    return item;
}

// After a tile: every thread's stores are issued (barrier), then one fence
// and the count (release).
__device__ __forceinline__ void flow_done(unsigned* done) {
    __syncthreads();
    if (threadIdx.x == 0 && done != nullptr) {
        __threadfence();
        atomicAdd(done, 1u);
    }
}

// OBS: the step returns the logging observables, so stage 4's x tiles run
// the reducing epilogue (XK_RKO: the last tile finalises, no x forward of
// the new state) instead of XK_RKF.
template <int L, bool OBS>
__global__ void __launch_bounds__(FLOW_THREADS, FLOW_MIN_BLOCKS) k_flow_step(const __grid_constant__ FlowArgs fa) {
    typedef FlowGeom<L> G;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned s_item;
    constexpr unsigned NT = G::NTX;
    constexpr unsigned N1 = NT * L, N2 = NT * L, N3 = NT * L, N4 = (L * L) / G::ROWS;
    constexpr unsigned NS = N1 + N2 + N3 + N4, TOTAL = 4 * NS;
    FlowSync* sy = fa.sync;
    const int set = fa.set;
    unsigned* cnt = &sy->cnt[set][0][0];
    if (!flow_begin(sy, set)) return;

    unsigned next = 0;
    if (threadIdx.x == 0) next = atomicAdd(&sy->ticket[set], 1u);
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned item = next;
            unsigned* w = nullptr;
            unsigned need = 0;
            if (item < TOTAL) {
                const unsigned s = item / NS, r = item % NS;
                const unsigned pass = r < N1 ? 0u : (r < N1 + N2 ? 1u : (r < N1 + N2 + N3 ? 2u : 3u));
                const unsigned j = pass == 0 ? r : (pass == 1 ? r - N1 : (pass == 2 ? r - N1 - N2 : r - N1 - N2 - N3));
                flow_deps<L>(cnt, s, pass, j, &w, &need);
            }
            s_item = flow_take(sy, set, next, TOTAL, w, need, fa.wait_bound, &fa.x[0].sc->status);
        }
        __syncthreads();
        const unsigned item = s_item;
        if (item >= TOTAL) break;
        const unsigned s = item / NS, r = item % NS;
        unsigned* done;
        if (r < N1) {
            const unsigned xb = r / L, z = r % L;
            spass2_tile<L, 1, G::TXP, 0>(fa.s[0], (int)NT, z * NT + xb, 0u, smem_raw);
            done = cnt + xb;
        } else if (r < N1 + N2) {
            const unsigned j = r - N1, xb = j / L, y = j % L;
            spass2_tile<L, 1, G::TXP, 0>(fa.s[1], (int)NT, y * NT + xb, 0u, smem_raw);
            done = cnt + FLOW_MAXC + xb;
        } else if (r < N1 + N2 + N3) {
            const unsigned j = r - N1 - N2, xb = j / L, z = j % L;
            spass2_tile<L, 1, G::TXP, 0>(fa.s[2], (int)NT, z * NT + xb, 0u, smem_raw);
            done = cnt + 2 * FLOW_MAXC + z;
        } else {
            const unsigned j = r - N1 - N2 - N3;
            if (OBS && s == 3)
                xpass_tile<float, L, 1, XK_RKO, BuiltinHam>(fa.x[3], G::ROWS, j, 0u, N4, smem_raw);
            else
                xpass_tile<float, L, 1, XK_RKF, BuiltinHam>(fa.x[s], G::ROWS, j, 0u, N4, smem_raw);
            done = cnt + 3 * FLOW_MAXC + (j * G::ROWS) / L;
        }
        flow_done(done);  // also frees the exchange storage for the next tile
    }
}

// Mode 2: the three strided passes of one stage (y forward, z forward *
// k-space * inverse, y inverse) in one launch, the x passes staying their
// own launches.  All three lists are x-block major and each pass depends on
// the previous one per x block only (the z tiles of block xb need its y
// forward tiles of every plane, the y-inverse tiles of xb its z tiles of
// every row), so the tiles stream without a corner turn: the z tiles of
// block 0 start once the first L y-forward tiles are done.  Registers: the
// paired strided tile alone (72, seven CTAs per SM).
constexpr int FLOW_S_MIN_BLOCKS = 7;

template <int L>
__global__ void __launch_bounds__(FLOW_THREADS, FLOW_S_MIN_BLOCKS) k_flow_strided(const __grid_constant__ FlowArgs fa) {
    typedef FlowGeom<L> G;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned s_item;
    constexpr unsigned NT = G::NTX, NP = NT * L, TOTAL = 3 * NP;
    FlowSync* sy = fa.sync;
    const int set = fa.set;
    unsigned* cnt = &sy->cnt[set][0][0];
    if (!flow_begin(sy, set)) return;

    unsigned next = 0;
    if (threadIdx.x == 0) next = atomicAdd(&sy->ticket[set], 1u);
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned item = next;
            unsigned* w = nullptr;
            unsigned need = L;
            if (item < TOTAL && item >= NP) w = cnt + (item < 2 * NP ? 0 : FLOW_MAXC) + (item % NP) / L;
            s_item = flow_take(sy, set, next, TOTAL, w, need, fa.wait_bound, &fa.s[0].sc->status);
        }
        __syncthreads();
        const unsigned item = s_item;
        if (item >= TOTAL) break;
        const unsigned pass = item / NP, j = item % NP, xb = j / L, o = j % L;
        spass2_tile<L, 1, G::TXP, 0>(fa.s[pass], (int)NT, o * NT + xb, 0u, smem_raw);
        flow_done(pass < 2 ? cnt + pass * FLOW_MAXC + xb : nullptr);
    }
}

template <int L, bool OBS>
cudaError_t launch_flow(const FlowArgs& fa, int grid, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(FLOW_THREADS);
    cfg.dynamicSmemBytes = FlowGeom<L>::SMEM;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_flow_step<L, OBS>, fa);
}

template <int L>
cudaError_t launch_flow_strided(const FlowArgs& fa, int grid, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(FLOW_THREADS);
    cfg.dynamicSmemBytes = FlowGeom<L>::SMEM_S;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_flow_strided<L>, fa);
}

template <int L>
int flow_strided_occupancy() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_flow_strided<L>, FLOW_THREADS, FlowGeom<L>::SMEM_S) !=
        cudaSuccess)
        return 0;
    return n;
}

template <int L>
int flow_occupancy() {
    int n = 0;
    int n2 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_flow_step<L, false>, FLOW_THREADS, FlowGeom<L>::SMEM) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n2, k_flow_step<L, true>, FLOW_THREADS, FlowGeom<L>::SMEM) !=
            cudaSuccess)
        return 0;
    return n < n2 ? n : n2;
}

}  // namespace gpe
