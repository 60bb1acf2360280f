// gpe_flow_args.cuh -- host/device arguments of the persistent RK4 step kernel
// (gpe_flow.cuh): one launch per real-time RK4 step of a complex64,
// one-component 3D handle, the sixteen axis passes of the step run as one
// ordered list of tiles with per-tile dependency counters.
#pragma once

#include "gpe_kernels.cuh"

namespace gpe {

constexpr int FLOW_THREADS = 128;  // every tile of the step uses 128 threads
constexpr int FLOW_MAXC = 512;     // counters per pass (x blocks or z planes)

// Completion counters of one launch: cnt[pass][index] counts the finished
// tiles of pass 0 (y forward) and 1 (z forward * k-space * inverse) per x
// block, of pass 2 (y inverse) and 3 (x inverse + stage + x forward) per z
// plane, summed over the step's four stages.  Launches alternate between two
// sets; a launch zeroes the other set after its wait on the previous grid.
struct FlowSync {
    unsigned cnt[2][4][FLOW_MAXC];
    unsigned ticket[2];  // next tile of the launch's list
    int status;          // GPE_ERR_TIMEOUT once a bounded wait expired (sticky)
    int pad;
};

struct FlowArgs {
    PassArgs<float> s[3];  // y forward, z forward * k-space * inverse, y inverse
    PassArgs<float> x[4];  // x inverse + RK4 stage 1..4 epilogue + x forward (mode 1 only)
    FlowSync* sync;
    int set;               // counter set of this launch (launch parity)
    int ntx;               // x blocks of a strided tile row
    int rows;              // x rows per x tile
    unsigned wait_bound;   // sleeps of a dependency wait before it gives up
};

// Cubic grids the kernel is compiled for (gpe_flow.cu).
bool flow_shape_supported(int nx, int ny, int nz);
// Tiles per x row and rows per x tile of the flow kernel at length L.
int flow_rows(int L);
int flow_ntx(int L);
// Resident CTAs per SM of the flow kernel for length L (0 if none).
int flow_ctas_per_sm(int L);
// The three strided passes of one stage in one launch (mode 2).
int flow_strided_ctas_per_sm(int L);
bool dispatch_flow_strided(int L, const FlowArgs& fa, int grid, cudaStream_t st, cudaError_t* err);
// obs: the step's stage 4 runs the reducing epilogue (logging observables).
bool dispatch_flow(int L, bool obs, const FlowArgs& fa, int grid, cudaStream_t st, cudaError_t* err);

}  // namespace gpe
