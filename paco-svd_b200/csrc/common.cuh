// Shared definitions for the sm_100a kernels of the paco-svd B200 library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/paco_svd.h"

#define PACO_WARP 32

// Device-side status block, the first bytes of every workspace.  Kernels never
// trap: they record what went wrong here and return, so the context stays
// usable and the host reads the cause after a synchronize.
struct DevStatus {
    int code;            // first fatal error code (PACO_ERR_*), 0 if none
    int info;            // detail for `code` (kernel-specific)
    int secular_nonconv; // secular roots that hit the iteration limit
    int wait_timeouts;   // bounded waits that gave up
    int counters[60];    // arrival tickets for last-block reductions
    int stage1_mark;     // PACO_STAGE1_MARK while a stage-1 run's status awaits stage 2
};

#define PACO_STAGE1_MARK 0x31474B42  // "BKG1"

// Opens a run on a workspace whose status block may hold anything.  Stage 1
// (stage = 1) starts a new factorization: the block is cleared and marked.
// Stage 2 (stage = 2) keeps the codes of a stage-1 run on the same workspace
// (the two-kernel flow reads both through one paco_sync_status) and clears
// them otherwise; either way the marker is consumed and the counters reset.
__global__ void dev_status_begin(DevStatus *st, int stage);

__device__ __forceinline__ void dev_fail(DevStatus *st, int code, int info)
{
    if (atomicCAS(&st->code, 0, code) == 0) st->info = info;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Last-block-done ticket: every block calls this once after writing its
// partial results; exactly one block (the last to arrive) gets `true` and may
// then read every other block's partials.  The counter is reset for reuse.
__device__ __forceinline__ bool last_block_ticket(int *counter, int nblocks, int *s_flag)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        int t = atomicAdd(counter, 1);
        *s_flag = (t == nblocks - 1);
        if (*s_flag) atomicExch(counter, 0);
    }
    __syncthreads();
    bool last = *s_flag != 0;
    if (last) __threadfence();
    return last;
}

// Host-side count of kernel launches issued by the library (paco_launch_count).
void paco_count_launch();

// Ordinal of the current device (0..PACO_MAX_DEVICES-1): the index of the
// per-device caches (kernel attributes, launch configurations, SM counts) a
// process that drives several GPUs keeps apart.
#define PACO_MAX_DEVICES 64
int paco_device();

// Shape-dependent choices of the single-matrix path (the tiling autotuner's
// output, paco_autotune): the persistent panel kernel or the two-kernel row /
// column passes, rows per CTA of a panel (sets the grid: fewer CTAs meet at
// each barrier, more CTAs stream more bandwidth), and whether the large
// products use the tcgen05 GEMM, and whether the last columns stay on the
// panel kernel instead of the cluster kernel (no_tail = 1); the tile shapes
// of the blocked products: reflectors per compact-WY block when U and V are
// formed (wy: 64 or 128), columns per QR block (qb: 32 or 64), and matrices
// per lockstep group of the multi-matrix form (mk: 1..8).  0 = the default.
struct PacoTune {
    int persistent, rows_per_cta, tc, no_tail;
    int wy, qb, mk;
    int ts;  // two-stage reduction: band width 32 or 64, 0 off
};
PacoTune paco_tune_for(int M, int N);

static inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }
static inline long round_up(long a, long b) { return (a + b - 1) / b * b; }
