// Common definitions for the Full Binary Pursuit CUDA kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cmath>
#include <stdint.h>

typedef uint32_t u32;
typedef uint8_t u8;
typedef uint16_t u16;
typedef unsigned long long u64;

namespace fbp {

// Block-wide tile of the ordered compaction: 256 threads x 16 bytes.
constexpr u32 kCompactThreads = 256;
constexpr u32 kCompactPerThread = 16;
constexpr u32 kCompactTile = kCompactThreads * kCompactPerThread;   // 4096

__host__ __device__ inline u32 ceil_div(u32 a, u32 b) { return (a + b - 1) / b; }
__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Device counters shared by the kernels of one chunk (one 128-byte line).
struct Counters {
    u32 n_win;        // windows in the active list of this pass
    u32 n_cand;       // overlap-recheck candidates of this pass
    u32 n_spk;        // spikes accepted in this pass
    u32 total;        // spikes written to the output so far
    u32 overflow;     // set when the output buffer is too small
    u32 scan_total;   // scratch: result of the last compaction
    u32 pool_total;   // overlap contenders appended this pass (may exceed the pool)
    u32 fb_count;     // overlap candidates sent to the exact kernel this pass
    u64 ov_items;     // overlap items evaluated (after the skip rules)
    u32 pad2;
    u32 tc_err;       // non-zero: a bounded wait in the tensor-core kernel gave up
    u32 tc_overflow;  // refinement list overflowed: the exact kernel redoes the pass
    u32 pad0;
    u64 lazy_ref;     // approximate likelihood entries refined on demand (whole chunk)
    u32 ov_ref;       // overlap contenders evaluated exactly this pass
    u32 pad1;
    u64 scan_next;    // work counter of the overlap scan
    u64 tc_refseg;    // tensor-core refinement list: entries queued (high half), tile segments (low half)
    u64 tc_seq;       // refinement entries whose sign needed the reference's own sum (whole chunk)
    u32 n_runs;       // runs of consecutive windows in the pass's list (wide tensor-core tiles)
    u32 n_stiles;     // tiles of the pass's window stream (wide tensor-core tiles)
    u32 pad[6];
};
static_assert(sizeof(Counters) == 128, "Counters is one 128-byte line");

// Warp-level inclusive prefix sum.
__device__ __forceinline__ u32 warp_incl_scan(u32 v) {
    const u32 lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        u32 y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= (u32)o) v += y;
    }
    return v;
}

// Block-wide exclusive scan for blockDim.x == kCompactThreads.  Returns the
// exclusive prefix of `v`; *total receives the block sum.
__device__ __forceinline__ u32 block_excl_scan(u32 v, u32 *total) {
    __shared__ u32 warp_sums[kCompactThreads / 32];
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u32 incl = warp_incl_scan(v);
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        u32 w = lane < kCompactThreads / 32 ? warp_sums[lane] : 0;
        u32 wi = warp_incl_scan(w);
        if (lane < kCompactThreads / 32) warp_sums[lane] = wi - w;
    }
    __syncthreads();
    u32 ex = warp_sums[warp] + incl - v;
    if (total) {
        __shared__ u32 tot;
        if (threadIdx.x == blockDim.x - 1) tot = ex + v;
        __syncthreads();
        *total = tot;
    }
    return ex;
}

}  // namespace fbp
