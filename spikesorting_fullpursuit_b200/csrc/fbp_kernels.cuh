// Full Binary Pursuit kernels for sm_100a.
//
// Each kernel restates one kernel of the reference
// (spikesorting_fullpursuit/kernels/binary_pursuit.cl) with the results a
// work-group size of 1 gives when work-items run in global-id order.  Where
// the reference's outcome depends on that order (neighbour flags, the
// overlap_recheck[id-2] read, overlapping residual subtractions), the order
// is resolved explicitly so that any thread schedule gives the same answer.
//
// Exact-order floating point: the likelihoods are accumulated with
// __fmul_rn/__fadd_rn (never contracted into FMA) in the reference's order,
// so every value is bit-identical to the reference's IEEE binary32 result.
#pragma once
#include "fbp_common.cuh"

namespace fbp {

// Per-window bounds written by the likelihood kernels (both paths) for the
// window argmax: wlb[w] the largest lower bound of an entry of window w,
// umax[w][t] the largest upper bound of template t's entries there (>= 0),
// wpos[w] whether any entry of the window is > 0.  Reset when the window is
// listed for recomputation; entries only move inside their intervals later.
struct WinBounds {
    float *wlb;
    float *umax;
    u8 *wpos;
};


// ---------------------------------------------------------------------------
// Ordered compaction: list of indices j < W with f[j] != 0, ascending.
// Three launches: per-tile counts, one-block scan of the tile counts, write.
// f must be readable up to align_up(W, kCompactTile) bytes.
// ---------------------------------------------------------------------------
__global__ void k_compact_count(const u8 *__restrict__ f, u32 W, u32 *__restrict__ tile_counts) {
    const u32 base = blockIdx.x * kCompactTile + threadIdx.x * kCompactPerThread;
    uint4 q = *reinterpret_cast<const uint4 *>(f + base);
    const u8 *b = reinterpret_cast<const u8 *>(&q);
    u32 c = 0;
#pragma unroll
    for (u32 i = 0; i < kCompactPerThread; i++) c += (base + i < W && b[i] != 0);
    u32 tot;
    block_excl_scan(c, &tot);
    if (threadIdx.x == 0) tile_counts[blockIdx.x] = tot;
}

// One block of kCompactThreads threads: exclusive scan of tile_counts in place.
__global__ void k_compact_scan(u32 *__restrict__ tile_counts, u32 n_tiles, u32 *__restrict__ total_out) {
    u32 carry = 0;
    for (u32 base = 0; base < n_tiles; base += kCompactThreads) {
        u32 i = base + threadIdx.x;
        u32 v = i < n_tiles ? tile_counts[i] : 0;
        u32 tot;
        u32 ex = block_excl_scan(v, &tot);
        if (i < n_tiles) tile_counts[i] = ex + carry;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_compact_write(const u8 *__restrict__ f, u32 W, const u32 *__restrict__ tile_offsets,
                                u32 *__restrict__ out) {
    const u32 base = blockIdx.x * kCompactTile + threadIdx.x * kCompactPerThread;
    uint4 q = *reinterpret_cast<const uint4 *>(f + base);
    const u8 *b = reinterpret_cast<const u8 *>(&q);
    u32 c = 0;
#pragma unroll
    for (u32 i = 0; i < kCompactPerThread; i++) c += (base + i < W && b[i] != 0);
    u32 off = tile_offsets[blockIdx.x] + block_excl_scan(c, nullptr);
#pragma unroll
    for (u32 i = 0; i < kCompactPerThread; i++)
        if (base + i < W && b[i] != 0) out[off++] = base + i;
}

// ---------------------------------------------------------------------------
// Pass setup.
// ---------------------------------------------------------------------------
__global__ void k_iota_windows(u32 *__restrict__ win, u8 *__restrict__ active, u32 W, Counters *cnt) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < W; i += gridDim.x * blockDim.x) {
        win[i] = i;
        active[i] = 1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt->n_win = W;
}

// active[j] = (flags[j] != 0) for the next pass.
// active = flags != 0; windows about to be recomputed also drop their
// lower bound (wlb, tensor-core path; may be NULL).
__global__ void k_mark_active(const u8 *__restrict__ flags, u8 *__restrict__ active, u32 W, WinBounds wb,
                              float *__restrict__ bm, u32 L, u32 n, u32 K) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < W; i += gridDim.x * blockDim.x) {
        active[i] = flags[i] != 0;
        if (!flags[i]) continue;
        if (wb.wlb) wb.wlb[i] = 0.0f;
        if (wb.wpos) wb.wpos[i] = 0;
        if (wb.umax)
            for (u32 t = 0; t < K; t++) wb.umax[(size_t)i * K + t] = 0.0f;
        if (bm)
            for (u32 s = i * L; s < min((i + 1) * L, n); s++) bm[s] = 0.0f;
    }
}

// ---------------------------------------------------------------------------
// Path (a): full likelihood, exact reference order on the FP32 pipes.
// compute_full_likelihood / compute_maximum_likelihood, binary_pursuit.cl:216-300.
//
// Work item = (listed window, group of 16 templates).  Block = 4 warps; warp
// q handles templates 4q..4q+3 of the group; lane l handles samples
// l + 32r (r < 4) of a 128-sample tile starting at the window.  The voltage
// strip of a channel chunk is staged in shared memory.  Each of the 16
// accumulators of a thread is an independent chain in (channel, lag) order,
// starting from float32(-0.5*SS) -- exactly the reference's sequence.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_max_float(float x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

constexpr int kLikThreads = 128;

// Per chunk: each template's non-zero channel range [lo, hi) (tsup), the
// template order sorted by (lo, id) (tperm), and per group of kLikTplPerBlock
// consecutive slots the union of their ranges (grange).  One block.
// Non-zero channel range of each template: one warp per template.
__global__ void k_template_ranges(const float *__restrict__ T, u32 K, u32 C, u32 L, u32 *__restrict__ tsup) {
    const u32 lane = threadIdx.x & 31;
    for (u32 t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < K; t += gridDim.x * (blockDim.x >> 5)) {
        u32 lo = C, hi = 0;
        for (u32 c = 0; c < C; c++) {
            const float *tp = T + ((size_t)t * C + c) * L;
            bool nz = false;
            for (u32 i = lane; i < L; i += 32) nz |= tp[i] != 0.0f;
            if (__any_sync(0xffffffffu, nz)) { lo = min(lo, c); hi = c + 1; }
        }
        if (hi == 0) lo = 0;                         // all-zero template: empty range
        if (lane == 0) {
            tsup[2 * t] = lo;
            tsup[2 * t + 1] = hi;
        }
    }
}

// The template order and group ranges from the supports (one block).
__global__ void k_template_support(const float *__restrict__ T, u32 K, u32 C, u32 L, u32 *__restrict__ tsup,
                                   u32 *__restrict__ tperm, u32 *__restrict__ grange, u32 group,
                                   u32 *__restrict__ grange2, u32 group2) {
    for (u32 t = threadIdx.x; t < K; t += blockDim.x) {
        const u32 lo = tsup[2 * t];
        u32 rank = 0;
        for (u32 o = 0; o < K; o++) {
            const u32 lo2 = tsup[2 * o];
            rank += (lo2 < lo || (lo2 == lo && o < t)) ? 1u : 0u;
        }
        tperm[rank] = t;
    }
    __syncthreads();
    for (int pass = 0; pass < 2; pass++) {
        const u32 gs = pass ? group2 : group;
        u32 *gr = pass ? grange2 : grange;
        if (!gr) continue;
        const u32 ng = (K + gs - 1) / gs;
        for (u32 g = threadIdx.x; g < ng; g += blockDim.x) {
            u32 lo = C, hi = 0;
            for (u32 j = g * gs; j < min(K, (g + 1) * gs); j++) {
                const u32 t = tperm[j];
                if (tsup[2 * t + 1] > tsup[2 * t]) {
                    lo = min(lo, tsup[2 * t]);
                    hi = max(hi, tsup[2 * t + 1]);
                }
            }
            if (hi == 0) lo = 0;
            gr[2 * g] = lo;
            gr[2 * g + 1] = hi;
        }
    }
}
constexpr int kLikQ = 4;             // templates per warp
constexpr int kLikR = 4;             // samples per lane
constexpr int kLikTile = 32 * kLikR; // 128 samples
constexpr int kLikTplPerBlock = (kLikThreads / 32) * kLikQ;   // 16
constexpr int kLikChanChunk = 8;

__global__ void __launch_bounds__(kLikThreads)
k_likelihood_fp32(const float *__restrict__ v, u32 n, u32 C, const float *__restrict__ T, u32 K, u32 L,
                  const float *__restrict__ tss, const u32 *__restrict__ win,
                  const u32 *__restrict__ n_win_dev, float *__restrict__ Lk, const u32 *__restrict__ gate,
                  u8 *__restrict__ apx, const u32 *__restrict__ tperm, const u32 *__restrict__ grange,
                  WinBounds wb) {
    extern __shared__ float strip[];   // kLikChanChunk x (kLikTile + L)
    if (gate && *gate == 0) return;    // only run when the gate asks for it
    const u32 n_win = *n_win_dev;
    const u32 kgroups = ceil_div(K, kLikTplPerBlock);
    const u32 stride = kLikTile + L;
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const u64 total = (u64)n_win * kgroups;
    for (u64 item = blockIdx.x; item < total; item += gridDim.x) {
        const u32 w = win[item / kgroups];
        const u32 kg = (u32)(item % kgroups);
        const u32 sw = w * L;
        const u32 ew = min((w + 1) * L, n);
        const u32 slot0 = kg * kLikTplPerBlock + warp * kLikQ;
        // templates of this warp (slot order sorted by support when masked)
        u32 tq[kLikQ];
#pragma unroll
        for (int q = 0; q < kLikQ; q++) {
            const u32 sl = min(slot0 + q, K - 1);
            tq[q] = tperm ? tperm[sl] : sl;
        }
        // channels where some template of the group is non-zero (the others
        // add exact zeros to the reference's sum)
        const u32 cbeg = grange ? grange[2 * kg] : 0u, cend = grange ? grange[2 * kg + 1] : C;
        for (u32 s0 = sw; s0 < ew; s0 += kLikTile) {
            float acc[kLikQ][kLikR];
#pragma unroll
            for (int q = 0; q < kLikQ; q++)
#pragma unroll
                for (int r = 0; r < kLikR; r++) acc[q][r] = (slot0 + q < K) ? tss[tq[q]] : 0.0f;
            for (u32 c0 = cbeg; c0 < cend; c0 += kLikChanChunk) {
                const u32 cc = min((u32)kLikChanChunk, cend - c0);
                __syncthreads();
                for (u32 e = threadIdx.x; e < cc * stride; e += blockDim.x) {
                    const u32 c = e / stride, x = e % stride;
                    const u32 g = s0 + x;
                    strip[c * stride + x] = g < n ? v[(size_t)(c0 + c) * n + g] : 0.0f;
                }
                __syncthreads();
                for (u32 c = 0; c < cc; c++) {
                    const float *sp = strip + c * stride + lane;
                    const float *tp[kLikQ];
#pragma unroll
                    for (int q = 0; q < kLikQ; q++) tp[q] = T + ((size_t)tq[q] * C + (c0 + c)) * L;
                    for (u32 i = 0; i < L; i++) {
                        float tv[kLikQ], vv[kLikR];
#pragma unroll
                        for (int q = 0; q < kLikQ; q++) tv[q] = __ldg(tp[q] + i);
#pragma unroll
                        for (int r = 0; r < kLikR; r++) vv[r] = sp[32 * r + i];
#pragma unroll
                        for (int q = 0; q < kLikQ; q++)
#pragma unroll
                            for (int r = 0; r < kLikR; r++)
                                acc[q][r] = __fadd_rn(acc[q][r], __fmul_rn(tv[q], vv[r]));
                    }
                }
            }
            if (wb.umax) {
                // window bounds: the values are exact (lower = upper bound)
                bool anypos = false;
#pragma unroll
                for (int q = 0; q < kLikQ; q++) {
                    float mq = 0.0f;
#pragma unroll
                    for (int r = 0; r < kLikR; r++) {
                        const u32 s = s0 + lane + 32 * r;
                        if (s < ew && s < s0 + kLikTile && s + L < n) mq = fmaxf(mq, acc[q][r]);
                    }
                    mq = warp_max_float(mq);
                    anypos |= mq > 0.0f;
                    if (lane == 0 && mq > 0.0f && slot0 + q < K) {
                        atomicMax(reinterpret_cast<int *>(wb.umax) + (size_t)w * K + tq[q], __float_as_int(mq));
                        atomicMax(reinterpret_cast<int *>(wb.wlb) + w, __float_as_int(mq));
                    }
                }
                if (lane == 0 && anypos) wb.wpos[w] = 1;
            }
#pragma unroll
            for (int q = 0; q < kLikQ; q++) {
                if (slot0 + q >= K) continue;
#pragma unroll
                for (int r = 0; r < kLikR; r++) {
                    const u32 s = s0 + lane + 32 * r;
                    if (s < ew && s < s0 + kLikTile) {
                        Lk[(size_t)tq[q] * n + s] = (s + L >= n) ? 0.0f : acc[q][r];
                        if (apx) apx[(size_t)tq[q] * n + s] = 0;
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Likelihood entries left approximate by the tensor-core path.  Certainly
// positive entries keep an approximate value and a flag; their interval is
// rebuilt from per-sample data (window norms and the tile's fp16 scale) and
// per-template data, and they are re-evaluated in the reference's order when
// a decision needs their value (exact values are written back).
// ---------------------------------------------------------------------------
// Likelihood entries the tensor-core path stored approximately.  apx[t][s]:
//   0     the stored value is the reference value, or an approximation that
//         is certainly <= 0 (only its sign is ever read);
//   1     approximate and certainly > 0; the interval is approx +- lazy_bound;
//   2, 3  was 1; the reference value was stored by a kernel of the pass with
//         that parity (tag = 2 + pass % 2).
// A kernel stores the value before the tag, so a reader in the SAME kernel
// that sees its own pass's tag may still read the old approximation: it
// treats the entry like a 1 (the interval holds both values).  A tag of the
// other parity was written by an earlier launch and is exact.
struct LazyLk {
    u8 *apx;                          // [K][n]; NULL: every entry is exact
    const float *wn, *wa;             // [n] window L2 / L1 norms at computation time
    const signed char *kx;            // [n] fp16 scale exponent of the tile
    const float *tnorm, *tabs, *tss;  // [K]
    const int *texp;                  // [K]
    const float *v, *T;               // voltage (residual) and templates
    u32 C, L;
    float kappa_b;                    // bound per unit of ||t|| ||window||
    float kappa_s;                    // bound per unit of |SS_t / 2| (the reference's running sum starts there)
    u64 *refined;                     // count of entries refined on demand (may be NULL)
    const float *wlb;                 // [W] largest lower bound over each window's entries
    const float *bm;                  // [n] largest bound of a flagged entry of each sample
    u32 tag;                          // 2 + pass % 2
    const u32 *tgrp;                  // [K] template group; wn/wa/kx are [group][n] (NULL: one group)
    u64 gstride;                      // n
    const u32 *tsup;                  // [K][2] non-zero channel range (NULL: all channels)
};

// The bound the tensor-core epilogue used for entry (t, s) (same formula).
__device__ __forceinline__ float lazy_bound(const LazyLk &z, u32 t, u32 s, float approx) {
    const size_t i = (z.tgrp ? (size_t)z.tgrp[t] * z.gstride : 0) + s;
    const float sub = 2.98023223876953125e-08f * (ldexpf(z.tabs[t], -(int)z.kx[i]) + ldexpf(z.wa[i], -z.texp[t])) * 1.001f;
    return z.kappa_b * z.tnorm[t] * z.wn[i] + sub + z.kappa_s * fabsf(z.tss[t]) +
           2.384185791015625e-07f * fabsf(approx);
}

// compute_maximum_likelihood (binary_pursuit.cl:216-252), reference order.
__device__ __forceinline__ float exact_likelihood(const LazyLk &z, u32 n, u32 t, u32 s) {
    float acc = z.tss[t];
    // channels outside the template's support add exact zeros
    const u32 clo = z.tsup ? z.tsup[2 * t] : 0u, chi = z.tsup ? z.tsup[2 * t + 1] : z.C;
    for (u32 c = clo; c < chi; c++) {
        const float *tp = z.T + ((size_t)t * z.C + c) * z.L;
        const float *vp = z.v + (size_t)c * n + s;
        for (u32 i = 0; i < z.L; i++) acc = __fadd_rn(acc, __fmul_rn(__ldg(tp + i), vp[i]));
    }
    return acc;
}

// The reference value of likelihood[t][pos] for a decision; not written back.
__device__ __forceinline__ float lk_exact(const LazyLk &z, const float *Lk, u32 n, u32 t, u32 pos) {
    const size_t e = (size_t)t * n + pos;
    if (z.apx && z.apx[e] == 1) return exact_likelihood(z, n, t, pos);
    return Lk[e];
}

// Warp-cooperative reference-order sums.  The products of a sum are
// independent, so the lanes form them (each rounded as in the reference)
// into a per-warp buffer; lane 0 then adds them in the reference's order --
// float addition is not associative, so the chain itself stays sequential,
// but its loads no longer wait on global memory one by one.
constexpr u32 kWarpChunk = 256;

__device__ __forceinline__ float warp_chain(float acc, const float *buf, u32 m) {
    u32 k = 0;
    for (; k + 8 <= m; k += 8) {
#pragma unroll
        for (int j = 0; j < 8; j++) acc = __fadd_rn(acc, buf[k + j]);
    }
    for (; k < m; k++) acc = __fadd_rn(acc, buf[k]);
    return acc;
}

// exact_likelihood(z, n, t, s) computed by the whole warp; every lane gets it.
// Each lane forms up to eight products of a chunk with its loads in flight
// together.
__device__ float warp_exact_likelihood(const LazyLk &z, u32 n, u32 t, u32 s, float *buf) {
    static_assert(kWarpChunk == 256, "eight products per lane");
    const u32 lane = threadIdx.x & 31;
    // the template's support: channels outside it add exact zeros
    const u32 clo = z.tsup ? z.tsup[2 * t] : 0u, chi = z.tsup ? z.tsup[2 * t + 1] : z.C;
    const u32 CL = (chi > clo ? chi - clo : 0u) * z.L;
    const float *tp = z.T + ((size_t)t * z.C + clo) * z.L;
    const float *vb = z.v + (size_t)clo * n;
    float acc = z.tss[t];
    for (u32 q0 = 0; q0 < CL; q0 += kWarpChunk) {
        const u32 m = min(kWarpChunk, CL - q0);
        float tv[8], vv[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const u32 k = lane + 32u * i;
            tv[i] = vv[i] = 0.0f;
            if (k < m) {
                const u32 q = q0 + k, c = q / z.L, j = q - c * z.L;
                tv[i] = __ldg(tp + q);
                vv[i] = vb[(size_t)c * n + s + j];
            }
        }
#pragma unroll
        for (int i = 0; i < 8; i++)
            if (lane + 32u * i < m) buf[lane + 32u * i] = __fmul_rn(tv[i], vv[i]);
        __syncwarp();
        if (lane == 0) acc = warp_chain(acc, buf, m);
        __syncwarp();
    }
    return __shfl_sync(0xffffffffu, acc, 0);
}

// lk_exact for a whole warp (all lanes pass the same entry).
__device__ __forceinline__ float warp_lk_exact(const LazyLk &z, const float *Lk, u32 n, u32 t, u32 pos, float *buf) {
    const size_t e = (size_t)t * n + pos;
    if (z.apx && z.apx[e] == 1) return warp_exact_likelihood(z, n, t, pos, buf);
    return Lk[e];
}

// Before the residual subtracts this pass's spikes: an approximate entry
// that reads a changing sample and whose window is not recomputed next pass
// keeps, in the reference, the value it was computed with; store that value
// now, from the voltage it was computed from.
__global__ void __launch_bounds__(256)
k_lazy_freeze(u32 n, u32 L, u32 K, const u32 *__restrict__ idx, const u32 *__restrict__ lab,
              const u32 *__restrict__ m_dev, const u8 *__restrict__ next_active, u32 W, float *__restrict__ Lk,
              LazyLk z) {
    const u32 m = *m_dev;
    __shared__ float fbuf[8][kWarpChunk];
    const u32 lane = threadIdx.x & 31;
    const u32 warps_per_block = blockDim.x >> 5;
    float *wbuf = fbuf[threadIdx.x >> 5];
    for (u32 g = blockIdx.x * warps_per_block + (threadIdx.x >> 5); g < m;
         g += gridDim.x * warps_per_block) {
        if (lab[g] >= K) continue;
        const u32 p = idx[g];
        const u32 lo = p + 1 > L ? p + 1 - L : 0;
        const u32 hi = min(n, p + L);
        u32 nref = 0;
        for (u32 s0 = lo; s0 < hi; s0 += 32) {
            const u32 s = s0 + lane;
            const u32 wd = s / L;
            const bool cand = s < hi && !(wd < W && next_active[wd]);   // not recomputed next pass
            for (u32 t = 0; t < K; t++) {
                const size_t e = (size_t)t * n + s;
                u32 nm = __ballot_sync(0xffffffffu, cand && z.apx[e] == 1);
                while (nm) {
                    const u32 src = __ffs(nm) - 1;
                    nm &= nm - 1;
                    const float x = warp_exact_likelihood(z, n, t, __shfl_sync(0xffffffffu, s, src), wbuf);
                    if (lane == src) {
                        Lk[e] = x;
                        __threadfence();
                        z.apx[e] = (u8)z.tag;
                        nref++;
                    }
                }
            }
        }
        if (z.refined && nref) atomicAdd(z.refined, (u64)nref);
    }
}

// ---------------------------------------------------------------------------
// Path (b): per-window argmax over all templates.
// compute_template_maximum_likelihood, binary_pursuit.cl:350-441, with the K
// per-template launches fused: one warp per listed window walks templates in
// order; within a template the warp finds the first sample holding the
// template's maximum, and the running best is replaced only on a strictly
// larger value -- the sequential scan's result.
// ---------------------------------------------------------------------------
constexpr int kArgmaxThreads = 256;
__global__ void __launch_bounds__(kArgmaxThreads)
k_window_argmax(u32 n, u32 L, u32 K, const u32 *__restrict__ win,
                                const u32 *__restrict__ n_win_dev, u32 *__restrict__ best_idx,
                                u32 *__restrict__ best_lab, float *__restrict__ best_ll,
                                u8 *__restrict__ flags, u8 *__restrict__ ovr,
                                u32 *__restrict__ ov_idx, u32 *__restrict__ ov_lab,
                                float *__restrict__ Lk, LazyLk z, WinBounds wb) {
    __shared__ float abuf[kArgmaxThreads / 32][kWarpChunk];
    const u32 n_win = *n_win_dev;
    const u32 lane = threadIdx.x & 31;
    const u32 warps_per_block = blockDim.x >> 5;
    float *wbuf = abuf[threadIdx.x >> 5];
    const u32 W = (n + L - 1) / L;
    for (u32 g = blockIdx.x * warps_per_block + (threadIdx.x >> 5); g < n_win;
         g += gridDim.x * warps_per_block) {
        const u32 id = win[g];
        const u32 sw = id * L, ew = (id + 1) * L;
        const u32 start = (L > sw) ? 0 : sw - L;
        const u32 stop = (ew + L) > n ? n : ew + L;
        if (ew >= n - L) continue;                       // .cl:380-383
        // Approximate entries (tensor-core path): lb = the largest lower
        // bound over windows id-1..id+1, which is the range [start, stop).
        // The maximum is >= lb, and an entry whose upper bound is below lb
        // cannot hold it, so only entries that reach lb need their
        // reference value; every other one is read as stored (< lb).
        float lb = 0.0f;
        if (wb.wlb) {
            lb = wb.wlb[id];
            if (id > 0) lb = fmaxf(lb, wb.wlb[id - 1]);
            if (id + 1 < W) lb = fmaxf(lb, wb.wlb[id + 1]);
        }
        // With window bounds only templates whose upper bound over windows
        // id-1..id+1 reaches lb (and 0) can hold the maximum or tie it: the
        // others are skipped, the rest scanned in template order.
        const bool bounded = wb.umax != nullptr;
        u32 nref = 0;
        float bl = 0.0f;                                 // .cl:389-393 (template 0 resets)
        u32 blab = best_lab[id], bidx = best_idx[id];
        bool check = bounded && wb.wpos[id] != 0;
        for (u32 t0 = 0; t0 < K; t0 += 32) {
          bool cand = t0 + lane < K;
          if (bounded && cand) {
              const u32 tt = t0 + lane;
              float u = wb.umax[(size_t)id * K + tt];
              if (id > 0) u = fmaxf(u, wb.umax[(size_t)(id - 1) * K + tt]);
              if (id + 1 < W) u = fmaxf(u, wb.umax[(size_t)(id + 1) * K + tt]);
              cand = u > 0.0f && u >= lb;
          }
          u32 tmask = __ballot_sync(0xffffffffu, cand);
          while (tmask) {
            const u32 t = t0 + __ffs(tmask) - 1;
            tmask &= tmask - 1;
            float *row = Lk + (size_t)t * n;
            float lv = -INFINITY;
            u32 li = 0xffffffffu;
            for (u32 s0 = start; s0 < stop; s0 += 32) {
                const u32 s = s0 + lane;
                const bool in = s < stop;
                float cur = in ? row[s] : -INFINITY;
                check |= in && cur > 0.0f && s >= sw && s < ew;   // a flagged entry is > 0 either way
                bool need = false;
                if (z.apx && in && cur + z.bm[s] >= lb) {
                    const u32 f = z.apx[(size_t)t * n + s];
                    need = (f == 1 || f == z.tag) && cur + lazy_bound(z, t, s, cur) >= lb;
                }
                u32 nm = __ballot_sync(0xffffffffu, need);
                while (nm) {                             // the warp refines them one by one
                    const u32 src = __ffs(nm) - 1;
                    nm &= nm - 1;
                    const float x = warp_exact_likelihood(z, n, t, __shfl_sync(0xffffffffu, s, src), wbuf);
                    if (lane == src) {
                        cur = x;
                        row[s] = x;
                        __threadfence();
                        z.apx[(size_t)t * n + s] = (u8)z.tag;
                        nref++;
                    }
                }
                if (in && cur > lv) { lv = cur; li = s; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const float ov = __shfl_xor_sync(0xffffffffu, lv, o);
                const u32 oi = __shfl_xor_sync(0xffffffffu, li, o);
                if (ov > lv || (ov == lv && oi < li)) { lv = ov; li = oi; }
            }
            if (lv > bl) { bl = lv; blab = t; bidx = li; }
          }
        }
        check = __any_sync(0xffffffffu, check);
        if (z.refined) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) nref += __shfl_xor_sync(0xffffffffu, nref, o);
            if (lane == 0 && nref) atomicAdd(z.refined, (u64)nref);
        }
        if (lane == 0) {
            if (check) flags[id] = 1;                    // .cl:419-422
            ovr[id] = (bl > 0.0f && bidx >= sw && bidx < ew) ? 1 : 0;   // .cl:423-433
            best_ll[id] = bl; best_lab[id] = blab; best_idx[id] = bidx;
            ov_idx[id] = bidx; ov_lab[id] = blab;        // .cl:435-439
        }
    }
}

// ---------------------------------------------------------------------------
// Overlap recheck, exact: overlap_recheck_indices + parse_overlap_recheck_indices
// (binary_pursuit.cl:444-815).  One block per candidate window; every
// (a, b, t) item is evaluated in the reference's order of operations; the
// block keeps the first item (lowest id) with the largest likelihood above
// the window's current best, which is what the parse kernel's strict-greater
// scan over single-item groups returns.
// ---------------------------------------------------------------------------
// Channels outside both templates' non-zero ranges [lo1, hi1), [lo2, hi2)
// add only exact zeros to the reference's sums (ss stays 0, so the -0.5 ss
// step is skipped there too) and are left out; the others keep the
// reference's channel order.
__device__ __forceinline__ float overlap_pair_exact(const float *__restrict__ vwin,   // [C][L] at bidx
                                                    const float *__restrict__ tk0,    // [C][L]
                                                    const float *__restrict__ tt,     // [C][L]
                                                    u32 C, u32 L, int fa, int sa, u32 lo1 = 0, u32 hi1 = ~0u,
                                                    u32 lo2 = 0, u32 hi2 = ~0u) {
    float cml = 0.0f;
    const u32 ffj = fa < 0 ? (u32)(-fa) : 0u;
    const u32 sfj = sa < 0 ? (u32)(-sa) : 0u;
    const u32 cend = min(C, max(hi1, hi2));
    for (u32 c = min(lo1, lo2); c < cend; c++) {
        if ((c < lo1 || c >= hi1) && (c < lo2 || c >= hi2)) continue;
        const float *f = tk0 + (size_t)c * L;
        const float *s = tt + (size_t)c * L;
        const float *vv = vwin + (size_t)c * L;
        float ss = 0.0f;
        for (u32 j = 0; j < L; j++) {
            float fv = 0.0f, sv = 0.0f;
            if (j >= ffj && (u32)(fa + (int)j) < L) fv = f[fa + (int)j];
            if (j >= sfj && (u32)(sa + (int)j) < L) sv = __ldg(s + sa + (int)j);
            const float sum = __fadd_rn(fv, sv);
            ss = __fadd_rn(ss, __fmul_rn(sum, sum));
            cml = __fadd_rn(cml, __fmul_rn(sum, vv[j]));
        }
        if ((double)ss > 0.0)                                          // .cl:627-630
            cml = __double2float_rn(__dsub_rn((double)cml, __dmul_rn(0.5, (double)ss)));
    }
    return cml;
}

// parse_overlap_recheck_indices' decision, binary_pursuit.cl:707-814, given
// the winning item and the reference values lf = L[lab][afix], ls = L[t][ashift].
__device__ __forceinline__ void overlap_parse_tail(u32 id, float best_group, u32 lab, u32 t, u32 afix, u32 ashift,
                                                   float lf, float ls, u32 *best_idx, u32 *best_lab,
                                                   float *best_ll, u32 *ov_idx, u32 *ov_lab, u8 *ovr,
                                                   const float *thr) {
    if (best_group < lf || best_group < ls) { ovr[id] = 0; return; }
    if (lf <= 0.0f || ls <= 0.0f) { ovr[id] = 0; return; }
    if (lf >= ls && lf > thr[lab]) {
        best_ll[id] = lf; ov_lab[id] = lab; ov_idx[id] = afix;
    } else if (ls > lf && ls > thr[t]) {
        best_ll[id] = ls; ov_lab[id] = t; ov_idx[id] = ashift;
    } else if (lf > thr[lab]) {
        best_ll[id] = lf; ov_lab[id] = lab; ov_idx[id] = afix;
    } else {
        ov_idx[id] = best_idx[id]; ov_lab[id] = best_lab[id]; ovr[id] = 0;
    }
}

// The same decision (best_group > best_ll[id] already established or not).
__device__ __forceinline__ void overlap_parse(u32 id, u32 n, u32 K, u32 S, u32 nmax, float best_group,
                                              u64 best_item, u32 *best_idx, u32 *best_lab,
                                              float *best_ll, u32 *ov_idx, u32 *ov_lab, u8 *ovr,
                                              const float *Lk, const float *thr, const LazyLk &z) {
    if (best_group <= best_ll[id] || best_group <= 0.0f) { ovr[id] = 0; return; }
    const u32 lab = best_lab[id], bidx = best_idx[id];
    const u32 t = (u32)(best_item % K);
    const u32 a = (u32)((best_item / K) % S);
    const u32 b = (u32)((best_item / ((u64)S * K)) % S);
    const u32 afix = bidx + a - nmax, ashift = bidx + b - nmax;
    const float lf = lk_exact(z, Lk, n, lab, afix);
    const float ls = lk_exact(z, Lk, n, t, ashift);
    overlap_parse_tail(id, best_group, lab, t, afix, ashift, lf, ls, best_idx, best_lab, best_ll, ov_idx, ov_lab,
                       ovr, thr);
}

constexpr int kOvThreads = 256;

__global__ void __launch_bounds__(kOvThreads)
k_overlap_exact(const float *__restrict__ v, u32 n, u32 C, const float *__restrict__ T, u32 K, u32 L,
                const u32 *__restrict__ cand, const u32 *__restrict__ n_cand_dev,
                u32 *__restrict__ best_idx, u32 *__restrict__ best_lab, float *__restrict__ best_ll,
                u32 *__restrict__ ov_idx, u32 *__restrict__ ov_lab, u8 *__restrict__ ovr,
                const float *__restrict__ Lk, u32 nmax, const float *__restrict__ thr,
                u64 *__restrict__ items_evaluated, LazyLk z, const u32 *__restrict__ tsup) {
    extern __shared__ float sm[];          // vwin [C*L], tk0 [C*L]
    __shared__ float red_v[kOvThreads / 32];
    __shared__ u64 red_i[kOvThreads / 32];
    const u32 n_cand = *n_cand_dev;
    const u32 S = 2 * nmax + 1;
    const u64 items = (u64)S * S * K;
    float *vwin = sm, *tk0 = sm + (size_t)C * L;
    for (u32 g = blockIdx.x; g < n_cand; g += gridDim.x) {
        const u32 id = cand[g];
        const u32 lab = best_lab[id], bidx = best_idx[id];
        const u32 lo_lab = tsup && lab < K ? tsup[2 * lab] : 0u, hi_lab = tsup && lab < K ? tsup[2 * lab + 1] : C;
        const float start_ll = best_ll[id];
        const float bll = Lk[(size_t)lab * n + bidx];
        const bool skip_all = (bll < thr[lab]) || (bidx >= n - L);   // .cl:518-527
        float bv = start_ll;
        u64 bi = ~0ull;
        u32 evaluated = 0;
        __syncthreads();
        if (!skip_all) {
            for (u32 e = threadIdx.x; e < C * L; e += blockDim.x) {
                const u32 c = e / L, j = e % L;
                vwin[e] = v[(size_t)c * n + bidx + j];
                tk0[e] = T[(size_t)lab * C * L + e];
            }
        }
        __syncthreads();
        if (!skip_all) {
            for (u64 it = threadIdx.x; it < items; it += blockDim.x) {
                const u32 t = (u32)(it % K);
                const u32 a = (u32)((it / K) % S);
                const u32 b = (u32)((it / ((u64)S * K)) % S);
                if (a + bidx < nmax || a + bidx >= n - L + nmax) continue;   // .cl:534-537
                if (b + bidx < nmax || b + bidx >= n - L + nmax) continue;   // .cl:538-541
                if (a > b && a - b > L) continue;                             // .cl:543-549
                if (b > a && b - a > L) continue;                             // .cl:550-556
                const u32 afix = bidx + a - nmax, ashift = bidx + b - nmax;
                const float lf = Lk[(size_t)lab * n + afix];
                const float ls = Lk[(size_t)t * n + ashift];
                if (lf <= 0.0f && ls <= 0.0f) continue;                       // .cl:572-576
                const float ll = overlap_pair_exact(vwin, tk0, T + (size_t)t * C * L, C, L,
                                                    (int)bidx - (int)afix, (int)bidx - (int)ashift, lo_lab, hi_lab,
                                                    tsup ? tsup[2 * t] : 0u, tsup ? tsup[2 * t + 1] : C);
                evaluated++;
                if (ll > bv) { bv = ll; bi = it; }
            }
        }
        if (items_evaluated) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) evaluated += __shfl_xor_sync(0xffffffffu, evaluated, o);
            if ((threadIdx.x & 31) == 0 && evaluated) atomicAdd(items_evaluated, (u64)evaluated);
        }
        // block argmax: larger value, then lower item id
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const u64 oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
        }
        if ((threadIdx.x & 31) == 0) { red_v[threadIdx.x >> 5] = bv; red_i[threadIdx.x >> 5] = bi; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (u32 w = 1; w < blockDim.x / 32; w++)
                if (red_v[w] > bv || (red_v[w] == bv && red_i[w] < bi)) { bv = red_v[w]; bi = red_i[w]; }
            overlap_parse(id, n, K, S, nmax, bv, bi == ~0ull ? 0 : bi, best_idx, best_lab, best_ll,
                          ov_idx, ov_lab, ovr, Lk, thr, z);
        }
    }
}

// ---------------------------------------------------------------------------
// check_overlap_reassignments, binary_pursuit.cl:822-875.  Window id reads
// overlap_recheck[id-2] after candidate id-2 has been processed; that value
// is reconstructed by walking the stride-2 chain of candidates that moved
// left.  The final overlap_recheck values go to ovr_out.
// ---------------------------------------------------------------------------
__device__ __forceinline__ u8 ovr_final(u32 k, u32 L, const u8 *ovr_in, const u32 *ov_idx) {
    u32 m = 0;
    while (ovr_in[k] == 1 && ov_idx[k] < k * L && k > 1) { k -= 2; m++; }
    const u8 base = ovr_in[k] == 1 ? 1 : 0;
    return (m & 1) ? (u8)(1 - base) : base;
}

__global__ void k_check_overlap(u32 n, u32 L, const u32 *__restrict__ cand, const u32 *__restrict__ n_cand_dev,
                                u32 *__restrict__ best_idx, u32 *__restrict__ best_lab,
                                u8 *__restrict__ flags, const u32 *__restrict__ ov_idx,
                                const u32 *__restrict__ ov_lab, const u8 *__restrict__ ovr,
                                u8 *__restrict__ ovr_out) {
    const u32 n_cand = *n_cand_dev;
    for (u32 g = blockIdx.x * blockDim.x + threadIdx.x; g < n_cand; g += gridDim.x * blockDim.x) {
        const u32 id = cand[g];
        const u32 sw = id * L, ew = (id + 1) * L;
        if (ovr[id] == 0) { ovr_out[id] = 0; continue; }
        best_idx[id] = ov_idx[id];
        best_lab[id] = ov_lab[id];
        u8 fin = 1;
        if (ov_idx[id] < sw && id > 1) {
            if (ovr_final(id - 2, L, ovr, ov_idx) == 1) {
                fin = 0;
                best_idx[id] = 0;
                flags[id - 1] = 2; flags[id] = 2; flags[id + 1] = 2;
            } else {
                flags[id - 2] = 2;
            }
        }
        if (ov_idx[id] >= ew && id + 2 < n / L) flags[id + 2] = 2;
        ovr_out[id] = fin;
    }
}

__global__ void k_copy_ovr(const u32 *__restrict__ cand, const u32 *__restrict__ n_cand_dev,
                           const u8 *__restrict__ src, u8 *__restrict__ dst) {
    const u32 n_cand = *n_cand_dev;
    for (u32 g = blockIdx.x * blockDim.x + threadIdx.x; g < n_cand; g += gridDim.x * blockDim.x)
        dst[cand[g]] = src[cand[g]];
}

// ---------------------------------------------------------------------------
// binary_pursuit kernel, binary_pursuit.cl:918-1063.
// k_accept_has: phase one (the accept decision) for every listed window.
// k_accept_flags: the flags after the kernel, for every window, reproducing
// the sequential reads of the neighbours' flags in phase two.
// ---------------------------------------------------------------------------
__global__ void k_accept_has(u32 n, u32 C, u32 L, const float *__restrict__ thr,
                             const u32 *__restrict__ win, const u32 *__restrict__ n_win_dev,
                             const u32 *__restrict__ best_idx, const u32 *__restrict__ best_lab,
                             const float *__restrict__ best_ll, const u8 *__restrict__ ovr,
                             u8 *__restrict__ has) {
    const u32 n_win = *n_win_dev;
    for (u32 g = blockIdx.x * blockDim.x + threadIdx.x; g < n_win; g += gridDim.x * blockDim.x) {
        const u32 id = win[g];
        const u32 sw = id * L, ew = (id + 1) * L;
        u32 lab = 0, idx = 0;
        float ml = 0.0f;
        if (ew < n - L && C > 0) { ml = best_ll[id]; lab = best_lab[id]; idx = best_idx[id]; }
        const bool o = ovr[id] == 1;
        has[id] = ((ml > thr[lab]) || o) && ((idx >= sw && idx < ew) || o);   // .cl:982-999
    }
}

struct AcceptView {
    u32 n, C, L, W, nfloor;
    const float *thr;
    const u32 *best_idx, *best_lab;
    const float *best_ll;
    const u8 *active, *has, *F0;
};

__device__ __forceinline__ bool acc_valid(const AcceptView &a, u32 k) {
    return ((k + 1) * a.L < a.n - a.L) && a.C > 0;
}
// flags[k] at the start of window k's phase two: window k-1's phase one may
// have set it to 3 (.cl:994-997); window k+1 has not run yet.
__device__ __forceinline__ u8 acc_f0(const AcceptView &a, u32 k) {
    return (k >= 1 && a.active[k - 1] && a.has[k - 1] && k < a.nfloor) ? (u8)3 : a.F0[k];
}
__device__ __forceinline__ bool acc_step3(const AcceptView &a, u32 k) {
    return a.best_ll[k] <= a.thr[a.best_lab[k]];
}
// Window k's left-prune (.cl:1024-1031) reads the final flag of window k-1.
__device__ __forceinline__ bool acc_left_dependent(const AcceptView &a, u32 k) {
    return k > 0 && a.active[k] && !a.has[k] && acc_valid(a, k) && acc_f0(a, k) == 1 &&
           a.best_idx[k] < k * a.L;
}
// flags[k] after windows 0..k ran, for a window that is not left-dependent.
__device__ __forceinline__ u8 acc_direct(const AcceptView &a, u32 k) {
    u8 f = acc_f0(a, k);
    if (!a.active[k]) return f;
    if (a.has[k]) return 3;
    if (!acc_valid(a, k)) return f;
    if (f == 1 && a.best_idx[k] >= (k + 1) * a.L && k + 1 < a.nfloor)     // .cl:1032-1039
        if (a.F0[k + 1] == 0) f = 0;
    if (acc_step3(a, k) && f < 3) f = 0;                                   // .cl:1040-1044
    return f;
}

__global__ void k_accept_flags(AcceptView a, u8 *__restrict__ flags_out) {
    for (u32 j = blockIdx.x * blockDim.x + threadIdx.x; j < a.W; j += gridDim.x * blockDim.x) {
        u8 P;
        if (!acc_left_dependent(a, j)) {
            P = acc_direct(a, j);
        } else {
            u32 k = j;
            while (acc_left_dependent(a, k)) k--;
            bool z = acc_direct(a, k) == 0;
            for (u32 q = k + 1; q <= j; q++) z = z || acc_step3(a, q);
            P = z ? 0 : 1;
        }
        // window j+1's phase one sets flags[j] = 3 (.cl:990-993)
        if (j + 1 < a.W && a.active[j + 1] && a.has[j + 1]) P = 3;
        flags_out[j] = P;
    }
}

// Spike payload of an accepting window (.cl:971-976, 1057-1061).
__global__ void k_gather_spikes(u32 n, u32 C, u32 L, const u32 *__restrict__ list,
                                const u32 *__restrict__ n_list_dev, const u32 *__restrict__ best_idx,
                                const u32 *__restrict__ best_lab, u32 *__restrict__ out_idx,
                                u32 *__restrict__ out_lab, u32 *__restrict__ out_win) {
    const u32 m = *n_list_dev;
    for (u32 g = blockIdx.x * blockDim.x + threadIdx.x; g < m; g += gridDim.x * blockDim.x) {
        const u32 id = list[g];
        const bool valid = ((id + 1) * L < n - L) && C > 0;
        out_idx[g] = valid ? best_idx[id] : 0;
        out_lab[g] = valid ? best_lab[id] : 0;
        if (out_win) out_win[g] = id;
    }
}

// Append this pass's spikes to the chunk output (device-side offset).
__global__ void k_append_spikes(const u32 *__restrict__ idx, const u32 *__restrict__ lab, Counters *cnt,
                                u32 *__restrict__ out_idx, u32 *__restrict__ out_lab, u32 cap) {
    const u32 m = cnt->n_spk, base = cnt->total;
    if (base + m > cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) cnt->overflow = 1;
        return;
    }
    for (u32 g = blockIdx.x * blockDim.x + threadIdx.x; g < m; g += gridDim.x * blockDim.x) {
        out_idx[base + g] = idx[g];
        out_lab[base + g] = lab[g];
    }
}

__global__ void k_commit_total(Counters *cnt, u32 cap) {
    if (cnt->total + cnt->n_spk <= cap) cnt->total += cnt->n_spk;
}

// ---------------------------------------------------------------------------
// Path (c): residual subtract, compute_residual (binary_pursuit.cl:57-102).
// Spikes of one pass can overlap (an overlap-recheck spike may move up to
// n_max_shift samples).  Each sample is written by the last listed spike
// covering it, which applies every covering spike's subtraction in list
// order -- the sequential reference's result, with no atomics.
// ---------------------------------------------------------------------------
// With template supports (tsup, may be NULL), a spike only touches its
// template's channels: elsewhere it subtracts zeros, which change nothing.
// Sample (c, x) is then written by the last covering spike whose support
// holds c, applying every such spike in list order.
__device__ __forceinline__ bool res_touches(const u32 *tsup, u32 lab, u32 c) {
    return !tsup || (c >= tsup[2 * lab] && c < tsup[2 * lab + 1]);
}
// One block per spike: its list neighbours j in [s - R, s + R] (position,
// label, channel range; an empty range for labels >= K) are staged in shared
// memory once, then warps take the spike's channels and lanes its L samples
// (no division per element, coalesced along samples).
constexpr u32 kResNb = 128;
__global__ void __launch_bounds__(256)
k_residual(float *__restrict__ v, u32 n, u32 C, const float *__restrict__ T, u32 K, u32 L,
           const u32 *__restrict__ idx, const u32 *__restrict__ lab, const u32 *__restrict__ n_spk_dev,
           u32 n_spk_host, u32 R, const u32 *__restrict__ tsup, float *__restrict__ vwmax = nullptr) {
    __shared__ u32 nb_p[kResNb], nb_lab[kResNb], nb_lo[kResNb], nb_hi[kResNb];
    const u32 m = n_spk_dev ? *n_spk_dev : n_spk_host;
    const u32 warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (u32 s = blockIdx.x; s < m; s += gridDim.x) {
        const u32 ls = lab[s];
        if (ls >= K) continue;                                           // .cl:78-81 (uniform in the block)
        const u32 jlo = s > R ? s - R : 0;
        const u32 jhi = min(m - 1, s + R);
        const u32 cnt = jhi - jlo + 1, self = s - jlo;
        const bool staged = cnt <= kResNb;
        __syncthreads();                                                 // the previous spike's readers are done
        if (staged) {
            for (u32 q = threadIdx.x; q < cnt; q += blockDim.x) {
                const u32 lj = lab[jlo + q];
                nb_p[q] = idx[jlo + q];
                nb_lab[q] = lj;
                nb_lo[q] = lj < K ? (tsup ? tsup[2 * lj] : 0u) : 1u;
                nb_hi[q] = lj < K ? (tsup ? tsup[2 * lj + 1] : C) : 0u;
            }
        }
        __syncthreads();
        // neighbour q covers (c, x) when its label is < K, c is in its
        // template's support and x lies in its clip
        auto covers = [&](u32 q, u32 c, u32 x) -> bool {
            u32 pq, lo, hi;
            if (staged) {
                pq = nb_p[q]; lo = nb_lo[q]; hi = nb_hi[q];
            } else {
                const u32 lj = lab[jlo + q];
                pq = idx[jlo + q];
                lo = lj < K ? (tsup ? tsup[2 * lj] : 0u) : 1u;
                hi = lj < K ? (tsup ? tsup[2 * lj + 1] : C) : 0u;
            }
            return c >= lo && c < hi && pq <= x && x < pq + L;
        };
        const u32 p = idx[s];
        const u32 clo = tsup ? tsup[2 * ls] : 0u, chi = tsup ? tsup[2 * ls + 1] : C;
        float mx = 0.0f;                                                 // largest |value| written
        for (u32 c = clo + warp; c < chi; c += nw) {
            for (u32 i = lane; i < L; i += 32) {
                const u32 x = p + i;
                if (x >= n) break;                                       // .cl:93-96
                bool owner = true;
                for (u32 q = self + 1; q < cnt && owner; q++) owner = !covers(q, c, x);
                if (!owner) continue;
                float val = v[(size_t)c * n + x];
                for (u32 q = 0; q <= self; q++) {
                    if (covers(q, c, x)) {
                        const u32 lq = staged ? nb_lab[q] : lab[jlo + q];
                        const u32 pq = staged ? nb_p[q] : idx[jlo + q];
                        val = __fsub_rn(val, T[((size_t)lq * C + c) * L + (x - pq)]);
                    }
                }
                v[(size_t)c * n + x] = val;
                mx = fmaxf(mx, fabsf(val));
            }
        }
        // the per-window bound on |v| of the wide tensor-core tiles stays an
        // upper bound (the clip covers windows p / L and (p + L - 1) / L)
        if (vwmax) {
            mx = warp_max_float(mx);
            if (lane == 0 && mx > 0.0f) {
                atomicMax(reinterpret_cast<int *>(vwmax) + p / L, __float_as_int(mx));
                atomicMax(reinterpret_cast<int *>(vwmax) + (p + L - 1) / L, __float_as_int(mx));
            }
        }
    }
}

// get_adjusted_clips, binary_pursuit.cl:1088-1130.
__global__ void k_adjusted_clips(const float *__restrict__ v, u32 n, u32 C, const float *__restrict__ T,
                                 u32 K, u32 L, const u32 *__restrict__ idx, const u32 *__restrict__ lab,
                                 u32 m, float *__restrict__ clips) {
    for (u32 s = blockIdx.x; s < m; s += gridDim.x) {
        const u32 p = idx[s], k = lab[s];
        if (k >= K) continue;
        for (u32 e = threadIdx.x; e < C * L; e += blockDim.x) {
            const u32 c = e / L, i = e % L;
            if (p + i >= n) continue;
            clips[(size_t)s * C * L + e] = __fadd_rn(v[(size_t)c * n + p + i], T[(size_t)k * C * L + e]);
        }
    }
}

}  // namespace fbp
