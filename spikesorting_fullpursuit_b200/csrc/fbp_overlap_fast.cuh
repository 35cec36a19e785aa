// Fast overlap recheck with exact refinement (sm_100a).
//
// The reference's overlap_recheck_indices (binary_pursuit.cl:444-654)
// evaluates, for each candidate window and every (a, b, t) item, the
// likelihood of the clipped sum of the best template k0 shifted by
// da = a - n_max and template t shifted by db = b - n_max, over the window
// [i0, i0+L), with C*L multiply-adds per item.  In exact arithmetic that
// value splits into
//
//     LL(t,a,b) = G(a) + H(t,b) - X(k0,t,a,b)
//     H(t,b)    = <t_t shifted by db, window>  - 0.5 * ||t_t clipped||^2   (G(a) = H(k0,a))
//     X         = <t_k0 shifted by da, t_t shifted by db>, both clipped to the window
//
// H is a small per-candidate correlation; X depends only on the templates
// and is read from prefix sums Q[k0][t][r][m] of the channel-summed product
// t_k0[m] * t_t[m+r] (r = da - db):  X = Q[hi] - Q[lo] with
// lo = max(0, -r, -da), hi = min(L, L-r, L-da).
//
// Each item gets an interval [lo, hi] guaranteed to contain the
// reference's IEEE-binary32 value: the reference's own rounding is bounded by
// gamma_n * (sum |s_j v_j| + sum s_j^2) with n the number of non-zero terms,
// and sum |s_j v_j| <= (||F_a|| + ||T_b||) * ||window||,
// sum s_j^2 <= ||F_a||^2 + ||T_b||^2 + 2|X|; kappa below covers twice that
// (the reference's error plus this approximation's).  Only items whose
// interval can reach the best one are re-evaluated exactly, in the
// reference's order; the parse kernel's strict-greater scan over single-item
// groups (.cl:699-706) then picks the same item as the reference.
#pragma once
#include "fbp_kernels.cuh"

namespace fbp {

// Contenders of all candidates of a pass share one pool of (slot, item)
// pairs; a candidate whose contenders do not fit goes to the exact kernel.
constexpr float kUnitRoundoff = 5.9604644775390625e-08f;   // 2^-24

// Constants of one chunk (computed on the device once per call).
struct OvConst {
    float kappa_ref;      // bound of the reference's rounding, per unit of sum|terms|
    float kappa_mine;     // bound of this approximation's rounding
    u32 cnz_max;          // max non-zero channels of a template
};

struct OvArgs {
    u32 n, C, K, L, nmax, S;
    const float *v, *T, *thr;
    float *Lk;
    const float *NT, *sNT, *tnorm;   // [K][S], [K][S], [K]
    const float *Q;                  // [K][K][2L-1][L+1]
    const float *XMr;                // [K][K][2L+1] upper bound of -X + kx|X| per lag r = a - b
    const float *XM;                 // [K][K]       its largest value over the lags
    const OvConst *oc;
    const u32 *cand, *n_cand;
    u32 *best_idx, *best_lab, *ov_idx, *ov_lab;
    float *best_ll;
    u8 *ovr;
    float *H;                        // [slot][K][S]
    float *vn;                       // [slot]
    u8 *cskip;                       // [slot]
    float *cand_lb;                  // [slot]     largest lower bound of an item (atomic max, >= 0)
    float *ga_lo, *ga_hi;            // [slot][S]  interval of G(a) = H[k0][a]
    u32 *ga_bits;                    // [slot][ceil(S/32)] rows a with L[k0][afix] not <= 0
    float *ga_max, *ga_abs;          // [slot]     largest in-bounds hi(a), largest |hi(a)|
    unsigned long long *scan_next;   // next (candidate, template) pair of the scan
    u32 *seed_a1;                    // [slot]     in-bounds row a of largest lower bound
    float *pair_mb, *pair_mabs;      // [slot][K]  per (candidate, template): largest in-bounds upper
                                     //            bound of a row b and of its magnitude (from the seed)
    const u32 *tsup;                 // [K][2] non-zero channel range of each template (may be NULL)
    u32 *pool_total;                 // appended entries this pass
    u32 pool_cap;
    u32 *pool_slot;                  // [pool_cap]
    u32 *pool_item;                  // [pool_cap]
    float *pool_hi;                  // [pool_cap] upper bound of the contender
    u32 *refined;                    // contenders evaluated exactly this pass
    u64 *best_key;                   // [slot] packed (value, ~item) of the best refined contender
    u8 *fallback;                    // [slot]
    u64 *items_evaluated;
    // H from the tensor cores: its rounding bound replaces kappa_mine, plus
    // the fp16 subnormal terms (see fbp_lik_tc.cuh)
    float km_override;               // > 0: bound of the tensor-core tables
    const float *tabs;               // [K] ||t||_1
    const int *texp;                 // [K] template scale exponents
    const int *kexp_tile;            // [group][slot][stiles] window scale exponents
    const u32 *tgrp;                 // [K] template group of the tensor-core tables (NULL: one group)
    u32 kt_slots;                    // slots per group in kexp_tile
    u32 stiles;
    float *ua;                       // [slot] ||window||_1
    LazyLk lazy;                     // approximate likelihood entries (tensor-core path)
};

__device__ __forceinline__ float warp_max_f(float x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

// ---------------------------------------------------------------- per chunk

// NT[t][b] = sum_c sum_{j in J(db)} T[t][c][j-db]^2 (clipped energy), sNT its
// square root, tnorm[t] = ||t||; kappa from the number of non-zero channels.
__global__ void k_ov_chunk_tables(const float *__restrict__ T, u32 K, u32 C, u32 L, u32 nmax,
                                  float *__restrict__ NT, float *__restrict__ sNT,
                                  float *__restrict__ tnorm, OvConst *oc, const u32 *__restrict__ tsup) {
    const u32 S = 2 * nmax + 1;
    for (u32 e = blockIdx.x * blockDim.x + threadIdx.x; e < K * S; e += gridDim.x * blockDim.x) {
        const u32 t = e / S, b = e % S;
        const int d = (int)b - (int)nmax;
        const int j0 = max(0, d), j1 = min((int)L, (int)L + d);
        double acc = 0.0;
        const u32 clo = tsup ? tsup[2 * t] : 0u, chi = tsup ? tsup[2 * t + 1] : C;
        for (u32 c = clo; c < chi; c++) {
            const float *tp = T + ((size_t)t * C + c) * L;
            for (int j = j0; j < j1; j++) {
                const double x = tp[j - d];
                acc += x * x;
            }
        }
        NT[e] = (float)(acc * (1.0 + 1e-6));
        sNT[e] = (float)(sqrt(acc) * (1.0 + 1e-6));
    }
    if (blockIdx.x == 0) {
        __shared__ u32 cmax;
        if (threadIdx.x == 0) cmax = 0;
        __syncthreads();
        for (u32 t = threadIdx.x; t < K; t += blockDim.x) {
            double ss = 0.0;
            u32 nz = 0;
            for (u32 c = 0; c < C; c++) {
                const float *tp = T + ((size_t)t * C + c) * L;
                bool any = false;
                for (u32 j = 0; j < L; j++) {
                    ss += (double)tp[j] * tp[j];
                    any |= tp[j] != 0.0f;
                }
                nz += any;
            }
            tnorm[t] = (float)(sqrt(ss) * (1.0 + 1e-6));
            atomicMax(&cmax, nz);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            oc->cnz_max = cmax;
            // gamma_n with n the reference's non-zero terms: products of two
            // templates' channels, the per-channel subtractions and sums of
            // squares, each product carrying two roundings
            const double u = (double)kUnitRoundoff;
            const double n_ref = 2.0 * cmax * L + C + 2.0 * L + 16.0;
            const double n_mine = (double)cmax * L + 8.0;
            oc->kappa_ref = (float)(1.05 * n_ref * u / (1.0 - n_ref * u));
            oc->kappa_mine = (float)(1.05 * n_mine * u / (1.0 - n_mine * u));
        }
    }
}

// Q[k0][t][ri][m] = sum_{m' < m} sum_c T[k0][c][m'] * T[t][c][m'+r], r = ri-(L-1).
// One thread per (k0, t, ri) row, accumulated in double, stored in float.
__global__ void k_ov_q_table(const float *__restrict__ T, u32 K, u32 C, u32 L, float *__restrict__ Q,
                             const u32 *__restrict__ tsup) {
    const u32 R = 2 * L - 1;
    const u64 rows = (u64)K * K * R;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < rows; e += (u64)gridDim.x * blockDim.x) {
        const u32 ri = (u32)(e % R);
        const u32 t = (u32)((e / R) % K);
        const u32 k0 = (u32)(e / ((u64)R * K));
        // channels where both templates can be non-zero (tsup: [lo, hi) per template)
        const u32 clo = tsup ? max(tsup[2 * k0], tsup[2 * t]) : 0u;
        const u32 chi = tsup ? min(tsup[2 * k0 + 1], tsup[2 * t + 1]) : C;
        const int r = (int)ri - (int)(L - 1);
        float *q = Q + e * (L + 1);
        double acc = 0.0;
        q[0] = 0.0f;
        for (u32 m = 0; m < L; m++) {
            const int mt = (int)m + r;
            if (mt >= 0 && mt < (int)L) {
                for (u32 c = clo; c < chi; c++)
                    acc += (double)T[((size_t)k0 * C + c) * L + m] * (double)T[((size_t)t * C + c) * L + mt];
            }
            q[m + 1] = (float)acc;
        }
    }
}

// ---------------------------------------------------------------- per pass

// One warp per candidate slot: skip rules of .cl:518-527, window energy,
// label histogram.
__global__ void k_ov_prep(OvArgs A) {
    const u32 nc = *A.n_cand;
    const u32 lane = threadIdx.x & 31;
    for (u32 g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < nc;
         g += gridDim.x * (blockDim.x >> 5)) {
        const u32 id = A.cand[g];
        const u32 lab = A.best_lab[id], bidx = A.best_idx[id];
        const float bll = A.Lk[(size_t)lab * A.n + bidx];
        const bool skip = (bll < A.thr[lab]) || (bidx >= A.n - A.L);
        double e = 0.0, e1 = 0.0;
        if (!skip)
            for (u32 q = lane; q < A.C * A.L; q += 32) {
                const double x = A.v[(size_t)(q / A.L) * A.n + bidx + q % A.L];
                e += x * x;
                e1 += fabs(x);
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            e += __shfl_xor_sync(0xffffffffu, e, o);
            e1 += __shfl_xor_sync(0xffffffffu, e1, o);
        }
        if (lane == 0) {
            A.cskip[g] = skip;
            A.vn[g] = (float)(sqrt(e) * (1.0 + 1e-6));
            if (A.ua) A.ua[g] = (float)(e1 * (1.0 + 1e-6));
            A.best_key[g] = 0ull;
            A.cand_lb[g] = 0.0f;
        }
    }
}

// H[g][t][b] for every template t and shift b of candidate g: correlation of
// t shifted by db with the window voltage (zero outside [i0, i0+L)), minus
// half the clipped energy.  FP32 FMA; its error is inside kappa.
// Thread tile: 8 shifts x 8 templates; per channel the window strip and the
// templates' channel slab ([m][t], t contiguous) are staged in shared memory.
constexpr int kTabThreads = 256;
__global__ void __launch_bounds__(kTabThreads)
k_ov_tables(OvArgs A) {
    extern __shared__ float sm[];
    const u32 S = A.S, K = A.K, L = A.L, C = A.C, nmax = A.nmax;
    const u32 Lp = (L + 7) & ~7u;                  // lags padded to 8
    const u32 Sg = (S + 7) / 8, Kg = (K + 7) / 8;  // output groups
    const u32 Sp = Sg * 8, Kp = Kg * 8;
    const u32 strip_len = Sp + Lp + 8;
    float *strip = sm;                             // [strip_len]
    float *slab = sm + strip_len;                  // [Lp][Kp]
    const u32 nc = *A.n_cand;
    const u32 groups = Sg * Kg;
    for (u32 g = blockIdx.x; g < nc; g += gridDim.x) {
        if (A.cskip[g]) continue;
        const u32 id = A.cand[g];
        const u32 bidx = A.best_idx[id];
        for (u32 gb = 0; gb < groups; gb += blockDim.x) {
            const u32 my = gb + threadIdx.x;
            const bool active = my < groups;
            const u32 sg = active ? my % Sg : 0, kg = active ? my / Sg : 0;
            float acc[8][8];
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = 0.0f;
            for (u32 c = 0; c < C; c++) {
                __syncthreads();
                // strip[x] = window voltage at position i0 - nmax + x (zero outside [i0, i0+L))
                for (u32 x = threadIdx.x; x < strip_len; x += blockDim.x) {
                    const int rel = (int)x - (int)nmax;   // position relative to i0
                    strip[x] = (rel >= 0 && rel < (int)L) ? A.v[(size_t)c * A.n + bidx + rel] : 0.0f;
                }
                for (u32 e = threadIdx.x; e < Lp * Kp; e += blockDim.x) {
                    const u32 m = e / Kp, t = e % Kp;
                    slab[e] = (m < L && t < K) ? A.T[((size_t)t * C + c) * L + m] : 0.0f;
                }
                __syncthreads();
                if (!active) continue;
                const float *sp = strip + sg * 8;
                const float *tp = slab + kg * 8;
                for (u32 m0 = 0; m0 < Lp; m0 += 8) {
                    float w[16];
#pragma unroll
                    for (int q = 0; q < 16; q++) w[q] = sp[m0 + q];
#pragma unroll
                    for (int mm = 0; mm < 8; mm++) {
                        const float4 t0 = *reinterpret_cast<const float4 *>(tp + (m0 + mm) * Kp);
                        const float4 t1 = *reinterpret_cast<const float4 *>(tp + (m0 + mm) * Kp + 4);
                        const float tv[8] = {t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z, t1.w};
#pragma unroll
                        for (int i = 0; i < 8; i++)
#pragma unroll
                            for (int j = 0; j < 8; j++) acc[i][j] = fmaf(tv[j], w[i + mm], acc[i][j]);
                    }
                }
            }
            if (active) {
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const u32 t = kg * 8 + j;
                    if (t >= K) continue;
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const u32 b = sg * 8 + i;
                        if (b < S)
                            A.H[((size_t)g * K + t) * S + b] = acc[i][j] - 0.5f * A.NT[(size_t)t * S + b];
                    }
                }
            }
        }
    }
}

// H[g][t][b] for masked templates (each non-zero on a narrow channel range):
// block = (candidate, group of 32 templates in support order); the group's
// channels of the window, zero-padded by n_max on both sides, are staged in
// chunks; warp w takes slots 4w..4w+3 of the group, lane l the shifts
// b = l + 32k, and each (channel, lag) step is one broadcast template value
// times a contiguous row of the window.  Only the templates' own channels
// are summed (the others add zero).  FP32 FMA in any order: the error bound
// of the tables covers it.
constexpr int kTabMThreads = 256;
constexpr int kTabMGroup = 32;
constexpr int kTabMChan = 16;            // staged channels per chunk
constexpr int kTabMShiftChunks = 16;     // S <= 512
__host__ __device__ inline size_t tables_m_smem_bytes(u32 S, u32 L) {
    return (size_t)kTabMChan * (S + L - 1) * 4;
}
__global__ void __launch_bounds__(kTabMThreads)
k_ov_tables_m(OvArgs A, const u32 *__restrict__ tperm, const u32 *__restrict__ tsup,
              const u32 *__restrict__ grange32) {
    extern __shared__ float wp[];                   // [kTabMChan][S + L - 1]
    const u32 S = A.S, K = A.K, L = A.L, nmax = A.nmax;
    const u32 P = S + L - 1;
    const u32 warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 nk = (S + 31) / 32;
    const u32 ng = (K + kTabMGroup - 1) / kTabMGroup;
    const u32 nc = *A.n_cand;
    for (u64 item = blockIdx.x; item < (u64)nc * ng; item += gridDim.x) {
        const u32 g = (u32)(item / ng), tg = (u32)(item % ng);
        if (A.cskip[g]) continue;
        const u32 i0 = A.best_idx[A.cand[g]];
        const u32 glo = grange32[2 * tg], ghi = grange32[2 * tg + 1];
        u32 tq[4], lo[4], hi[4];
        u32 wlo = 0xffffffffu, whi = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const u32 sl = tg * kTabMGroup + warp * 4 + q;
            tq[q] = sl < K ? tperm[sl] : 0u;
            lo[q] = sl < K ? tsup[2 * tq[q]] : 0u;
            hi[q] = sl < K ? tsup[2 * tq[q] + 1] : 0u;
            if (hi[q] > lo[q]) { wlo = min(wlo, lo[q]); whi = max(whi, hi[q]); }
        }
        float acc[4][kTabMShiftChunks];
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
            for (int k = 0; k < kTabMShiftChunks; k++) acc[q][k] = 0.0f;
        for (u32 c0 = glo; c0 < ghi; c0 += kTabMChan) {
            const u32 cc = min((u32)kTabMChan, ghi - c0);
            __syncthreads();
            for (u32 e = threadIdx.x; e < cc * P; e += blockDim.x) {
                const u32 c = e / P, x = e % P;
                const int rel = (int)x - (int)nmax;          // position relative to i0
                wp[e] = (rel >= 0 && rel < (int)L) ? A.v[(size_t)(c0 + c) * A.n + i0 + rel] : 0.0f;
            }
            __syncthreads();
            const u32 cb = max(c0, wlo), ce = min(c0 + cc, whi);
            for (u32 c = cb; c < ce; c++) {
                const float *row = wp + (size_t)(c - c0) * P + lane;
                const float *tp[4];
                bool on[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    on[q] = c >= lo[q] && c < hi[q];
                    tp[q] = A.T + ((size_t)tq[q] * A.C + c) * L;
                }
                for (u32 m = 0; m < L; m++) {
                    float tv[4];
#pragma unroll
                    for (int q = 0; q < 4; q++) tv[q] = on[q] ? __ldg(tp[q] + m) : 0.0f;
#pragma unroll
                    for (int k = 0; k < kTabMShiftChunks; k++) {
                        if ((u32)k >= nk) break;
                        // m + b <= P - 1 for every b < S; lanes past S read nothing
                        const float wv = (lane + 32u * k < S) ? row[m + 32 * k] : 0.0f;
#pragma unroll
                        for (int q = 0; q < 4; q++) acc[q][k] = fmaf(tv[q], wv, acc[q][k]);
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const u32 sl = tg * kTabMGroup + warp * 4 + q;
            if (sl >= K) continue;
            const u32 t = tq[q];
#pragma unroll
            for (int k = 0; k < kTabMShiftChunks; k++) {
                const u32 b = lane + 32 * k;
                if ((u32)k < nk && b < S)
                    A.H[((size_t)g * K + t) * S + b] = acc[q][k] - 0.5f * A.NT[(size_t)t * S + b];
            }
        }
    }
}

constexpr int kScanThreads = 256;
// Per-warp scratch of the scan: ga_lo, ga_hi, hb_lo, hb_hi (S floats each),
// the a and b row lists (S u16 each), and the bitmasks of rows a with
// L[k0][afix] not <= 0 and rows b with L[t][ashift] not <= 0 (S bits each).
__host__ __device__ inline size_t sweep_warp_bytes(u32 S) {
    return align_up((size_t)20 * S + (size_t)(S + 31) / 32 * 8, 16);
}
__host__ __device__ inline size_t scan_smem_bytes(u32 S) {
    return (size_t)(kScanThreads / 32) * sweep_warp_bytes(S);
}
// k_ov_xm stages one template pair's prefix table.
__host__ __device__ inline size_t xm_smem_bytes(u32 L) { return (size_t)(2 * L - 1) * (L + 1) * 4; }
__host__ __device__ inline size_t tables_smem_bytes(u32 S, u32 K, u32 L) {
    const size_t Lp = (L + 7) & ~7u, Sp = (size_t)(S + 7) / 8 * 8, Kp = (size_t)(K + 7) / 8 * 8;
    return (Sp + Lp + 8 + Lp * Kp) * 4;
}
constexpr int kSeedThreads = 256;

// Interval of one item from its row-invariant and moving parts.
__device__ __forceinline__ float ov_x(const float *__restrict__ q, u32 L, int a_minus_nmax, int r) {
    float X = 0.0f;
    if (r > -(int)L && r < (int)L) {
        const int lo_m = max(max(0, -r), -a_minus_nmax);
        const int hi_m = min(min((int)L, (int)L - r), (int)L - a_minus_nmax);
        if (lo_m < hi_m) {
            const float *qr = q + (size_t)(r + (int)L - 1) * (L + 1);
            X = qr[hi_m] - qr[lo_m];
        }
    }
    return X;
}
__device__ __forceinline__ void ov_item_bounds(const float *__restrict__ q, u32 L, int a_minus_nmax, int r,
                                               float loA, float hiA, float loB, float hiB, float kx,
                                               float &lo, float &hi) {
    const float X = ov_x(q, L, a_minus_nmax, r);
    const float ex = kx * fabsf(X);
    hi = hiA + hiB - X + ex;
    lo = loA + loB - X - ex;
}

// Interval of a row term: G(a) = H[k0][a] (extra = 0) or H[t][b] (extra =
// the cross term's own rounding), with the fp16 subnormal terms of
// tensor-core tables (sub0 / sub1 scaled by the tile's voltage exponent).
__device__ __forceinline__ void ov_row_interval(const OvArgs &A, u32 g, u32 tmpl, u32 x, float Hv, float nt,
                                                float snt, float vn, float krm, float extra, float sub0, float sub1,
                                                float &lo, float &hi) {
    float sx = 0.0f;
    if (A.kexp_tile) {
        // scale exponent of the table tile: per template group, candidate, tile of 128 shifts
        const size_t grp = A.tgrp ? (size_t)A.tgrp[tmpl] * A.kt_slots : 0;
        sx = sub0 * ldexpf(1.0f, -A.kexp_tile[(grp + g) * A.stiles + x / 128]) + sub1;
    }
    const float e = krm * (snt * vn + nt) + 4.0f * kUnitRoundoff * fabsf(Hv) + extra + sx;
    lo = Hv - e;
    hi = Hv + e;
}

// Per-candidate constants of the row intervals.
struct OvCand {
    u32 id, k0, bidx, xlo, xhi_ex;
    float lbest, vn, subA0, subA1;
};
__device__ __forceinline__ OvCand ov_cand(const OvArgs &A, u32 g) {
    OvCand c;
    c.id = A.cand[g];
    c.k0 = A.best_lab[c.id];
    c.bidx = A.best_idx[c.id];
    c.lbest = A.best_ll[c.id];
    c.vn = A.vn[g];
    c.xlo = c.bidx >= A.nmax ? 0u : A.nmax - c.bidx;          // in-bounds shifts (.cl:534-541)
    c.xhi_ex = A.n - A.L + A.nmax - c.bidx;                    // first out-of-bounds shift
    c.subA0 = c.subA1 = 0.0f;
    if (A.kexp_tile) {
        c.subA1 = 2.98023224e-08f * 1.001f * ldexpf(A.ua[g], -A.texp[c.k0]);
        c.subA0 = 2.98023224e-08f * 1.001f * A.tabs[c.k0];
    }
    return c;
}
__device__ __forceinline__ void ov_sub_b(const OvArgs &A, u32 g, u32 t, float &subB0, float &subB1) {
    subB0 = subB1 = 0.0f;
    if (A.kexp_tile) {
        subB1 = 2.98023224e-08f * 1.001f * ldexpf(A.ua[g], -A.texp[t]);
        subB0 = 2.98023224e-08f * 1.001f * A.tabs[t];
    }
}
__device__ __forceinline__ float ov_kx(const OvArgs &A) { return 2.0f * A.oc->kappa_ref + 4.0f * kUnitRoundoff; }
__device__ __forceinline__ float ov_krm(const OvArgs &A) {
    return A.oc->kappa_ref + (A.km_override > 0.0f ? A.km_override : A.oc->kappa_mine);
}
// Slack for the float roundings of the pruning sums (2^-18 relative).
constexpr float kPruneSlack = 3.814697265625e-06f;

// Per chunk: XMr[k0][t][r + L] = an upper bound of -X + kx|X| over every
// shift a of an item with lag r = a - b (X = 0 where the clipped templates
// do not overlap), and XM[k0][t] = its maximum over r.  Then
//     hi(a, b) <= hiA(a) + hiB(b) + XMr[a - b]
// bounds every item's interval without its cross term.
__global__ void __launch_bounds__(256)
k_ov_xm(const float *__restrict__ Q, u32 K, u32 L, u32 nmax, const OvConst *__restrict__ oc,
        float *__restrict__ XMr, float *__restrict__ XM) {
    extern __shared__ float xm_sm[];                 // Q[k0][t]: [2L-1][L+1]
    const u32 R = 2 * L - 1, S = 2 * nmax + 1, NR = 2 * L + 1;
    const float kx = 2.0f * oc->kappa_ref + 4.0f * kUnitRoundoff;
    __shared__ float red[8];
    for (u32 pair = blockIdx.x; pair < K * K; pair += gridDim.x) {
        const float *qg = Q + (size_t)pair * R * (L + 1);
        __syncthreads();
        for (u32 e = threadIdx.x; e < R * (L + 1); e += blockDim.x) xm_sm[e] = qg[e];
        __syncthreads();
        float pm = -INFINITY;
        for (u32 ri = threadIdx.x; ri < NR; ri += blockDim.x) {
            const int r = (int)ri - (int)L;
            float m = -INFINITY;
            for (u32 a = 0; a < S; a++) {
                const float X = ov_x(xm_sm, L, (int)a - (int)nmax, r);
                m = fmaxf(m, -X + kx * fabsf(X));
            }
            m += kPruneSlack * fabsf(m);
            XMr[(size_t)pair * NR + ri] = m;
            pm = fmaxf(pm, m);
        }
        pm = warp_max_f(pm);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = pm;
        __syncthreads();
        if (threadIdx.x == 0) {
            float v = red[0];
            for (u32 w = 1; w < blockDim.x / 32; w++) v = fmaxf(v, red[w]);
            XM[pair] = v;
        }
    }
}

// Warp argmax: larger value, then lower index.
__device__ __forceinline__ void warp_argmax(float &v, u32 &i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, v, o);
        const u32 oi = __shfl_xor_sync(0xffffffffu, i, o);
        if (ov > v || (ov == v && oi < i)) { v = ov; i = oi; }
    }
}

// Rows a of each candidate (one warp per candidate): the intervals of
// G(a) = H[k0][a], the L[k0][afix] > 0 bits, the largest in-bounds upper
// bound and |upper bound|, and the row of largest lower bound (a1), for the
// seed and the scan.
__global__ void __launch_bounds__(kSeedThreads)
k_ov_rows(OvArgs A) {
    const u32 nc = *A.n_cand;
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const u32 S = A.S, n = A.n, nmax = A.nmax, NB = (S + 31) / 32;
    const float krm = ov_krm(A);
    for (u32 g = blockIdx.x * (kSeedThreads / 32) + warp; g < nc; g += gridDim.x * (kSeedThreads / 32)) {
        if (A.cskip[g]) continue;
        const OvCand c = ov_cand(A, g);
        const float *Hg = A.H + ((size_t)g * A.K + c.k0) * S;
        float va = -INFINITY, mA = -INFINITY, mabs = 0.0f;
        u32 a1 = 0;
        for (u32 x0 = 0; x0 < S; x0 += 32) {
            const u32 x = x0 + lane;
            bool ap = false;
            if (x < S) {
                float lo, hi;
                ov_row_interval(A, g, c.k0, x, Hg[x], A.NT[(size_t)c.k0 * S + x], A.sNT[(size_t)c.k0 * S + x], c.vn,
                                krm, 0.0f, c.subA0, c.subA1, lo, hi);
                A.ga_lo[(size_t)g * S + x] = lo;
                A.ga_hi[(size_t)g * S + x] = hi;
                if (x >= c.xlo && x < c.xhi_ex) {
                    ap = !(A.Lk[(size_t)c.k0 * n + c.bidx + x - nmax] <= 0.0f);
                    if (lo > va) { va = lo; a1 = x; }
                    mA = fmaxf(mA, hi);
                    mabs = fmaxf(mabs, fabsf(hi));
                }
            }
            const u32 m = __ballot_sync(0xffffffffu, ap);
            if (lane == 0) A.ga_bits[(size_t)g * NB + x0 / 32] = m;
        }
        warp_argmax(va, a1);
        mA = warp_max_f(mA);
        mabs = warp_max_f(mabs);
        if (lane == 0) {
            A.ga_max[g] = mA;
            A.ga_abs[g] = mabs;
            A.seed_a1[g] = a1;
        }
    }
}

// Seed of each candidate's best lower bound, one warp per (candidate,
// template t): the items (a1, b1), (a1, b2), (a3, b1) with b1 the row b of
// largest lower bound, b2 the best row b within L of a1 and a3 the best row a
// within L of b1.  Any item's lower bound is a valid lower bound of the best
// item, and these are close to the largest one, so the scan can prune
// against it from the start.
__global__ void __launch_bounds__(kSeedThreads)
k_ov_seed(OvArgs A) {
    const u32 nc = *A.n_cand;
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const u32 S = A.S, K = A.K, L = A.L, nmax = A.nmax, n = A.n, R = 2 * L - 1, NB = (S + 31) / 32;
    const float krm = ov_krm(A), kx = ov_kx(A);
    const u64 total = (u64)nc * K;
    const u64 nwarps = (u64)gridDim.x * (kSeedThreads / 32);
    for (u64 e = (u64)blockIdx.x * (kSeedThreads / 32) + warp; e < total; e += nwarps) {
        const u32 g = (u32)(e / K), t = (u32)(e % K);
        if (A.cskip[g] || A.ga_max[g] == -INFINITY) continue;   // skipped, or no in-bounds row
        const OvCand c = ov_cand(A, g);
        const u32 a1 = A.seed_a1[g];
        const float *ga_lo = A.ga_lo + (size_t)g * S;
        const float va = ga_lo[a1];
        const float *Hg = A.H + ((size_t)g * K + t) * S;
        float subB0, subB1;
        ov_sub_b(A, g, t, subB0, subB1);
        const float eqt = 4.0f * kUnitRoundoff * A.tnorm[c.k0] * A.tnorm[t];
        const u32 xend = min(S, c.xhi_ex);
        float v1 = -INFINITY, v2 = -INFINITY, mB = -INFINITY, mabs = 0.0f;
        u32 b1 = 0, b2 = 0;
        for (u32 x = c.xlo + lane; x < xend; x += 32) {
            float lo, hi;
            ov_row_interval(A, g, t, x, Hg[x], A.NT[(size_t)t * S + x], A.sNT[(size_t)t * S + x], c.vn, krm, eqt,
                            subB0, subB1, lo, hi);
            if (lo > v1) { v1 = lo; b1 = x; }
            if ((x > a1 ? x - a1 : a1 - x) <= L && lo > v2) { v2 = lo; b2 = x; }
            mB = fmaxf(mB, hi);
            mabs = fmaxf(mabs, fabsf(hi));
        }
        warp_argmax(v1, b1);
        warp_argmax(v2, b2);
        mB = warp_max_f(mB);
        mabs = warp_max_f(mabs);
        if (lane == 0) {                                 // the scan's pair test, before its row pass
            A.pair_mb[e] = mB;
            A.pair_mabs[e] = mabs;
        }
        float v3 = -INFINITY;
        u32 a3 = 0;
        for (u32 x = c.xlo + lane; x < xend; x += 32)
            if ((x > b1 ? x - b1 : b1 - x) <= L && ga_lo[x] > v3) { v3 = ga_lo[x]; a3 = x; }
        warp_argmax(v3, a3);
        float seed = 0.0f;
        if (lane < 3) {
            const u32 a = lane == 2 ? a3 : a1, b = lane == 1 ? b2 : b1;
            const float lb_b = lane == 1 ? v2 : v1;
            const float lb_a = lane == 2 ? v3 : va;
            if ((a > b ? a - b : b - a) <= L && lb_a > -INFINITY && lb_b > -INFINITY) {
                const bool fp = (A.ga_bits[(size_t)g * NB + (a >> 5)] >> (a & 31)) & 1u;
                const bool sp = !(A.Lk[(size_t)t * n + c.bidx + b - nmax] <= 0.0f);
                if (fp || sp) {                          // .cl:572-576
                    const float *q = A.Q + ((size_t)c.k0 * K + t) * R * (L + 1);
                    const float X = ov_x(q, L, (int)a - (int)nmax, (int)a - (int)b);
                    seed = lb_a + lb_b - X - kx * fabsf(X);
                }
            }
        }
        seed = warp_max_f(seed);
        if (lane == 0 && seed > 0.0f) atomicMax(reinterpret_cast<int *>(A.cand_lb) + g, __float_as_int(seed));
    }
}

// One warp per (candidate, template t): every item (a, b, t) the reference
// evaluates (.cl:534-576) either gets its interval here or is shown to have
// hi < TH, TH = max(best lower bound so far, current best likelihood):
//   - the whole pair is skipped when max hiA + max hiB + XM < TH;
//   - rows a / b whose bound with the other side's maximum is below TH drop;
//   - of the remaining pairs, those that pass the skip rules and
//     hiA + hiB + XMr[a-b] >= TH get their interval from the prefix table.
// An item that is never enumerated can neither be the best item (whose value
// is >= every lower bound) nor beat the current best.  Items with
// hi >= TH and hi > current best go to the contender pool with their hi;
// their lower bounds raise the candidate's best lower bound.
__global__ void __launch_bounds__(kScanThreads)
k_ov_scan(OvArgs A) {
    extern __shared__ float sm[];
    const u32 S = A.S, K = A.K, L = A.L, nmax = A.nmax, n = A.n;
    const u32 R = 2 * L - 1, NR = 2 * L + 1, NB = (S + 31) / 32;
    const u32 warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *ga_lo = (float *)((char *)sm + (size_t)warp * sweep_warp_bytes(S));
    float *ga_hi = ga_lo + S, *hb_lo = ga_hi + S, *hb_hi = hb_lo + S;
    u16 *alist = (u16 *)(hb_hi + S);
    u16 *blist = alist + S;
    u32 *abits = (u32 *)((char *)ga_lo + (size_t)20 * S);
    u32 *bbits = abits + NB;
    const u32 nc = *A.n_cand;
    const u64 total = (u64)nc * K;
    const float krm = ov_krm(A), kx = ov_kx(A);
    u32 evaluated = 0;
    for (;;) {
        // pairs are taken dynamically: their cost varies by orders of magnitude
        u64 e = 0;
        if (lane == 0) e = atomicAdd(A.scan_next, 1ull);
        e = __shfl_sync(0xffffffffu, e, 0);
        if (e >= total) break;
        const u32 g = (u32)(e / K), t = (u32)(e % K);
        if (A.cskip[g]) continue;
        const float mA = A.ga_max[g];
        if (mA == -INFINITY) continue;                  // no in-bounds row
        const OvCand c = ov_cand(A, g);
        const float LB = *(volatile const float *)(A.cand_lb + g);
        const float TH = fmaxf(LB, c.lbest);
        const size_t pair = (size_t)c.k0 * K + t;
        const float XM = A.XM[pair];
        {
            // the pair test below with the seed's row maxima (the same values
            // the row pass computes): a pair that fails it needs no row pass
            const float mB0 = A.pair_mb[e];
            const float mabs0 = fmaxf(A.ga_abs[g], A.pair_mabs[e]);
            const float slack0 = kPruneSlack * (2.0f * mabs0 + fabsf(TH) + fabsf(XM));
            if (!(mA + mB0 + XM + slack0 >= TH)) continue;
        }
        const float *Hg = A.H + ((size_t)g * K + t) * S;
        float subB0, subB1;
        ov_sub_b(A, g, t, subB0, subB1);
        const float eqt = 4.0f * kUnitRoundoff * A.tnorm[c.k0] * A.tnorm[t];
        // rows b: intervals and the L[t][ashift] > 0 bits; rows a: copied
        float mB = -INFINITY, mabs = A.ga_abs[g];
        for (u32 x0 = 0; x0 < S; x0 += 32) {
            const u32 x = x0 + lane;
            bool bp = false;
            if (x < S) {
                ga_lo[x] = A.ga_lo[(size_t)g * S + x];
                ga_hi[x] = A.ga_hi[(size_t)g * S + x];
                float lo, hi;
                ov_row_interval(A, g, t, x, Hg[x], A.NT[(size_t)t * S + x], A.sNT[(size_t)t * S + x], c.vn, krm, eqt,
                                subB0, subB1, lo, hi);
                hb_lo[x] = lo;
                hb_hi[x] = hi;
                if (x >= c.xlo && x < c.xhi_ex) {
                    bp = !(A.Lk[(size_t)t * n + c.bidx + x - nmax] <= 0.0f);
                    mB = fmaxf(mB, hi);
                    mabs = fmaxf(mabs, fabsf(hi));
                }
            }
            const u32 mb = __ballot_sync(0xffffffffu, bp);
            if (lane == 0) {
                bbits[x0 / 32] = mb;
                abits[x0 / 32] = A.ga_bits[(size_t)g * NB + x0 / 32];
            }
        }
        mB = warp_max_f(mB);
        mabs = warp_max_f(mabs);
        const float slack = kPruneSlack * (2.0f * mabs + fabsf(TH) + fabsf(XM));
        if (!(mA + mB + XM + slack >= TH)) continue;
        // rows that can reach TH with the other side's best
        u32 na = 0, nb = 0;
        for (u32 x0 = 0; x0 < S; x0 += 32) {
            const u32 x = x0 + lane;
            const bool inb = x < S && x >= c.xlo && x < c.xhi_ex;
            const bool ka = inb && ga_hi[x] + mB + XM + slack >= TH;
            const bool kb = inb && hb_hi[x] + mA + XM + slack >= TH;
            const u32 ma = __ballot_sync(0xffffffffu, ka), mb = __ballot_sync(0xffffffffu, kb);
            if (ka) alist[na + __popc(ma & ((1u << lane) - 1u))] = (u16)x;
            if (kb) blist[nb + __popc(mb & ((1u << lane) - 1u))] = (u16)x;
            na += __popc(ma);
            nb += __popc(mb);
        }
        __syncwarp();
        const float *xmr = A.XMr + pair * NR;
        const float *q = A.Q + pair * R * (L + 1);
        const u32 P = na * nb;
        float lbmax = -INFINITY;
        // pair p = ai * nb + bi; each lane steps its (ai, bi) by 32 pairs
        u32 ai = 0, bi = lane, dq = 0, dr = 32;
        if (nb) {
            ai = lane / nb; bi = lane - ai * nb;
            dq = 32 / nb; dr = 32 - dq * nb;
        }
        for (u32 p0 = 0; p0 < P; p0 += 32) {
            const u32 p = p0 + lane;
            bool valid = false;
            u32 a = 0, b = 0;
            if (p < P) {
                a = alist[ai];
                b = blist[bi];
                valid = (a > b ? a - b : b - a) <= L &&                                    // .cl:543-556
                        (((abits[a >> 5] >> (a & 31)) | (bbits[b >> 5] >> (b & 31))) & 1u);  // .cl:572-576
                if (valid) {
                    const float xr = __ldg(xmr + (int)a - (int)b + (int)L);
                    valid = ga_hi[a] + hb_hi[b] + xr + slack + kPruneSlack * fabsf(xr) >= TH;
                }
            }
            ai += dq;
            bi += dr;
            if (bi >= nb) { bi -= nb; ai++; }
            float lo = -INFINITY, hi = -INFINITY;
            if (valid) {
                ov_item_bounds(q, L, (int)a - (int)nmax, (int)a - (int)b, ga_lo[a], ga_hi[a], hb_lo[b], hb_hi[b],
                               kx, lo, hi);
                evaluated++;
            }
            lbmax = fmaxf(lbmax, lo);
            const bool keep = valid && hi >= TH && hi > c.lbest;
            const u32 mk = __ballot_sync(0xffffffffu, keep);
            if (mk) {
                u32 base = 0;
                if (lane == 0) base = atomicAdd(A.pool_total, (u32)__popc(mk));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (keep) {
                    const u32 pp = base + __popc(mk & ((1u << lane) - 1u));
                    if (pp < A.pool_cap) {
                        A.pool_slot[pp] = g;
                        A.pool_item[pp] = t + K * (a + S * b);
                        A.pool_hi[pp] = hi;
                    } else {
                        A.fallback[g] = 1;
                    }
                }
            }
        }
        lbmax = warp_max_f(lbmax);
        if (lane == 0 && lbmax > 0.0f) atomicMax(reinterpret_cast<int *>(A.cand_lb) + g, __float_as_int(lbmax));
        __syncwarp();
    }
    if (A.items_evaluated) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) evaluated += __shfl_xor_sync(0xffffffffu, evaluated, o);
        if (lane == 0 && evaluated) atomicAdd(A.items_evaluated, (u64)evaluated);
    }
}

// Order-preserving key: larger value first, then lower item id.
__device__ __forceinline__ u64 ov_pack(float v, u32 item) {
    u32 u = __float_as_uint(v);
    u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ((u64)u << 32) | (u64)(0xffffffffu - item);
}
__device__ __forceinline__ float ov_unpack_value(u64 key) {
    u32 u = (u32)(key >> 32);
    u = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    return __uint_as_float(u);
}

// Exact value of one item (overlap_recheck_indices, .cl:583-646), in the
// reference's order of operations; loads are issued eight lags at a time so
// the two sequential sums do not wait on each one.
__device__ float overlap_item_exact_global(const OvArgs &A, u32 lab, u32 bidx, u32 t, u32 a, u32 b) {
    const u32 L = A.L, C = A.C;
    const u32 afix = bidx + a - A.nmax, ashift = bidx + b - A.nmax;
    const int fa = (int)bidx - (int)afix, sa = (int)bidx - (int)ashift;
    // channels where either template is non-zero, in channel order: the two
    // supports as one range when they meet, else one after the other
    // (elsewhere both terms are 0 and the reference's sums do not change)
    u32 r0 = 0, r1 = C, r2 = C, r3 = C;
    if (A.tsup) {
        u32 al = A.tsup[2 * lab], ah = A.tsup[2 * lab + 1], bl = A.tsup[2 * t], bh = A.tsup[2 * t + 1];
        if (ah <= al) { al = bl; ah = bh; }
        if (bh <= bl) { bl = al; bh = ah; }
        if (bl < al) { u32 x = al; al = bl; bl = x; x = ah; ah = bh; bh = x; }
        if (bl <= ah) { r0 = al; r1 = max(ah, bh); r2 = r3 = r1; }
        else { r0 = al; r1 = ah; r2 = bl; r3 = bh; }
    }
    float cml = 0.0f;
    for (u32 c = r0; c < r3; c = (c + 1 == r1) ? r2 : c + 1) {
        const float *f = A.T + ((size_t)lab * C + c) * L;
        const float *sp = A.T + ((size_t)t * C + c) * L;
        const float *vv = A.v + (size_t)c * A.n + bidx;
        float ss = 0.0f;
        for (u32 j0 = 0; j0 < L; j0 += 8) {
            float fv[8], sv[8], wv[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int j = (int)j0 + i;
                const int jf = fa + j, js = sa + j;
                fv[i] = (j < (int)L && jf >= 0 && jf < (int)L) ? __ldg(f + jf) : 0.0f;
                sv[i] = (j < (int)L && js >= 0 && js < (int)L) ? __ldg(sp + js) : 0.0f;
                wv[i] = j < (int)L ? __ldg(vv + j) : 0.0f;
            }
#pragma unroll
            for (int i = 0; i < 8; i++) {
                if (j0 + i < L) {
                    const float sum = __fadd_rn(fv[i], sv[i]);
                    ss = __fadd_rn(ss, __fmul_rn(sum, sum));
                    cml = __fadd_rn(cml, __fmul_rn(sum, wv[i]));
                }
            }
        }
        if ((double)ss > 0.0) cml = __double2float_rn(__dsub_rn((double)cml, __dmul_rn(0.5, (double)ss)));
    }
    return cml;
}

constexpr int kRefineThreads = 256;

// Exact values of the pooled contenders whose upper bound reaches their
// candidate's final lower bound, one thread each (the sums are sequential,
// so many items in flight hide them best); each candidate keeps the largest
// value above its current best, lowest item id on ties (the parse kernel's
// strict-greater scan over single-item groups, .cl:699-706).
__global__ void __launch_bounds__(kRefineThreads)
k_ov_refine(OvArgs A) {
    const u32 m = min(*A.pool_total, A.pool_cap);
    for (u32 e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        const u32 g = A.pool_slot[e];
        if (A.fallback[g]) continue;
        if (A.pool_hi[e] < A.cand_lb[g]) continue;      // below another item's lower bound
        atomicAdd(A.refined, 1u);
        const u32 it = A.pool_item[e];
        const u32 id = A.cand[g];
        const u32 t = it % A.K, a = (it / A.K) % A.S, b = it / (A.K * A.S);
        const float ll = overlap_item_exact_global(A, A.best_lab[id], A.best_idx[id], t, a, b);
        if (ll > A.best_ll[id]) atomicMax(&A.best_key[g], ov_pack(ll, it));
    }
}

// One warp per candidate slot: the parse decision (.cl:707-814) for the
// winning contender, or "no improvement".
__global__ void __launch_bounds__(kRefineThreads)
k_ov_finalize(OvArgs A) {
    __shared__ float fbuf[kRefineThreads / 32][kWarpChunk];
    const u32 lane = threadIdx.x & 31;
    float *buf = fbuf[threadIdx.x >> 5];
    const u32 nc = *A.n_cand;
    const u32 nwarps = gridDim.x * (blockDim.x >> 5);
    for (u32 g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < nc; g += nwarps) {
        if (A.fallback[g]) continue;
        const u32 id = A.cand[g];
        const u64 key = A.best_key[g];
        float bv = A.best_ll[id];
        u64 bi = 0;
        if (key != 0ull) {
            bv = ov_unpack_value(key);
            bi = 0xffffffffu - (u32)(key & 0xffffffffu);
        }
        if (bv <= A.best_ll[id] || bv <= 0.0f) {
            if (lane == 0) A.ovr[id] = 0;
            continue;
        }
        const u32 lab = A.best_lab[id], bidx = A.best_idx[id];
        const u32 t = (u32)(bi % A.K);
        const u32 a = (u32)((bi / A.K) % A.S);
        const u32 b = (u32)((bi / ((u64)A.S * A.K)) % A.S);
        const u32 afix = bidx + a - A.nmax, ashift = bidx + b - A.nmax;
        const float lf = warp_lk_exact(A.lazy, A.Lk, A.n, lab, afix, buf);
        const float ls = warp_lk_exact(A.lazy, A.Lk, A.n, t, ashift, buf);
        if (lane == 0)
            overlap_parse_tail(id, bv, lab, t, afix, ashift, lf, ls, A.best_idx, A.best_lab, A.best_ll, A.ov_idx,
                               A.ov_lab, A.ovr, A.thr);
    }
}

// Window ids of the candidates that overflowed a contender list.
__global__ void k_ov_fallback_list(OvArgs A, const u32 *__restrict__ slots, const u32 *__restrict__ n_slots,
                                   u32 *__restrict__ out) {
    const u32 m = *n_slots;
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        out[i] = A.cand[slots[i]];
}

}  // namespace fbp
