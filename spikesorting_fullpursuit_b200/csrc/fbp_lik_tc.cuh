// Path (a) on the tensor cores: tcgen05 likelihood (16-bit operands, FP32
// accumulation) with exact refinement.
//
// likelihood[t][s] = -0.5*SS_t + sum_c sum_m T[t][c][m] * v[c][s+m]
// (compute_full_likelihood, binary_pursuit.cl:216-300) is the product of a
// Toeplitz voltage operand (rows = samples, K = (channel, lag)) and the
// template matrix.  The voltage strip of a tile lives in shared memory as
// rows of 8 channels (16 bytes, fp16): that is the K-major, no-swizzle
// canonical UMMA layout, and the operand for lag m is the same strip started
// m rows later -- so the contraction is L accumulating
// tcgen05.mma (M = 128 samples, N = templates, K = 16 channels) per channel
// pair, with no im2col.  Templates ([lag][channel group][template][8]) are
// copied into shared memory once per CTA with one bulk asynchronous copy.
// Accumulators are FP32 in tensor memory.
//
// Operands are IEEE fp16 after exact power-of-two scaling (per tile for the
// voltage, per template for the templates), undone exactly in the epilogue;
// fp16's 11 significant bits give a 2^-10 product bound where bf16 would give
// 2^-7, with the same shared-memory footprint.
//
// Exactness: every value is either re-evaluated in the reference's order
// (IEEE binary32, .cl:239-249) or provably <= 0.  With
//   E(t,s) = kappa * ||t|| * ||window(s)|| + 2^-25 (||t||_1 / s_v + |window|_1 / s_t)
//            + 2^-22 (|SS_t/2| + |approx|)
// bounding |approx - reference| (fp16 rounding of both operands including
// subnormals, FP32 accumulation in any order, and the reference's own
// rounding), entries
// with approx + E > 0 go to the refinement list; the rest are stored as
// approx, which is < 0 like the reference value.  Every later decision reads
// such an entry only through "> 0" / "<= 0" tests (window argmax, check flag,
// overlap skip rules and parse), so the pursuit is unchanged.
#pragma once
#include <cuda_fp16.h>
#include "fbp_kernels.cuh"

namespace fbp {

constexpr int kTcThreads = 128;      // 4 warps: warp w owns TMEM lanes [32w, 32w+32)
constexpr int kTcM = 128;            // samples per tile

struct TcArgs {
    u32 n, C, K, L;
    u32 Cg2;                         // channel groups of 8, padded to even
    u32 Np;                          // templates padded to a multiple of 16
    u32 rows_pad;                    // strip rows (128 + L - 1) padded to 8
    u32 tmem_cols;
    float kappa_b;
    const float *v;                  // [C][n]
    const float *T;                  // [K][C][L] (exact refinement)
    const float *tss;                // [K]
    const float *tnorm;              // [K] ||t||_2
    const float *tabs;               // [K] ||t||_1
    const int *texp;                 // [K] power-of-two scale of template t's fp16 copy
    const uint4 *Tb;                 // [L][Cg2][Np] x 8 fp16 (scaled)
    u32 tb_bytes;
    const u32 *win;
    const u32 *n_win;
    float *Lk;                       // [K][n]
    u32 *ref_t, *ref_s;              // refinement list (one contiguous segment per tile)
    u32 *ref_count;
    u32 ref_cap;
    u32 *seg_s0, *seg_base, *seg_cnt;  // tile segments of the refinement list
    u32 *seg_count, *seg_overflow;
    u32 seg_cap;
    u32 *err;                        // non-zero: a bounded wait gave up
    u8 *apx;                         // [K][n] approximate-entry flags
    float *wn_s, *wa_s;              // [n] per-sample window norms
    float *bm_s;                     // [n] largest bound of a flagged entry of the sample
    float *wlb;                      // [W] largest lower bound over a window's entries
    signed char *kx_s;               // [n] per-sample fp16 scale exponent
    // overlap-table tiles (MODE 1): rows are the shifts b of a candidate window
    u32 S, nmax, stiles;
    const u32 *cand, *n_cand, *best_idx;
    const u8 *cskip;
    const float *NT;                 // [K][S]
    float *H;                        // [slot][K][S]
    int *kexp_tile;                  // [slot][stiles] voltage scale of each tile
};

__host__ __device__ inline size_t tc_smem_bytes(u32 L, u32 Cg2, u32 Np) {
    const size_t rows_pad = (kTcM + L - 1 + 7) / 8 * 8;
    return (size_t)L * Cg2 * Np * 16          // templates
           + rows_pad * Cg2 * 16              // voltage strip
           + rows_pad * 4 * 2                 // row energies / absolute sums, their prefix sums
           + 64                               // mbarriers, tmem address, scan scratch
           + (size_t)Np * 4;                  // per-template counters
}

__device__ __forceinline__ u32 smem_u32(const void *p) { return (u32)__cvta_generic_to_shared(p); }

// Exclusive scan over the 128 threads of the tensor-core kernel.
__device__ __forceinline__ u32 tc_block_excl_scan(u32 v, u32 *total, u32 *tmp) {
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u32 incl = warp_incl_scan(v);
    if (lane == 31) tmp[warp] = incl;
    __syncthreads();
    u32 off = 0, tot = 0;
    for (u32 w = 0; w < kTcThreads / 32; w++) {
        if (w < warp) off += tmp[w];
        tot += tmp[w];
    }
    __syncthreads();
    *total = tot;
    return off + incl - v;
}

// K-major, no swizzle: rows 16 B apart, 8-row groups SBO apart, K chunks LBO apart.
__device__ __forceinline__ u64 umma_desc(u32 saddr, u32 lbo, u32 sbo) {
    u64 d = 0;
    d |= (u64)((saddr >> 4) & 0x3FFF);
    d |= (u64)((lbo >> 4) & 0x3FFF) << 16;
    d |= (u64)((sbo >> 4) & 0x3FFF) << 32;
    d |= (u64)1 << 46;                         // descriptor version for sm_100
    return d;                                  // base offset 0, swizzle none
}

__device__ __forceinline__ void mbar_init(u32 bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ bool mbar_try_wait(u32 bar, u32 parity) {
    u32 ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}
// Bounded wait: gives up after `limit` polls (each poll may itself suspend).
__device__ __forceinline__ bool mbar_wait_bounded(u32 bar, u32 parity, u32 limit) {
    for (u32 i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// MODE 0: likelihood tiles (128 samples of a listed window).
// MODE 1: overlap tables -- tile = (candidate, 128 shifts b); the strip is the
//         candidate window [i0, i0+L) with zeros around it, so row b of the
//         product is the correlation of every template shifted by b - n_max
//         with the window (H of the fast overlap recheck, without refinement:
//         its error bound goes into the overlap intervals).
template <int MODE>
__global__ void __launch_bounds__(kTcThreads, 1)
k_lik_tc(TcArgs A) {
    extern __shared__ __align__(128) unsigned char tsm[];
    const u32 L = A.L, Cg2 = A.Cg2, Np = A.Np, rows_pad = A.rows_pad, n = A.n;
    unsigned char *Bs = tsm;
    unsigned char *As = Bs + (size_t)L * Cg2 * Np * 16;
    float *rowsq = (float *)(As + (size_t)rows_pad * Cg2 * 16);   // prefix of sum_c v^2 after the scan
    float *rowab = rowsq + rows_pad;                              // prefix of sum_c |v|
    u64 *bars = (u64 *)(rowab + rows_pad);     // [0] templates loaded, [1] MMA done
    u32 *tmem_slot = (u32 *)(bars + 2);
    u32 *seg_info = tmem_slot + 1;
    u32 *scan_tmp = seg_info + 1;              // 4 warps + total
    int *tile_exp = (int *)(scan_tmp + 5);     // power-of-two scale of this tile's voltage
    u32 *tcnt = (u32 *)(tile_exp + 3);         // [Np] per-template counters of the tile
    const u32 tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const u32 bar_b = smem_u32(&bars[0]), bar_mma = smem_u32(&bars[1]);
    const u32 kWaitLimit = 1u << 24;

    if (tid == 0) {
        mbar_init(bar_b, 1);
        mbar_init(bar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"(A.tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const u32 tmem = *tmem_slot;

    // templates: one bulk asynchronous copy global -> shared
    if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_b), "r"(A.tb_bytes)
                     : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(smem_u32(Bs)), "l"(A.Tb), "r"(A.tb_bytes), "r"(bar_b) : "memory");
    }
    bool ok = mbar_wait_bounded(bar_b, 0, kWaitLimit);
    ok = __syncthreads_and(ok);                  // block-uniform from here on
    if (!ok) {
        if (tid == 0) atomicExch(A.err, 1u);
        mbar_wait_bounded(bar_b, 0, kWaitLimit);  // let the copy land before leaving
    }

    // instruction descriptor: D f32, A/B f16, both K-major, M = 128, N = Np
    const u32 idesc = (1u << 4) | ((Np >> 3) << 17) | ((u32)(kTcM >> 4) << 24);
    const u32 lbo_a = rows_pad * 16, lbo_b = Np * 16;
    const u32 a_base = smem_u32(As), b_base = smem_u32(Bs);
    const float kappa_b = A.kappa_b;
    const u32 sub = MODE == 0 ? (L + kTcM - 1) / kTcM : A.stiles;   // tiles per window / candidate
    const u64 nitems = (u64)(MODE == 0 ? *A.n_win : *A.n_cand) * sub;
    u32 phase = 0;

    for (u64 item = blockIdx.x; ok && item < nitems; item += gridDim.x) {
        // strip row x holds sample s0 + x (MODE 1: signed, masked to [m_lo, m_hi))
        long long s0;
        u32 ew = 0, g = 0;
        long long m_lo = 0, m_hi = n;
        if (MODE == 0) {
            const u32 w = A.win[item / sub];
            s0 = (long long)w * L + (u32)(item % sub) * kTcM;
            ew = min((w + 1) * L, n);
        } else {
            g = (u32)(item / sub);
            if (A.cskip[g]) continue;
            const u32 i0 = A.best_idx[A.cand[g]];
            s0 = (long long)i0 - (long long)A.nmax + (long long)(item % sub) * kTcM;
            m_lo = i0;
            m_hi = (long long)i0 + L;
        }
        // ---- row sums (energy, absolute) and the tile's largest magnitude
        float mx = 0.0f;
        for (u32 x = tid; x < rows_pad; x += blockDim.x) {
            const long long pos = s0 + x;
            float e2 = 0.0f, ab = 0.0f;
            if (pos >= m_lo && pos < m_hi && pos < n)
                for (u32 c = 0; c < A.C; c++) {
                    const float f = A.v[(size_t)c * n + pos];
                    e2 = fmaf(f, f, e2);
                    ab += fabsf(f);
                    mx = fmaxf(mx, fabsf(f));
                }
            rowsq[x] = e2;
            rowab[x] = ab;
        }
        mx = warp_max_f(mx);
        if (lane == 0) scan_tmp[warp] = __float_as_uint(mx);
        __syncthreads();
        if (tid == 0) {
            float m = 0.0f;
            for (int q = 0; q < kTcThreads / 32; q++) m = fmaxf(m, __uint_as_float(scan_tmp[q]));
            int e = 0;
            if (m > 0.0f) {
                frexpf(m, &e);                       // m < 2^e
                e = 14 - e;                          // scaled magnitudes < 2^14
                e = max(-127, min(127, e));          // stored as int8 with the entries
            }
            *tile_exp = e;
            if (MODE == 1) A.kexp_tile[(size_t)g * sub + (u32)(item % sub)] = e;
        }
        __syncthreads();
        const int kexp = *tile_exp;
        // ---- stage the strip: rows x -> samples s0 + x, 8 fp16 channels per row
        for (u32 e = tid; e < rows_pad * Cg2; e += blockDim.x) {
            const u32 x = e % rows_pad, cg = e / rows_pad;
            const long long pos = s0 + x;
            const bool inside = pos >= m_lo && pos < m_hi && pos < n;
            u16 h[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const u32 c = cg * 8 + j;
                const float f = (c < A.C && inside) ? A.v[(size_t)c * n + pos] : 0.0f;
                h[j] = __half_as_ushort(__float2half_rn(ldexpf(f, kexp)));
            }
            uint4 q;
            q.x = ((u32)h[1] << 16) | h[0];
            q.y = ((u32)h[3] << 16) | h[2];
            q.z = ((u32)h[5] << 16) | h[4];
            q.w = ((u32)h[7] << 16) | h[6];
            *reinterpret_cast<uint4 *>(As + ((size_t)cg * rows_pad + x) * 16) = q;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        // ---- issue the MMAs: for each lag m, each channel pair j
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (u32 m = 0; m < L; m++) {
                for (u32 j = 0; j < Cg2 / 2; j++) {
                    const u64 da = umma_desc(a_base + 2 * j * lbo_a + m * 16, lbo_a, 128);
                    const u64 db = umma_desc(b_base + (m * Cg2 + 2 * j) * lbo_b, lbo_b, 128);
                    const u32 acc = (m | j) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                        ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(bar_mma) : "memory");
        }
        // ---- meanwhile: prefix sums of the row sums (warp 1: energies, warp 2: absolute)
        if (MODE == 0 && (warp == 1 || warp == 2)) {
            float *arr = warp == 1 ? rowsq : rowab;
            float carry = 0.0f;
            for (u32 x0 = 0; x0 < rows_pad; x0 += 32) {
                float val = (x0 + lane < rows_pad) ? arr[x0 + lane] : 0.0f;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const float y = __shfl_up_sync(0xffffffffu, val, o);
                    if (lane >= (u32)o) val += y;
                }
                __syncwarp();
                if (x0 + lane < rows_pad) arr[x0 + lane] = carry + val;
                carry += __shfl_sync(0xffffffffu, val, 31);
            }
        }
        const bool done = __syncthreads_and(mbar_wait_bounded(bar_mma, phase, kWaitLimit));
        if (!done) {
            if (tid == 0) atomicExch(A.err, 2u);
            mbar_wait_bounded(bar_mma, phase, kWaitLimit);   // MMAs must finish before TMEM is freed
            ok = false;
            break;
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (MODE == 1) {
            // H[g][t][b] = correlation - 0.5 * clipped energy, b = shift row
            const u32 row = warp * 32 + lane;
            const u32 b = (u32)(item % sub) * kTcM + row;
            for (u32 c0 = 0; c0 < Np; c0 += 16) {
                u32 r[16];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                    "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                      "=r"(r[14]), "=r"(r[15])
                    : "r"(tmem + ((warp * 32u) << 16) + c0));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (b < A.S) {
#pragma unroll
                    for (int q = 0; q < 16; q++) {
                        const u32 t = c0 + q;
                        if (t >= A.K) continue;
                        A.H[((size_t)g * A.K + t) * A.S + b] =
                            ldexpf(__uint_as_float(r[q]), -(kexp + A.texp[t])) - 0.5f * A.NT[(size_t)t * A.S + b];
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            continue;
        }
        // ---- epilogue: warp w reads rows 32w..32w+31 (one sample per thread)
        const u32 row = warp * 32 + lane;
        const u32 s = (u32)s0 + row;
        const bool in_win = s < ew && row < kTcM;
        float wn = 0.0f, wa = 0.0f;
        if (in_win) {
            const u32 hi_i = min(row + L, rows_pad) - 1;
            wn = sqrtf(fmaxf(rowsq[hi_i] - (row ? rowsq[row - 1] : 0.0f), 0.0f)) * 1.0001f + 1e-30f;
            wa = fmaxf(rowab[hi_i] - (row ? rowab[row - 1] : 0.0f), 0.0f) * 1.0001f + 1e-30f;
        }
        // phase 1: store the values whose sign is certain, mark the others
        u32 wantbits[8] = {0, 0, 0, 0, 0, 0, 0, 0};      // Np <= 256
        u32 nwant = 0;
        float lomax = 0.0f, bmax = 0.0f;                 // this sample's lower bounds / flagged bounds
        if (in_win) {                                    // interval data of this sample
            A.wn_s[s] = wn;
            A.wa_s[s] = wa;
            A.kx_s[s] = (signed char)kexp;
        }
        for (u32 c0 = 0; c0 < Np; c0 += 16) {
            u32 r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(tmem + ((warp * 32u) << 16) + c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const u32 t = c0 + q;
                if (!in_win || t >= A.K) continue;
                float *dst = A.Lk + (size_t)t * n + s;
                u8 *fl = A.apx + (size_t)t * n + s;
                if (s + L >= n) { *dst = 0.0f; *fl = 0; continue; }     // .cl:231-234
                const float tssv = A.tss[t];
                const int je = A.texp[t];
                const float approx = ldexpf(__uint_as_float(r[q]), -(kexp + je)) + tssv;
                const float sub = 2.98023223876953125e-08f *          // 2^-25: fp16 subnormal spacing / 2
                                  (ldexpf(A.tabs[t], -kexp) + ldexpf(wa, -je)) * 1.001f;
                const float E = kappa_b * A.tnorm[t] * wn + sub +
                                2.384185791015625e-07f * (fabsf(tssv) + fabsf(approx));
                lomax = fmaxf(lomax, approx - E);
                if (approx + E <= 0.0f) {            // certainly <= 0: only its sign is read
                    *dst = approx;
                    *fl = 0;
                } else if (approx - E > 0.0f) {      // certainly > 0: refined when a decision needs it
                    *dst = approx;
                    *fl = 1;
                    bmax = fmaxf(bmax, E);
                } else {                             // sign uncertain: refined now
                    wantbits[t >> 5] |= 1u << (t & 31);
                    nwant++;
                    *fl = 0;
                }
            }
        }
        if (in_win) {
            A.bm_s[s] = bmax;
            if (lomax > 0.0f) atomicMax(reinterpret_cast<int *>(A.wlb) + s / L, __float_as_int(lomax));
        }
        // phase 2: one contiguous segment of (template, sample) entries per
        // tile, ordered by template so the refinement shares template rows
        for (u32 t = tid; t < Np; t += blockDim.x) tcnt[t] = 0;
        __syncthreads();
        for (u32 wd = 0; wd < 8; wd++) {
            u32 bits = wantbits[wd];
            while (bits) {
                const u32 b = __ffs(bits) - 1;
                bits &= bits - 1;
                atomicAdd(&tcnt[wd * 32 + b], 1u);
            }
        }
        u32 seg_total;
        (void)tc_block_excl_scan(nwant, &seg_total, scan_tmp);
        if (tid == 0) {
            seg_info[0] = seg_total ? atomicAdd(A.ref_count, seg_total) : 0u;
            u32 off = 0;                            // template offsets inside the segment
            for (u32 t = 0; t < Np; t++) {
                const u32 c = tcnt[t];
                tcnt[t] = off;
                off += c;
            }
        }
        __syncthreads();
        const u32 seg_base = seg_info[0];
        if (seg_total && tid == 0 && seg_base + seg_total <= A.ref_cap) {
            const u32 si = atomicAdd(A.seg_count, 1u);
            if (si < A.seg_cap) {
                A.seg_s0[si] = (u32)s0;
                A.seg_base[si] = seg_base;
                A.seg_cnt[si] = seg_total;
            } else {
                atomicExch(A.seg_overflow, 1u);
            }
        }
        if (nwant && seg_base + seg_total <= A.ref_cap) {
            for (u32 wd = 0; wd < 8; wd++) {
                u32 bits = wantbits[wd];
                while (bits) {
                    const u32 b = __ffs(bits) - 1;
                    bits &= bits - 1;
                    const u32 t = wd * 32 + b;
                    const u32 p = seg_base + atomicAdd(&tcnt[t], 1u);
                    A.ref_t[p] = t;
                    A.ref_s[p] = s;
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(A.tmem_cols));
}

// Templates in the UMMA B layout: Tb[m][g][t] = 8 fp16 channels 8g..8g+7 of
// template t at lag m, scaled by 2^texp[t] (zero padding for channels >= C
// and t >= K).
__global__ void k_tc_pack_templates(const float *__restrict__ T, u32 K, u32 C, u32 L, u32 Cg2, u32 Np,
                                    const int *__restrict__ texp, uint4 *__restrict__ Tb) {
    const u64 total = (u64)L * Cg2 * Np;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (u64)gridDim.x * blockDim.x) {
        const u32 t = (u32)(e % Np), g = (u32)((e / Np) % Cg2), m = (u32)(e / ((u64)Np * Cg2));
        u16 h[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const u32 c = g * 8 + j;
            const float f = (t < K && c < C) ? ldexpf(T[((size_t)t * C + c) * L + m], texp[t]) : 0.0f;
            h[j] = __half_as_ushort(__float2half_rn(f));
        }
        uint4 q;
        q.x = ((u32)h[1] << 16) | h[0];
        q.y = ((u32)h[3] << 16) | h[2];
        q.z = ((u32)h[5] << 16) | h[4];
        q.w = ((u32)h[7] << 16) | h[6];
        Tb[e] = q;
    }
}

// Exact reference-order values of the refinement list
// (compute_maximum_likelihood, binary_pursuit.cl:216-252).  One tile
// segment per block; its entries are ordered by template.  The tile's
// voltage (all channels) is staged once; each warp takes 32 consecutive
// entries -- mostly one template, so the template reads are broadcasts --
// and every lane advances its own entry's chain in the reference's
// channel-major, lag-minor order.
constexpr int kRefThreads = 256;
__host__ __device__ inline size_t tc_refine_smem_bytes(u32 C, u32 L) {
    return ((size_t)C * (kTcM + L) + 8) * 4;
}
__global__ void __launch_bounds__(kRefThreads)
k_tc_refine(const float *__restrict__ v, u32 n, u32 C, const float *__restrict__ T, u32 K, u32 L,
            const float *__restrict__ tss, const u32 *__restrict__ ref_t, const u32 *__restrict__ ref_s,
            const u32 *__restrict__ seg_s0, const u32 *__restrict__ seg_base, const u32 *__restrict__ seg_cnt,
            const u32 *__restrict__ seg_count, u32 seg_cap, float *__restrict__ Lk) {
    extern __shared__ float rsm[];
    const u32 rl = kTcM + L;               // strip row length
    const u32 nseg = min(*seg_count, seg_cap);
    for (u32 sg = blockIdx.x; sg < nseg; sg += gridDim.x) {
        const u32 s0 = seg_s0[sg], base = seg_base[sg], cnt = seg_cnt[sg];
        __syncthreads();
        for (u32 x = threadIdx.x; x < C * rl; x += blockDim.x) {
            const u32 c = x / rl, i = x % rl, pos = s0 + i;
            rsm[x] = pos < n ? v[(size_t)c * n + pos] : 0.0f;
        }
        __syncthreads();
        for (u32 e = threadIdx.x; e < cnt; e += blockDim.x) {
            const u32 t = ref_t[base + e], so = ref_s[base + e] - s0;
            float acc = tss[t];
            for (u32 c = 0; c < C; c++) {
                const float *tp = T + ((size_t)t * C + c) * L;
                const float *sp = rsm + (size_t)c * rl + so;
                for (u32 i = 0; i < L; i++) acc = __fadd_rn(acc, __fmul_rn(__ldg(tp + i), sp[i]));
            }
            Lk[(size_t)t * n + s0 + so] = acc;
        }
    }
}

}  // namespace fbp
