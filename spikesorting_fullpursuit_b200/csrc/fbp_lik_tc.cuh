// Path (a) on the tensor cores: BF16 tcgen05 likelihood with exact refinement.
//
// likelihood[t][s] = -0.5*SS_t + sum_c sum_m T[t][c][m] * v[c][s+m]
// (compute_full_likelihood, binary_pursuit.cl:216-300) is the product of a
// Toeplitz voltage operand (rows = samples, K = (channel, lag)) and the
// template matrix.  The voltage strip of a tile lives in shared memory as
// rows of 8 channels (16 bytes, bf16): that is the K-major, no-swizzle
// canonical UMMA layout, and the operand for lag m is the same strip started
// m rows later -- so the contraction is L accumulating
// tcgen05.mma (M = 128 samples, N = templates, K = 16 channels) per channel
// pair, with no im2col.  Templates ([lag][channel group][template][8]) are
// copied into shared memory once per CTA with one bulk asynchronous copy.
// Accumulators are FP32 in tensor memory.
//
// Exactness: every value is either re-evaluated in the reference's order
// (IEEE binary32, .cl:239-249) or provably <= 0.  With
//   E(t,s) = kappa_b * ||t|| * ||window(s)|| + 2^-22 (|SS_t/2| + |approx|)
// bounding |approx - reference| (bf16 rounding of both operands, FP32
// accumulation in any order, and the reference's own rounding), entries
// with approx + E > 0 go to the refinement list; the rest are stored as
// approx, which is < 0 like the reference value.  Every later decision reads
// such an entry only through "> 0" / "<= 0" tests (window argmax, check flag,
// overlap skip rules and parse), so the pursuit is unchanged.
#pragma once
#include <cuda_bf16.h>
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
    const float *tnorm;              // [K]
    const uint4 *Tb;                 // [L][Cg2][Np] x 8 bf16
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
};

__host__ __device__ inline size_t tc_smem_bytes(u32 L, u32 Cg2, u32 Np) {
    const size_t rows_pad = (kTcM + L - 1 + 7) / 8 * 8;
    return (size_t)L * Cg2 * Np * 16          // templates
           + rows_pad * Cg2 * 16              // voltage strip
           + rows_pad * 4 * 2                 // row energies and their prefix sums
           + 64;                              // mbarriers, tmem address, scan scratch
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

__global__ void __launch_bounds__(kTcThreads, 1)
k_lik_tc(TcArgs A) {
    extern __shared__ __align__(128) unsigned char tsm[];
    const u32 L = A.L, Cg2 = A.Cg2, Np = A.Np, rows_pad = A.rows_pad, n = A.n;
    unsigned char *Bs = tsm;
    unsigned char *As = Bs + (size_t)L * Cg2 * Np * 16;
    float *rowsq = (float *)(As + (size_t)rows_pad * Cg2 * 16);
    float *wpre = rowsq + rows_pad;
    u64 *bars = (u64 *)(wpre + rows_pad);      // [0] templates loaded, [1] MMA done
    u32 *tmem_slot = (u32 *)(bars + 2);
    u32 *seg_info = tmem_slot + 1;
    u32 *scan_tmp = seg_info + 1;              // 4 warps + total
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

    // instruction descriptor: D f32, A/B bf16, both K-major, M = 128, N = Np
    const u32 idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((Np >> 3) << 17) | ((u32)(kTcM >> 4) << 24);
    const u32 lbo_a = rows_pad * 16, lbo_b = Np * 16;
    const u32 a_base = smem_u32(As), b_base = smem_u32(Bs);
    const float kappa_b = A.kappa_b;
    const u32 n_win = *A.n_win;
    const u32 sub = (L + kTcM - 1) / kTcM;       // 128-sample tiles per window
    u32 phase = 0;

    for (u64 item = blockIdx.x; ok && item < (u64)n_win * sub; item += gridDim.x) {
        const u32 w = A.win[item / sub];
        const u32 s0 = w * L + (u32)(item % sub) * kTcM;
        const u32 ew = min((w + 1) * L, n);
        // ---- stage the strip: rows x -> samples s0 + x, bf16 channels, row energies
        for (u32 e = tid; e < rows_pad * Cg2; e += blockDim.x) {
            const u32 x = e % rows_pad, g = e / rows_pad;
            const u32 pos = s0 + x;
            float f[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const u32 c = g * 8 + j;
                f[j] = (c < A.C && pos < n) ? A.v[(size_t)c * n + pos] : 0.0f;
            }
            uint4 q;
            q.x = ((u32)__bfloat16_as_ushort(__float2bfloat16_rn(f[1])) << 16) | __bfloat16_as_ushort(__float2bfloat16_rn(f[0]));
            q.y = ((u32)__bfloat16_as_ushort(__float2bfloat16_rn(f[3])) << 16) | __bfloat16_as_ushort(__float2bfloat16_rn(f[2]));
            q.z = ((u32)__bfloat16_as_ushort(__float2bfloat16_rn(f[5])) << 16) | __bfloat16_as_ushort(__float2bfloat16_rn(f[4]));
            q.w = ((u32)__bfloat16_as_ushort(__float2bfloat16_rn(f[7])) << 16) | __bfloat16_as_ushort(__float2bfloat16_rn(f[6]));
            *reinterpret_cast<uint4 *>(As + ((size_t)g * rows_pad + x) * 16) = q;
        }
        for (u32 x = tid; x < rows_pad; x += blockDim.x) {
            const u32 pos = s0 + x;
            float e2 = 0.0f;
            if (pos < n)
                for (u32 c = 0; c < A.C; c++) {
                    const float f = A.v[(size_t)c * n + pos];
                    e2 = fmaf(f, f, e2);
                }
            rowsq[x] = e2;
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
        // ---- meanwhile: window energies ||v[s .. s+L)||^2 by prefix sums (warp 1)
        if (warp == 1) {
            float carry = 0.0f;
            for (u32 x0 = 0; x0 < rows_pad; x0 += 32) {
                float val = (x0 + lane < rows_pad) ? rowsq[x0 + lane] : 0.0f;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const float y = __shfl_up_sync(0xffffffffu, val, o);
                    if (lane >= (u32)o) val += y;
                }
                if (x0 + lane < rows_pad) wpre[x0 + lane] = carry + val;
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
        // ---- epilogue: warp w reads rows 32w..32w+31 (one sample per thread)
        const u32 row = warp * 32 + lane;
        const u32 s = s0 + row;
        const bool in_win = s < ew && row < kTcM;
        float wn = 0.0f;
        if (in_win) {
            const float hi = wpre[min(row + L, rows_pad) - 1];
            const float lo = row ? wpre[row - 1] : 0.0f;
            wn = sqrtf(fmaxf(hi - lo, 0.0f)) * 1.0001f + 1e-30f;
        }
        // phase 1: store the provably-negative values, mark the others
        u32 wantbits[8] = {0, 0, 0, 0, 0, 0, 0, 0};      // Np <= 256
        u32 nwant = 0;
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
                if (s + L >= n) { *dst = 0.0f; continue; }               // .cl:231-234
                const float tssv = A.tss[t];
                const float approx = __uint_as_float(r[q]) + tssv;
                const float E = kappa_b * A.tnorm[t] * wn + 2.384185791015625e-07f * (fabsf(tssv) + fabsf(approx));
                if (approx + E > 0.0f) {
                    wantbits[t >> 5] |= 1u << (t & 31);
                    nwant++;
                } else {
                    *dst = approx;
                }
            }
        }
        // phase 2: one contiguous segment of (template, sample) entries per tile
        u32 seg_total;
        const u32 my_off = tc_block_excl_scan(nwant, &seg_total, scan_tmp);
        if (tid == 0) {
            seg_info[0] = seg_total ? atomicAdd(A.ref_count, seg_total) : 0u;
        }
        __syncthreads();
        const u32 seg_base = seg_info[0];
        if (seg_total && tid == 0 && seg_base + seg_total <= A.ref_cap) {
            const u32 si = atomicAdd(A.seg_count, 1u);
            if (si < A.seg_cap) {
                A.seg_s0[si] = s0;
                A.seg_base[si] = seg_base;
                A.seg_cnt[si] = seg_total;
            } else {
                atomicExch(A.seg_overflow, 1u);
            }
        }
        if (nwant && seg_base + seg_total <= A.ref_cap) {
            u32 p = seg_base + my_off;
            for (u32 wd = 0; wd < 8; wd++) {
                u32 bits = wantbits[wd];
                while (bits) {
                    const u32 b = __ffs(bits) - 1;
                    bits &= bits - 1;
                    A.ref_t[p] = wd * 32 + b;
                    A.ref_s[p] = s;
                    p++;
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(A.tmem_cols));
}

// Templates in the UMMA B layout: Tb[m][g][t] = 8 bf16 channels 8g..8g+7 of
// template t at lag m (zero padding for channels >= C and t >= K).
__global__ void k_tc_pack_templates(const float *__restrict__ T, u32 K, u32 C, u32 L, u32 Cg2, u32 Np,
                                    uint4 *__restrict__ Tb) {
    const u64 total = (u64)L * Cg2 * Np;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (u64)gridDim.x * blockDim.x) {
        const u32 t = (u32)(e % Np), g = (u32)((e / Np) % Cg2), m = (u32)(e / ((u64)Np * Cg2));
        u16 h[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const u32 c = g * 8 + j;
            const float f = (t < K && c < C) ? T[((size_t)t * C + c) * L + m] : 0.0f;
            h[j] = __bfloat16_as_ushort(__float2bfloat16_rn(f));
        }
        uint4 q;
        q.x = ((u32)h[1] << 16) | h[0];
        q.y = ((u32)h[3] << 16) | h[2];
        q.z = ((u32)h[5] << 16) | h[4];
        q.w = ((u32)h[7] << 16) | h[6];
        Tb[e] = q;
    }
}

// Exact reference-order values of the refinement list, one tile segment per
// block (compute_maximum_likelihood, binary_pursuit.cl:216-252): channel by
// channel, the tile's voltage row and all templates' channel row are staged
// in shared memory, and every entry's chain advances through that channel's
// lags -- the reference's channel-major, lag-minor order.  Each thread keeps
// up to kRefIlp independent chains.
constexpr int kRefThreads = 256;
constexpr int kRefIlp = 4;
__host__ __device__ inline size_t tc_refine_smem_bytes(u32 K, u32 L) {
    return ((size_t)K * L + kTcM + L + 8) * 4;
}
__global__ void __launch_bounds__(kRefThreads)
k_tc_refine(const float *__restrict__ v, u32 n, u32 C, const float *__restrict__ T, u32 K, u32 L,
            const float *__restrict__ tss, const u32 *__restrict__ ref_t, const u32 *__restrict__ ref_s,
            const u32 *__restrict__ seg_s0, const u32 *__restrict__ seg_base, const u32 *__restrict__ seg_cnt,
            const u32 *__restrict__ seg_count, u32 seg_cap, float *__restrict__ Lk) {
    extern __shared__ float rsm[];
    float *Ts = rsm;                     // [K][L] channel c of every template
    float *strip = rsm + (size_t)K * L;  // [kTcM + L] voltage of channel c from s0
    const u32 nseg = min(*seg_count, seg_cap);
    for (u32 sg = blockIdx.x; sg < nseg; sg += gridDim.x) {
        const u32 s0 = seg_s0[sg], base = seg_base[sg], cnt = seg_cnt[sg];
        for (u32 e0 = 0; e0 < cnt; e0 += blockDim.x * kRefIlp) {
            u32 tt[kRefIlp], ss[kRefIlp];
            float acc[kRefIlp];
            bool act[kRefIlp];
#pragma unroll
            for (int q = 0; q < kRefIlp; q++) {
                const u32 e = e0 + q * blockDim.x + threadIdx.x;
                act[q] = e < cnt;
                tt[q] = act[q] ? ref_t[base + e] : 0;
                ss[q] = act[q] ? ref_s[base + e] - s0 : 0;
                acc[q] = act[q] ? tss[tt[q]] : 0.0f;
            }
            for (u32 c = 0; c < C; c++) {
                __syncthreads();
                for (u32 x = threadIdx.x; x < K * L; x += blockDim.x) Ts[x] = T[((size_t)(x / L) * C + c) * L + x % L];
                for (u32 x = threadIdx.x; x < kTcM + L; x += blockDim.x) {
                    const u32 pos = s0 + x;
                    strip[x] = pos < n ? v[(size_t)c * n + pos] : 0.0f;
                }
                __syncthreads();
                const float *tp[kRefIlp], *sp[kRefIlp];
#pragma unroll
                for (int q = 0; q < kRefIlp; q++) {
                    tp[q] = Ts + (size_t)tt[q] * L;
                    sp[q] = strip + ss[q];
                }
                for (u32 i = 0; i < L; i++) {
#pragma unroll
                    for (int q = 0; q < kRefIlp; q++) acc[q] = __fadd_rn(acc[q], __fmul_rn(tp[q][i], sp[q][i]));
                }
            }
#pragma unroll
            for (int q = 0; q < kRefIlp; q++)
                if (act[q]) Lk[(size_t)tt[q] * n + s0 + ss[q]] = acc[q];
        }
    }
}

}  // namespace fbp
