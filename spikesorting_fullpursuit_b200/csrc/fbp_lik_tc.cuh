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
// Exactness.  With
//   E(t,s) = kappa * ||t|| * ||window(s)|| + 2^-25 (||t||_1 / s_v + |window|_1 / s_t) * 1.001
//            + kappa_s * |SS_t/2| + 2^-22 |approx|
// bounding |approx - reference| -- fp16 rounding of both operands including
// subnormals, FP32 accumulation in any order, and the reference's own
// recursive sum (.cl:239-249), whose running value starts at -SS_t/2 and so
// carries up to n*u*|SS_t/2| besides n*u*sum|t v| -- every entry is one of
//   certainly <= 0  (approx + E <= 0): stored as approx; only its sign is
//                   ever read (window argmax, check flag, overlap skip rules
//                   and parse);
//   certainly > 0   (approx - E > 0): stored as approx with a flag; its
//                   reference value is computed when a decision needs it
//                   (see LazyLk in fbp_kernels.cuh);
//   uncertain       : queued and re-evaluated in the reference's order.
// So the pursuit reads the reference's values wherever they matter.
#pragma once
#include <cuda_fp16.h>
#include "fbp_kernels.cuh"

namespace fbp {

// Warp roles of the tensor-core kernel: warps 0-7 stage tiles (the fp16
// strip, row sums, per-tile factors), warp 8 issues the MMAs, warps 9-16
// drain accumulators (epilogue).  Epilogue warp w reads TMEM lanes
// [32(w%4), 32(w%4)+32) -- the lanes a warp may access -- and every other
// 16-column chunk starting at 16 * ((w-9)/4).
constexpr int kTcProdWarps = 8;
constexpr int kTcMmaWarp = kTcProdWarps;
constexpr int kTcEpiWarps = 8;
constexpr int kTcEpiWarp0 = kTcMmaWarp + 1;
constexpr int kTcThreads = 32 * (kTcProdWarps + 1 + kTcEpiWarps);
constexpr int kTcProdThreads = 32 * kTcProdWarps;
constexpr int kTcEpiThreads = 32 * kTcEpiWarps;
constexpr int kTcM = 128;            // samples per tile
// Polls of the waits a CTA makes before it exits: for its template copy to
// land and for MMAs it issued to finish.  These stay long even when a test
// shortens the pipeline waits: shared memory and TMEM are released only
// after the asynchronous work into them is done.
constexpr u32 kTcDrainPolls = 1u << 24;

struct TcArgs {
    u32 n, C, K, L;                  // C: the group's channels; K: the group's templates
    const u32 *trow;                 // [K] template of each group column (NULL: column = template)
    u32 Kall;                        // templates of the chunk (row stride of the overlap tables)
    u32 tstride;                     // floats between consecutive templates in T (all channels)
    u32 Cg2;                         // channel groups of 8, padded to even
    u32 Np;                          // templates padded to a multiple of 16
    u32 rows_pad;                    // strip rows (128 + L - 1) padded to 8
    u32 nbuf;                        // strip / accumulator buffers (2: staging overlaps the epilogue)
    u32 tmem_cols;
    float kappa_b;                   // bound per unit of ||t|| ||window||
    float kappa_s;                   // bound per unit of |SS_t / 2|
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
    u32 wpt;                         // MODE 0: windows per tile (> 1: tiles are aligned blocks of
                                     // wpt windows, of which the listed ones are computed)
    const u8 *active;                // [W] window listed in this pass (block tiles)
    float *Lk;                       // [K][n]
    u32 *ref_t, *ref_s;              // refinement list (one contiguous segment per tile)
    unsigned long long *refseg;      // entries queued (high half) and tile segments (low half)
    u32 ref_cap;
    u32 *seg_s0, *seg_base, *seg_cnt;  // tile segments of the refinement list
    u32 *seg_grp;                      // template group of each segment
    u32 grp;                           // this launch's template group
    u32 *seg_overflow;
    u32 seg_cap;
    u32 *err;                        // non-zero: a bounded wait gave up
    u32 wait_polls;                  // polls before a pipeline wait gives up (final drains use kTcDrainPolls)
    float *dbgE;                     // MODE 0, testing: when set, the bound E of every entry ([K][n])
    u8 *apx;                         // [K][n] approximate-entry flags
    float *wn_s, *wa_s;              // [n] per-sample window norms
    float *bm_s;                     // [n] largest bound of a flagged entry of the sample
    float *wlb;                      // [W] largest lower bound over a window's entries
    float *umax;                     // [W][Kall] largest upper bound of a template's entries in a window
    u8 *wpos;                        // [W] some entry of the window is > 0
    signed char *kx_s;               // [n] per-sample fp16 scale exponent
    // overlap-table tiles (MODE 1): rows are the shifts b of a candidate window
    u32 S, nmax, stiles;
    const u32 *cand, *n_cand, *best_idx;
    const u8 *cskip;
    const float *NT;                 // [K][S]
    float *H;                        // [slot][K][S]
    int *kexp_tile;                  // [slot][stiles] voltage scale of each tile
};

// Shared memory of the tensor-core kernel (nbuf strip buffers).
struct TcSmem {
    size_t Bs, As, rowsq, rowab, tsc, tsa, ctk, ctb, ctss, cta, ctrow, tinfo, bars, misc, tcnt, bmh, total;
};
__host__ __device__ inline TcSmem tc_smem_layout(u32 L, u32 Cg2, u32 Np, u32 nbuf) {
    const size_t rows_pad = (kTcM + L - 1 + 7) / 8 * 8;
    TcSmem m;
    size_t o = 0;
    m.Bs = o;    o += (size_t)L * Cg2 * Np * 16;            // templates
    m.As = o;    o += (size_t)nbuf * rows_pad * Cg2 * 16;   // voltage strips
    m.rowsq = o; o += (size_t)nbuf * rows_pad * 4;          // row energies -> prefix sums
    m.rowab = o; o += (size_t)nbuf * rows_pad * 4;          // row absolute sums -> prefix sums
    m.tsc = o;   o += (size_t)nbuf * Np * 4;                // per tile: 2^-(kexp + texp[t]) (0: use ldexpf)
    m.tsa = o;   o += (size_t)nbuf * Np * 4;                // per tile: 2^-25 * 1.001 * |t|_1 * 2^-kexp
    m.ctk = o;   o += (size_t)Np * 4;                       // kappa * ||t||
    m.ctb = o;   o += (size_t)Np * 4;                       // 2^-25 * 1.001 * 2^-texp[t]
    m.ctss = o;  o += (size_t)Np * 4;                       // -SS_t / 2
    m.cta = o;   o += (size_t)Np * 4;                       // kappa_s * |SS_t / 2|
    m.ctrow = o; o += (size_t)Np * 4;                       // template of each column
    m.tinfo = o; o += (size_t)nbuf * 32;                    // per buffer: s0, ew, g, kexp
    o = (o + 7) / 8 * 8;
    m.bars = o;  o += 8 * 8;                                // full[2], empty[2], staged[2], templates
    m.misc = o;  o += 64;                                   // tmem slot, segment info, reductions, abort
    m.tcnt = o;  o += (size_t)Np * 4;                       // per-template counters of the tile
    m.bmh = o;   o += (size_t)kTcM * 4;                     // second half's largest flagged bound per row
    m.total = o;
    return m;
}
__host__ __device__ inline size_t tc_smem_bytes(u32 L, u32 Cg2, u32 Np, u32 nbuf = 1) {
    return tc_smem_layout(L, Cg2, Np, nbuf).total;
}

__device__ __forceinline__ u32 smem_u32(const void *p) { return (u32)__cvta_generic_to_shared(p); }

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
__device__ __forceinline__ void named_bar(u32 id, u32 count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
// Named barrier that also returns the OR of a predicate over its threads
// (the same value in every thread, so a loop can leave it uniformly).
__device__ __forceinline__ bool named_bar_or(u32 id, u32 count, bool v) {
    u32 r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r) : "r"((u32)v), "r"(id), "r"(count) : "memory");
    return r != 0;
}
__device__ __forceinline__ void mbar_arrive(u32 bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// Bounded wait: gives up after `limit` polls (each poll may itself suspend).
__device__ __forceinline__ bool mbar_wait_bounded(u32 bar, u32 parity, u32 limit) {
    for (u32 i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Max over the warp of 16 values per lane, all 16 columns at once: at each
// step a lane keeps half of its columns (the half picked by its lane bit)
// and takes the partner's values for them, so 8 + 4 + 2 + 1 shuffles leave
// column (lane >> 1) & 15 reduced over the lanes that differ in bits 1-4;
// a last shuffle adds bit 0.  Returns that column's maximum.
__device__ __forceinline__ float warp_max16(float (&v)[16], u32 lane) {
#pragma unroll
    for (int o = 16, h = 8; h >= 1; o >>= 1, h >>= 1) {
        const bool hi = (lane & (u32)o) != 0;
#pragma unroll
        for (int i = 0; i < h; i++) {
            const float send = hi ? v[i] : v[i + h];
            const float keep = hi ? v[i + h] : v[i];
            v[i] = fmaxf(keep, __shfl_xor_sync(0xffffffffu, send, o));
        }
    }
    return fmaxf(v[0], __shfl_xor_sync(0xffffffffu, v[0], 1));
}

// The same for 8 values per lane: after 4 + 2 + 1 shuffles column
// (lane >> 2) & 7 is reduced over lane bits 2-4, two more add bits 0-1.
__device__ __forceinline__ float warp_max8(float (&v)[8], u32 lane) {
#pragma unroll
    for (int o = 16, h = 4; h >= 1; o >>= 1, h >>= 1) {
        const bool hi = (lane & (u32)o) != 0;
#pragma unroll
        for (int i = 0; i < h; i++) {
            const float send = hi ? v[i] : v[i + h];
            const float keep = hi ? v[i + h] : v[i];
            v[i] = fmaxf(keep, __shfl_xor_sync(0xffffffffu, send, o));
        }
    }
    const float a = fmaxf(v[0], __shfl_xor_sync(0xffffffffu, v[0], 2));
    return fmaxf(a, __shfl_xor_sync(0xffffffffu, a, 1));
}

// CW consecutive accumulator columns of this warp's 32 TMEM lanes.
template <int CW>
__device__ __forceinline__ void tmem_ld(u32 (&r)[CW], u32 taddr) {
    if constexpr (CW == 16) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
              "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
              "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
    } else {
        static_assert(CW == 8, "8 or 16 columns");
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                       "=r"(r[7])
                     : "r"(taddr));
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

template <int CW> struct ColW { static constexpr int value = CW; };

// MODE 0: likelihood tiles (128 samples of a listed window).
// MODE 1: overlap tables -- tile = (candidate, 128 shifts b); the strip is the
//         candidate window [i0, i0+L) with zeros around it, so row b of the
//         product is the correlation of every template shifted by b - n_max
//         with the window (H of the fast overlap recheck, without refinement:
//         its error bound goes into the overlap intervals).
//
// Persistent, one CTA per SM.  Producer warps stage tile i into strip buffer
// i % nbuf; the MMA warp multiplies it into accumulator i % nbuf while the
// producers stage tile i+1 and the epilogue warps drain tile i-1.
// staged[b] completes when the producers have written buffer b; full[b] when
// the MMA warp has published it (one arrive) and its MMAs are done
// (tcgen05.commit); empty[b] when all epilogue warps have read accumulator b
// and the buffer's row sums.  Every wait is bounded; a wait that gives up
// sets err and the abort flag, and every role leaves its loop.
template <int MODE>
__global__ void __launch_bounds__(kTcThreads, 1)
k_lik_tc(const TcArgs *__restrict__ gargs, u32 ngroups) {
    // CTAs are split over the template groups in proportion (the first
    // gridDim % ngroups groups get one more); a CTA loads its group's
    // templates once and takes that group's tiles bi, bi + cnt, ...
    u32 gi, bi, cnt;
    {
        const u32 b = blockIdx.x, base = gridDim.x / ngroups, rem = gridDim.x % ngroups;
        if (base == 0) {
            gi = b; bi = 0; cnt = 1;
        } else if (b < rem * (base + 1)) {
            gi = b / (base + 1); bi = b % (base + 1); cnt = base + 1;
        } else {
            const u32 b2 = b - rem * (base + 1);
            gi = rem + b2 / base; bi = b2 % base; cnt = base;
        }
        if (gi >= ngroups) return;
    }
    const TcArgs &A = gargs[gi];
    extern __shared__ __align__(128) unsigned char tsm[];
    const u32 L = A.L, Cg2 = A.Cg2, Np = A.Np, rows_pad = A.rows_pad, n = A.n, nbuf = A.nbuf;
    const TcSmem lay = tc_smem_layout(L, Cg2, Np, nbuf);
    unsigned char *Bs = tsm + lay.Bs;
    float *rowsq_all = (float *)(tsm + lay.rowsq), *rowab_all = (float *)(tsm + lay.rowab);
    float *tsc_all = (float *)(tsm + lay.tsc), *tsa_all = (float *)(tsm + lay.tsa);
    float *ctk = (float *)(tsm + lay.ctk), *ctb = (float *)(tsm + lay.ctb);
    float *ctss = (float *)(tsm + lay.ctss), *cta = (float *)(tsm + lay.cta);
    u32 *ctrow = (u32 *)(tsm + lay.ctrow);
    int *tinfo = (int *)(tsm + lay.tinfo);                 // [nbuf][8]: s0 lo, s0 hi, ew, g, kexp
    u64 *bars = (u64 *)(tsm + lay.bars);
    u32 *misc = (u32 *)(tsm + lay.misc);
    u32 *tmem_slot = misc, *seg_info = misc + 1, *pred = misc + 4, *abort_flag = misc + 12;
    u32 *tcnt = (u32 *)(tsm + lay.tcnt);
    float *bmh = (float *)(tsm + lay.bmh);
    const u32 tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const u32 wlim = A.wait_polls;                   // pipeline waits (a test may shorten them)
    // MODE 0 tiles: one listed window (L > 64 may take several tiles), or
    // with wpt > 1 the aligned block of windows [wpt q, wpt q + wpt) when
    // one of them is listed (short templates: both windows' rows in one tile)
    const u32 wpt = MODE == 0 ? A.wpt : 1u;
    const u32 Wn = (n + L - 1) / L;
    const u32 sub = MODE == 0 ? (wpt > 1 ? 1u : (L + kTcM - 1) / kTcM) : A.stiles;   // tiles per window / candidate
    const u64 nitems = MODE == 0 ? (wpt > 1 ? (u64)((Wn + wpt - 1) / wpt) : (u64)*A.n_win * sub)
                                 : (u64)*A.n_cand * sub;
    if ((u64)bi >= nitems) return;                   // no tile for this CTA: no set-up at all
    // every role skips the same items: candidates without a table (MODE 1),
    // blocks without a listed window (MODE 0, wpt > 1)
    auto live = [&](u64 item) -> bool {
        if (MODE == 1) return !A.cskip[(u32)(item / sub)];
        if (wpt <= 1) return true;
        const u32 w0 = (u32)item * wpt;
        bool any = false;
        for (u32 k = 0; k < wpt && w0 + k < Wn; k++) any |= A.active[w0 + k] != 0;
        return any;
    };
    auto bar_full = [&](u32 b) { return smem_u32(&bars[b]); };
    auto bar_empty = [&](u32 b) { return smem_u32(&bars[2 + b]); };
    auto bar_staged = [&](u32 b) { return smem_u32(&bars[4 + b]); };
    const u32 bar_tb = smem_u32(&bars[6]);

    if (tid == 0) {
        for (u32 b = 0; b < 2; b++) {
            mbar_init(bar_full(b), 2);                // MMA warp arrive + MMA commit
            mbar_init(bar_empty(b), kTcEpiWarps);     // one arrive per epilogue warp
            mbar_init(bar_staged(b), 1);              // producers (after their barrier)
        }
        mbar_init(bar_tb, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"(A.tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // per-chunk template constants (epilogue); tile counters start at zero
    for (u32 t = tid; t < Np; t += blockDim.x) {
        tcnt[t] = 0;
        const bool real = t < A.K;
        const u32 gt = real ? (A.trow ? A.trow[t] : t) : 0u;
        ctrow[t] = gt;
        if (MODE == 0) {
            ctk[t] = real ? A.kappa_b * A.tnorm[gt] : 0.0f;
            ctb[t] = real ? 2.98023223876953125e-08f * 1.001f * ldexpf(1.0f, -A.texp[gt]) : 0.0f;
            ctss[t] = real ? A.tss[gt] : 0.0f;
            cta[t] = real ? A.kappa_s * fabsf(A.tss[gt]) : 0.0f;
        }
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const u32 tmem = *tmem_slot;

    // templates: one bulk asynchronous copy global -> shared
    if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_tb), "r"(A.tb_bytes)
                     : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(smem_u32(Bs)), "l"(A.Tb), "r"(A.tb_bytes), "r"(bar_tb) : "memory");
    }

    u32 lfp0 = 2u, lfp1 = 2u;                         // MMA thread: parity of the last commit per buffer
    bool tb_ready = false;                           // MMA thread: the template copy has landed

    if (warp < kTcProdWarps) {
        // =========================== producer ===========================
        const u32 pt = tid;                          // 0..255
        u32 use0 = 0u, use1 = 0u;                    // uses of each buffer so far
        u32 it = 0;
        for (u64 item = bi; item < nitems; item += cnt) {
            long long s0;
            u32 ew = 0, g = 0;
            long long m_lo = 0, m_hi = n;
            if (!live(item)) continue;
            if (MODE == 0 && wpt > 1) {
                const u32 w0 = (u32)item * wpt;
                s0 = (long long)w0 * L;
                ew = (u32)min((u64)(w0 + wpt) * L, (u64)n);
            } else if (MODE == 0) {
                const u32 w = A.win[item / sub];
                s0 = (long long)w * L + (u32)(item % sub) * kTcM;
                ew = min((w + 1) * L, n);
            } else {
                g = (u32)(item / sub);
                const u32 i0 = A.best_idx[A.cand[g]];
                s0 = (long long)i0 - (long long)A.nmax + (long long)(item % sub) * kTcM;
                m_lo = i0;
                m_hi = (long long)i0 + L;
            }
            const u32 b = nbuf == 2 ? (it & 1u) : 0u;
            it++;
            const u32 ub = b ? use1 : use0;
            if (ub > 0) {
                bool ok = mbar_wait_bounded(bar_empty(b), (ub - 1) & 1u, wlim);
                if (!ok) { atomicExch(A.err, 3u); atomicExch(abort_flag, 1u); }
            }
            if (named_bar_or(1, kTcProdThreads, *(volatile u32 *)abort_flag != 0)) break;
            float *rowsq = rowsq_all + (size_t)b * rows_pad, *rowab = rowab_all + (size_t)b * rows_pad;
            unsigned char *As = tsm + lay.As + (size_t)b * rows_pad * Cg2 * 16;
            // ---- the next tile's voltage rows into L2 (one 128-byte line per thread)
            {
                const u64 nx = item + cnt;
                if (MODE == 0 && nx < nitems) {
                    const long long p0 = wpt > 1 ? (long long)nx * wpt * L
                                                 : (long long)A.win[nx / sub] * L + (u32)(nx % sub) * kTcM;
                    const u32 lines = (rows_pad + 31) / 32;
                    for (u32 e = pt; e < A.C * lines; e += kTcProdThreads) {
                        const u32 c = e / lines, ln = e % lines;
                        const long long pos = p0 + (long long)ln * 32;
                        if (pos < n) asm volatile("prefetch.global.L2 [%0];" ::"l"(A.v + (size_t)c * n + pos));
                    }
                }
            }
            // ---- row sums (energy, absolute) and the tile's largest magnitude
            float mx = 0.0f;
            for (u32 x = pt; x < rows_pad; x += kTcProdThreads) {
                const long long pos = s0 + x;
                float e2 = 0.0f, ab = 0.0f;
                if (pos >= m_lo && pos < m_hi && pos < n) {
                    const float *vp = A.v + pos;
                    u32 c = 0;
                    for (; c + 8 <= A.C; c += 8) {
                        float f[8];
#pragma unroll
                        for (int j = 0; j < 8; j++) f[j] = vp[(size_t)(c + j) * n];
#pragma unroll
                        for (int j = 0; j < 8; j++) {
                            e2 = fmaf(f[j], f[j], e2);
                            ab += fabsf(f[j]);
                            mx = fmaxf(mx, fabsf(f[j]));
                        }
                    }
                    for (; c < A.C; c++) {
                        const float f = vp[(size_t)c * n];
                        e2 = fmaf(f, f, e2);
                        ab += fabsf(f);
                        mx = fmaxf(mx, fabsf(f));
                    }
                }
                rowsq[x] = e2;
                rowab[x] = ab;
            }
            mx = warp_max_f(mx);
            if (lane == 0) pred[warp] = __float_as_uint(mx);
            named_bar(1, kTcProdThreads);
            int kexp = 0;
            {
                float m = 0.0f;
                for (int q = 0; q < kTcProdWarps; q++) m = fmaxf(m, __uint_as_float(pred[q]));
                if (m > 0.0f) {
                    int e;
                    frexpf(m, &e);                   // m < 2^e
                    kexp = max(-126, min(126, 14 - e));   // scaled magnitudes < 2^14
                }
            }
            if (MODE == 1 && pt == 0) A.kexp_tile[(size_t)g * sub + (u32)(item % sub)] = kexp;
            // ---- the strip: rows x -> samples s0 + x, 8 fp16 channels per row
            const float kscale = ldexpf(1.0f, kexp);         // exact: |kexp| <= 126
            for (u32 e = pt; e < rows_pad * Cg2; e += kTcProdThreads) {
                const u32 x = e % rows_pad, cg = e / rows_pad;
                const long long pos = s0 + x;
                const bool inside = pos >= m_lo && pos < m_hi && pos < n;
                u16 h[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const u32 c = cg * 8 + j;
                    const float f = (c < A.C && inside) ? A.v[(size_t)c * n + pos] : 0.0f;
                    h[j] = __half_as_ushort(__float2half_rn(__fmul_rn(f, kscale)));
                }
                uint4 q;
                q.x = ((u32)h[1] << 16) | h[0];
                q.y = ((u32)h[3] << 16) | h[2];
                q.z = ((u32)h[5] << 16) | h[4];
                q.w = ((u32)h[7] << 16) | h[6];
                *reinterpret_cast<uint4 *>(As + ((size_t)cg * rows_pad + x) * 16) = q;
            }
            // ---- per-tile template factors; prefix sums of the row sums
            for (u32 t = pt; t < Np; t += kTcProdThreads) {
                float sc = 0.0f;
                if (t < A.K) {
                    const u32 gt = ctrow[t];
                    const int ex = -(kexp + A.texp[gt]);
                    if (ex >= -149 && ex <= 127) sc = ldexpf(1.0f, ex);   // exact power of two
                    if (MODE == 0) tsa_all[(size_t)b * Np + t] =
                                       2.98023223876953125e-08f * 1.001f * ldexpf(A.tabs[gt], -kexp);
                }
                tsc_all[(size_t)b * Np + t] = sc;
            }
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
            if (pt == 0) {
                int *ti = tinfo + b * 8;
                ti[0] = (int)(s0 & 0xffffffffll);
                ti[1] = (int)(s0 >> 32);
                ti[2] = (int)ew;
                ti[3] = (int)g;
                ti[4] = kexp;
                ti[5] = (int)(item % sub);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            named_bar(1, kTcProdThreads);
            if (pt == 0) mbar_arrive(bar_staged(b));   // release: the barrier ordered every write
            if (b) use1++; else use0++;
        }
    } else if (warp == kTcMmaWarp) {
        // =========================== MMA issue ===========================
        // instruction descriptor: D f32, A/B f16, both K-major, M = 128, N = Np
        const u32 idesc = (1u << 4) | ((Np >> 3) << 17) | ((u32)(kTcM >> 4) << 24);
        const u32 lbo_a = rows_pad * 16, lbo_b = Np * 16;
        // descriptors differ only in their start address (16-byte units,
        // low 14 bits; every operand lies below 256 KB of shared memory)
        const u64 db0 = umma_desc(smem_u32(Bs), lbo_b, 128);
        u32 use0 = 0u, use1 = 0u;
        u32 it = 0;
        for (u64 item = bi; item < nitems; item += cnt) {
            if (!live(item)) continue;
            const u32 b = nbuf == 2 ? (it & 1u) : 0u;
            it++;
            const u32 ub = b ? use1 : use0;
            u32 ok = 1;
            if (lane == 0) {
                ok = mbar_wait_bounded(bar_staged(b), ub & 1u, wlim) ? 1u : 0u;
                if (!ok) atomicExch(A.err, 4u);
                if (ok && !tb_ready) {
                    tb_ready = mbar_wait_bounded(bar_tb, 0, wlim);
                    if (!tb_ready) { atomicExch(A.err, 1u); ok = 0; }
                }
                if (!ok) atomicExch(abort_flag, 1u);
                if (*(volatile u32 *)abort_flag) ok = 0;
            }
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) break;
            if (lane == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const u64 da0 = umma_desc(smem_u32(tsm + lay.As + (size_t)b * rows_pad * Cg2 * 16), lbo_a, 128);
                const u32 dst = tmem + b * Np;
                // The issuing thread is the limit (each MMA of a small N is
                // shorter than the instructions between two issues), so the
                // inner loop only steps both descriptors by constants: lag m
                // moves the strip one row (16 B) and the templates one lag
                // block.  The first MMA overwrites the accumulator.
                const u64 bstep = (u64)Cg2 * Np;
                u32 acc = 0u;
                for (u32 j = 0; j < Cg2 / 2; j++) {
                    u64 da = da0 + (u64)(2 * j * rows_pad);
                    u64 db = db0 + (u64)(2 * j * Np);
#pragma unroll 4
                    for (u32 m = 0; m < L; m++) {
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                            ::"r"(dst), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
                        acc = 1u;
                        da += 1u;
                        db += bstep;
                    }
                }
                mbar_arrive(bar_full(b));
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             ::"r"(bar_full(b)) : "memory");
                if (b) lfp1 = ub & 1u; else lfp0 = ub & 1u;
            }
            __syncwarp();
            if (b) use1++; else use0++;
        }
    } else {
        // =========================== epilogue ===========================
        const u32 et = tid - 32 * kTcEpiWarp0;       // 0..255
        const u32 ew_ = warp - kTcEpiWarp0;          // 0..7
        const u32 quad = warp & 3u;                  // TMEM lanes [32 quad, 32 quad + 32)
        const u32 half = ew_ >> 2;                   // column chunks 16 * (half + 2k)
        const u32 row = quad * 32 + lane;
        u32 use0 = 0u, use1 = 0u;
        u32 it = 0;
        for (u64 item = bi; item < nitems; item += cnt) {
            if (!live(item)) continue;
            const u32 b = nbuf == 2 ? (it & 1u) : 0u;
            it++;
            const bool ok = mbar_wait_bounded(bar_full(b), (b ? use1 : use0) & 1u, wlim);
            if (b) use1++; else use0++;
            if (!ok) { atomicExch(A.err, 2u); atomicExch(abort_flag, 1u); }
            if (named_bar_or(2, kTcEpiThreads, *(volatile u32 *)abort_flag != 0)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int *ti = tinfo + b * 8;
            const long long s0 = (long long)(((unsigned long long)(u32)ti[1] << 32) | (u32)ti[0]);
            const u32 ewin = (u32)ti[2], g = (u32)ti[3];
            const int kexp = ti[4];
            const u32 subi = (u32)ti[5];
            const float *tsc = tsc_all + (size_t)b * Np;
            const u32 acc0 = tmem + ((quad * 32u) << 16) + b * Np;
            if (MODE == 1) {
                // H[g][t][b] = correlation - 0.5 * clipped energy, b = shift row
                const u32 brow = subi * kTcM + row;
                auto table_cols = [&](auto cwc, u32 c0) {
                    constexpr int CW = decltype(cwc)::value;
                    u32 r[CW];
                    tmem_ld<CW>(r, acc0 + c0);
                    if (brow < A.S) {
#pragma unroll
                        for (int q = 0; q < CW; q++) {
                            const u32 t = c0 + q;
                            if (t >= A.K) continue;
                            const u32 gt = ctrow[t];
                            const float a = __uint_as_float(r[q]);
                            const float sc = tsc[t];
                            const float x = sc != 0.0f ? __fmul_rn(a, sc) : ldexpf(a, -(kexp + A.texp[gt]));
                            A.H[((size_t)g * A.Kall + gt) * A.S + brow] = x - 0.5f * A.NT[(size_t)gt * A.S + brow];
                        }
                    }
                };
                if (Np == 16) {
                    table_cols(ColW<8>{}, 8 * half);       // both warps of the quadrant: 8 columns each
                } else {
                    for (u32 c0 = 16 * half; c0 < Np; c0 += 32) table_cols(ColW<16>{}, c0);
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(bar_empty(b));
                continue;
            }
            // ---- MODE 0 epilogue: one sample per TMEM lane
            const float *rowsq = rowsq_all + (size_t)b * rows_pad, *rowab = rowab_all + (size_t)b * rows_pad;
            const float *tsa = tsa_all + (size_t)b * Np;
            const u32 s = (u32)s0 + row;
            // block tiles: rows of a window that is not listed keep the values
            // an earlier pass left (the reference recomputes listed windows only)
            const bool in_win = s < ewin && row < kTcM && (wpt <= 1 || A.active[s / L] != 0);
            float wn = 0.0f, wa = 0.0f;
            if (in_win) {
                const u32 hi_i = min(row + L, rows_pad) - 1;
                wn = sqrtf(fmaxf(rowsq[hi_i] - (row ? rowsq[row - 1] : 0.0f), 0.0f)) * 1.0001f + 1e-30f;
                wa = fmaxf(rowab[hi_i] - (row ? rowab[row - 1] : 0.0f), 0.0f) * 1.0001f + 1e-30f;
            }
            if (in_win && half == 0) {                   // interval data of this sample
                A.wn_s[s] = wn;
                A.wa_s[s] = wa;
                A.kx_s[s] = (signed char)kexp;
            }
            // phase 1: every entry gets its approximation and flag; the ones
            // whose sign is uncertain are marked for refinement (which
            // overwrites them before anything reads them).  Branch-free, and
            // every index is known at compile time (no local memory).
            u32 wantbits[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // Np <= 256: word k holds chunks k of both halves
            float lomax = 0.0f, bmax = 0.0f;
            const bool tail = s + L >= n;                // .cl:231-234
            // this warp's rows lie in windows wlo..whi (one window per tile
            // when wpt == 1; with block tiles L >= 32, so at most two)
            const u32 wlo = wpt > 1 ? ((u32)s0 + 32u * quad) / L : (u32)(s0 / L);
            const u32 whi = wpt > 1 ? ((u32)s0 + 32u * quad + 31u) / L : wlo;
            const u32 myw = s / L;
            bool anypos = false;
            // One chunk of CW columns starting at c0; its uncertain entries
            // set bits `shift`.. of `word`.  CW = 16: the two warps of a
            // quadrant take alternate 16-column chunks; groups of exactly 16
            // templates use CW = 8, so both warps drain 8 columns each.
            auto chunk = [&](auto cwc, u32 c0, u32 &word, u32 shift) {
                constexpr int CW = decltype(cwc)::value;
                float uq[CW];
#pragma unroll
                for (int q = 0; q < CW; q++) uq[q] = 0.0f;
                u32 r[CW];
                tmem_ld<CW>(r, acc0 + c0);
                u32 cw = 0;
                if (in_win) {
#pragma unroll
                for (int q = 0; q < CW; q++) {
                    const u32 t = c0 + q;
                    // padding columns (t >= K) are computed and dropped, so the
                    // loop has no exit and its shared-memory reads can be issued early
                    const bool real = t < A.K;
                    const u32 gt = ctrow[t];
                    float *dst = A.Lk + (size_t)gt * n + s;
                    u8 *fl = A.apx + (size_t)gt * n + s;
                    const float a = __uint_as_float(r[q]);
                    const float sc = tsc[t];
                    const float approx = __fadd_rn(sc != 0.0f ? __fmul_rn(a, sc) : ldexpf(a, -(kexp + A.texp[gt])),
                                                   ctss[t]);
                    // E = kappa ||t|| ||w|| + 2^-25 (|t|_1 / s_v + |w|_1 / s_t) * 1.001
                    //     + kappa_s |SS/2| + 2^-22 |approx|
                    const float E = fmaf(ctk[t], wn, fmaf(ctb[t], wa, tsa[t]) + cta[t] +
                                                         2.384185791015625e-07f * fabsf(approx));
                    const bool pos = approx - E > 0.0f;      // certainly > 0: refined when a decision needs it
                    const bool neg = approx + E <= 0.0f;     // certainly <= 0: only its sign is read
                    lomax = real ? fmaxf(lomax, approx - E) : lomax;
                    bmax = (real && pos) ? fmaxf(bmax, E) : bmax;
                    cw |= (real && !tail && !pos && !neg) ? (1u << q) : 0u;
                    if (real) {
                        *dst = tail ? 0.0f : approx;
                        *fl = (!tail && pos) ? (u8)1 : (u8)0;
                        if (A.dbgE) A.dbgE[(size_t)gt * n + s] = tail ? 0.0f : E;
                    }
                    uq[q] = (real && !tail) ? fmaxf(0.0f, approx + E) : 0.0f;
                    anypos |= real && !tail && pos;
                }
                if (tail) lomax = 0.0f, bmax = 0.0f;
                word |= cw << shift;
                }
                // per (window, template): the largest upper bound over the
                // tile's rows -- the CW columns reduced over the warp together
                {
                    constexpr u32 per = 32 / CW;               // lanes holding one column's result
                    const u32 col = (lane / per) & (CW - 1);
                    float vv[CW];
#pragma unroll
                    for (int q = 0; q < CW; q++) vv[q] = myw == wlo ? uq[q] : 0.0f;
                    float u;
                    if constexpr (CW == 16) u = warp_max16(vv, lane); else u = warp_max8(vv, lane);
                    if ((lane % per) == 0 && u > 0.0f && c0 + col < A.K)
                        atomicMax(reinterpret_cast<int *>(A.umax) + (size_t)wlo * A.Kall + ctrow[c0 + col],
                                  __float_as_int(u));
                    if (whi != wlo) {                    // uniform in the warp
#pragma unroll
                        for (int q = 0; q < CW; q++) vv[q] = myw == whi ? uq[q] : 0.0f;
                        float u2;
                        if constexpr (CW == 16) u2 = warp_max16(vv, lane); else u2 = warp_max8(vv, lane);
                        if ((lane % per) == 0 && u2 > 0.0f && c0 + col < A.K)
                            atomicMax(reinterpret_cast<int *>(A.umax) + (size_t)whi * A.Kall + ctrow[c0 + col],
                                      __float_as_int(u2));
                    }
                }
            };
            if (Np == 16) {
                // bit t of word 0 is column t, as phase 2 decodes it
                chunk(ColW<8>{}, 8 * half, wantbits[0], 8 * half);
            } else {
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const u32 c0 = 16 * half + 32 * k;
                    if (c0 >= Np) break;                 // uniform in the warp
                    chunk(ColW<16>{}, c0, wantbits[k], 16 * half);
                }
            }
            if (__any_sync(0xffffffffu, anypos && myw == wlo) && lane == 0) A.wpos[wlo] = 1;
            if (whi != wlo && __any_sync(0xffffffffu, anypos && myw == whi) && lane == 0) A.wpos[whi] = 1;
            // accumulator b and the row sums are no longer needed
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(bar_empty(b));
            if (in_win && lomax > 0.0f) atomicMax(reinterpret_cast<int *>(A.wlb) + s / L, __float_as_int(lomax));
            if (half == 1) bmh[row] = bmax;
            u32 nwant = 0;
#pragma unroll
            for (int wd = 0; wd < 8; wd++) nwant += __popc(wantbits[wd]);
            const bool anywant = named_bar_or(2, kTcEpiThreads, nwant != 0);   // also publishes bmh
            // largest flagged bound of the sample over every template group
            // (reset when its window is listed for recomputation)
            if (half == 0 && in_win) {
                const float bmv = fmaxf(bmax, bmh[row]);
                if (bmv > 0.0f) atomicMax(reinterpret_cast<int *>(A.bm_s) + s, __float_as_int(bmv));
            }
            if (anywant) {
                // phase 2: one contiguous segment of (template, sample)
                // entries per tile, ordered by template so the refinement
                // shares template rows (tcnt is zero here)
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    u32 bits = wantbits[k];
                    while (bits) {                       // word k: chunk k of each half
                        const u32 bb = __ffs(bits) - 1;
                        bits &= bits - 1;
                        atomicAdd(&tcnt[32 * k + (bb & 15) + 16 * (bb >> 4)], 1u);
                    }
                }
                named_bar(2, kTcEpiThreads);
                if (ew_ == 0) {
                    // template offsets: lane l scans templates [8l, 8l+8)
                    u32 c[8], sum = 0;
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const u32 t = lane * 8 + i;
                        c[i] = t < Np ? tcnt[t] : 0u;
                        sum += c[i];
                    }
                    const u32 incl = warp_incl_scan(sum);
                    u32 off = incl - sum;
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const u32 t = lane * 8 + i;
                        if (t < Np) tcnt[t] = off;
                        off += c[i];
                    }
                    const u32 total = __shfl_sync(0xffffffffu, incl, 31);
                    if (lane == 0) {
                        // one atomic reserves the entries and the segment slot
                        const unsigned long long old =
                            atomicAdd(A.refseg, ((unsigned long long)total << 32) | 1ull);
                        const u32 base = (u32)(old >> 32), si = (u32)old;
                        seg_info[0] = base;
                        seg_info[1] = total;
                        seg_info[2] = 0;
                        if (base + total <= A.ref_cap && si < A.seg_cap) {
                            A.seg_s0[si] = (u32)s0;
                            A.seg_base[si] = base;
                            A.seg_cnt[si] = total;
                            A.seg_grp[si] = A.grp;
                            seg_info[2] = 1;
                        } else {
                            atomicExch(A.seg_overflow, 1u);
                        }
                    }
                }
                named_bar(2, kTcEpiThreads);
                const u32 seg_base = seg_info[0];
                if (seg_info[2]) {
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        u32 bits = wantbits[k];
                        while (bits) {
                            const u32 bb = __ffs(bits) - 1;
                            bits &= bits - 1;
                            const u32 t = 32 * k + (bb & 15) + 16 * (bb >> 4);
                            const u32 p = seg_base + atomicAdd(&tcnt[t], 1u);
                            A.ref_t[p] = t;
                            A.ref_s[p] = s;
                        }
                    }
                }
                named_bar(2, kTcEpiThreads);         // tcnt / seg_info are done with
                for (u32 t = et; t < Np; t += kTcEpiThreads) tcnt[t] = 0;
            }
        }
    }
    __syncthreads();
    if (tid == 32 * kTcMmaWarp) {
        // the template copy must land before this CTA's shared memory is released
        if (!tb_ready) mbar_wait_bounded(bar_tb, 0, kTcDrainPolls);
        // MMAs must finish before their TMEM is freed
        if (*(volatile u32 *)abort_flag) {
            if (lfp0 < 2u) mbar_wait_bounded(bar_full(0), lfp0, kTcDrainPolls);
            if (lfp1 < 2u) mbar_wait_bounded(bar_full(1), lfp1, kTcDrainPolls);
        }
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(A.tmem_cols));
}

// Templates in the UMMA B layout: Tb[m][g][t] = 8 fp16 channels 8g..8g+7
// (of the group's range, starting at channel clo) of template trow[t] at lag
// m, scaled by 2^texp (zero padding for channels >= Cg and columns >= K).
__global__ void k_tc_pack_templates(const float *__restrict__ T, u32 K, u32 Call, u32 clo, u32 Cg, u32 L,
                                    u32 Cg2, u32 Np, const int *__restrict__ texp, const u32 *__restrict__ trow,
                                    uint4 *__restrict__ Tb) {
    const u64 total = (u64)L * Cg2 * Np;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (u64)gridDim.x * blockDim.x) {
        const u32 t = (u32)(e % Np), g = (u32)((e / Np) % Cg2), m = (u32)(e / ((u64)Np * Cg2));
        const u32 gt = t < K ? (trow ? trow[t] : t) : 0u;
        u16 h[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const u32 c = g * 8 + j;
            const float f = (t < K && c < Cg) ? ldexpf(T[((size_t)gt * Call + clo + c) * L + m], texp[gt]) : 0.0f;
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

// The refinement list (entries whose tensor-core interval straddles 0).
// One tile segment per block; its entries are ordered by template (so the
// template reads of neighbouring warps hit the same lines); a warp takes one
// entry, its lanes reading the voltage coalesced:
//   1. its lanes form X = -SS_t/2 + sum t*v and S = |SS_t/2| + sum |t*v| in
//      double (each product exact, the sums' own error negligible);
//      the reference value R (compute_maximum_likelihood,
//      binary_pursuit.cl:216-252) satisfies |R - X| <= gamma * S;
//   2. X + gamma S <= 0: R <= 0, stored as float(X) (only its sign is read);
//      X - gamma S > 0: R > 0, stored as float(X) and flagged approximate --
//      the lazy bound E of the entry covers gamma * S, so its reference
//      value is computed when a decision needs it;
//   3. otherwise the warp computes R itself: lanes form the products (each
//      rounded as in the reference), lane 0 adds them in the reference's
//      order.
constexpr int kRefThreads = 256;
__host__ __device__ inline size_t tc_refine_smem_bytes(u32 C, u32 L) {
    (void)C; (void)L;
    return (size_t)(kRefThreads / 32) * kWarpChunk * 4;
}
__global__ void __launch_bounds__(kRefThreads)
k_tc_refine(const float *__restrict__ vall, u32 n, u32 Call, u32 Cmax, const float *__restrict__ Tall, u32 K,
            u32 L, const float *__restrict__ tss, const u32 *__restrict__ ref_t, const u32 *__restrict__ ref_s,
            const u32 *__restrict__ seg_s0, const u32 *__restrict__ seg_base, const u32 *__restrict__ seg_cnt,
            const u32 *__restrict__ seg_grp, const u32 *__restrict__ gdesc, const u32 *__restrict__ tperm,
            const u32 *__restrict__ seg_count, u32 seg_cap, float *__restrict__ Lk, LazyLk z, double gamma,
            u64 *__restrict__ n_seq, u8 *__restrict__ wpos, const u32 *__restrict__ overflow, u32 ref_cap) {
    extern __shared__ float rsm[];
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *wbuf = rsm + (size_t)warp * kWarpChunk;
    // A tile whose entries did not fit reserved its segment but wrote no
    // record of it; the FP32 kernel then redoes the whole pass, so nothing
    // here is needed (and the unwritten records must not be read).
    if (*overflow) return;
    const u32 nseg = min(*seg_count, seg_cap);
    const u32 tstride = Call * L;          // floats between templates in T
    u32 nseq = 0;
    for (u32 sg = blockIdx.x; sg < nseg; sg += gridDim.x) {
        const u32 s0 = seg_s0[sg], base = seg_base[sg], cnt = seg_cnt[sg];
        if (base > ref_cap || cnt > ref_cap - base) continue;   // never true for a written record
        // the segment's template group: columns t0.., channels [clo, clo + C)
        const u32 gi = seg_grp[sg];
        const u32 t0 = gdesc[3 * gi], clo = gdesc[3 * gi + 1], C = gdesc[3 * gi + 2];
        const float *v = vall + (size_t)clo * n;
        const float *T = Tall + (size_t)clo * L;
        const u32 *trow = tperm ? tperm + t0 : nullptr;
        const u32 CL = C * L;
        for (u32 e = warp; e < cnt; e += kRefThreads / 32) {
            const u32 t = trow ? trow[ref_t[base + e]] : ref_t[base + e], so = ref_s[base + e] - s0;
            const float *tp = T + (size_t)t * tstride;      // the group's channels of template t
            double X = 0.0, S = 0.0;
            for (u32 q = lane; q < CL; q += 32) {
                const u32 c = q / L, i = q - c * L;
                const double p = (double)__ldg(tp + q) * (double)__ldg(v + (size_t)c * n + s0 + so + i);
                X += p;
                S += fabs(p);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                X += __shfl_xor_sync(0xffffffffu, X, o);
                S += __shfl_xor_sync(0xffffffffu, S, o);
            }
            X += (double)tss[t];
            S += fabs((double)tss[t]);
            const double bnd = gamma * S;
            const size_t idx = (size_t)t * n + s0 + so;
            if (X + bnd <= 0.0 || X - bnd > 0.0) {
                if (lane == 0) {
                    const float xf = (float)X;
                    Lk[idx] = xf;
                    if (X - bnd > 0.0) {                 // certainly > 0: refined on demand
                        z.apx[idx] = 1;
                        wpos[(s0 + so) / L] = 1;
                        const u32 s = s0 + so;
                        atomicMax(reinterpret_cast<int *>(const_cast<float *>(z.bm)) + s,
                                  __float_as_int(lazy_bound(z, t, s, xf)));
                    }
                }
                continue;
            }
            // sign still uncertain: the reference's own sum
            float acc = tss[t];
            for (u32 q0 = 0; q0 < CL; q0 += kWarpChunk) {
                const u32 m = min(kWarpChunk, CL - q0);
                for (u32 k = lane; k < m; k += 32) {
                    const u32 q = q0 + k, c = q / L, i = q - c * L;
                    wbuf[k] = __fmul_rn(__ldg(tp + q), __ldg(v + (size_t)c * n + s0 + so + i));
                }
                __syncwarp();
                if (lane == 0) acc = warp_chain(acc, wbuf, m);
                __syncwarp();
            }
            if (lane == 0) {
                Lk[idx] = acc;
                if (acc > 0.0f) wpos[(s0 + so) / L] = 1;
                nseq++;
            }
        }
    }
    if (n_seq && nseq) atomicAdd(n_seq, (u64)nseq);
}

}  // namespace fbp
