// Path (a) on the tensor cores, wide tiles: the likelihood of every listed
// window as one tcgen05 contraction per (channel, 16-lag block) with
// M = 128 = 16 templates x 8 sample shifts and N = 256 blocks of 8 samples.
//
// likelihood[t][s] = -0.5*SS_t + sum_c sum_m T[t][c][m] * v[c][s+m]
// (compute_full_likelihood, binary_pursuit.cl:216-300).  Write s = s0 + 8u + d
// (d < 8) and j = m + d.  Then
//     sum_m T[t][c][m] v[c][s+m] = sum_j A[(t,d)][j] * B[u][j],
//     A[(t,d)][j] = T[t][c][j-d]  (zero outside 0 <= j-d < L),
//     B[u][j]     = v[c][s0 + 8u + j],
// with j < 16 * nkc, nkc = ceil((L + 7) / 16).  B is the channel's voltage
// stream itself: in the K-major no-swizzle UMMA layout a row is 16 bytes
// (8 fp16 samples), so rows 16 bytes apart (SBO 128 per 8 rows) and K halves
// 16 bytes apart (LBO 16) make row u start at sample 8u and read 16 samples.
// No im2col, and one MMA does 128 x 256 x 16 products where the
// sample-major kernel (fbp_lik_tc.cuh) does 128 x (templates in a group) x 16.
// A (the shifted templates) is packed once per chunk (k_tcw_pack) and
// streamed per channel into a ring of shared-memory stages with one bulk
// asynchronous copy.  The channel's fp32 voltage reaches a staging slot by
// coalesced 4-byte asynchronous copies, kWDepth - 1 channels ahead, and the
// producers convert it to fp16 into the stage.  Accumulators are FP32 in
// tensor memory (two tiles of 256 columns).
//
// The stream.  A pass lists windows w (ascending).  Their outputs are laid
// end to end: listed window i of the list starts at stream position
//     pos_i = i * L + R_i * (L - 1),
// R_i = the number of runs of consecutive windows before it, so a run is
// contiguous and every run is followed by L - 1 positions that continue its
// recording samples (the lags of its last outputs).  Those positions, and
// whatever lies past the last run, compute values that are dropped.  A tile
// is 2048 consecutive stream positions; dense passes fill it with ~33
// windows of L = 61, isolated windows still use about half of it.
//
// Exactness is the argument of fbp_lik_tc.cuh: the same bound E per entry
// (fp16 operands after exact power-of-two scaling, FP32 accumulation in any
// order -- a zero product adds and rounds nothing, so the count of rounded
// terms is the template support times L -- and the reference's recursive
// sum), the same three classes of entries and the same refinement list.
// The tile's voltage scale comes from a per-window bound on |v| over all
// channels (vwmax, kept by k_residual), covering every sample a kept output
// multiplies by a non-zero template value; other staged samples are clamped
// to the fp16 range, so no inf reaches a product with a zero template value.
#pragma once
#include <cuda_fp16.h>
#include <type_traits>
#include "fbp_lik_tc.cuh"

namespace fbp {

constexpr u32 kWN = 256;                 // MMA N: blocks of 8 samples per tile
constexpr u32 kWPos = 8 * kWN;           // 2048 stream positions per tile
constexpr u32 kWTwMax = 136;             // listed windows a tile can touch (L >= kWMinL)
constexpr u32 kWMinL = 16;
constexpr u32 kWMaxStages = 8;
constexpr u32 kWATile = 4096;            // one A tile: 128 rows x 16 lags x fp16
constexpr u32 kWDepth = 3;               // channels of voltage in flight (fp32 staging slots)
constexpr u32 kWTail = 0x80000000u;      // stream table: a kept output in the zeroed tail (n < 2^31)

__host__ __device__ inline u32 tcw_nkc(u32 L) { return (L + 7 + 15) / 16; }
__host__ __device__ inline u32 tcw_px(u32 L) { return kWPos + 16 * tcw_nkc(L); }   // staged positions

struct TcwArgs {
    u32 n, Cg, nt, L, nkc, ns, px, Kall, W;
    const u32 *trow;                 // [nt] template of each group column
    float kappa_b, kappa_s;
    const float *v;                  // channel clo of the recording ([Cg][n] from there)
    const float *tss, *tnorm, *tabs;
    const int *texp;
    const unsigned char *Aw;         // [Cg][nkc] A tiles of this group
    const float *vwmax;              // [W + 2] largest |v| of each window over all channels
    const u32 *win, *n_win;          // the pass's window list
    const u32 *pos, *first, *n_stiles;   // stream position of each listed window; first listed
                                         // window of each tile; tiles of the stream
    float *Lk;                       // [Kall][n]
    u8 *apx;                         // [Kall][n]
    float *dbgE;                     // testing: when set, the bound E of every entry ([Kall][n])
    float *wn_s, *wa_s;              // [n] this group's window norms
    signed char *kx_s;               // [n] this group's fp16 scale exponents
    float *bm_s, *wlb, *umax;
    u8 *wpos;
    u32 *ref_t, *ref_s;
    unsigned long long *refseg;
    u32 ref_cap;
    u32 *seg_s0, *seg_base, *seg_cnt, *seg_grp;
    u32 grp;
    u32 *seg_overflow;
    u32 seg_cap;
    u32 *err;
    u32 wait_polls;
};

static_assert(sizeof(TcwArgs) % 4 == 0, "TcwArgs is copied as 32-bit words");
struct TcwSmem {
    size_t args, ring, stage, a_bytes, vst, spos, wnwa, wrel, tw, cw, tf, ti, psq, pab, tpos, twin, xs, xe, ct, bars,
        misc, tcnt, total;
};
__host__ __device__ inline TcwSmem tcw_smem_layout(u32 L, u32 ns) {
    const size_t nkc = tcw_nkc(L), px = tcw_px(L);
    TcwSmem m;
    m.a_bytes = nkc * kWATile;
    m.stage = align_up(m.a_bytes + align_up(px * 2, 16), 128);
    size_t o = 0;
    m.args = o;  o += align_up(sizeof(TcwArgs), 128);     // the launch arguments (shared-memory copy)
    m.ring = o;  o += ns * m.stage;                       // A tiles + voltage stream per channel
    m.vst = o;   o += (size_t)kWDepth * px * 4;            // producers: fp32 voltage of the next channels
    m.spos = o;  o += 2 * (size_t)kWPos * 4;               // per tile: sample of a kept output, else ~0
    m.wnwa = o;  o += 2 * (size_t)kWPos * 8;               // per tile: window L2 / L1 norms
    m.wrel = o;  o += 2 * (size_t)kWPos;                   // per tile: table entry of a kept output, else 0xff
    m.tw = o;    o += 2 * (size_t)kWTwMax * 4;             // per tile: window of each table entry
    m.cw = o;    o += 2 * 16 * 4;                          // per tile, per 128 positions: first | last entry << 16
    m.tf = o;    o += 2 * 32 * 4;                          // per tile: tsc[16], tsa[16]
    m.ti = o;    o += 2 * 16;                              // per tile: kexp
    o = align_up(o, 8);
    m.psq = o;   o += (px + 1) * 8;                        // producers: prefix sums of row energies
    m.pab = o;   o += (px + 1) * 8;                        //            and of row absolute sums
    m.tpos = o;  o += (size_t)(kWTwMax + 1) * 4;           //            tile table: stream position
    m.twin = o;  o += (size_t)(kWTwMax + 1) * 4;           //            and window of each entry
    m.xs = o;    o += (px - kWPos) * 4;                    //            samples of the positions past 2048
    m.xe = o;    o += 2 * (px - kWPos) * 4;                //            and their energy / absolute sums
    m.ct = o;    o += 16 * 4 * 5;                          // template constants
    o = align_up(o, 8);
    m.bars = o;  o += (size_t)(2 * ns + 9) * 8;
    m.misc = o;  o += 256;
    m.tcnt = o;  o += 16 * 4;
    m.total = o;
    return m;
}

__device__ __forceinline__ void mbar_expect_tx(u32 bar, u32 bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ u32 named_bar_popc(u32 id, u32 count, bool v) {
    u32 r;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.popc.u32 %0, %2, %3, p;\n\t}"
        : "=r"(r) : "r"((u32)v), "r"(id), "r"(count) : "memory");
    return r;
}
__device__ __forceinline__ double warp_incl_scan_d(double v, u32 lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= (u32)o) v += y;
    }
    return v;
}
// 4-byte asynchronous copy global -> shared; src_bytes 0 writes a zero
// (nothing is read)
__device__ __forceinline__ void cp_async4(u32 dst, const float *src, u32 src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ u16 half_bits_clamped(float f) {
    return __half_as_ushort(__float2half_rn(fminf(fmaxf(f, -65504.0f), 65504.0f)));
}

// Persistent, one CTA per SM, 17 warps: 8 producers (tile tables, voltage
// stream per channel, window norms), 1 MMA warp, 8 epilogue warps (two per
// TMEM lane quadrant, one half of the 256 columns each).  The launch
// arguments are copied into shared memory first.  Barriers:
//   stage_full[s]  producers wrote the stream (one arrive) and the A copy landed (tx);
//   stage_empty[s] the MMAs that read stage s are done (tcgen05.commit);
//   acc_full[b]    the tile's MMAs are done (commit);
//   acc_empty[b]   the epilogue read accumulator b (one arrive per epilogue warp);
//   info_full[b]   the producers wrote tile b's tables and norms (one arrive);
//   buf_empty[b]   the epilogue is done with tile b's tables (one arrive per warp).
// Every wait is bounded; a wait that gives up sets err and the abort flag.
__global__ void __launch_bounds__(kTcThreads, 1)
k_lik_tcw(const TcwArgs *__restrict__ gargs, u32 ngroups) {
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
    const TcwArgs &Ag = gargs[gi];
    const u32 ntiles = *Ag.n_stiles;
    if (bi >= ntiles) return;                        // no tile for this CTA: no set-up at all
    extern __shared__ __align__(128) unsigned char wsm[];
    // the roles read their arguments from a shared-memory copy (a reload
    // costs a shared-memory access, not a global one)
    for (u32 i = threadIdx.x; i < (u32)(sizeof(TcwArgs) / 4); i += blockDim.x)
        reinterpret_cast<u32 *>(wsm)[i] = reinterpret_cast<const u32 *>(&Ag)[i];
    const TcwArgs &A = *reinterpret_cast<const TcwArgs *>(wsm);   // valid after the first __syncthreads
    const u32 L = Ag.L, nkc = Ag.nkc, ns = Ag.ns, px = Ag.px, n = Ag.n, Cg = Ag.Cg;
    const TcwSmem lay = tcw_smem_layout(L, ns);
    unsigned char *ring = wsm + lay.ring;
    u32 *spos_all = (u32 *)(wsm + lay.spos);
    float2 *wnwa_all = (float2 *)(wsm + lay.wnwa);
    u8 *wrel_all = wsm + lay.wrel;
    u32 *tw_all = (u32 *)(wsm + lay.tw);
    u32 *cw_all = (u32 *)(wsm + lay.cw);
    float *tf_all = (float *)(wsm + lay.tf);
    int *ti_all = (int *)(wsm + lay.ti);
    double *psq = (double *)(wsm + lay.psq), *pab = (double *)(wsm + lay.pab);
    int *tpos = (int *)(wsm + lay.tpos);
    u32 *twin = (u32 *)(wsm + lay.twin);
    u32 *xs = (u32 *)(wsm + lay.xs);
    float *xe2 = (float *)(wsm + lay.xe), *xab = xe2 + (px - kWPos);
    float *ctk = (float *)(wsm + lay.ct), *ctb = ctk + 16, *ctss = ctk + 32, *cta = ctk + 48;
    u32 *ctrow = (u32 *)(ctk + 64);
    u64 *bars = (u64 *)(wsm + lay.bars);
    u32 *misc = (u32 *)(wsm + lay.misc);
    u32 *tmem_slot = misc, *seg_info = misc + 1, *abort_flag = misc + 4;
    float *pred = (float *)(misc + 8);               // [8] producer warp maxima
    double *dsum = (double *)(misc + 16);            // [16] producer warp sums (two arrays)
    u32 *tcnt = (u32 *)(wsm + lay.tcnt);
    const u32 tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const u32 wlim = Ag.wait_polls;
    auto bar_sfull = [&](u32 s) { return smem_u32(&bars[s]); };
    auto bar_sempty = [&](u32 s) { return smem_u32(&bars[ns + s]); };
    auto bar_afull = [&](u32 b) { return smem_u32(&bars[2 * ns + b]); };
    auto bar_aempty = [&](u32 b) { return smem_u32(&bars[2 * ns + 2 + b]); };
    auto bar_ifull = [&](u32 b) { return smem_u32(&bars[2 * ns + 4 + b]); };
    auto bar_bempty = [&](u32 b) { return smem_u32(&bars[2 * ns + 6 + b]); };
    const u32 bar_fin = smem_u32(&bars[2 * ns + 8]);

    if (tid == 0) {
        for (u32 s = 0; s < ns; s++) {
            mbar_init(bar_sfull(s), 1);
            mbar_init(bar_sempty(s), 1);
        }
        for (u32 b = 0; b < 2; b++) {
            mbar_init(bar_afull(b), 1);
            mbar_init(bar_aempty(b), kTcEpiWarps);
            mbar_init(bar_ifull(b), 1);
            mbar_init(bar_bempty(b), kTcEpiWarps);
        }
        mbar_init(bar_fin, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"(2 * kWN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    for (u32 t = tid; t < 16; t += blockDim.x) {
        tcnt[t] = 0;
        const bool real = t < Ag.nt;
        const u32 gt = real ? Ag.trow[t] : 0u;
        ctrow[t] = gt;
        ctk[t] = real ? Ag.kappa_b * Ag.tnorm[gt] : 0.0f;
        ctb[t] = real ? 2.98023223876953125e-08f * 1.001f * ldexpf(1.0f, -Ag.texp[gt]) : 0.0f;
        ctss[t] = real ? Ag.tss[gt] : 0.0f;
        cta[t] = real ? Ag.kappa_s * fabsf(Ag.tss[gt]) : 0.0f;
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const u32 tmem = *tmem_slot;
    u32 gstage = 0;                                  // producers / MMA: stages used so far

    if (warp < kTcProdWarps) {
        // =========================== producers ===========================
        const u32 pt = tid;                          // 0..255
        const u32 m = *A.n_win;
        const u32 nB = px - kWPos;                   // staged positions past 2048
        const bool hasB = 8 * pt < nB;               // this thread packs 8 of them
        float *vst = (float *)(wsm + lay.vst);       // [kWDepth][px] fp32 voltage (cp.async)
        u32 use0 = 0u, use1 = 0u;
        u32 it = 0;
        for (u32 q = bi; q < ntiles; q += cnt, it++) {
            const u32 b = it & 1u;
            const u32 ub = b ? use1 : use0;
            if (ub > 0 && !mbar_wait_bounded(bar_bempty(b), (ub - 1) & 1u, wlim)) {
                atomicExch(A.err, 13u);
                atomicExch(abort_flag, 1u);
            }
            if (named_bar_or(1, kTcProdThreads, *(volatile u32 *)abort_flag != 0)) break;
            u32 *spos = spos_all + (size_t)b * kWPos;
            float2 *wnwa = wnwa_all + (size_t)b * kWPos;
            u8 *wrel = wrel_all + (size_t)b * kWPos;
            u32 *tw = tw_all + (size_t)b * kWTwMax;
            u32 *cw = cw_all + b * 16;
            float *tsc = tf_all + b * 32, *tsa = tsc + 16;
            // ---- the tile's table: listed windows whose outputs or lags meet
            //      stream positions [Q0, Q0 + px)
            const long long Q0 = (long long)q * kWPos;
            const u32 i_lo = A.first[q];
            bool in = false;
            if (pt <= kWTwMax) {
                const u32 i = i_lo + pt;
                in = i < m && (long long)A.pos[i] < Q0 + (long long)px;
                if (in && pt < kWTwMax) {
                    tpos[pt] = (int)((long long)A.pos[i] - Q0);
                    twin[pt] = A.win[i];
                    tw[pt] = A.win[i];
                }
                if (in && pt == kWTwMax) {           // cannot happen for L >= kWMinL
                    atomicExch(A.err, 15u);
                    atomicExch(abort_flag, 1u);
                }
            }
            const u32 nw = named_bar_popc(1, kTcProdThreads, in && pt < kWTwMax);   // also publishes the table
            if (nw == 0 || tpos[0] > 0) {            // the stream kernels guarantee an entry at or before Q0
                if (pt == 0) { atomicExch(A.err, 16u); atomicExch(abort_flag, 1u); }
                break;
            }
            // ---- positions -> samples (this thread: 8pt.. in registers and,
            //      past 2048, 2048 + 8pt.. in shared memory)
            u32 smpA[8], smpB[8];
            auto map8 = [&](u32 x0, u32 (&smp)[8], bool kept_out) -> u32 {
                // last entry with tpos <= x0 (binary search), then step
                u32 lo = 0, hi = nw - 1;
                while (lo < hi) {
                    const u32 mid = (lo + hi + 1) >> 1;
                    if (tpos[mid] <= (int)x0) lo = mid; else hi = mid - 1;
                }
                u32 j = lo, kept = 0;
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const u32 x = x0 + e;
                    while (j + 1 < nw && tpos[j + 1] <= (int)x) j++;
                    const u32 o = (u32)((int)x - tpos[j]);
                    const u32 s = twin[j] * L + o;
                    smp[e] = s;
                    if (kept_out) {
                        const bool k = o < L && s < n;
                        // bit 31: the output is the reference's zeroed tail (.cl:231-234)
                        spos[x] = k ? (s | (s + L >= n ? kWTail : 0u)) : 0xffffffffu;
                        wrel[x] = k ? (u8)j : (u8)0xff;
                        kept |= k ? (1u << e) : 0u;
                    }
                }
                return kept;
            };
            map8(8 * pt, smpA, true);              // spos / wrel of this thread's positions
            if (hasB) {
                map8(kWPos + 8 * pt, smpB, false);
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    xs[8 * pt + e] = smpB[e];
                    xe2[8 * pt + e] = 0.0f;
                    xab[8 * pt + e] = 0.0f;
                }
            }
            // per 128-position chunk: the table entries whose outputs meet it
            if (pt < 16) {
                const int c0 = 128 * (int)pt, c1 = c0 + 128;
                u32 lo = 0, hi = nw - 1;             // last entry starting at or before c0
                while (lo < hi) {
                    const u32 mid = (lo + hi + 1) >> 1;
                    if (tpos[mid] <= c0) lo = mid; else hi = mid - 1;
                }
                const u32 wf = (tpos[lo] + (int)L > c0) ? lo : lo + 1;
                u32 wl = lo;                         // last entry starting before c1
                while (wl + 1 < nw && tpos[wl + 1] < c1) wl++;
                cw[pt] = wf | (wl << 16);
            }
            // ---- the tile's fp16 scale: every sample a kept output multiplies
            //      by a non-zero template value lies in its window or the next
            float mx = 0.0f;
            if (pt < nw) mx = fmaxf(A.vwmax[twin[pt]], A.vwmax[twin[pt] + 1]);
            mx = warp_max_float(mx);
            if (lane == 0) pred[warp] = mx;
            named_bar(1, kTcProdThreads);
            int kexp = 0;
            {
                float mm = 0.0f;
                for (int w8 = 0; w8 < kTcProdWarps; w8++) mm = fmaxf(mm, pred[w8]);
                if (mm > 0.0f) {
                    int e;
                    frexpf(mm, &e);                  // mm < 2^e
                    kexp = max(-126, min(126, 14 - e));   // scaled magnitudes < 2^14
                }
            }
            if (pt == 0) ti_all[b * 4] = kexp;
            if (pt < 16) {
                float sc = 0.0f, sa = 0.0f;
                if (pt < A.nt) {
                    const u32 gt = ctrow[pt];
                    const int ex = -(kexp + A.texp[gt]);
                    if (ex >= -149 && ex <= 127) sc = ldexpf(1.0f, ex);   // exact power of two
                    sa = 2.98023223876953125e-08f * 1.001f * ldexpf(A.tabs[gt], -kexp);
                }
                tsc[pt] = sc;
                tsa[pt] = sa;
            }
            // ---- the voltage stream, one channel per ring stage.  Each channel
            //      is copied (fp32) into a staging slot by coalesced 4-byte
            //      asynchronous copies -- thread pt copies positions pt + 256 e --
            //      kWDepth - 1 channels ahead of the one being packed; a thread
            //      packs positions 8 pt .. 8 pt + 7 (and 2048 + 8 pt .. when hasB).
            u32 lidx[8];                             // sample of position pt + 256 e, ~0 past the recording
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const int x = (int)(pt + 256u * e);
                u32 lo = 0, hi = nw - 1;             // last entry with tpos <= x
                while (lo < hi) {
                    const u32 mid = (lo + hi + 1) >> 1;
                    if (tpos[mid] <= x) lo = mid; else hi = mid - 1;
                }
                const u32 sx = twin[lo] * L + (u32)(x - tpos[lo]);
                lidx[e] = sx < n ? sx : 0xffffffffu;
            }
            auto issue = [&](u32 c) {
                float *dst = vst + (size_t)(c % kWDepth) * px;
                const float *vc = A.v + (size_t)c * n;
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const bool ok = lidx[e] != 0xffffffffu;
                    cp_async4(smem_u32(dst + pt + 256u * e), vc + (ok ? lidx[e] : 0u), ok ? 4u : 0u);
                }
                for (u32 x = pt; x < nB; x += kTcProdThreads) {
                    const u32 sb = xs[x];
                    cp_async4(smem_u32(dst + kWPos + x), vc + (sb < n ? sb : 0u), sb < n ? 4u : 0u);
                }
            };
            const float kscale = ldexpf(1.0f, kexp);     // exact: |kexp| <= 126
            float e2A[8], abA[8];
#pragma unroll
            for (int e = 0; e < 8; e++) e2A[e] = abA[e] = 0.0f;
#pragma unroll
            for (u32 j = 0; j + 1 < kWDepth; j++) {
                if (j < Cg) issue(j);
                cp_async_commit();
            }
            cp_async_wait<kWDepth - 2>();            // channel 0: this thread's copies
            named_bar(1, kTcProdThreads);            // and every thread's
            bool stop = false;
            for (u32 c = 0; c < Cg; c++) {
                if (c + kWDepth - 1 < Cg) issue(c + kWDepth - 1);
                cp_async_commit();                   // one group per channel (empty past the last)
                const float *src = vst + (size_t)(c % kWDepth) * px;
                uint4 qa, qb = make_uint4(0u, 0u, 0u, 0u);
                {
                    const float4 f0 = *reinterpret_cast<const float4 *>(src + 8 * pt);
                    const float4 f1 = *reinterpret_cast<const float4 *>(src + 8 * pt + 4);
                    const float f[8] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w};
                    u16 h[8];
#pragma unroll
                    for (int e = 0; e < 8; e++) {
                        e2A[e] = fmaf(f[e], f[e], e2A[e]);
                        abA[e] += fabsf(f[e]);
                        h[e] = half_bits_clamped(__fmul_rn(f[e], kscale));
                    }
                    qa.x = ((u32)h[1] << 16) | h[0];
                    qa.y = ((u32)h[3] << 16) | h[2];
                    qa.z = ((u32)h[5] << 16) | h[4];
                    qa.w = ((u32)h[7] << 16) | h[6];
                }
                if (hasB) {
                    const float4 f0 = *reinterpret_cast<const float4 *>(src + kWPos + 8 * pt);
                    const float4 f1 = *reinterpret_cast<const float4 *>(src + kWPos + 8 * pt + 4);
                    const float f[8] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w};
                    u16 h[8];
#pragma unroll
                    for (int e = 0; e < 8; e++) {
                        xe2[8 * pt + e] = fmaf(f[e], f[e], xe2[8 * pt + e]);
                        xab[8 * pt + e] += fabsf(f[e]);
                        h[e] = half_bits_clamped(__fmul_rn(f[e], kscale));
                    }
                    qb.x = ((u32)h[1] << 16) | h[0];
                    qb.y = ((u32)h[3] << 16) | h[2];
                    qb.z = ((u32)h[5] << 16) | h[4];
                    qb.w = ((u32)h[7] << 16) | h[6];
                }
                const u32 s = gstage % ns, u = gstage / ns;
                if (u > 0 && !mbar_wait_bounded(bar_sempty(s), (u - 1) & 1u, wlim)) {
                    atomicExch(A.err, 11u);
                    atomicExch(abort_flag, 1u);
                }
                if (named_bar_or(1, kTcProdThreads, *(volatile u32 *)abort_flag != 0)) { stop = true; break; }
                gstage++;
                unsigned char *stg = ring + (size_t)s * lay.stage;
                if (pt == 0) {
                    const u32 bytes = nkc * kWATile;
                    mbar_expect_tx(bar_sfull(s), bytes);
                    asm volatile(
                        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                        ::"r"(smem_u32(stg)), "l"(A.Aw + (size_t)c * bytes), "r"(bytes), "r"(bar_sfull(s))
                        : "memory");
                }
                *reinterpret_cast<uint4 *>(stg + lay.a_bytes + 16 * (size_t)pt) = qa;
                if (hasB) *reinterpret_cast<uint4 *>(stg + lay.a_bytes + 16 * (size_t)(kWN + pt)) = qb;
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                cp_async_wait<kWDepth - 2>();        // channel c + 1: this thread's copies
                named_bar(1, kTcProdThreads);        // every thread's; the stage is written
                if (pt == 0) mbar_arrive(bar_sfull(s));  // release: the barrier ordered every write
            }
            cp_async_wait<0>();                      // no copy lands after the loop (abort path)
            if (stop) break;
            // ---- window norms: prefix sums (double) over the staged positions
#pragma unroll
            for (int e = 0; e < 8; e++) {
                psq[8 * pt + e] = e2A[e];
                pab[8 * pt + e] = abA[e];
                if (hasB) {
                    psq[kWPos + 8 * pt + e] = xe2[8 * pt + e];
                    pab[kWPos + 8 * pt + e] = xab[8 * pt + e];
                }
            }
            named_bar(1, kTcProdThreads);
            {
                const u32 per = (px + kTcProdThreads - 1) / kTcProdThreads;
                const u32 lo = min(px, pt * per), hi = min(px, lo + per);
                double a = 0.0, bb = 0.0;
                for (u32 x = lo; x < hi; x++) { a += psq[x]; bb += pab[x]; }
                const double ia = warp_incl_scan_d(a, lane), ib = warp_incl_scan_d(bb, lane);
                if (lane == 31) { dsum[warp] = ia; dsum[8 + warp] = ib; }
                named_bar(1, kTcProdThreads);
                double ca = ia - a, cb = ib - bb;
                for (u32 w8 = 0; w8 < warp; w8++) { ca += dsum[w8]; cb += dsum[8 + w8]; }
                for (u32 x = lo; x < hi; x++) {
                    ca += psq[x]; cb += pab[x];
                    psq[x] = ca; pab[x] = cb;
                }
            }
            named_bar(1, kTcProdThreads);
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const u32 x = 8 * pt + e, hi_x = x + L - 1;    // < px
                const u32 sp = spos[x];              // the sample of a kept output
                if (sp == 0xffffffffu) continue;
                const u32 smp = sp & ~kWTail;
                const double pa = psq[hi_x], pb = pab[hi_x];
                const double da = pa - (x ? psq[x - 1] : 0.0), db = pb - (x ? pab[x - 1] : 0.0);
                // the double sums' own rounding (< 2 px 2^-53 of the prefix) is added back
                const float wn = (float)sqrt(fmax(da, 0.0) + 1e-12 * pa) * 1.0001f + 1e-30f;
                const float wa = (float)(fmax(db, 0.0) + 1e-12 * pb) * 1.0001f + 1e-30f;
                wnwa[x] = make_float2(wn, wa);
                A.wn_s[smp] = wn;
                A.wa_s[smp] = wa;
                A.kx_s[smp] = (signed char)kexp;
            }
            named_bar(1, kTcProdThreads);
            if (pt == 0) mbar_arrive(bar_ifull(b));
            if (b) use1++; else use0++;
        }
        // the last copies into the ring land before the CTA exits
        if (pt == 0) {
            for (u32 s = 0; s < ns; s++) {
                const u32 uses = gstage / ns + (s < gstage % ns ? 1u : 0u);
                if (uses > 0) mbar_wait_bounded(bar_sfull(s), (uses - 1) & 1u, kTcDrainPolls);
            }
        }
    } else if (warp == kTcMmaWarp) {
        // =========================== MMA issue ===========================
        // D f32, A/B f16, both K-major, M = 128, N = 256
        const u32 idesc = (1u << 4) | ((kWN >> 3) << 17) | ((u32)(kTcM >> 4) << 24);
        const u64 a0 = umma_desc(smem_u32(ring), kWATile / 2, 128);       // K halves 2048 B apart
        const u64 b0 = umma_desc(smem_u32(ring) + (u32)lay.a_bytes, 16, 128);   // rows 8 samples apart
        const u64 sstep = (u64)(lay.stage >> 4);
        u32 use0 = 0u, use1 = 0u;
        u32 it = 0;
        bool issued = false;
        for (u32 q = bi; q < ntiles; q += cnt, it++) {
            const u32 b = it & 1u;
            const u32 ub = b ? use1 : use0;
            u32 ok = 1;
            if (lane == 0) {
                if (ub > 0 && !mbar_wait_bounded(bar_aempty(b), (ub - 1) & 1u, wlim)) {
                    atomicExch(A.err, 12u);
                    ok = 0;
                }
                if (!ok) atomicExch(abort_flag, 1u);
                if (*(volatile u32 *)abort_flag) ok = 0;
            }
            if (!__shfl_sync(0xffffffffu, ok, 0)) break;
            const u32 dst = tmem + b * kWN;
            for (u32 c = 0; c < Cg && ok; c++) {
                const u32 s = gstage % ns, u = gstage / ns;
                gstage++;
                if (lane == 0) {
                    if (!mbar_wait_bounded(bar_sfull(s), u & 1u, wlim)) {
                        atomicExch(A.err, 14u);
                        ok = 0;
                    }
                    if (!ok) atomicExch(abort_flag, 1u);
                    if (*(volatile u32 *)abort_flag) ok = 0;
                    if (ok) {
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        u64 da = a0 + s * sstep, db = b0 + s * sstep;
                        for (u32 k = 0; k < nkc; k++) {
                            const u32 acc = (c | k) != 0 ? 1u : 0u;   // the first MMA overwrites
                            asm volatile(
                                "{\n\t.reg .pred p;\n\t"
                                "setp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                                ::"r"(dst), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
                            da += (u64)(kWATile >> 4);           // next A tile
                            db += 2u;                            // 16 samples (32 bytes) later
                        }
                        issued = true;
                        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                                     ::"r"(bar_sempty(s)) : "memory");
                    }
                }
                ok = __shfl_sync(0xffffffffu, ok, 0);
            }
            if (!ok) break;
            if (lane == 0)
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             ::"r"(bar_afull(b)) : "memory");
            __syncwarp();
            if (b) use1++; else use0++;
        }
        // every MMA issued here is done before TMEM and the ring are released
        if (lane == 0 && issued) {
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(bar_fin) : "memory");
            mbar_wait_bounded(bar_fin, 0, kTcDrainPolls);
        }
        __syncwarp();
    } else {
        // =========================== epilogue ===========================
        const u32 ew_ = warp - kTcEpiWarp0;          // 0..7
        const u32 quad = warp & 3u;                  // TMEM lanes [32 quad, 32 quad + 32)
        const u32 half = ew_ >> 2;                   // columns [128 half, 128 half + 128)
        const u32 row = quad * 32 + lane;
        const u32 tl = row >> 3, d = row & 7u;       // template column, sample shift
        const bool real = tl < A.nt;
        const u32 gt = ctrow[tl];
        const float ck = ctk[tl], cb = ctb[tl], css = ctss[tl], ca = cta[tl];
        const int texp_t = real ? A.texp[gt] : 0;
        // this lane's template row of the likelihood and flag buffers
        float *const Lk_t = A.Lk + (size_t)gt * n;
        u8 *const apx_t = A.apx + (size_t)gt * n;
        float *const dbg_t = A.dbgE ? A.dbgE + (size_t)gt * n : nullptr;
        int *const bm_i = reinterpret_cast<int *>(A.bm_s);
        u32 use0 = 0u, use1 = 0u;
        u32 it = 0;
        for (u32 q = bi; q < ntiles; q += cnt, it++) {
            const u32 b = it & 1u;
            const u32 ub = b ? use1 : use0;
            bool ok = mbar_wait_bounded(bar_afull(b), ub & 1u, wlim);
            ok = ok && mbar_wait_bounded(bar_ifull(b), ub & 1u, wlim);
            if (!ok) { atomicExch(A.err, 10u); atomicExch(abort_flag, 1u); }
            if (named_bar_or(2, kTcEpiThreads, *(volatile u32 *)abort_flag != 0)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const u32 *spos = spos_all + (size_t)b * kWPos;
            const float2 *wnwa = wnwa_all + (size_t)b * kWPos;
            const u8 *wrel = wrel_all + (size_t)b * kWPos;
            const u32 *tw = tw_all + (size_t)b * kWTwMax;
            const u32 *cw = cw_all + b * 16;
            const int kexp = ti_all[b * 4];
            const float tsc = tf_all[b * 32 + tl], tsa = tf_all[b * 32 + 16 + tl];
            const u32 acc0 = tmem + ((quad * 32u) << 16) + b * kWN;
            // the rare cases (a scale outside the float range, the testing
            // output of E) take a separate, warp-uniform copy of the loop
            const bool rare = __any_sync(0xffffffffu, tsc == 0.0f) || dbg_t != nullptr;
            u32 want[8];
            // one 16-column chunk: classify and store its entries; per
            // (window, template) the largest upper bound, per window the
            // largest lower bound and whether some entry is > 0
            auto chunk = [&](const int k, auto RARE) {
                constexpr bool kRare = decltype(RARE)::value;
                const u32 c0 = 128 * half + 16 * k;
                u32 r[16];
                tmem_ld<16>(r, acc0 + c0);
                float uq[16], lq[16];
                u32 wbits = 0, pbits = 0;
                bool any = false;
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const u32 x = 8 * (c0 + j) + d;
                    const u32 sp = spos[x];
                    const bool kept = real && sp != 0xffffffffu;
                    const bool tail = (sp & kWTail) != 0u;          // .cl:231-234 (kept outputs only)
                    const u32 s = sp & ~kWTail;
                    const float2 nwa = wnwa[x];
                    const float a = __uint_as_float(r[j]);
                    float sa = __fmul_rn(a, tsc);
                    if (kRare && tsc == 0.0f) sa = ldexpf(a, -(kexp + texp_t));
                    const float approx = __fadd_rn(sa, css);
                    // E = kappa ||t|| ||w|| + 2^-25 (|t|_1 / s_v + |w|_1 / s_t) * 1.001
                    //     + kappa_s |SS/2| + 2^-22 |approx|
                    const float E = fmaf(ck, nwa.x, fmaf(cb, nwa.y, tsa) + ca + 2.384185791015625e-07f * fabsf(approx));
                    const bool pos = approx - E > 0.0f;        // certainly > 0: refined when a decision needs it
                    const bool neg = approx + E <= 0.0f;       // certainly <= 0: only its sign is read
                    const bool live = kept && !tail;
                    if (kept) {
                        Lk_t[s] = tail ? 0.0f : approx;
                        apx_t[s] = (live && pos) ? (u8)1 : (u8)0;
                        if (kRare && dbg_t) dbg_t[s] = tail ? 0.0f : E;
                    }
                    if (live && pos) atomicMax(bm_i + s, __float_as_int(E));
                    wbits |= (live && !pos && !neg) ? (1u << j) : 0u;
                    pbits |= (live && pos) ? (1u << j) : 0u;
                    uq[j] = live ? fmaxf(0.0f, approx + E) : 0.0f;
                    lq[j] = live ? approx - E : 0.0f;
                    any |= live && !neg;
                }
                want[k] = wbits;
                if (__any_sync(0xffffffffu, any)) {
                    const u32 cwv = cw[half * 8 + k];
                    const u32 wf = cwv & 0xffffu, wl = cwv >> 16;
                    for (u32 w = wf; w <= wl; w++) {
                        float mu = 0.0f, ml = 0.0f;
                        bool mp = false;
#pragma unroll
                        for (int j = 0; j < 16; j++) {
                            const bool here = wrel[8 * (c0 + j) + d] == w;
                            mu = here ? fmaxf(mu, uq[j]) : mu;
                            ml = here ? fmaxf(ml, lq[j]) : ml;
                            mp |= here && ((pbits >> j) & 1u);
                        }
#pragma unroll
                        for (int o = 1; o < 8; o <<= 1) mu = fmaxf(mu, __shfl_xor_sync(0xffffffffu, mu, o));
#pragma unroll
                        for (int o = 1; o < 32; o <<= 1) ml = fmaxf(ml, __shfl_xor_sync(0xffffffffu, ml, o));
                        const u32 wa = tw[w];
                        if (d == 0 && real && mu > 0.0f)
                            atomicMax(reinterpret_cast<int *>(A.umax) + (size_t)wa * A.Kall + gt, __float_as_int(mu));
                        if (lane == 0 && ml > 0.0f) atomicMax(reinterpret_cast<int *>(A.wlb) + wa, __float_as_int(ml));
                        if (__any_sync(0xffffffffu, mp) && lane == 0) A.wpos[wa] = 1;
                    }
                }
            };
            if (rare) {
#pragma unroll
                for (int k = 0; k < 8; k++) chunk(k, std::true_type{});
            } else {
#pragma unroll
                for (int k = 0; k < 8; k++) chunk(k, std::false_type{});
            }
            // accumulator b is no longer needed
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(bar_aempty(b));
            u32 nwant = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) nwant += __popc(want[k]);
            if (named_bar_or(2, kTcEpiThreads, nwant != 0)) {
                // one contiguous segment of (template, sample) entries per
                // tile, ordered by template (tcnt is zero here)
                if (nwant) atomicAdd(&tcnt[tl], nwant);
                named_bar(2, kTcEpiThreads);
                if (ew_ == 0) {
                    const u32 cnt_t = lane < 16 ? tcnt[lane] : 0u;
                    const u32 incl = warp_incl_scan(cnt_t);
                    if (lane < 16) tcnt[lane] = incl - cnt_t;
                    const u32 total = __shfl_sync(0xffffffffu, incl, 31);
                    if (lane == 0) {
                        const unsigned long long old = atomicAdd(A.refseg, ((unsigned long long)total << 32) | 1ull);
                        const u32 base = (u32)(old >> 32), si = (u32)old;
                        seg_info[0] = base;
                        seg_info[2] = 0;
                        if (base + total <= A.ref_cap && si < A.seg_cap) {
                            A.seg_s0[si] = 0;                // entries carry their absolute samples
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
                if (seg_info[2] && nwant) {
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        u32 bits = want[k];
                        while (bits) {
                            const u32 j = __ffs(bits) - 1;
                            bits &= bits - 1;
                            const u32 x = 8 * (128 * half + 16 * k + j) + d;
                            const u32 p = seg_base + atomicAdd(&tcnt[tl], 1u);
                            A.ref_t[p] = tl;
                            A.ref_s[p] = spos[x] & ~kWTail;
                        }
                    }
                }
                named_bar(2, kTcEpiThreads);         // tcnt / seg_info are done with
                if (ew_ == 0 && lane < 16) tcnt[lane] = 0;
            }
            // the tile's tables are no longer needed
            __syncwarp();
            if (lane == 0) mbar_arrive(bar_bempty(b));
            if (b) use1++; else use0++;
        }
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kWN));
}

// A tiles of one template group: Aw[c][k] = 128 rows (template tl = row / 8,
// shift d = row % 8) x 16 lags j = 16k + jj, holding T[trow[tl]][clo + c][j - d]
// scaled by 2^texp (zero outside 0 <= j - d < L and for tl >= nt), in the
// K-major no-swizzle layout: K half (jj / 8) 2048 bytes apart, 8-row groups
// 128 bytes apart, rows 16 bytes apart.
__global__ void k_tcw_pack(const float *__restrict__ T, u32 Call, u32 L, u32 nkc, const u32 *__restrict__ trow,
                           u32 nt, u32 clo, u32 Cg, const int *__restrict__ texp, u16 *__restrict__ Aw) {
    const u64 total = (u64)Cg * nkc * (kWATile / 2);
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (u64)gridDim.x * blockDim.x) {
        const u32 within = (u32)(e % (kWATile / 2)), tile = (u32)(e / (kWATile / 2));
        const u32 c = tile / nkc, k = tile % nkc;
        const u32 h = within >> 10, tl = (within >> 6) & 15u, d = (within >> 3) & 7u, el = within & 7u;
        const int lag = (int)(16 * k + 8 * h + el) - (int)d;
        float f = 0.0f;
        if (tl < nt && lag >= 0 && lag < (int)L) {
            const u32 t = trow[tl];
            f = ldexpf(T[((size_t)t * Call + clo + c) * L + (u32)lag], texp[t]);
        }
        Aw[e] = __half_as_ushort(__float2half_rn(f));
    }
}

// Largest |v| of each window over all channels; two zero pads past the end.
__global__ void k_window_vmax(const float *__restrict__ v, u32 n, u32 C, u32 L, u32 W, float *__restrict__ vwmax) {
    const u32 lane = threadIdx.x & 31;
    const u32 nwarps = (gridDim.x * blockDim.x) >> 5;
    for (u32 w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < W + 2; w += nwarps) {
        float m = 0.0f;
        if (w < W) {
            for (u32 c = 0; c < C; c++) {
                const float *vc = v + (size_t)c * n + (size_t)w * L;
                for (u32 i = lane; i < L; i += 32)
                    if ((size_t)w * L + i < n) m = fmaxf(m, fabsf(vc[i]));
            }
        }
        m = warp_max_float(m);
        if (lane == 0) vwmax[w] = m;
    }
}

// The stream of a pass.  brk[i] = 1 where listed window i starts a run
// (entries past the list are 0, as the ordered compaction reads them).
__global__ void k_ws_breaks(const u32 *__restrict__ win, const u32 *__restrict__ n_win, u32 nbytes,
                            u8 *__restrict__ brk) {
    const u32 m = *n_win;
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < nbytes; i += gridDim.x * blockDim.x)
        brk[i] = (i < m && (i == 0 || win[i] != win[i - 1] + 1)) ? 1 : 0;
}

// pos[i] = i L + R_i (L - 1), R_i = runs before listed window i (runs[] =
// list index of each run's first window); first[q] = the last listed window
// with pos <= 2048 q; *n_stiles = tiles that hold kept outputs.
__global__ void k_ws_pos(const u32 *__restrict__ n_win, const u8 *__restrict__ brk, const u32 *__restrict__ runs,
                         const u32 *__restrict__ n_runs, u32 L, u32 *__restrict__ pos, u32 *__restrict__ first,
                         u32 *__restrict__ n_stiles) {
    const u32 m = *n_win, nr = *n_runs;
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g == 0 && m == 0) *n_stiles = 0;
    for (u32 i = g; i < m; i += gridDim.x * blockDim.x) {
        u32 lo = 0, hi = nr;                         // first run starting after i
        while (lo < hi) {
            const u32 mid = (lo + hi) >> 1;
            if (runs[mid] <= i) lo = mid + 1; else hi = mid;
        }
        const u32 R = lo - 1;                        // runs[0] = 0 <= i
        const u32 p = i * L + R * (L - 1);
        pos[i] = p;
        const u64 next = i + 1 < m ? (u64)p + L + (brk[i + 1] ? L - 1 : 0) : ~0ull;
        const u64 qt = ((u64)p + kWPos - 1) / kWPos;  // the one tile start in [p, next), if any
        if (qt * kWPos < next && (i + 1 < m || qt * kWPos < (u64)p + L)) first[qt] = i;
        if (i + 1 == m) *n_stiles = (u32)(((u64)p + L + kWPos - 1) / kWPos);
    }
}

}  // namespace fbp
