// C ABI and per-chunk driver of the Full Binary Pursuit library (sm_100a).
//
// fbp_pursuit_chunk replaces the iterate-until-converged loop of the
// reference host driver (spikesorting_fullpursuit/parallel/
// binary_pursuit_parallel.py:386-736): the window lists that the reference
// builds on the host with np.nonzero after every pass are compacted on the
// device, and the host reads back one count per pass.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fbp_b200.h"
#include "fbp_overlap_fast.cuh"
#include "fbp_lik_tc.cuh"
#include "fbp_lik_tcw.cuh"

using namespace fbp;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

}  // namespace

// Error text for the entry points of the other translation unit
// (fbp_prepost.cu): one per-thread string for the whole library.
namespace fbp {
int set_last_error(int code, const char *msg) {
    g_last_error = msg ? msg : "";
    return code;
}
}  // namespace fbp

namespace {

#define FBP_CUDA(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(FBP_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));     \
    } while (0)

#define FBP_LAUNCH_CHECK()                                                                 \
    do {                                                                                   \
        cudaError_t e_ = cudaGetLastError();                                               \
        if (e_ != cudaSuccess)                                                             \
            return fail(FBP_ERR_CUDA, "kernel launch failed at %s:%d: %s", __FILE__,       \
                        __LINE__, cudaGetErrorString(e_));                                 \
    } while (0)

// Testing limits (fbp_set_test_limits): capacities of the refinement list
// and the contender pool (0: the workspace's), polls of the tensor-core
// kernel's pipeline waits.
std::atomic<u32> g_lim_refine{0}, g_lim_pool{0}, g_lim_wait{FBP_DEFAULT_WAIT_POLLS};
// Tensor-core template group size chosen by a tuner for the calling thread
// (fbp_set_tc_group_size; 0: the planner's cost model).
thread_local u32 t_tc_group_size = 0;
// Layout of the tensor-core likelihood for the calling thread
// (fbp_set_tc_layout): FBP_TC_LAYOUT_AUTO, _SAMPLES or _WIDE.
thread_local int t_tc_layout = FBP_TC_LAYOUT_AUTO;

int sm_count() {
    // initialised once, thread-safely (calls may come from several host threads)
    static const int cached = [] {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n > 0 ? n : 148;
    }();
    return cached;
}

// Raises the dynamic shared memory limit of `func` to the device's opt-in
// maximum, once per kernel and device.  The limit is a process-wide kernel
// attribute: setting it per call to the call's own size would let one host
// thread shrink it under another thread's launch (or captured graph) of the
// same kernel with a larger size.
std::mutex g_attr_mu;
std::vector<std::pair<const void *, int>> g_attr_done;
int allow_smem(const void *func) {
    int dev = 0;
    FBP_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_attr_mu);
    for (const auto &d : g_attr_done)
        if (d.first == func && d.second == dev) return FBP_OK;
    int mx = 0;
    FBP_CUDA(cudaDeviceGetAttribute(&mx, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa;
    FBP_CUDA(cudaFuncGetAttributes(&fa, func));          // the kernel's static shared memory counts too
    FBP_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  mx - (int)fa.sharedSizeBytes));
    g_attr_done.emplace_back(func, dev);
    return FBP_OK;
}
#define FBP_ALLOW_SMEM(kern)                                                               \
    do {                                                                                   \
        const int rc_ = allow_smem((const void *)&kern);                                 \
        if (rc_ != FBP_OK) return rc_;                                                     \
    } while (0)

// A template group of the tensor-core likelihood: columns t0..t0+nt of the
// support order (tperm), channels [clo, clo + Cg) of the recording.
struct TcGroup {
    u32 t0, nt, clo, Cg, Cg2, Np, nbuf, cols;
    size_t tb_off;                   // offset of its packed templates in Tb (uint4 units)
};

// Device workspace of one chunk: sub-buffers at 256-byte boundaries.
struct Workspace {
    float *Lk;
    u32 *best_idx, *best_lab, *ov_idx, *ov_lab, *win, *cand, *acc_list;
    u32 *spk_idx, *spk_lab, *spk_win, *tile_counts;
    float *best_ll;
    u8 *flags, *flags_out, *ovr, *ovr2, *active, *has;
    Counters *cnt;
    // fast overlap recheck (present when `fast`)
    bool fast;
    u32 slots;
    float *NT, *sNT, *tnorm, *Q, *XMr, *XM, *H, *vn, *cand_lb, *ga_lo, *ga_hi, *ga_max, *ga_abs, *pool_hi;
    u32 *ga_bits, *seed_a1;
    float *pair_mb, *pair_mabs;
    Counters *snap;                  // counts of the last pass
    u32 *tsup, *tperm, *grange;      // template channel supports, order, group ranges
    u32 *grange32;                   // group ranges of 32 slots (masked overlap tables)
    bool masked_tables = false;      // templates occupy narrow channel ranges
    OvConst *oc;
    u8 *cskip, *fallback, *need;
    u32 *pool_slot, *pool_item, *fb_slots, *fb_list;
    u64 *best_key;
    u32 pool_cap;
    float *ua;
    int *kexp_tile;
    u32 stiles;
    // tensor-core likelihood (present when `tc`)
    bool tc;
    u32 tc_ref_cap;
    u32 tc_gmax;                     // template groups the buffers hold
    std::vector<TcGroup> tcg;        // this chunk's groups (planned from the template supports)
    u32 tc_cg2max, tc_cmax;          // largest channel groups / channels of a group
    u32 tc_nz;                       // widest template support (channels): only non-zero products round
    u32 *tc_gdesc;                   // [group][3]: t0, clo, Cg (device)
    TcArgs *tc_args0, *tc_args1;     // [group] launch arguments: likelihood tiles, overlap tables (device)
    size_t tc_smem;                  // dynamic shared memory of the largest group
    u32 *tgrp;                       // [K] group of each template (device)
    u32 *tc_seg_grp;                 // [seg_cap] group of each refinement segment
    uint4 *Tb;
    float *tc_tnorm, *tc_tabs;
    int *tc_texp;
    u8 *apx;
    float *wn_s, *wa_s, *bm_s, *wlb;
    float *umax;                     // [W][K] largest upper bound of a template's entries per window
    u8 *wpos;                        // [W] some entry of the window is > 0
    signed char *kx_s;
    u32 *tc_ref_t, *tc_ref_s, *tc_seg_s0, *tc_seg_base, *tc_seg_cnt;
    u32 tc_seg_cap;
    // wide tiles (fbp_lik_tcw.cuh): groups of 16 templates, window streams
    bool tcw = false;                // this chunk's likelihood passes use k_lik_tcw
    u32 tcw_ns = 0;                  // ring stages
    std::vector<TcGroup> tcwg;       // wide groups (tb_off: offset of its A tiles, 4 KB units)
    float *vwmax;                    // [W + 2] bound on |v| per window (all channels)
    u8 *ws_brk;                      // [window bytes] run starts of the pass's list
    u32 *ws_runs, *ws_pos, *ws_first;
    unsigned char *Aw;               // packed A tiles of every wide group
    u32 *tgrp_w;                     // [K] wide group of each template
    u32 *tcw_gdesc;                  // [group][3]: t0, clo, Cg (device)
    TcwArgs *tcw_args;               // [group] (device)
    size_t tcw_smem;
    u32 n;                           // samples of the chunk
    size_t bytes;
};

// The fast overlap recheck is used when its shared-memory tiles fit and the
// shift range is at most 4L+1 (production uses S = 2L-1).
bool fast_overlap_fits(u32 K, u32 L, u32 nmax) {
    const u64 S = 2 * (u64)nmax + 1;
    if (S > 4 * (u64)L + 1 || S > 65535) return false;
    if (xm_smem_bytes(L) > 227 * 1024 || scan_smem_bytes((u32)S) > 227 * 1024) return false;
    if (tables_smem_bytes((u32)S, K, L) > 227 * 1024) return false;
    return true;
}

size_t window_bytes_u8(u32 W) { return align_up((size_t)W + FBP_WINDOW_PAD, kCompactTile); }

// Tensor-core template groups.  Templates in support order (tperm) are cut
// into groups of GS consecutive columns; a group's channel range is the union
// of its templates' supports.  Every GS from all templates down to 16 is
// tried; the plan whose groups all fit shared memory (templates, two or one
// strip buffers; the refinement's strip) with the least padded MMA work per
// tile (columns x channel groups, plus a fixed cost per group) wins.
bool plan_tc_groups(const std::vector<u32> &tsup, const std::vector<u32> &tperm, u32 K, u32 C, u32 L, u32 gmax,
                    std::vector<TcGroup> &out) {
    double best = 1e300;
    std::vector<TcGroup> cur;
    const u32 kall = (K + 15) / 16 * 16;
    const u32 sizes[] = {kall, 256, 128, 64, 32, 16};
    const u32 forced = t_tc_group_size;
    bool forced_fits = false;                        // a forced size that does not fit: the cost model
    for (int pass = forced ? 0 : 1; pass < 2 && !forced_fits; pass++)
    for (u32 GS : sizes) {
        if (GS > 256 || GS == 0) continue;
        if (pass == 0 && GS != std::min(forced, kall)) continue;
        if ((K + GS - 1) / GS > gmax) continue;
        cur.clear();
        double cost = 0;
        bool ok = true;
        size_t off = 0;
        for (u32 t0 = 0; t0 < K && ok; t0 += GS) {
            TcGroup g{};
            g.t0 = t0;
            g.nt = std::min(GS, K - t0);
            u32 lo = C, hi = 0;
            for (u32 j = t0; j < t0 + g.nt; j++) {
                const u32 t = tperm[j];
                if (tsup[2 * t + 1] > tsup[2 * t]) {
                    lo = std::min(lo, tsup[2 * t]);
                    hi = std::max(hi, tsup[2 * t + 1]);
                }
            }
            if (hi <= lo) { lo = 0; hi = std::min(C, 8u); }   // all-zero templates: zero products
            g.clo = lo;
            g.Cg = hi - lo;
            g.Cg2 = (g.Cg + 15) / 16 * 2;
            g.Np = (g.nt + 15) / 16 * 16;
            if (tc_smem_bytes(L, g.Cg2, g.Np, 2) <= 227 * 1024) g.nbuf = 2;
            else if (tc_smem_bytes(L, g.Cg2, g.Np, 1) <= 227 * 1024) g.nbuf = 1;
            else ok = false;
            if (tc_refine_smem_bytes(g.Cg, L) > 227 * 1024) ok = false;
            g.cols = 32;
            while (g.cols < g.nbuf * g.Np) g.cols <<= 1;
            g.tb_off = off;
            off += (size_t)L * g.Cg2 * g.Np;
            cost += (double)g.Np * g.Cg2 + 8.0 * g.Cg2 + 2.0 * g.Np + 64.0;
            cur.push_back(g);
        }
        if (ok && cost < best) {
            best = cost;
            out = cur;
            if (pass == 0) forced_fits = true;
        }
    }
    return best < 1e300;
}

// Wide-tile groups (fbp_lik_tcw.cuh): templates in support order (tperm)
// cut into groups of 16 (M = 16 templates x 8 sample shifts); a group's
// channels are the union of its templates' supports.  Returns the ring
// stages that fit shared memory, 0 when the wide layout does not apply.
u32 plan_tcw_groups(const std::vector<u32> &tsup, const std::vector<u32> &tperm, u32 K, u32 C, u32 L,
                    std::vector<TcGroup> &out) {
    out.clear();
    if (L < kWMinL || L > 1024) return 0;
    u32 ns = 0;
    for (u32 s = kWMaxStages; s >= 2; s--)
        if (tcw_smem_layout(L, s).total <= 227 * 1024) { ns = s; break; }
    if (ns == 0) return 0;
    size_t off = 0;
    for (u32 t0 = 0; t0 < K; t0 += 16) {
        TcGroup g{};
        g.t0 = t0;
        g.nt = std::min(16u, K - t0);
        u32 lo = C, hi = 0;
        for (u32 j = t0; j < t0 + g.nt; j++) {
            const u32 t = tperm[j];
            if (tsup[2 * t + 1] > tsup[2 * t]) {
                lo = std::min(lo, tsup[2 * t]);
                hi = std::max(hi, tsup[2 * t + 1]);
            }
        }
        if (hi <= lo) { lo = 0; hi = 1; }               // all-zero templates: zero products
        g.clo = lo;
        g.Cg = hi - lo;
        g.tb_off = off;
        off += (size_t)g.Cg * tcw_nkc(L);
        out.push_back(g);
    }
    return ns;
}

Workspace layout(char *base, u32 n, u32 K, u32 L, u32 nmax, bool want_fast, u32 C = 0, bool want_tc = false) {
    Workspace w{};
    const u32 W = ceil_div(n, L);
    const size_t Wp = (size_t)W + FBP_WINDOW_PAD;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char *p = base ? base + off : nullptr;
        off = align_up(off + bytes, 256);
        return p;
    };
    w.cnt = (Counters *)take(sizeof(Counters));
    w.snap = (Counters *)take(sizeof(Counters));
    w.wlb = (float *)take((size_t)W * 4);
    w.umax = (float *)take((size_t)W * K * 4);
    w.wpos = (u8 *)take((size_t)W);
    w.tsup = (u32 *)take((size_t)K * 8);
    w.tperm = (u32 *)take((size_t)K * 4);
    w.grange = (u32 *)take((size_t)ceil_div(K, kLikTplPerBlock) * 8);
    w.grange32 = (u32 *)take((size_t)ceil_div(K, kTabMGroup) * 8);
    w.Lk = (float *)take((size_t)K * n * sizeof(float));
    w.best_idx = (u32 *)take(Wp * 4);
    w.best_lab = (u32 *)take(Wp * 4);
    w.best_ll = (float *)take(Wp * 4);
    w.ov_idx = (u32 *)take(Wp * 4);
    w.ov_lab = (u32 *)take(Wp * 4);
    w.win = (u32 *)take(Wp * 4);
    w.cand = (u32 *)take(Wp * 4);
    w.acc_list = (u32 *)take(Wp * 4);
    w.spk_idx = (u32 *)take(Wp * 4);
    w.spk_lab = (u32 *)take(Wp * 4);
    w.spk_win = (u32 *)take(Wp * 4);
    w.tile_counts = (u32 *)take((size_t)(ceil_div(W, kCompactTile) + 1) * 4);
    const size_t wb = window_bytes_u8(W);
    w.flags = (u8 *)take(wb);
    w.flags_out = (u8 *)take(wb);
    w.ovr = (u8 *)take(wb);
    w.ovr2 = (u8 *)take(wb);
    w.active = (u8 *)take(wb);
    w.has = (u8 *)take(wb);
    w.fast = want_fast && fast_overlap_fits(K, L, nmax);
    if (w.fast) {
        const u32 S = 2 * nmax + 1;
        // at most every other window is a candidate (their bests cannot
        // both lie in their own windows)
        w.slots = W / 2 + 2;
        const size_t sl = w.slots;
        w.oc = (OvConst *)take(sizeof(OvConst));
        w.NT = (float *)take((size_t)K * S * 4);
        w.sNT = (float *)take((size_t)K * S * 4);
        w.tnorm = (float *)take((size_t)K * 4);
        w.Q = (float *)take((size_t)K * K * (2 * L - 1) * (L + 1) * 4);
        w.XMr = (float *)take((size_t)K * K * (2 * L + 1) * 4);
        w.XM = (float *)take((size_t)K * K * 4);
        w.H = (float *)take(sl * K * S * 4);
        w.vn = (float *)take(sl * 4);
        w.cskip = (u8 *)take(sl);
        w.fallback = (u8 *)take(align_up(sl + FBP_WINDOW_PAD, kCompactTile));
        w.ga_lo = (float *)take(sl * S * 4);
        w.ga_hi = (float *)take(sl * S * 4);
        w.ga_bits = (u32 *)take(sl * ((S + 31) / 32) * 4);
        w.ga_max = (float *)take(sl * 4);
        w.ga_abs = (float *)take(sl * 4);
        w.seed_a1 = (u32 *)take(sl * 4);
        w.pair_mb = (float *)take(sl * K * 4);
        w.pair_mabs = (float *)take(sl * K * 4);
        w.cand_lb = (float *)take(sl * 4);
        w.best_key = (u64 *)take(sl * 8);
        w.pool_cap = (u32)std::min<u64>(0x7fffffffull, std::max<u64>(1u << 22, (u64)sl * 128));
        w.pool_slot = (u32 *)take((size_t)w.pool_cap * 4);
        w.pool_item = (u32 *)take((size_t)w.pool_cap * 4);
        w.pool_hi = (float *)take((size_t)w.pool_cap * 4);
        w.fb_slots = (u32 *)take(sl * 4);
        w.fb_list = (u32 *)take(sl * 4);
        w.ua = (float *)take(sl * 4);
        w.stiles = (S + kTcM - 1) / kTcM;
        w.kexp_tile = (int *)take(sl * w.stiles * 4 * (want_tc ? std::max(1u, ceil_div(K, 16)) : 1u));
    }
    w.tc = want_tc && C > 0;
    if (w.tc) {
        // buffers for up to one group per 16 templates (the plan is made per
        // chunk from the template supports)
        w.tc_gmax = std::max(1u, ceil_div(K, 16));
        const u32 cg2all = ceil_div(C, 16) * 2;
        w.Tb = (uint4 *)take((size_t)L * cg2all * (2 * (size_t)K + 16) * 16);
        w.apx = (u8 *)take((size_t)K * n);
        w.wn_s = (float *)take((size_t)w.tc_gmax * n * 4);
        w.bm_s = (float *)take((size_t)n * 4);
        w.wa_s = (float *)take((size_t)w.tc_gmax * n * 4);
        w.kx_s = (signed char *)take((size_t)w.tc_gmax * n);
        w.tc_tnorm = (float *)take((size_t)K * 4);
        w.tc_tabs = (float *)take((size_t)K * 4);
        w.tc_texp = (int *)take((size_t)K * 4);
        w.tc_ref_cap = (u32)std::min<u64>(0x7fffffffull, std::max<u64>(1u << 20, (u64)n * K / 4));
        w.tc_ref_t = (u32 *)take((size_t)w.tc_ref_cap * 4);
        w.tc_ref_s = (u32 *)take((size_t)w.tc_ref_cap * 4);
        w.tc_seg_cap = (W * ((L + kTcM - 1) / kTcM) + 16) * w.tc_gmax;
        w.tc_seg_s0 = (u32 *)take((size_t)w.tc_seg_cap * 4);
        w.tc_seg_base = (u32 *)take((size_t)w.tc_seg_cap * 4);
        w.tc_seg_cnt = (u32 *)take((size_t)w.tc_seg_cap * 4);
        w.tc_seg_grp = (u32 *)take((size_t)w.tc_seg_cap * 4);
        w.tc_gdesc = (u32 *)take((size_t)w.tc_gmax * 12);
        w.tgrp = (u32 *)take((size_t)K * 4);
        w.tc_args0 = (TcArgs *)take((size_t)w.tc_gmax * sizeof(TcArgs));
        w.tc_args1 = (TcArgs *)take((size_t)w.tc_gmax * sizeof(TcArgs));
        // wide tiles: per-window |v| bound, the pass's stream, A tiles of
        // every group of 16 templates (at most all C channels each)
        w.vwmax = (float *)take(((size_t)W + 2) * 4);
        w.ws_brk = (u8 *)take(window_bytes_u8(W));
        w.ws_runs = (u32 *)take(Wp * 4);
        w.ws_pos = (u32 *)take(Wp * 4);
        w.ws_first = (u32 *)take(((size_t)W * (2 * (size_t)L) / kWPos + 4) * 4);
        w.Aw = (unsigned char *)take((size_t)w.tc_gmax * C * tcw_nkc(L) * kWATile);
        w.tgrp_w = (u32 *)take((size_t)K * 4);
        w.tcw_gdesc = (u32 *)take((size_t)w.tc_gmax * 12);
        w.tcw_args = (TcwArgs *)take((size_t)w.tc_gmax * sizeof(TcwArgs));
    }
    w.n = n;
    w.bytes = off;
    return w;
}

int grid_for(u64 items, int threads, int per_sm = 8) {
    u64 b = (items + threads - 1) / threads;
    u64 cap = (u64)sm_count() * per_sm;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// Ordered compaction of f[0..W) into list; count written to *count_dev.
int compact(const u8 *f, u32 W, u32 *list, u32 *count_dev, u32 *tile_counts, cudaStream_t st) {
    const u32 tiles = ceil_div(W, kCompactTile);
    if (tiles == 0) {
        FBP_CUDA(cudaMemsetAsync(count_dev, 0, 4, st));
        return FBP_OK;
    }
    k_compact_count<<<tiles, kCompactThreads, 0, st>>>(f, W, tile_counts);
    k_compact_scan<<<1, kCompactThreads, 0, st>>>(tile_counts, tiles, count_dev);
    k_compact_write<<<tiles, kCompactThreads, 0, st>>>(f, W, tile_counts, list);
    FBP_LAUNCH_CHECK();
    return FBP_OK;
}

int launch_likelihood(const float *v, u32 n, u32 C, const float *T, u32 K, u32 L, const float *tss,
                      const u32 *win, const u32 *n_win_dev, u32 max_windows, float *Lk,
                      cudaStream_t st, const u32 *gate = nullptr, u8 *apx = nullptr,
                      const u32 *tperm = nullptr, const u32 *grange = nullptr, WinBounds wb = WinBounds{}) {
    const size_t smem = (size_t)kLikChanChunk * (kLikTile + L) * sizeof(float);
    if (smem > 48 * 1024) {
        FBP_ALLOW_SMEM(k_likelihood_fp32);
    }
    const u64 items = (u64)max_windows * ceil_div(K, kLikTplPerBlock);
    const int grid = grid_for(items * kLikThreads, kLikThreads, 16);
    k_likelihood_fp32<<<grid, kLikThreads, smem, st>>>(v, n, C, T, K, L, tss, win, n_win_dev, Lk, gate, apx,
                                                       tperm, grange, wb);
    FBP_LAUNCH_CHECK();
    return FBP_OK;
}

int launch_argmax(u32 n, u32 L, u32 K, const u32 *win, const u32 *n_win_dev, u32 max_windows,
                  const fbp_window_state &s, float *Lk, cudaStream_t st, const LazyLk &z = LazyLk{},
                  WinBounds wb = WinBounds{}) {
    const int threads = kArgmaxThreads;
    const int grid = grid_for((u64)max_windows * 32, threads, 8);
    k_window_argmax<<<grid, threads, 0, st>>>(n, L, K, win, n_win_dev, s.best_idx, s.best_lab, s.best_ll,
                                              s.flags, s.overlap_recheck, s.ov_idx, s.ov_lab, Lk, z, wb);
    FBP_LAUNCH_CHECK();
    return FBP_OK;
}

int launch_overlap(const float *v, u32 n, u32 C, const float *T, u32 K, u32 L, const u32 *cand,
                   const u32 *n_cand_dev, u32 max_cand, const fbp_window_state &s, float *Lk,
                   u32 nmax, const float *thr, u64 *items_evaluated, cudaStream_t st,
                   const LazyLk &z = LazyLk{}, const u32 *tsup = nullptr) {
    const size_t smem = (size_t)2 * C * L * sizeof(float);
    if (smem > 227 * 1024)
        return fail(FBP_ERR_BAD_ARG, "overlap recheck: C*L = %u too large for shared memory", C * L);
    if (smem > 48 * 1024) {
        FBP_ALLOW_SMEM(k_overlap_exact);
    }
    const int grid = grid_for((u64)max_cand * kOvThreads, kOvThreads, 4);
    k_overlap_exact<<<grid, kOvThreads, smem, st>>>(v, n, C, T, K, L, cand, n_cand_dev, s.best_idx,
                                                    s.best_lab, s.best_ll, s.ov_idx, s.ov_lab,
                                                    s.overlap_recheck, Lk, nmax, thr, items_evaluated, z, tsup);
    FBP_LAUNCH_CHECK();
    return FBP_OK;
}

int launch_check_overlap(u32 n, u32 L, const u32 *cand, const u32 *n_cand_dev, u32 max_cand,
                         const fbp_window_state &s, u8 *scratch, cudaStream_t st) {
    const int threads = 256;
    const int grid = grid_for(max_cand, threads, 8);
    k_check_overlap<<<grid, threads, 0, st>>>(n, L, cand, n_cand_dev, s.best_idx, s.best_lab, s.flags,
                                              s.ov_idx, s.ov_lab, s.overlap_recheck, scratch);
    k_copy_ovr<<<grid, threads, 0, st>>>(cand, n_cand_dev, scratch, s.overlap_recheck);
    FBP_LAUNCH_CHECK();
    return FBP_OK;
}

int launch_accept(u32 n, u32 C, u32 L, const float *thr, const u32 *win, const u32 *n_win_dev,
                  u32 max_windows, const fbp_window_state &s, const u8 *active, u8 *has, u8 *flags_out,
                  u32 *acc_list, u32 *spk_idx, u32 *spk_lab, u32 *spk_win, u32 *n_spk_dev,
                  u32 *tile_counts, cudaStream_t st) {
    const u32 W = ceil_div(n, L);
    const int threads = 256;
    FBP_CUDA(cudaMemsetAsync(has, 0, window_bytes_u8(W), st));
    k_accept_has<<<grid_for(max_windows, threads), threads, 0, st>>>(
        n, C, L, thr, win, n_win_dev, s.best_idx, s.best_lab, s.best_ll, s.overlap_recheck, has);
    AcceptView a{n, C, L, W, n / L, thr, s.best_idx, s.best_lab, s.best_ll, active, has, s.flags};
    k_accept_flags<<<grid_for(W, threads), threads, 0, st>>>(a, flags_out);
    FBP_LAUNCH_CHECK();
    int rc = compact(has, W, acc_list, n_spk_dev, tile_counts, st);
    if (rc) return rc;
    k_gather_spikes<<<grid_for(W, threads), threads, 0, st>>>(n, C, L, acc_list, n_spk_dev, s.best_idx,
                                                              s.best_lab, spk_idx, spk_lab, spk_win);
    FBP_LAUNCH_CHECK();
    return FBP_OK;
}

float tc_kappa(u32 C, u32 L, u32 Cg2);
float tc_kappa_s(u32 C, u32 L);
TcArgs tc_group_args(const Workspace &w, u32 gi, const float *v, u32 n, u32 C, const float *T, u32 K, u32 L,
                     const float *tss, float *Lk, Counters *cnt);

// Context for likelihood entries the tensor-core path left approximate.
LazyLk lazy_ctx(const Workspace &w, const float *v, const float *T, const float *tss, u32 C, u32 L, u32 pass) {
    LazyLk z{};
    if (!w.tc) return z;
    z.apx = w.apx; z.wn = w.wn_s; z.wa = w.wa_s; z.kx = w.kx_s;
    z.tnorm = w.tc_tnorm; z.tabs = w.tc_tabs; z.tss = tss; z.texp = w.tc_texp;
    z.v = v; z.T = T; z.C = C; z.L = L;
    z.kappa_b = tc_kappa(w.tc_nz, L, ceil_div(w.tc_nz, 8));
    z.kappa_s = tc_kappa_s(w.tc_nz, L);
    z.tgrp = w.tcw ? w.tgrp_w : w.tgrp; z.gstride = w.n; z.tsup = w.tsup;
    z.refined = &w.cnt->lazy_ref;
    z.wlb = w.wlb; z.bm = w.bm_s;
    z.tag = 2u + (pass & 1u);
    return z;
}

OvArgs ov_args(const Workspace &w, const float *v, u32 n, u32 C, const float *T, u32 K, u32 L, u32 nmax,
               const float *thr, const fbp_window_state &s, float *Lk, const u32 *cand,
               const u32 *n_cand, Counters *cnt, const float *tss) {
    OvArgs A{};
    A.n = n; A.C = C; A.K = K; A.L = L; A.nmax = nmax; A.S = 2 * nmax + 1;
    A.v = v; A.T = T; A.Lk = Lk; A.thr = thr;
    A.NT = w.NT; A.sNT = w.sNT; A.tnorm = w.tnorm; A.Q = w.Q; A.XMr = w.XMr; A.XM = w.XM; A.oc = w.oc;
    A.cand = cand; A.n_cand = n_cand;
    A.best_idx = s.best_idx; A.best_lab = s.best_lab; A.ov_idx = s.ov_idx; A.ov_lab = s.ov_lab;
    A.best_ll = s.best_ll; A.ovr = s.overlap_recheck;
    A.H = w.H; A.vn = w.vn; A.cskip = w.cskip;
    A.cand_lb = w.cand_lb;
    A.ga_lo = w.ga_lo; A.ga_hi = w.ga_hi; A.ga_bits = w.ga_bits; A.ga_max = w.ga_max; A.ga_abs = w.ga_abs;
    A.seed_a1 = w.seed_a1;
    A.pair_mb = w.pair_mb; A.pair_mabs = w.pair_mabs;
    A.tsup = w.tsup;
    A.pool_slot = w.pool_slot; A.pool_item = w.pool_item; A.pool_hi = w.pool_hi; A.pool_cap = w.pool_cap;
    A.refined = &cnt->ov_ref;
    A.scan_next = &cnt->scan_next;
    A.best_key = w.best_key; A.fallback = w.fallback;
    A.items_evaluated = &cnt->ov_items;
    A.pool_total = &cnt->pool_total;
    A.ua = w.ua;
    A.lazy = lazy_ctx(w, v, T, tss, C, L, 0);   // read only: the tag is not used
    if (w.tc) {                      // H from the tensor cores
        A.km_override = tc_kappa(w.tc_nz, L, ceil_div(w.tc_nz, 8));
        A.tgrp = w.tgrp;
        A.kt_slots = w.slots;
        A.tabs = w.tc_tabs;
        A.texp = w.tc_texp;
        A.kexp_tile = w.kexp_tile;
        A.stiles = w.stiles;
    }
    return A;
}

// Per-chunk tables of the fast overlap recheck (templates are fixed).
int ov_chunk_setup(const Workspace &w, const float *T, u32 K, u32 C, u32 L, u32 nmax, cudaStream_t st) {
    const u32 S = 2 * nmax + 1;
    k_ov_chunk_tables<<<grid_for((u64)K * S, 256), 256, 0, st>>>(T, K, C, L, nmax, w.NT, w.sNT, w.tnorm, w.oc,
                                                                  w.tsup);
    const u64 rows = (u64)K * K * (2 * L - 1);
    k_ov_q_table<<<grid_for(rows, 128, 16), 128, 0, st>>>(T, K, C, L, w.Q, w.tsup);
    const size_t xm_smem = (size_t)(2 * L - 1) * (L + 1) * 4;
    if (xm_smem > 48 * 1024)
        FBP_ALLOW_SMEM(k_ov_xm);
    k_ov_xm<<<(int)std::min<u64>((u64)K * K, (u64)sm_count() * 2), 256, xm_smem, st>>>(w.Q, K, L, nmax, w.oc, w.XMr,
                                                                                        w.XM);
    FBP_LAUNCH_CHECK();
    return FBP_OK;
}

// One pass of the fast overlap recheck over the candidate list (device count
// n_cand).  Returns the number of kernels launched in *launches.
int ov_fast_tables(const Workspace &w, const OvArgs &A, Counters *cnt, cudaStream_t st, int *launches) {
    const u32 slots = w.slots;
    const u32 S = A.S;
    FBP_CUDA(cudaMemsetAsync(w.fallback, 0, align_up((size_t)slots + FBP_WINDOW_PAD, kCompactTile), st));
    FBP_CUDA(cudaMemsetAsync(&cnt->pool_total, 0, 4, st));
    FBP_CUDA(cudaMemsetAsync(&cnt->ov_ref, 0, 4, st));
    FBP_CUDA(cudaMemsetAsync(&cnt->scan_next, 0, 8, st));
    k_ov_prep<<<grid_for((u64)slots * 32, 256), 256, 0, st>>>(A);
    FBP_LAUNCH_CHECK();
    if (w.tc) {
        FBP_ALLOW_SMEM(k_lik_tc<1>);
        const u32 G = (u32)w.tcg.size();
        k_lik_tc<1><<<std::max<u32>(sm_count(), G), kTcThreads, w.tc_smem, st>>>(w.tc_args1, G);
        FBP_LAUNCH_CHECK();
    } else if (w.masked_tables) {
        const size_t smem = tables_m_smem_bytes(S, A.L);
        if (smem > 48 * 1024)
            FBP_ALLOW_SMEM(k_ov_tables_m);
        k_ov_tables_m<<<grid_for((u64)slots * ceil_div(A.K, kTabMGroup) * kTabMThreads, kTabMThreads, 4),
                        kTabMThreads, smem, st>>>(A, w.tperm, w.tsup, w.grange32);
        FBP_LAUNCH_CHECK();
    } else {
        const size_t smem = tables_smem_bytes(S, A.K, A.L);
        if (smem > 48 * 1024)
            FBP_ALLOW_SMEM(k_ov_tables);
        k_ov_tables<<<grid_for((u64)slots * kTabThreads, kTabThreads, 4), kTabThreads, smem, st>>>(A);
        FBP_LAUNCH_CHECK();
    }
    *launches = 2;
    return FBP_OK;
}

// The search over the tables: rows, seed, scan, exact refinement of the
// contenders, parse, and the exact kernel for candidates whose contenders did
// not fit.
int ov_fast_pass(const Workspace &w, const OvArgs &A, Counters *cnt, cudaStream_t st, int *launches) {
    const u32 slots = w.slots;
    const u32 S = A.S;
    k_ov_rows<<<grid_for((u64)slots * 32, kSeedThreads, 8), kSeedThreads, 0, st>>>(A);
    k_ov_seed<<<grid_for((u64)slots * A.K * 32, kSeedThreads, 8), kSeedThreads, 0, st>>>(A);
    const size_t scan_smem = scan_smem_bytes(S);
    if (scan_smem > 48 * 1024)
        FBP_ALLOW_SMEM(k_ov_scan);
    k_ov_scan<<<grid_for((u64)slots * A.K * 32, kScanThreads, 8), kScanThreads, scan_smem, st>>>(A);
    k_ov_refine<<<(int)sm_count() * 16, kRefineThreads, 0, st>>>(A);
    k_ov_finalize<<<grid_for((u64)slots * 32, kRefineThreads, 8), kRefineThreads, 0, st>>>(A);
    FBP_LAUNCH_CHECK();
    int rc = compact(w.fallback, slots, w.fb_slots, &cnt->fb_count, w.tile_counts, st);
    if (rc) return rc;
    k_ov_fallback_list<<<grid_for(slots, 256), 256, 0, st>>>(A, w.fb_slots, &cnt->fb_count, w.fb_list);
    FBP_LAUNCH_CHECK();
    fbp_window_state s{A.best_idx, A.best_lab, A.best_ll, A.ov_idx, A.ov_lab, nullptr, A.ovr};
    rc = launch_overlap(A.v, A.n, A.C, A.T, A.K, A.L, w.fb_list, &cnt->fb_count, slots, s, A.Lk, A.nmax, A.thr,
                        A.items_evaluated, st, A.lazy, w.tsup);
    *launches = 10;
    return rc;
}

// Per template: ||t||_2, ||t||_1 (rounded up) and the power-of-two scale that
// brings its largest magnitude just under 2^14 in fp16.  One warp per
// template: lanes stride over its C*L values, double sums reduced over the
// warp (the 1e-6 margin covers any summation order's rounding).
__global__ void k_tnorm(const float *__restrict__ T, u32 K, u32 CL, float *__restrict__ out,
                        float *__restrict__ out1, int *__restrict__ texp) {
    const u32 lane = threadIdx.x & 31u, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (u32 t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < K; t += nwarps) {
        double ss = 0.0, s1 = 0.0;
        float mx = 0.0f;
        for (u32 i = lane; i < CL; i += 32) {
            const float x = T[(size_t)t * CL + i];
            ss += (double)x * x;
            s1 += fabs((double)x);
            mx = fmaxf(mx, fabsf(x));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ss += __shfl_xor_sync(0xffffffffu, ss, o);
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        if (lane == 0) {
            out[t] = (float)(sqrt(ss) * (1.0 + 1e-6));
            out1[t] = (float)(s1 * (1.0 + 1e-6));
            int e = 0;
            if (mx > 0.0f) {
                frexpf(mx, &e);
                e = 14 - e;
            }
            texp[t] = e;
        }
    }
}

__global__ void k_tc_gate(Counters *cnt, u32 cap, u32 seg_cap) {
    const u64 rs = cnt->tc_refseg;
    cnt->tc_overflow = ((u32)(rs >> 32) > cap || (u32)rs > seg_cap) ? 1u : 0u;
}

int tc_chunk_setup(const Workspace &w, const float *v, u32 n, const float *T, u32 K, u32 C, u32 L,
                   cudaStream_t st) {
    k_tnorm<<<grid_for((u64)K * 32, 256), 256, 0, st>>>(T, K, C * L, w.tc_tnorm, w.tc_tabs, w.tc_texp);
    for (const TcGroup &g : w.tcg) {
        const u64 total = (u64)L * g.Cg2 * g.Np;
        k_tc_pack_templates<<<grid_for(total, 256), 256, 0, st>>>(T, g.nt, C, g.clo, g.Cg, L, g.Cg2, g.Np,
                                                                   w.tc_texp, w.tperm + g.t0, w.Tb + g.tb_off);
    }
    if (w.tcw) {
        const u32 nkc = tcw_nkc(L);
        for (const TcGroup &g : w.tcwg) {
            const u64 total = (u64)g.Cg * nkc * (kWATile / 2);
            k_tcw_pack<<<grid_for(total, 256), 256, 0, st>>>(T, C, L, nkc, w.tperm + g.t0, g.nt, g.clo, g.Cg,
                                                              w.tc_texp, (u16 *)(w.Aw + g.tb_off * kWATile));
        }
        const u32 W = ceil_div(n, L);
        k_window_vmax<<<grid_for((u64)(W + 2) * 32, 256, 8), 256, 0, st>>>(v, n, C, L, W, w.vwmax);
    }
    FBP_LAUNCH_CHECK();
    return FBP_OK;
}

// Launch arguments of one wide-tile group.
TcwArgs tcw_group_args(const Workspace &w, u32 gi, const float *v, u32 n, u32 C, u32 K, u32 L, const float *tss,
                       float *Lk, Counters *cnt) {
    const TcGroup &g = w.tcwg[gi];
    TcwArgs A{};
    A.n = n; A.Cg = g.Cg; A.nt = g.nt; A.L = L;
    A.nkc = tcw_nkc(L); A.ns = w.tcw_ns; A.px = tcw_px(L); A.Kall = K; A.W = ceil_div(n, L);
    A.trow = w.tperm + g.t0;
    A.kappa_b = tc_kappa(w.tc_nz, L, ceil_div(w.tc_nz, 8));
    A.kappa_s = tc_kappa_s(w.tc_nz, L);
    A.v = v + (size_t)g.clo * n;
    A.tss = tss; A.tnorm = w.tc_tnorm; A.tabs = w.tc_tabs; A.texp = w.tc_texp;
    A.Aw = w.Aw + g.tb_off * kWATile;
    A.vwmax = w.vwmax;
    A.win = w.win; A.n_win = &cnt->n_win;
    A.pos = w.ws_pos; A.first = w.ws_first; A.n_stiles = &cnt->n_stiles;
    A.Lk = Lk; A.apx = w.apx;
    A.wn_s = w.wn_s + (size_t)gi * n; A.wa_s = w.wa_s + (size_t)gi * n; A.kx_s = w.kx_s + (size_t)gi * n;
    A.bm_s = w.bm_s; A.wlb = w.wlb; A.umax = w.umax; A.wpos = w.wpos;
    A.ref_t = w.tc_ref_t; A.ref_s = w.tc_ref_s; A.refseg = &cnt->tc_refseg; A.ref_cap = w.tc_ref_cap;
    A.seg_s0 = w.tc_seg_s0; A.seg_base = w.tc_seg_base; A.seg_cnt = w.tc_seg_cnt; A.seg_grp = w.tc_seg_grp;
    A.grp = gi;
    A.seg_overflow = &cnt->tc_overflow; A.seg_cap = w.tc_seg_cap;
    A.err = &cnt->tc_err;
    A.wait_polls = g_lim_wait.load();
    return A;
}

// Launch arguments of one template group of the tensor-core kernel.
TcArgs tc_group_args(const Workspace &w, u32 gi, const float *v, u32 n, u32 C, const float *T, u32 K, u32 L,
                     const float *tss, float *Lk, Counters *cnt) {
    const TcGroup &g = w.tcg[gi];
    TcArgs A{};
    A.n = n; A.C = g.Cg; A.K = g.nt; A.L = L;
    A.trow = w.tperm + g.t0; A.Kall = K; A.tstride = C * L;
    A.Cg2 = g.Cg2; A.Np = g.Np;
    A.rows_pad = (kTcM + L - 1 + 7) / 8 * 8;
    A.tmem_cols = g.cols;
    A.nbuf = g.nbuf;
    A.kappa_b = tc_kappa(w.tc_nz, L, ceil_div(w.tc_nz, 8));
    A.kappa_s = tc_kappa_s(w.tc_nz, L);
    A.v = v + (size_t)g.clo * n; A.T = T; A.tss = tss;
    A.tnorm = w.tc_tnorm; A.tabs = w.tc_tabs; A.texp = w.tc_texp;
    A.Tb = w.Tb + g.tb_off;
    A.tb_bytes = (u32)((size_t)L * g.Cg2 * g.Np * 16);
    A.Lk = Lk;
    A.ref_t = w.tc_ref_t; A.ref_s = w.tc_ref_s; A.refseg = &cnt->tc_refseg; A.ref_cap = w.tc_ref_cap;
    A.seg_s0 = w.tc_seg_s0; A.seg_base = w.tc_seg_base; A.seg_cnt = w.tc_seg_cnt; A.seg_grp = w.tc_seg_grp;
    A.grp = gi;
    A.seg_overflow = &cnt->tc_overflow; A.seg_cap = w.tc_seg_cap;
    A.err = &cnt->tc_err;
    A.wait_polls = g_lim_wait.load();
    A.apx = w.apx; A.bm_s = w.bm_s; A.wlb = w.wlb; A.umax = w.umax; A.wpos = w.wpos;
    A.wn_s = w.wn_s + (size_t)gi * n; A.wa_s = w.wa_s + (size_t)gi * n; A.kx_s = w.kx_s + (size_t)gi * n;
    return A;
}

// Bound on |tensor-core value - reference value| per unit of
// ||t|| * ||window||: both operands rounded to fp16 (normal range; the
// subnormal part is a separate absolute term), FP32 accumulation of every
// product allowed one ulp of error, and the reference's own recursive sum.
// C is the number of channels whose products can be non-zero (a template's
// support): zero products add nothing and round nothing.
float tc_kappa(u32 C, u32 L, u32 Cg2) {
    const double u_h = 1.0 / 2048.0, u = 1.0 / 16777216.0;
    const double prod = 2.0 * u_h + u_h * u_h;
    const double n_acc = (double)Cg2 * 8 * L + 1;
    const double n_ref = (double)C * L + 2;
    const double k = prod + (1.0 + 4 * u_h) * n_acc * 2.0 * u + 1.01 * n_ref * u;
    return (float)(k * 1.01);
}

// Bound per unit of |SS_t / 2|: the reference's running sum starts at
// -SS_t/2, and each of its C*L + 1 roundings is relative to a partial sum
// that may be as large as |SS_t/2| + sum|t v| (the sum|t v| part is in
// tc_kappa); plus the final fp32 addition of the approximation.
float tc_kappa_s(u32 C, u32 L) {
    const double u = 1.0 / 16777216.0;
    const double n_ref = (double)C * L + 2;
    return (float)((1.01 * n_ref * u + 4.0 * u) * 1.01);
}

// One pass of the tensor-core likelihood over the listed windows: the tiles,
// one launch per template group.
int tc_likelihood_pass(const Workspace &w, const float *v, u32 n, u32 C, const float *T, u32 K, u32 L,
                       const float *tss, const u32 *win, const u32 *n_win, u32 max_windows, float *Lk,
                       Counters *cnt, cudaStream_t st, int *launches) {
    (void)max_windows;
    FBP_CUDA(cudaMemsetAsync(&cnt->tc_refseg, 0, 8, st));
    FBP_CUDA(cudaMemsetAsync(&cnt->tc_overflow, 0, 4, st));   // set by the tiles when the list overflows
    (void)v; (void)C; (void)T; (void)K; (void)tss; (void)Lk;
    if (w.tcw) {
        // the pass's window stream: run starts, their list, stream positions
        const u32 W = ceil_div(n, L);
        const size_t wbb = window_bytes_u8(W);
        k_ws_breaks<<<grid_for(wbb, 256), 256, 0, st>>>(win, n_win, (u32)wbb, w.ws_brk);
        FBP_LAUNCH_CHECK();
        if (int rc = compact(w.ws_brk, W, w.ws_runs, &cnt->n_runs, w.tile_counts, st)) return rc;
        k_ws_pos<<<grid_for(W, 256), 256, 0, st>>>(n_win, w.ws_brk, w.ws_runs, &cnt->n_runs, L, w.ws_pos,
                                                    w.ws_first, &cnt->n_stiles);
        FBP_LAUNCH_CHECK();
        FBP_ALLOW_SMEM(k_lik_tcw);
        const u32 G = (u32)w.tcwg.size();
        k_lik_tcw<<<std::max<u32>(sm_count(), G), kTcThreads, w.tcw_smem, st>>>(w.tcw_args, G);
        FBP_LAUNCH_CHECK();
        *launches = 6;
        return FBP_OK;
    }
    (void)win; (void)n_win;
    FBP_ALLOW_SMEM(k_lik_tc<0>);
    const u32 G = (u32)w.tcg.size();
    k_lik_tc<0><<<std::max<u32>(sm_count(), G), kTcThreads, w.tc_smem, st>>>(w.tc_args0, G);
    FBP_LAUNCH_CHECK();
    *launches = 1;
    return FBP_OK;
}

// The same pass: the refinement list, and the FP32 kernel over the listed
// windows when that list overflowed.
int tc_refine_pass(const Workspace &w, const float *v, u32 n, u32 C, const float *T, u32 K, u32 L,
                   const float *tss, const u32 *win, const u32 *n_win, u32 max_windows, float *Lk,
                   Counters *cnt, cudaStream_t st, int *launches) {
    const size_t rsmem = tc_refine_smem_bytes(w.tc_cmax, L);
    if (rsmem > 48 * 1024)
        FBP_ALLOW_SMEM(k_tc_refine);
    // gamma: the reference's recursive sum of C*L + 1 terms (products
    // rounded once each), plus the double sums' own error
    const double u = 1.0 / 16777216.0, nr = (double)w.tc_nz * L + 2;
    const double gamma = 1.01 * (nr * u / (1.0 - nr * u)) + 4.0 * nr * 1.1102230246251565e-16;
    k_tc_refine<<<sm_count() * 8, kRefThreads, rsmem, st>>>(
        v, n, C, w.tc_cmax, T, K, L, tss, w.tc_ref_t, w.tc_ref_s, w.tc_seg_s0, w.tc_seg_base, w.tc_seg_cnt,
        w.tc_seg_grp, w.tcw ? w.tcw_gdesc : w.tc_gdesc, w.tperm, reinterpret_cast<const u32 *>(&cnt->tc_refseg), w.tc_seg_cap, Lk,
        lazy_ctx(w, v, T, tss, C, L, 0), gamma, &cnt->tc_seq, w.wpos, &cnt->tc_overflow, w.tc_ref_cap);
    k_tc_gate<<<1, 1, 0, st>>>(cnt, w.tc_ref_cap, w.tc_seg_cap);
    FBP_LAUNCH_CHECK();
    int rc = launch_likelihood(v, n, C, T, K, L, tss, win, n_win, max_windows, Lk, st, &cnt->tc_overflow, w.apx,
                               w.tperm, w.grange, WinBounds{w.wlb, w.umax, w.wpos});
    *launches = 3;
    return rc;
}

// CUDA-event timing of the stages of a pass.  Events come from a pool that
// is drained after every host synchronisation (collect()).
class StageTimer {
  public:
    StageTimer(bool on, cudaStream_t st, fbp_stage_stats *s) : on_(on), st_(st), s_(s) {}
    ~StageTimer() {
        for (auto &e : pool_) cudaEventDestroy(e);
    }
    void begin(int stage) {
        if (!on_) return;
        cur_stage_ = stage;
        cur_begin_ = next();
        cudaEventRecord(cur_begin_, st_);
    }
    void end(int stage) {
        if (!on_) return;
        cudaEvent_t e = next();
        cudaEventRecord(e, st_);
        pending_.push_back({stage, cur_begin_, e});
    }
    void collect() {
        if (!on_) return;
        for (auto &p : pending_) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, p.b, p.e) == cudaSuccess) s_->ms[p.stage] += ms;
        }
        pending_.clear();
        used_ = 0;
    }

  private:
    struct Pending { int stage; cudaEvent_t b, e; };
    cudaEvent_t next() {
        if (used_ == pool_.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            pool_.push_back(e);
        }
        return pool_[used_++];
    }
    bool on_;
    cudaStream_t st_;
    fbp_stage_stats *s_;
    std::vector<cudaEvent_t> pool_;
    std::vector<Pending> pending_;
    size_t used_ = 0;
    int cur_stage_ = 0;
    cudaEvent_t cur_begin_ = nullptr;
};

u32 overlap_neighbours(u32 L, u32 nmax) {
    // spikes of one pass lie within n_max_shift of their window; two of them
    // can overlap only if their windows are fewer than 2 + 2*nmax/L apart.
    return 3 + ceil_div(2 * nmax, L);
}

// Instantiated pass graphs of recent calls.  A graph holds the pointers and
// sizes it was captured with, so it is reused only by a call with all of them
// equal (device, buffers, sizes and modes): it then enqueues exactly the
// launches a fresh capture would.
struct PassGraphs {
    std::vector<uint64_t> key;
    cudaGraphExec_t gx[2] = {nullptr, nullptr};
    uint64_t launches[2][FBP_N_STAGES] = {};
};
std::mutex g_graph_mu;
std::vector<PassGraphs> g_graphs;            // most recent last
constexpr size_t kGraphCacheSize = 8;

// Pinned host copy of the counters and a capture stream, per thread and device.
struct HostScratch {
    int dev = -1;
    u32 *counts = nullptr;
    cudaStream_t capture = nullptr;
};
thread_local HostScratch t_scratch;
int host_scratch(HostScratch **out) {
    int dev = 0;
    FBP_CUDA(cudaGetDevice(&dev));
    HostScratch &h = t_scratch;
    if (h.dev != dev) {
        if (!h.counts) FBP_CUDA(cudaMallocHost(&h.counts, sizeof(Counters)));
        h.capture = nullptr;                 // streams belong to the device they were made on
        FBP_CUDA(cudaStreamCreateWithFlags(&h.capture, cudaStreamNonBlocking));
        h.dev = dev;
    }
    *out = &h;
    return FBP_OK;
}

// Per-chunk set-up shared by fbp_pursuit_chunk and fbp_tc_likelihood_bounds:
// state zeroed as the reference's buffers start (.py:387, :412-423), every
// window listed, template supports and order, the tensor-core group plan and
// launch arguments (dbg_bound: the testing output of the bound E), and the
// fast overlap recheck's template tables.
int prepare_chunk(Workspace &w, float *voltage, u32 n, u32 C, const float *templates, u32 K, u32 L,
                  const float *neg_half_ss, u32 nmax, int do_overlap_recheck, cudaStream_t st,
                  fbp_stage_stats &S, StageTimer &timer, float *dbg_bound) {
    const u32 W = ceil_div(n, L);
    const size_t Wp = (size_t)W + FBP_WINDOW_PAD;
    const size_t wb = window_bytes_u8(W);
    // reference buffers start zeroed (.py:387, :412-423)
    timer.begin(FBP_STAGE_LISTS);
    FBP_CUDA(cudaMemsetAsync(w.cnt, 0, sizeof(Counters), st));
    FBP_CUDA(cudaMemsetAsync(w.Lk, 0, (size_t)K * n * sizeof(float), st));
    FBP_CUDA(cudaMemsetAsync(w.best_idx, 0, Wp * 4, st));
    FBP_CUDA(cudaMemsetAsync(w.best_lab, 0, Wp * 4, st));
    FBP_CUDA(cudaMemsetAsync(w.best_ll, 0, Wp * 4, st));
    FBP_CUDA(cudaMemsetAsync(w.ov_idx, 0, Wp * 4, st));
    FBP_CUDA(cudaMemsetAsync(w.ov_lab, 0, Wp * 4, st));
    FBP_CUDA(cudaMemsetAsync(w.flags, 0, wb, st));
    FBP_CUDA(cudaMemsetAsync(w.ovr, 0, wb, st));
    FBP_CUDA(cudaMemsetAsync(w.ovr2, 0, wb, st));
    FBP_CUDA(cudaMemsetAsync(w.active, 0, wb, st));
    FBP_CUDA(cudaMemsetAsync(w.wlb, 0, (size_t)W * 4, st));
    FBP_CUDA(cudaMemsetAsync(w.umax, 0, (size_t)W * K * 4, st));
    FBP_CUDA(cudaMemsetAsync(w.wpos, 0, (size_t)W, st));
    k_iota_windows<<<grid_for(W, 256), 256, 0, st>>>(w.win, w.active, W, w.cnt);
    k_template_ranges<<<grid_for((u64)K * 32, 256), 256, 0, st>>>(templates, K, C, L, w.tsup);
    k_template_support<<<1, 256, 0, st>>>(templates, K, C, L, w.tsup, w.tperm, w.grange, kLikTplPerBlock,
                                          w.grange32, kTabMGroup);
    FBP_LAUNCH_CHECK();
    if (w.tc || (w.fast && do_overlap_recheck)) {
        // template supports on the host (one small read-back per chunk): the
        // tensor-core group plan and the choice of overlap-table kernel
        const u32 ng = ceil_div(K, kTabMGroup);
        std::vector<u32> tsup(2 * (size_t)K), tperm(K), gr(2 * (size_t)ng);
        FBP_CUDA(cudaMemcpyAsync(tsup.data(), w.tsup, tsup.size() * 4, cudaMemcpyDeviceToHost, st));
        FBP_CUDA(cudaMemcpyAsync(tperm.data(), w.tperm, tperm.size() * 4, cudaMemcpyDeviceToHost, st));
        FBP_CUDA(cudaMemcpyAsync(gr.data(), w.grange32, gr.size() * 4, cudaMemcpyDeviceToHost, st));
        FBP_CUDA(cudaStreamSynchronize(st));
        if (w.tc) {
            if (!plan_tc_groups(tsup, tperm, K, C, L, w.tc_gmax, w.tcg)) {
                w.tc = false;                        // no group fits: the FP32 kernel
            } else {
                w.tc_cg2max = w.tc_cmax = 0;
                // adding an exact zero product is exact (in the reference's
                // sum and in any accumulation order), so the rounding bounds
                // count the widest support's products, not C*L
                w.tc_nz = 1;
                for (u32 t = 0; t < K; t++)
                    if (tsup[2 * t + 1] > tsup[2 * t]) w.tc_nz = std::max(w.tc_nz, tsup[2 * t + 1] - tsup[2 * t]);
                std::vector<u32> gdesc(3 * w.tcg.size()), tgrp(K);
                for (u32 gi = 0; gi < (u32)w.tcg.size(); gi++) {
                    const TcGroup &g = w.tcg[gi];
                    w.tc_cg2max = std::max(w.tc_cg2max, g.Cg2);
                    w.tc_cmax = std::max(w.tc_cmax, g.Cg);
                    gdesc[3 * gi] = g.t0; gdesc[3 * gi + 1] = g.clo; gdesc[3 * gi + 2] = g.Cg;
                    for (u32 j = g.t0; j < g.t0 + g.nt; j++) tgrp[tperm[j]] = gi;
                }
                FBP_CUDA(cudaMemcpyAsync(w.tc_gdesc, gdesc.data(), gdesc.size() * 4, cudaMemcpyHostToDevice, st));
                FBP_CUDA(cudaMemcpyAsync(w.tgrp, tgrp.data(), tgrp.size() * 4, cudaMemcpyHostToDevice, st));
                // the likelihood passes' layout: wide tiles where they apply
                w.tcw = false;
                if (t_tc_layout != FBP_TC_LAYOUT_SAMPLES) {
                    w.tcw_ns = plan_tcw_groups(tsup, tperm, K, C, L, w.tcwg);
                    // the stream table marks tail outputs in bit 31 of a sample
                    w.tcw = w.tcw_ns > 0 && n < 0x80000000u;
                }
                std::vector<u32> gdesc_w(3 * w.tcwg.size()), tgrp_w(K);
                if (w.tcw) {
                    for (u32 gi = 0; gi < (u32)w.tcwg.size(); gi++) {
                        const TcGroup &g = w.tcwg[gi];
                        w.tc_cmax = std::max(w.tc_cmax, g.Cg);
                        gdesc_w[3 * gi] = g.t0; gdesc_w[3 * gi + 1] = g.clo; gdesc_w[3 * gi + 2] = g.Cg;
                        for (u32 j = g.t0; j < g.t0 + g.nt; j++) tgrp_w[tperm[j]] = gi;
                    }
                    FBP_CUDA(cudaMemcpyAsync(w.tcw_gdesc, gdesc_w.data(), gdesc_w.size() * 4,
                                             cudaMemcpyHostToDevice, st));
                    FBP_CUDA(cudaMemcpyAsync(w.tgrp_w, tgrp_w.data(), tgrp_w.size() * 4, cudaMemcpyHostToDevice,
                                             st));
                }
                FBP_CUDA(cudaStreamSynchronize(st));   // the host vectors go out of scope
            }
        }
        if (w.fast && do_overlap_recheck && !w.tc) {
            // the masked overlap tables pay off when the template groups
            // touch well under all channels
            u64 span = 0;
            for (u32 g = 0; g < ng; g++) span += gr[2 * g + 1] - gr[2 * g];
            w.masked_tables = 2 * span < (u64)ng * C && 2 * nmax + 1 <= 32u * kTabMShiftChunks;
        }
    }
    S.launches[FBP_STAGE_LISTS] += 1;
    timer.end(FBP_STAGE_LISTS);
    if (w.tc) {
        timer.begin(FBP_STAGE_LIKELIHOOD);
        FBP_CUDA(cudaMemsetAsync(w.apx, 0, (size_t)K * n, st));
        FBP_CUDA(cudaMemsetAsync(w.bm_s, 0, (size_t)n * 4, st));
        int rc0 = tc_chunk_setup(w, voltage, n, templates, K, C, L, st);
        if (rc0) return rc0;
        // launch arguments of every template group (constant for the chunk)
        {
            const u32 G = (u32)w.tcg.size();
            std::vector<TcArgs> a0(G), a1(G);
            w.tc_smem = 0;
            for (u32 gi = 0; gi < G; gi++) {
                a0[gi] = tc_group_args(w, gi, voltage, n, C, templates, K, L, neg_half_ss, w.Lk, w.cnt);
                a0[gi].win = w.win;
                a0[gi].n_win = &w.cnt->n_win;
                // short templates: a tile holds the rows of wpt aligned windows
                a0[gi].wpt = (L >= 32 && 2 * L <= (u32)kTcM) ? (u32)kTcM / L : 1u;
                a0[gi].active = w.active;
                a0[gi].dbgE = dbg_bound;
                a1[gi] = tc_group_args(w, gi, voltage, n, C, templates, K, L, nullptr, nullptr, w.cnt);
                if (w.fast && do_overlap_recheck) {
                    a1[gi].S = 2 * nmax + 1; a1[gi].nmax = nmax; a1[gi].stiles = w.stiles;
                    a1[gi].cand = w.cand; a1[gi].n_cand = &w.cnt->n_cand; a1[gi].best_idx = w.best_idx;
                    a1[gi].cskip = w.cskip; a1[gi].NT = w.NT; a1[gi].H = w.H;
                    a1[gi].kexp_tile = w.kexp_tile + (size_t)gi * w.slots * w.stiles;
                }
                w.tc_smem = std::max(w.tc_smem, tc_smem_bytes(L, a0[gi].Cg2, a0[gi].Np, a0[gi].nbuf));
            }
            FBP_CUDA(cudaMemcpyAsync(w.tc_args0, a0.data(), G * sizeof(TcArgs), cudaMemcpyHostToDevice, st));
            FBP_CUDA(cudaMemcpyAsync(w.tc_args1, a1.data(), G * sizeof(TcArgs), cudaMemcpyHostToDevice, st));
            std::vector<TcwArgs> aw(w.tcwg.size());
            if (w.tcw) {
                for (u32 gi = 0; gi < (u32)aw.size(); gi++) {
                    aw[gi] = tcw_group_args(w, gi, voltage, n, C, K, L, neg_half_ss, w.Lk, w.cnt);
                    aw[gi].dbgE = dbg_bound;
                }
                FBP_CUDA(cudaMemcpyAsync(w.tcw_args, aw.data(), aw.size() * sizeof(TcwArgs), cudaMemcpyHostToDevice,
                                         st));
                w.tcw_smem = tcw_smem_layout(L, w.tcw_ns).total;
            }
            FBP_CUDA(cudaStreamSynchronize(st));   // the host vectors go out of scope
        }
        S.tc_layout = w.tcw ? FBP_TC_LAYOUT_WIDE : FBP_TC_LAYOUT_SAMPLES;
        S.launches[FBP_STAGE_LIKELIHOOD] += 2;
        timer.end(FBP_STAGE_LIKELIHOOD);
    }
    if (w.fast && do_overlap_recheck) {
        timer.begin(FBP_STAGE_OVERLAP);
        int rc0 = ov_chunk_setup(w, templates, K, C, L, nmax, st);
        if (rc0) return rc0;
        S.launches[FBP_STAGE_OVERLAP] += 3;
        timer.end(FBP_STAGE_OVERLAP);
    }

    return FBP_OK;
}

}  // namespace

extern "C" {

int fbp_version(void) { return 100; }

const char *fbp_last_error(void) { return g_last_error.c_str(); }

size_t fbp_scan_scratch_bytes(uint32_t n_windows) {
    return (size_t)(ceil_div(n_windows, kCompactTile) + 1) * 4;
}

size_t fbp_window_u8_bytes(uint32_t n_windows) { return window_bytes_u8(n_windows); }

int fbp_pursuit_workspace_bytes(uint32_t n, uint32_t C, uint32_t K, uint32_t L, uint32_t nmax,
                                int precision, size_t *bytes_out) {
    if (!bytes_out || n == 0 || C == 0 || K == 0 || L == 0)
        return fail(FBP_ERR_BAD_ARG, "workspace size: bad arguments");
    *bytes_out = layout(nullptr, n, K, L, nmax, true, C, precision == FBP_PREC_BF16_REFINE).bytes;
    return FBP_OK;
}

int fbp_pursuit_chunk(float *voltage, uint32_t n, uint32_t C, const float *templates, uint32_t K,
                      uint32_t L, const float *neg_half_ss, const float *thresholds, uint32_t nmax,
                      int do_overlap_recheck, int precision, int overlap_method, uint32_t max_passes,
                      void *workspace, size_t workspace_bytes, uint32_t *spike_idx, uint32_t *spike_lab,
                      uint32_t spike_cap, uint32_t *pass_counts, uint32_t *n_spikes_host,
                      uint32_t *n_passes_host, int profile, fbp_stage_stats *stats, void *stream) {
    g_last_error.clear();
    if (!voltage || !templates || !neg_half_ss || !thresholds || !workspace || !spike_idx ||
        !spike_lab || !n_spikes_host || !n_passes_host)
        return fail(FBP_ERR_BAD_ARG, "fbp_pursuit_chunk: null pointer argument");
    if (n == 0 || C == 0 || K == 0 || L == 0)
        return fail(FBP_ERR_BAD_ARG, "fbp_pursuit_chunk: zero size (n=%u C=%u K=%u L=%u)", n, C, K, L);
    if (precision != FBP_PREC_FP32 && precision != FBP_PREC_BF16_REFINE)
        return fail(FBP_ERR_BAD_ARG, "fbp_pursuit_chunk: unknown precision %d", precision);
    if ((u64)2 * nmax + 1 > 0xffffffffull)
        return fail(FBP_ERR_BAD_ARG, "fbp_pursuit_chunk: n_max_shift too large");
    if (overlap_method != FBP_OVERLAP_FAST && overlap_method != FBP_OVERLAP_EXACT)
        return fail(FBP_ERR_BAD_ARG, "fbp_pursuit_chunk: unknown overlap method %d", overlap_method);
    Workspace w = layout((char *)workspace, n, K, L, nmax, overlap_method == FBP_OVERLAP_FAST, C,
                         precision == FBP_PREC_BF16_REFINE);
    if (workspace_bytes < w.bytes)
        return fail(FBP_ERR_BAD_ARG, "fbp_pursuit_chunk: workspace has %zu bytes, needs %zu",
                    workspace_bytes, w.bytes);
    const u32 lim_refine = g_lim_refine.load(), lim_pool = g_lim_pool.load(), lim_wait = g_lim_wait.load();
    if (lim_refine && w.tc) w.tc_ref_cap = std::min(w.tc_ref_cap, lim_refine);
    if (lim_pool && w.fast) w.pool_cap = std::min(w.pool_cap, lim_pool);
    cudaStream_t st = (cudaStream_t)stream;
    const u32 W = ceil_div(n, L);
    const size_t wb = window_bytes_u8(W);
    fbp_window_state s{w.best_idx, w.best_lab, w.best_ll, w.ov_idx, w.ov_lab, w.flags, w.ovr};
    fbp_stage_stats local_stats;
    fbp_stage_stats &S = stats ? *stats : local_stats;
    memset(&S, 0, sizeof(S));
    StageTimer timer(profile != 0, st, &S);

    if (int e = prepare_chunk(w, voltage, n, C, templates, K, L, neg_half_ss, nmax, do_overlap_recheck, st, S,
                              timer, nullptr))
        return e;
    HostScratch *hs = nullptr;
    if (int e = host_scratch(&hs)) return e;
    u32 *h_counts = hs->counts;
    const u32 R = overlap_neighbours(L, nmax);
    int rc = FBP_OK;
    u32 passes = 0;
    // One pass (.py:538-731), entirely device-driven: every kernel reads its
    // counts from device memory, so the same launches serve every pass.  The
    // counts of the pass are snapshotted (w.snap) before the next pass's
    // window list overwrites them.  `launched` receives the launches per stage.
    auto enqueue_pass = [&](u32 pass, uint64_t *launched, cudaStream_t q) -> int {
        int rc2 = FBP_OK;
        // 1. likelihood over the listed windows (.py:538-549)
        timer.begin(FBP_STAGE_LIKELIHOOD);
        if (w.tc) {
            int nl = 0;
            if ((rc2 = tc_likelihood_pass(w, voltage, n, C, templates, K, L, neg_half_ss, w.win, &w.cnt->n_win, W,
                                          w.Lk, w.cnt, q, &nl)))
                return rc2;
            launched[FBP_STAGE_LIKELIHOOD] += nl;
            timer.end(FBP_STAGE_LIKELIHOOD);
            timer.begin(FBP_STAGE_LIK_REFINE);
            if ((rc2 = tc_refine_pass(w, voltage, n, C, templates, K, L, neg_half_ss, w.win, &w.cnt->n_win, W,
                                      w.Lk, w.cnt, q, &nl)))
                return rc2;
            launched[FBP_STAGE_LIK_REFINE] += nl;
            timer.end(FBP_STAGE_LIK_REFINE);
            timer.begin(FBP_STAGE_LIKELIHOOD);
        } else {
            if ((rc2 = launch_likelihood(voltage, n, C, templates, K, L, neg_half_ss, w.win, &w.cnt->n_win, W,
                                         w.Lk, q, nullptr, nullptr, w.tperm, w.grange,
                                         WinBounds{w.wlb, w.umax, w.wpos})))
                return rc2;
            launched[FBP_STAGE_LIKELIHOOD] += 1;
        }
        timer.end(FBP_STAGE_LIKELIHOOD);
        // 2. per-window argmax over all templates (.py:551-562)
        timer.begin(FBP_STAGE_ARGMAX);
        const LazyLk lz = lazy_ctx(w, voltage, templates, neg_half_ss, C, L, pass);
        if ((rc2 = launch_argmax(n, L, K, w.win, &w.cnt->n_win, W, s, w.Lk, q, lz, WinBounds{w.wlb, w.umax, w.wpos})))
            return rc2;
        launched[FBP_STAGE_ARGMAX] += 1;
        timer.end(FBP_STAGE_ARGMAX);
        // 3. candidates = nonzero(overlap_recheck) (.py:565-569), 4. recheck (.py:570-661)
        if (do_overlap_recheck) {
            timer.begin(FBP_STAGE_LISTS);
            if ((rc2 = compact(w.ovr, W, w.cand, &w.cnt->n_cand, w.tile_counts, q))) return rc2;
            launched[FBP_STAGE_LISTS] += 3;
            timer.end(FBP_STAGE_LISTS);
            timer.begin(FBP_STAGE_OVERLAP);
            if (w.fast) {
                int nl = 0;
                OvArgs A = ov_args(w, voltage, n, C, templates, K, L, nmax, thresholds, s, w.Lk, w.cand,
                                   &w.cnt->n_cand, w.cnt, neg_half_ss);
                timer.end(FBP_STAGE_OVERLAP);
                timer.begin(FBP_STAGE_OVERLAP_TABLES);
                if ((rc2 = ov_fast_tables(w, A, w.cnt, q, &nl))) return rc2;
                launched[FBP_STAGE_OVERLAP_TABLES] += nl;
                timer.end(FBP_STAGE_OVERLAP_TABLES);
                timer.begin(FBP_STAGE_OVERLAP);
                if ((rc2 = ov_fast_pass(w, A, w.cnt, q, &nl))) return rc2;
                launched[FBP_STAGE_OVERLAP] += nl;
            } else {
                if ((rc2 = launch_overlap(voltage, n, C, templates, K, L, w.cand, &w.cnt->n_cand, W, s, w.Lk,
                                          nmax, thresholds, &w.cnt->ov_items, q, lz, w.tsup)))
                    return rc2;
                launched[FBP_STAGE_OVERLAP] += 1;
            }
            timer.end(FBP_STAGE_OVERLAP);
            timer.begin(FBP_STAGE_CHECK);
            if ((rc2 = launch_check_overlap(n, L, w.cand, &w.cnt->n_cand, W, s, w.ovr2, q))) return rc2;
            launched[FBP_STAGE_CHECK] += 2;
            timer.end(FBP_STAGE_CHECK);
        }
        // 5. accept (.py:663-671)
        timer.begin(FBP_STAGE_ACCEPT);
        if ((rc2 = launch_accept(n, C, L, thresholds, w.win, &w.cnt->n_win, W, s, w.active, w.has,
                                 w.flags_out, w.acc_list, w.spk_idx, w.spk_lab, w.spk_win, &w.cnt->n_spk,
                                 w.tile_counts, q)))
            return rc2;
        launched[FBP_STAGE_ACCEPT] += 6;
        timer.end(FBP_STAGE_ACCEPT);
        // 6. the pass's counts (.py:673-676 stops when nothing was added)
        FBP_CUDA(cudaMemcpyAsync(w.snap, w.cnt, sizeof(Counters), cudaMemcpyDeviceToDevice, q));
        // 7. reset overlap flags, next list = nonzero(flags), reset flags (.py:678-700)
        timer.begin(FBP_STAGE_LISTS);
        FBP_CUDA(cudaMemsetAsync(w.ovr, 0, wb, q));
        if ((rc2 = compact(w.flags_out, W, w.win, &w.cnt->n_win, w.tile_counts, q))) return rc2;
        k_mark_active<<<grid_for(W, 256), 256, 0, q>>>(w.flags_out, w.active, W, WinBounds{w.wlb, w.umax, w.wpos},
                                                       w.tc ? w.bm_s : nullptr, L, n, K);
        FBP_CUDA(cudaMemsetAsync(w.flags, 0, wb, q));
        // 8. keep the spikes (.py:702-710)
        k_append_spikes<<<grid_for(W, 256), 256, 0, q>>>(w.spk_idx, w.spk_lab, w.cnt, spike_idx, spike_lab,
                                                           spike_cap);
        k_commit_total<<<1, 1, 0, q>>>(w.cnt, spike_cap);
        FBP_LAUNCH_CHECK();
        launched[FBP_STAGE_LISTS] += 6;
        timer.end(FBP_STAGE_LISTS);
        // 9. subtract them (.py:712-731)
        timer.begin(FBP_STAGE_RESIDUAL);
        if (lz.apx) {
            k_lazy_freeze<<<grid_for((u64)W * 32, 256, 8), 256, 0, q>>>(n, L, K, w.spk_idx, w.spk_lab,
                                                                        &w.cnt->n_spk, w.active, W, w.Lk, lz);
            FBP_LAUNCH_CHECK();
            launched[FBP_STAGE_RESIDUAL] += 1;
        }
        k_residual<<<grid_for((u64)W * 256, 256, 16), 256, 0, q>>>(voltage, n, C, templates, K, L, w.spk_idx,
                                                                    w.spk_lab, &w.cnt->n_spk, 0, R, w.tsup,
                                                                    w.tcw ? w.vwmax : nullptr);
        FBP_LAUNCH_CHECK();
        launched[FBP_STAGE_RESIDUAL] += 1;
        timer.end(FBP_STAGE_RESIDUAL);
        return FBP_OK;
    };
    // Without per-stage timing each pass is one CUDA graph launch (one graph
    // per pass parity: the parity is the only thing that differs).  Graphs
    // are captured on a private stream (the caller's may be the legacy
    // default stream, which cannot capture) and launched on the caller's.
    const bool use_graph = profile == 0;
    PassGraphs pg;
    if (use_graph) {
        int dev = 0;
        cudaGetDevice(&dev);
        pg.key = {(uint64_t)dev, (uint64_t)(uintptr_t)voltage, n, C, (uint64_t)(uintptr_t)templates, K, L,
                  (uint64_t)(uintptr_t)neg_half_ss, (uint64_t)(uintptr_t)thresholds, nmax,
                  (uint64_t)do_overlap_recheck, (uint64_t)precision, (uint64_t)overlap_method,
                  (uint64_t)(uintptr_t)workspace, (uint64_t)workspace_bytes, (uint64_t)(uintptr_t)spike_idx,
                  (uint64_t)(uintptr_t)spike_lab, spike_cap, (uint64_t)w.masked_tables, (uint64_t)w.tc,
                  lim_refine, lim_pool, lim_wait, (uint64_t)w.tcw, w.tcw_ns};
        for (const TcGroup &g : w.tcg)               // the group plan follows the template supports
            if (w.tc) pg.key.insert(pg.key.end(), {g.t0, g.nt, g.clo, g.Cg, g.nbuf});
        std::lock_guard<std::mutex> lk(g_graph_mu);
        for (size_t i = 0; i < g_graphs.size(); i++)
            if (g_graphs[i].key == pg.key) {
                pg = g_graphs[i];
                g_graphs.erase(g_graphs.begin() + i);   // back in the cache when this call ends
                break;
            }
    }
    cudaGraphExec_t *gx = pg.gx;
    uint64_t (*glaunch)[FBP_N_STAGES] = pg.launches;
    cudaStream_t cs = hs->capture;
    for (;;) {
        if (passes >= max_passes) { rc = fail(FBP_ERR_ITER_CAP, "no convergence after %u passes", passes); break; }
        passes++;
        const u32 par = passes & 1u;
        if (use_graph) {
            if (!gx[par]) {
                cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
                if (e != cudaSuccess) { rc = fail(FBP_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e)); break; }
                const int rc2 = enqueue_pass(passes, glaunch[par], cs);
                cudaGraph_t g = nullptr;
                e = cudaStreamEndCapture(cs, &g);
                if (rc2) { if (g) cudaGraphDestroy(g); rc = rc2; break; }
                if (e == cudaSuccess) e = cudaGraphInstantiate(&gx[par], g, 0);
                if (g) cudaGraphDestroy(g);
                if (e != cudaSuccess) { rc = fail(FBP_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e)); break; }
            }
            cudaError_t e = cudaGraphLaunch(gx[par], st);
            if (e != cudaSuccess) { rc = fail(FBP_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e)); break; }
            for (int k = 0; k < FBP_N_STAGES; k++) S.launches[k] += glaunch[par][k];
        } else {
            if ((rc = enqueue_pass(passes, S.launches, st))) break;
        }
        {
            cudaError_t e = cudaMemcpyAsync(h_counts, w.snap, sizeof(Counters), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) { rc = fail(FBP_ERR_CUDA, "pass %u: %s", passes, cudaGetErrorString(e)); break; }
        }
        timer.collect();
        const u32 added = h_counts[2];
        const u32 nwin = h_counts[0];
        if (w.tc) {
            const Counters *hc = (const Counters *)h_counts;
            if (hc->tc_err) {
                rc = fail(FBP_ERR_TIMEOUT, "tensor-core kernel: bounded wait (role code %u) gave up", hc->tc_err);
                break;
            }
            S.lik_refined += std::min((u32)(hc->tc_refseg >> 32), w.tc_ref_cap);
            S.work[FBP_STAGE_LIK_REFINE] += std::min((u32)(hc->tc_refseg >> 32), w.tc_ref_cap);
            S.lik_exact_passes += hc->tc_overflow;
        }
        S.work[FBP_STAGE_LIKELIHOOD] += (u64)nwin * L * K;
        S.work[FBP_STAGE_ARGMAX] += (u64)nwin * 3 * L * K;
        S.work[FBP_STAGE_ACCEPT] += nwin;
        S.work[FBP_STAGE_RESIDUAL] += added;
        if (do_overlap_recheck) {
            S.work[FBP_STAGE_CHECK] += h_counts[1];
            S.candidates += h_counts[1];
            if (w.fast) S.work[FBP_STAGE_OVERLAP_TABLES] += h_counts[1];
            if (w.fast) {
                S.refined_items += ((const Counters *)h_counts)->ov_ref;
                S.fallback_candidates += h_counts[7];
            }
        }
        if (pass_counts)
            FBP_CUDA(cudaMemcpyAsync(pass_counts + passes - 1, &w.snap->n_spk, 4, cudaMemcpyDeviceToDevice, st));
        if (added == 0) break;
    }
    if (use_graph && (gx[0] || gx[1])) {
        std::lock_guard<std::mutex> lk(g_graph_mu);
        g_graphs.push_back(pg);
        if (g_graphs.size() > kGraphCacheSize) {
            for (auto &g : g_graphs.front().gx)
                if (g) cudaGraphExecDestroy(g);
            g_graphs.erase(g_graphs.begin());
        }
    }
    if (rc == FBP_OK || rc == FBP_ERR_ITER_CAP) {
        cudaError_t e = cudaMemcpyAsync(h_counts, w.cnt, sizeof(Counters), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = fail(FBP_ERR_CUDA, "final readback: %s", cudaGetErrorString(e));
        else {
            timer.collect();
            *n_spikes_host = h_counts[3];
            S.spikes = h_counts[3];
            S.work[FBP_STAGE_OVERLAP] = *(const u64 *)(h_counts + 8);
            S.lik_lazy_refined = ((const Counters *)h_counts)->lazy_ref;
            S.lik_seq_refined = ((const Counters *)h_counts)->tc_seq;
            if (h_counts[4]) rc = fail(FBP_ERR_CAPACITY, "spike output holds %u spikes; more were found", spike_cap);
        }
    }
    *n_passes_host = passes;
    S.passes = passes;
    return rc;
}

int fbp_set_tc_group_size(uint32_t templates_per_group) {
    g_last_error.clear();
    if (templates_per_group != 0 && (templates_per_group % 16 != 0 || templates_per_group > 256))
        return fail(FBP_ERR_BAD_ARG, "fbp_set_tc_group_size: %u is not 0 or a multiple of 16 up to 256",
                    templates_per_group);
    t_tc_group_size = templates_per_group;
    return FBP_OK;
}

int fbp_set_tc_layout(int layout) {
    g_last_error.clear();
    if (layout != FBP_TC_LAYOUT_AUTO && layout != FBP_TC_LAYOUT_SAMPLES && layout != FBP_TC_LAYOUT_WIDE)
        return fail(FBP_ERR_BAD_ARG, "fbp_set_tc_layout: unknown layout %d", layout);
    t_tc_layout = layout;
    return FBP_OK;
}

int fbp_set_test_limits(const fbp_test_limits *lim) {
    g_last_error.clear();
    g_lim_refine.store(lim ? lim->refine_list_cap : 0u);
    g_lim_pool.store(lim ? lim->contender_pool_cap : 0u);
    g_lim_wait.store(lim ? lim->wait_polls : FBP_DEFAULT_WAIT_POLLS);
    return FBP_OK;
}

int fbp_tc_likelihood_bounds(const float *voltage, uint32_t n, uint32_t C, const float *templates, uint32_t K,
                             uint32_t L, const float *neg_half_ss, void *workspace, size_t workspace_bytes,
                             float *approx, float *bound, void *stream) {
    g_last_error.clear();
    if (!voltage || !templates || !neg_half_ss || !workspace || !approx || !bound)
        return fail(FBP_ERR_BAD_ARG, "fbp_tc_likelihood_bounds: null pointer argument");
    if (n == 0 || C == 0 || K == 0 || L == 0)
        return fail(FBP_ERR_BAD_ARG, "fbp_tc_likelihood_bounds: zero size");
    Workspace w = layout((char *)workspace, n, K, L, 0, false, C, true);
    if (workspace_bytes < w.bytes)
        return fail(FBP_ERR_BAD_ARG, "fbp_tc_likelihood_bounds: workspace has %zu bytes, needs %zu",
                    workspace_bytes, w.bytes);
    cudaStream_t st = (cudaStream_t)stream;
    fbp_stage_stats S;
    memset(&S, 0, sizeof(S));
    StageTimer timer(false, st, &S);
    FBP_CUDA(cudaMemsetAsync(bound, 0, (size_t)K * n * 4, st));
    if (int e = prepare_chunk(w, const_cast<float *>(voltage), n, C, templates, K, L, neg_half_ss, 0, 0, st, S,
                              timer, bound))
        return e;
    if (!w.tc) return fail(FBP_ERR_BAD_ARG, "fbp_tc_likelihood_bounds: no tensor-core plan for this shape");
    int nl = 0;
    if (int e = tc_likelihood_pass(w, voltage, n, C, templates, K, L, neg_half_ss, w.win, &w.cnt->n_win,
                                   ceil_div(n, L), w.Lk, w.cnt, st, &nl))
        return e;
    FBP_CUDA(cudaMemcpyAsync(approx, w.Lk, (size_t)K * n * 4, cudaMemcpyDeviceToDevice, st));
    u32 err = 0;
    FBP_CUDA(cudaMemcpyAsync(&err, &w.cnt->tc_err, 4, cudaMemcpyDeviceToHost, st));
    FBP_CUDA(cudaStreamSynchronize(st));
    if (err) return fail(FBP_ERR_TIMEOUT, "tensor-core kernel: bounded wait (role code %u) gave up", err);
    return FBP_OK;
}

int fbp_compute_residual(float *voltage, uint32_t n, uint32_t C, const float *templates, uint32_t K,
                         uint32_t L, const uint32_t *spike_idx, const uint32_t *spike_lab,
                         uint32_t n_spikes, uint32_t max_overlap_neighbours, void *stream) {
    g_last_error.clear();
    if (n_spikes == 0 || C == 0) return FBP_OK;
    if (!voltage || !templates || !spike_idx || !spike_lab)
        return fail(FBP_ERR_BAD_ARG, "fbp_compute_residual: null pointer argument");
    k_residual<<<grid_for((u64)n_spikes * 256, 256, 16), 256, 0, (cudaStream_t)stream>>>(
        voltage, n, C, templates, K, L, spike_idx, spike_lab, nullptr, n_spikes, max_overlap_neighbours, nullptr);
    FBP_LAUNCH_CHECK();
    return FBP_OK;
}

int fbp_get_adjusted_clips(const float *voltage, uint32_t n, uint32_t C, const float *templates,
                           uint32_t K, uint32_t L, const uint32_t *spike_idx, const uint32_t *spike_lab,
                           uint32_t n_spikes, float *clips, void *stream) {
    g_last_error.clear();
    if (n_spikes == 0 || C == 0) return FBP_OK;
    if (!voltage || !templates || !spike_idx || !spike_lab || !clips)
        return fail(FBP_ERR_BAD_ARG, "fbp_get_adjusted_clips: null pointer argument");
    k_adjusted_clips<<<grid_for((u64)n_spikes * 256, 256, 16), 256, 0, (cudaStream_t)stream>>>(
        voltage, n, C, templates, K, L, spike_idx, spike_lab, n_spikes, clips);
    FBP_LAUNCH_CHECK();
    return FBP_OK;
}

int fbp_compute_full_likelihood(const float *voltage, uint32_t n, uint32_t C, const float *templates,
                                uint32_t K, uint32_t L, const float *neg_half_ss,
                                const uint32_t *window_list, const uint32_t *n_windows_dev,
                                uint32_t max_windows, float *likelihood, int precision, void *stream) {
    g_last_error.clear();
    if (!voltage || !templates || !neg_half_ss || !window_list || !n_windows_dev || !likelihood)
        return fail(FBP_ERR_BAD_ARG, "fbp_compute_full_likelihood: null pointer argument");
    if (C == 0 || max_windows == 0) return FBP_OK;
    (void)precision;
    return launch_likelihood(voltage, n, C, templates, K, L, neg_half_ss, window_list, n_windows_dev,
                             max_windows, likelihood, (cudaStream_t)stream);
}

int fbp_window_argmax(uint32_t n, uint32_t L, uint32_t K, const uint32_t *window_list,
                      const uint32_t *n_windows_dev, uint32_t max_windows, const fbp_window_state *st,
                      const float *likelihood, void *stream) {
    g_last_error.clear();
    if (!st || !window_list || !n_windows_dev || !likelihood)
        return fail(FBP_ERR_BAD_ARG, "fbp_window_argmax: null pointer argument");
    if (max_windows == 0) return FBP_OK;
    return launch_argmax(n, L, K, window_list, n_windows_dev, max_windows, *st, const_cast<float *>(likelihood),
                         (cudaStream_t)stream);
}

int fbp_overlap_recheck(const float *voltage, uint32_t n, uint32_t C, const float *templates, uint32_t K,
                        uint32_t L, const uint32_t *cand_list, const uint32_t *n_cand_dev, uint32_t max_cand,
                        const fbp_window_state *st, const float *likelihood, uint32_t nmax,
                        const float *thresholds, void *stream) {
    g_last_error.clear();
    if (!voltage || !templates || !cand_list || !n_cand_dev || !st || !likelihood || !thresholds)
        return fail(FBP_ERR_BAD_ARG, "fbp_overlap_recheck: null pointer argument");
    if (max_cand == 0) return FBP_OK;
    return launch_overlap(voltage, n, C, templates, K, L, cand_list, n_cand_dev, max_cand, *st,
                          const_cast<float *>(likelihood), nmax, thresholds, nullptr, (cudaStream_t)stream);
}

int fbp_check_overlap_reassignments(uint32_t n, uint32_t L, const uint32_t *cand_list,
                                    const uint32_t *n_cand_dev, uint32_t max_cand,
                                    const fbp_window_state *st, uint8_t *scratch, void *stream) {
    g_last_error.clear();
    if (!cand_list || !n_cand_dev || !st || !scratch)
        return fail(FBP_ERR_BAD_ARG, "fbp_check_overlap_reassignments: null pointer argument");
    if (max_cand == 0) return FBP_OK;
    return launch_check_overlap(n, L, cand_list, n_cand_dev, max_cand, *st, scratch, (cudaStream_t)stream);
}

int fbp_binary_pursuit_accept(uint32_t n, uint32_t C, uint32_t L, const float *thresholds,
                              const uint32_t *window_list, const uint32_t *n_windows_dev,
                              uint32_t max_windows, const fbp_window_state *st, const uint8_t *active,
                              uint8_t *has, uint8_t *flags_out, uint32_t *spike_idx, uint32_t *spike_lab,
                              uint32_t *spike_win, uint32_t *n_spikes_dev, void *scan_scratch,
                              void *stream) {
    g_last_error.clear();
    if (!thresholds || !window_list || !n_windows_dev || !st || !active || !has || !flags_out ||
        !spike_idx || !spike_lab || !n_spikes_dev || !scan_scratch)
        return fail(FBP_ERR_BAD_ARG, "fbp_binary_pursuit_accept: null pointer argument");
    // the compaction list reuses spike_win when given, else spike_idx as scratch is unsafe
    if (!spike_win) return fail(FBP_ERR_BAD_ARG, "fbp_binary_pursuit_accept: spike_win is required");
    return launch_accept(n, C, L, thresholds, window_list, n_windows_dev, max_windows, *st, active, has,
                         flags_out, spike_win, spike_idx, spike_lab, nullptr, n_spikes_dev,
                         (u32 *)scan_scratch, (cudaStream_t)stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free accept: the scratch of fbp_binary_pursuit_accept (the
// per-window accept bytes and the compaction's tile offsets) in a file-scope
// device array, for callers that cannot allocate device memory.
// ---------------------------------------------------------------------------
namespace {

static __device__ __align__(256) unsigned char g_accept_scratch[FBP_NOALLOC_SCRATCH_BYTES];

constexpr size_t kNoallocHasBytes = 4194304;   // align_up(FBP_NOALLOC_MAX_WINDOWS + pad, 4096)
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char *g_noalloc_ptr[kMaxDevices] = {nullptr};

// Device address of g_accept_scratch on the current device, looked up once
// per device.  Host code must not use the symbol itself as a pointer.
int noalloc_scratch(unsigned char **out) {
    int dev = 0;
    FBP_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(FBP_ERR_BAD_ARG, "device index %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_accept_scratch);
        if (e != cudaSuccess || !p)
            return fail(FBP_ERR_CUDA, "cudaGetSymbolAddress(accept scratch) failed: %s", cudaGetErrorString(e));
        g_noalloc_ptr[dev] = (unsigned char *)p;
    }
    *out = g_noalloc_ptr[dev];
    return FBP_OK;
}

}  // namespace

static_assert(kNoallocHasBytes >= ((size_t)FBP_NOALLOC_MAX_WINDOWS + FBP_WINDOW_PAD + kCompactTile - 1) /
                                       kCompactTile * kCompactTile,
              "accept bytes do not fit the no-alloc scratch");
static_assert(FBP_NOALLOC_SCRATCH_BYTES - kNoallocHasBytes >=
                  (size_t)((FBP_NOALLOC_MAX_WINDOWS + kCompactTile - 1) / kCompactTile + 1) * 4,
              "tile offsets do not fit the no-alloc scratch");

extern "C" int fbp_binary_pursuit_accept_noalloc(uint32_t n, uint32_t C, uint32_t L, const float *thresholds,
                                                 const uint32_t *window_list, const uint32_t *n_windows_dev,
                                                 uint32_t max_windows, const fbp_window_state *st,
                                                 const uint8_t *active, uint8_t *flags_out, uint32_t *spike_idx,
                                                 uint32_t *spike_lab, uint32_t *spike_win, uint32_t *n_spikes_dev,
                                                 void *stream) {
    g_last_error.clear();
    if (!thresholds || !window_list || !n_windows_dev || !st || !active || !flags_out || !spike_idx ||
        !spike_lab || !spike_win || !n_spikes_dev)
        return fail(FBP_ERR_BAD_ARG, "fbp_binary_pursuit_accept_noalloc: null pointer argument");
    if (L == 0) return fail(FBP_ERR_BAD_ARG, "fbp_binary_pursuit_accept_noalloc: template_len is 0");
    const u32 W = ceil_div(n, L);
    if (W > FBP_NOALLOC_MAX_WINDOWS)
        return fail(FBP_ERR_BAD_ARG,
                    "fbp_binary_pursuit_accept_noalloc: %u windows exceed the fixed scratch limit of %u "
                    "windows (use fbp_binary_pursuit_accept with caller-provided scratch)",
                    W, FBP_NOALLOC_MAX_WINDOWS);
    unsigned char *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    u8 *has = scratch;                                        // cleared by launch_accept
    u32 *tile_offsets = (u32 *)(scratch + kNoallocHasBytes);  // fully rewritten by the compaction
    return launch_accept(n, C, L, thresholds, window_list, n_windows_dev, max_windows, *st, active, has, flags_out,
                         spike_win, spike_idx, spike_lab, nullptr, n_spikes_dev, tile_offsets,
                         (cudaStream_t)stream);
}

