/*
 * Oracle: CPU restatement of Full Binary Pursuit (TEST INFRASTRUCTURE ONLY).
 *
 * This file restates, in plain C, the device kernels of the reference
 * (spikesorting_fullpursuit/kernels/binary_pursuit.cl) and the per-chunk host
 * loop that drives them (spikesorting_fullpursuit/parallel/
 * binary_pursuit_parallel.py:386-736).  It is the checker the CUDA product is
 * compared against; nothing in the product links or calls it.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 *
 * Execution semantics.  The reference's result depends on the OpenCL
 * scheduler at three places: the neighbour-flag reads/writes inside the
 * `binary_pursuit` kernel (.cl:1009-1045), the `overlap_recheck[id-2]` read in
 * `check_overlap_reassignments` (.cl:852), and the non-atomic residual
 * subtraction (.cl:89-97); and on the work-group size at exact ties of the
 * overlap tree reduction (.cl:167-186).  The only deterministic reading is
 * the one a work-group size of 1 gives when work-items run one after another
 * in global-id order.  This oracle implements exactly that reading, and the
 * unmodified reference kernels compiled for CPU (oracle/ref_launch.c) run the
 * same way; tests pin the two against each other.
 *
 * Arithmetic.  Every floating-point operation is the reference's, in the
 * reference's order, in IEEE binary32 with no contraction (build with
 * -ffp-contract=off).  The one double-precision step is the per-channel
 * `-= 0.5 * summed_chan_ss` of the overlap recheck (.cl:627-630), where the
 * literal 0.5 promotes the expression to double.
 *
 * Parity: pinned against the reference's own host code and kernels run in
 * this container (tests/golden/make_golden.py, tests/test_oracle_pin.py).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint32_t u32;
typedef uint8_t u8;

/* Work counters (for profiling the algorithm, not part of its semantics):
 * [0] likelihood samples x templates evaluated, [1] overlap candidates,
 * [2] overlap (a, b, t) items that survive the skip rules, [3] passes. */
static unsigned long long g_counters[8];
void bpo_counters(unsigned long long *out, int reset)
{
    for (int i = 0; i < 8; i++) { out[i] = g_counters[i]; if (reset) g_counters[i] = 0; }
}

/* compute_maximum_likelihood, binary_pursuit.cl:216-252.  Start from
 * -0.5*SS (already scaled on the host, binary_pursuit_parallel.py:199), then
 * channel-outer, sample-inner accumulation of t*v. */
static float ml_at(const float *v, u32 n, u32 C, const float *T, u32 K, u32 L,
                   u32 index, u32 k, const float *tss)
{
    float m = 0.0f;
    if (index + L >= n) return m;               /* .cl:231-234 */
    if (k >= K) return m;                       /* .cl:235-238 */
    m = tss[k];                                 /* .cl:239 */
    for (u32 c = 0; c < C; c++) {               /* .cl:242-250 */
        const float *t = T + (size_t)k * L * C + (size_t)c * L;
        const float *vv = v + index + (size_t)n * c;
        for (u32 i = 0; i < L; i++) m = m + t[i] * vv[i];
    }
    return m;
}

/* compute_full_likelihood, binary_pursuit.cl:255-300: for every listed window
 * and every template, write the likelihood at each sample of the window. */
void bpo_compute_full_likelihood(const float *v, u32 n, u32 C, const float *T,
                                 u32 K, u32 L, const float *tss, const u32 *win,
                                 u32 nwin, float *Lk, int nthreads)
{
    if (C == 0) return;
    long long total = (long long)nwin * K;
    __atomic_fetch_add(&g_counters[0], (unsigned long long)total * L, __ATOMIC_RELAXED);
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads > 0 ? nthreads : 1)
    for (long long g = 0; g < total; g++) {
        u32 w = (u32)(g / K), k = (u32)(g % K);
        u32 id = win[w];
        u32 s0 = id * L;
        u32 s1 = ((id + 1) * L) > n ? n : (id + 1) * L;
        for (u32 i = 0; i < s1 - s0; i++)
            Lk[(size_t)k * n + s0 + i] = ml_at(v, n, C, T, K, L, s0 + i, k, tss);
    }
}

/* compute_template_maximum_likelihood, binary_pursuit.cl:350-441, launched
 * once per template in template order (binary_pursuit_parallel.py:551-562).
 * The K launches are folded into one loop per window; the per-window state
 * carries across templates exactly as the global buffers do. */
void bpo_template_maximum_likelihood(u32 n, u32 L, u32 K, const u32 *win, u32 nwin,
                                     u32 *best_idx, u32 *best_lab, float *best_ll,
                                     u8 *flags, u8 *ovr, u32 *ov_idx, u32 *ov_lab,
                                     const float *Lk)
{
    for (u32 k = 0; k < K; k++) {
        for (u32 g = 0; g < nwin; g++) {
            u32 id = win[g];
            u32 sw = id * L, ew = (id + 1) * L;
            u32 start = (L > sw) ? 0 : sw - L;
            u32 stop = (ew + L) > n ? n : ew + L;
            if (ew >= n - L) continue;                       /* .cl:380-383 */
            float bl = best_ll[id];
            u32 blab = best_lab[id], bidx = best_idx[id];
            if (k == 0) bl = 0.0f;                           /* .cl:389-393 */
            u8 check = 0;
            const float *row = Lk + (size_t)k * n + start;
            for (u32 i = 0; i < stop - start; i++) {         /* .cl:399-418 */
                float cur = row[i];
                if (cur > bl) { bl = cur; blab = k; bidx = start + i; }
                if (cur > 0.0f && start + i >= sw && start + i < ew) check = 1;
            }
            if (check) flags[id] = 1;                        /* .cl:419-422 */
            ovr[id] = 0;                                     /* .cl:423 */
            if (bl > 0.0f && bidx >= sw && bidx < ew) ovr[id] = 1; /* .cl:430-433 */
            best_ll[id] = bl; best_lab[id] = blab; best_idx[id] = bidx;
            ov_idx[id] = bidx; ov_lab[id] = blab;            /* .cl:435-439 */
        }
    }
}

/* Likelihood of the sum of the best template at shift a and template t at
 * shift b, clipped to [bidx, bidx+L): the body of overlap_recheck_indices,
 * binary_pursuit.cl:578-632. */
static float overlap_pair_ll(const float *v, u32 n, u32 C, const float *T, u32 L,
                             u32 lab, u32 bidx, u32 t, u32 afix, u32 ashift)
{
    float cml = 0.0f;
    int fa = (int)bidx - (int)afix;                  /* .cl:585 */
    u32 ffj = fa < 0 ? (u32)(-fa) : 0;
    int sa = (int)bidx - (int)ashift;                /* .cl:591 */
    u32 sfj = sa < 0 ? (u32)(-sa) : 0;
    for (u32 c = 0; c < C; c++) {
        const float *tf = T + (size_t)lab * L * C + (size_t)c * L;
        const float *ts = T + (size_t)t * L * C + (size_t)c * L;
        const float *vv = v + bidx + (size_t)n * c;
        float ss = 0.0f;
        for (u32 j = 0; j < L; j++) {
            float fv = 0.0f, sv = 0.0f;
            if (j >= ffj && (u32)(fa + (int)j) < L) fv = tf[fa + (int)j];
            if (j >= sfj && (u32)(sa + (int)j) < L) sv = ts[sa + (int)j];
            float s = fv + sv;
            ss += s * s;
            cml += s * vv[j];
        }
        if (ss > 0.0) cml = (float)((double)cml - 0.5 * (double)ss); /* .cl:627-630 */
    }
    return cml;
}

/* overlap_recheck_indices (binary_pursuit.cl:444-654) followed by
 * parse_overlap_recheck_indices (.cl:657-815), with a work-group size of 1:
 * each (a, b, t) work-item is its own group, so the parse kernel's scan over
 * group results (.cl:699-706) is a strict-greater scan over work-items in
 * ascending id, starting from the window's current best likelihood. */
void bpo_overlap_recheck(const float *v, u32 n, u32 C, const float *T, u32 K, u32 L,
                         const u32 *cand, u32 ncand, u32 *best_idx, u32 *best_lab,
                         float *best_ll, u32 *ov_idx, u32 *ov_lab, const float *Lk,
                         u32 nmax, const float *thr, u8 *ovr, int nthreads)
{
    const size_t S = 2 * (size_t)nmax + 1;
    const size_t items = S * S * K;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
    for (long long ci = 0; ci < (long long)ncand; ci++) {
        u32 id = cand[ci];
        u32 lab = best_lab[id], bidx = best_idx[id];
        float bll = Lk[(size_t)lab * n + bidx];
        int skip_all = 0;
        if (bll < thr[lab]) skip_all = 1;                    /* .cl:518-522 */
        if (bidx >= n - L) skip_all = 1;                     /* .cl:524-527 */
        float best_group = best_ll[id];                      /* .cl:690-694 */
        size_t best_item = 0;
        unsigned long long evaluated = 0;
        if (!skip_all) {
            for (size_t it = 0; it < items; it++) {
                u32 t = (u32)(it % K);                       /* .cl:530-532 */
                u32 a = (u32)((it / K) % S);
                u32 b = (u32)((it / (S * K)) % S);
                if (a + bidx < nmax || a + bidx >= n - L + nmax) continue;   /* .cl:534-537 */
                if (b + bidx < nmax || b + bidx >= n - L + nmax) continue;   /* .cl:538-541 */
                if (a > b && a - b > L) continue;            /* .cl:543-549 */
                if (b > a && b - a > L) continue;            /* .cl:550-556 */
                u32 afix = bidx + a - nmax, ashift = bidx + b - nmax;
                float lf = Lk[(size_t)lab * n + afix];
                float ls = Lk[(size_t)t * n + ashift];
                if (lf <= 0 && ls <= 0) continue;            /* .cl:572-576 */
                float ll = overlap_pair_ll(v, n, C, T, L, lab, bidx, t, afix, ashift);
                evaluated++;
                if (ll > best_group) { best_group = ll; best_item = it; }
            }
        }
        __atomic_fetch_add(&g_counters[1], 1ULL, __ATOMIC_RELAXED);
        __atomic_fetch_add(&g_counters[2], evaluated, __ATOMIC_RELAXED);
        /* parse_overlap_recheck_indices, .cl:707-814 */
        if (best_group <= best_ll[id] || best_group <= 0.0f) { ovr[id] = 0; continue; }
        u32 t = (u32)(best_item % K);
        u32 a = (u32)((best_item / K) % S);
        u32 b = (u32)((best_item / (S * K)) % S);
        u32 afix = bidx + a - nmax, ashift = bidx + b - nmax;
        float lf = Lk[(size_t)lab * n + afix];
        float ls = Lk[(size_t)t * n + ashift];
        if (best_group < lf || best_group < ls) { ovr[id] = 0; continue; }
        if (lf <= 0.0f || ls <= 0.0f) { ovr[id] = 0; continue; }
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
}

/* check_overlap_reassignments, binary_pursuit.cl:822-875, work-items in
 * candidate order. */
void bpo_check_overlap_reassignments(u32 n, u32 L, const u32 *cand, u32 ncand,
                                     u32 *best_idx, u32 *best_lab, u8 *flags,
                                     const u32 *ov_idx, const u32 *ov_lab, u8 *ovr)
{
    for (u32 g = 0; g < ncand; g++) {
        u32 id = cand[g];
        u32 sw = id * L, ew = (id + 1) * L;
        if (ovr[id] == 0) continue;
        best_idx[id] = ov_idx[id];
        best_lab[id] = ov_lab[id];
        if (ov_idx[id] < sw && id > 1) {
            if (ovr[id - 2] == 1) {
                ovr[id] = 0;
                best_idx[id] = 0;
                flags[id - 1] = 2; flags[id] = 2; flags[id + 1] = 2;
            } else {
                flags[id - 2] = 2;
            }
        }
        if (ov_idx[id] >= ew && id + 2 < n / L) flags[id + 2] = 2;
    }
}

/* binary_pursuit kernel, binary_pursuit.cl:918-1063, work-group size 1,
 * work-items in window-list order.  Returns the number of spikes appended. */
u32 bpo_binary_pursuit(u32 n, u32 C, u32 L, const float *thr, const u32 *win, u32 nwin,
                       const u32 *best_idx, const u32 *best_lab, const float *best_ll,
                       u32 *out_idx, u32 *out_lab, const u8 *ovr, u8 *flags)
{
    u32 count = 0;
    const u32 nw_floor = n / L;
    for (u32 g = 0; g < nwin; g++) {
        u32 id = win[g];
        u32 sw = id * L, ew = (id + 1) * L;
        u32 lab = 0, idx = 0;
        float ml = 0.0f;
        int valid = (ew < n - L) && C > 0;
        if (valid) { ml = best_ll[id]; lab = best_lab[id]; idx = best_idx[id]; }
        int has = 0;
        if (ml > thr[lab] || ovr[id] == 1) {                 /* .cl:982-999 */
            if ((idx >= sw && idx < ew) || ovr[id] == 1) {
                has = 1;
                flags[id] = 3;
                if (id > 0) flags[id - 1] = 3;
                if (id + 1 < nw_floor) flags[id + 1] = 3;
            }
        }
        if (valid && !has) {                                 /* .cl:1009-1045 */
            if (idx < sw && flags[id] == 1 && id > 0)
                if (flags[id - 1] == 0) flags[id] = 0;
            if (idx >= ew && flags[id] == 1 && id + 1 < nw_floor)
                if (flags[id + 1] == 0) flags[id] = 0;
            if (ml <= thr[lab] && flags[id] < 3) flags[id] = 0;
        }
        if (has) { out_idx[count] = idx; out_lab[count] = lab; count++; }
    }
    return count;
}

/* compute_residual, binary_pursuit.cl:57-102, spikes in list order. */
void bpo_compute_residual(float *v, u32 n, u32 C, const float *T, u32 K, u32 L,
                          const u32 *idx, const u32 *lab, u32 count)
{
    if (C == 0) return;
    for (u32 s = 0; s < count; s++) {
        if (lab[s] >= K) continue;
        for (u32 c = 0; c < C; c++) {
            float *vv = v + idx[s] + (size_t)n * c;
            const float *t = T + (size_t)lab[s] * L * C + (size_t)c * L;
            for (u32 i = 0; i < L; i++) {
                if (idx[s] + i >= n) break;
                vv[i] -= t[i];
            }
        }
    }
}

/* get_adjusted_clips, binary_pursuit.cl:1088-1130: clips must arrive zeroed. */
void bpo_get_adjusted_clips(const float *v, u32 n, u32 C, const float *T, u32 K, u32 L,
                            const u32 *idx, const u32 *lab, u32 count, float *clips)
{
    if (C == 0) return;
    for (u32 s = 0; s < count; s++) {
        if (lab[s] >= K) continue;
        for (u32 c = 0; c < C; c++) {
            const float *vv = v + idx[s] + (size_t)n * c;
            const float *t = T + (size_t)lab[s] * L * C + (size_t)c * L;
            float *o = clips + (size_t)s * L * C + (size_t)c * L;
            for (u32 i = 0; i < L; i++) {
                if (idx[s] + i >= n) break;
                o[i] = vv[i] + t[i];
            }
        }
    }
}

/* Per-chunk iterate-until-converged loop, binary_pursuit_parallel.py:386-736.
 * `v` (C x n, channel-major) is turned into the residual in place.  Spikes
 * are appended to out_idx/out_lab in pass order, window order within a pass
 * (the compaction order a work-group size of 1 produces).  pass_counts (may
 * be NULL) receives the spikes added per pass.  Returns the number of
 * spikes, or -1 if `cap` was too small, or -2 on allocation failure. */
long long bpo_pursuit_chunk(float *v, u32 n, u32 C, const float *T, u32 K, u32 L,
                            const float *tss, const float *thr, u32 nmax,
                            int do_overlap_recheck, u32 *out_idx, u32 *out_lab,
                            u32 cap, u32 *n_passes, u32 *pass_counts, u32 max_passes,
                            int nthreads)
{
    const u32 W = (n + L - 1) / L;                       /* :402 */
    const size_t Wp = (size_t)W + 4;                     /* padded state arrays */
    float *Lk = (float *)calloc((size_t)n * K, sizeof(float));   /* :387 */
    u32 *best_idx = (u32 *)calloc(Wp, 4), *best_lab = (u32 *)calloc(Wp, 4);
    float *best_ll = (float *)calloc(Wp, 4);
    u32 *ov_idx = (u32 *)calloc(Wp, 4), *ov_lab = (u32 *)calloc(Wp, 4);
    u8 *flags = (u8 *)calloc(Wp, 1), *ovr = (u8 *)calloc(Wp, 1);
    u32 *win = (u32 *)calloc(Wp, 4), *cand = (u32 *)calloc(Wp, 4);
    u32 *add_idx = (u32 *)calloc(Wp, 4), *add_lab = (u32 *)calloc(Wp, 4);
    long long total = 0;
    if (!Lk || !best_idx || !best_lab || !best_ll || !ov_idx || !ov_lab || !flags ||
        !ovr || !win || !cand || !add_idx || !add_lab) { total = -2; goto done; }
    u32 nwin = W;
    for (u32 i = 0; i < W; i++) win[i] = i;              /* :418 */
    u32 passes = 0;
    for (;;) {
        passes++;
        g_counters[3]++;
        bpo_compute_full_likelihood(v, n, C, T, K, L, tss, win, nwin, Lk, nthreads);
        bpo_template_maximum_likelihood(n, L, K, win, nwin, best_idx, best_lab, best_ll,
                                        flags, ovr, ov_idx, ov_lab, Lk);
        u32 ncand = 0;                                   /* :565-569 */
        for (u32 i = 0; i < W; i++) if (ovr[i]) cand[ncand++] = i;
        if (ncand > 0 && do_overlap_recheck) {           /* :570-661 */
            bpo_overlap_recheck(v, n, C, T, K, L, cand, ncand, best_idx, best_lab, best_ll,
                                ov_idx, ov_lab, Lk, nmax, thr, ovr, nthreads);
            bpo_check_overlap_reassignments(n, L, cand, ncand, best_idx, best_lab, flags,
                                            ov_idx, ov_lab, ovr);
        }
        u32 cnt = bpo_binary_pursuit(n, C, L, thr, win, nwin, best_idx, best_lab, best_ll,
                                     add_idx, add_lab, ovr, flags);
        if (pass_counts && passes <= max_passes) pass_counts[passes - 1] = cnt;
        if (cnt == 0) break;                             /* :673-676 */
        memset(ovr, 0, Wp);                              /* :679-680 */
        nwin = 0;                                        /* :683-689 */
        for (u32 i = 0; i < W; i++) if (flags[i]) win[nwin++] = i;
        memset(flags, 0, Wp);                            /* :699-700 */
        if (total + cnt > cap) { total = -1; goto done; }
        memcpy(out_idx + total, add_idx, (size_t)cnt * 4);   /* :702-710 */
        memcpy(out_lab + total, add_lab, (size_t)cnt * 4);
        total += cnt;
        bpo_compute_residual(v, n, C, T, K, L, add_idx, add_lab, cnt);   /* :712-731 */
    }
    if (n_passes) *n_passes = passes;
done:
    free(Lk); free(best_idx); free(best_lab); free(best_ll); free(ov_idx); free(ov_lab);
    free(flags); free(ovr); free(win); free(cand); free(add_idx); free(add_lab);
    return total;
}

/* Reference value (binary_pursuit.cl:578-632) of listed overlap items of one
 * candidate, whatever the skip rules say: item = t + K*(a + S*b). */
void bpo_overlap_items(const float *v, u32 n, u32 C, const float *T, u32 K, u32 L, u32 lab,
                       u32 bidx, u32 nmax, const unsigned long long *items, u32 count, float *out)
{
    const size_t S = 2 * (size_t)nmax + 1;
    for (u32 q = 0; q < count; q++) {
        unsigned long long it = items[q];
        u32 t = (u32)(it % K), a = (u32)((it / K) % S), b = (u32)((it / (S * K)) % S);
        u32 afix = bidx + a - nmax, ashift = bidx + b - nmax;
        out[q] = overlap_pair_ll(v, n, C, T, L, lab, bidx, t, afix, ashift);
    }
}
