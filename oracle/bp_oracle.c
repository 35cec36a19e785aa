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

/* Non-zero template rows.  A product t*v with t == 0 is +-0 (finite
 * voltage), and adding +-0 leaves a sum unchanged unless the sum is -0.  The
 * likelihood sum starts at float32(-0.5*SS) != 0 for a non-zero template and
 * the overlap sum at +0; neither can become -0 afterwards (in
 * round-to-nearest x + y is -0 only for -0 + -0).  So channels on which a
 * template's row is all zeros add nothing and are skipped -- a bit-exact
 * shortcut that matters for masked templates (e.g. 16 of 384 channels).
 * Rows are stored with P zeros on each side, so the overlap recheck's
 * shifted reads need no range tests (.cl:585-603 read 0 outside [0, L)). */
typedef struct {
    u32 K, C, L, P;
    float *pad;          /* padded non-zero rows, L + 2P floats each, then one zero row */
    const float **row;   /* [K*C]: index P of the padded row (or of the zero row) */
    u32 *nzc;            /* [K*C]: non-zero channels of template k, ascending */
    u32 *nnz;            /* [K]: how many */
    u8 *dense;           /* [K]: the template is all zeros (SS == 0): no skipping */
} TplRows;

static void tpl_rows_free(TplRows *r)
{
    free(r->pad); free((void *)r->row); free(r->nzc); free(r->nnz); free(r->dense);
    memset(r, 0, sizeof(*r));
}

static int tpl_rows_init(TplRows *r, const float *T, u32 K, u32 C, u32 L, u32 P)
{
    memset(r, 0, sizeof(*r));
    r->K = K; r->C = C; r->L = L; r->P = P;
    r->row = (const float **)calloc((size_t)K * C + 1, sizeof(float *));
    r->nzc = (u32 *)calloc((size_t)K * C + 1, 4);
    r->nnz = (u32 *)calloc((size_t)K + 1, 4);
    r->dense = (u8 *)calloc((size_t)K + 1, 1);
    size_t rows = 0;
    if (!r->row || !r->nzc || !r->nnz || !r->dense) { tpl_rows_free(r); return -1; }
    for (u32 k = 0; k < K; k++)
        for (u32 c = 0; c < C; c++) {
            const float *t = T + (size_t)k * L * C + (size_t)c * L;
            int nz = 0;
            for (u32 i = 0; i < L && !nz; i++) nz = t[i] != 0.0f;
            if (nz) r->nzc[(size_t)k * C + r->nnz[k]++] = c;
        }
    for (u32 k = 0; k < K; k++) {
        if (r->nnz[k] == 0) {            /* all-zero template: visit every channel */
            r->dense[k] = 1;
            for (u32 c = 0; c < C; c++) r->nzc[(size_t)k * C + c] = c;
            r->nnz[k] = C;
        }
        rows += r->nnz[k];
    }
    const size_t w = (size_t)L + 2 * (size_t)P;
    r->pad = (float *)calloc((rows + 1) * w, sizeof(float));
    if (!r->pad) { tpl_rows_free(r); return -1; }
    const float *zero = r->pad + rows * w + P;
    for (size_t q = 0; q < (size_t)K * C; q++) r->row[q] = zero;
    size_t q = 0;
    for (u32 k = 0; k < K; k++)
        for (u32 j = 0; j < r->nnz[k]; j++, q++) {
            const u32 c = r->nzc[(size_t)k * C + j];
            float *dst = r->pad + q * w + P;
            memcpy(dst, T + (size_t)k * L * C + (size_t)c * L, (size_t)L * sizeof(float));
            r->row[(size_t)k * C + c] = dst;
        }
    return 0;
}

/* compute_maximum_likelihood, binary_pursuit.cl:216-252.  Start from
 * -0.5*SS (already scaled on the host, binary_pursuit_parallel.py:199), then
 * channel-outer, sample-inner accumulation of t*v (zero rows skipped, see
 * TplRows). */
static float ml_at(const float *v, u32 n, const TplRows *R, const float *tss, u32 index, u32 k)
{
    float m = 0.0f;
    const u32 L = R->L, C = R->C;
    if (index + L >= n) return m;               /* .cl:231-234 */
    if (k >= R->K) return m;                    /* .cl:235-238 */
    m = tss[k];                                 /* .cl:239 */
    const u32 *chans = R->nzc + (size_t)k * C;
    for (u32 j = 0; j < R->nnz[k]; j++) {       /* .cl:242-250 */
        const u32 c = chans[j];
        const float *t = R->row[(size_t)k * C + c];
        const float *vv = v + index + (size_t)n * c;
        for (u32 i = 0; i < L; i++) m = m + t[i] * vv[i];
    }
    return m;
}

/* compute_full_likelihood, binary_pursuit.cl:255-300: for every listed window
 * and every template, write the likelihood at each sample of the window. */
static void full_likelihood(const float *v, u32 n, const TplRows *R, const float *tss,
                            const u32 *win, u32 nwin, float *Lk, int nthreads)
{
    const u32 K = R->K, L = R->L;
    long long total = (long long)nwin * K;
    __atomic_fetch_add(&g_counters[0], (unsigned long long)total * L, __ATOMIC_RELAXED);
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads > 0 ? nthreads : 1)
    for (long long g = 0; g < total; g++) {
        u32 w = (u32)(g / K), k = (u32)(g % K);
        u32 id = win[w];
        u32 s0 = id * L;
        u32 s1 = ((id + 1) * L) > n ? n : (id + 1) * L;
        for (u32 i = 0; i < s1 - s0; i++)
            Lk[(size_t)k * n + s0 + i] = ml_at(v, n, R, tss, s0 + i, k);
    }
}

void bpo_compute_full_likelihood(const float *v, u32 n, u32 C, const float *T,
                                 u32 K, u32 L, const float *tss, const u32 *win,
                                 u32 nwin, float *Lk, int nthreads)
{
    if (C == 0) return;
    TplRows R;
    if (tpl_rows_init(&R, T, K, C, L, 0)) return;
    full_likelihood(v, n, &R, tss, win, nwin, Lk, nthreads);
    tpl_rows_free(&R);
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
 * binary_pursuit.cl:578-632.  Channels run in ascending order over the union
 * of the two templates' non-zero rows (the others add nothing, see
 * TplRows); the rows are read through their zero padding (P >= n_max). */
static float overlap_pair_ll(const float *v, u32 n, const TplRows *R, u32 lab, u32 bidx, u32 t,
                             int fa, int sa)
{
    float cml = 0.0f;
    const u32 L = R->L, C = R->C;
    const u32 *ca = R->nzc + (size_t)lab * C, *cb = R->nzc + (size_t)t * C;
    const u32 na = R->nnz[lab], nb = R->nnz[t];
    u32 ia = 0, ib = 0;
    while (ia < na || ib < nb) {
        u32 c;
        if (ib >= nb || (ia < na && ca[ia] < cb[ib])) c = ca[ia++];
        else if (ia >= na || cb[ib] < ca[ia]) c = cb[ib++];
        else { c = ca[ia]; ia++; ib++; }
        const float *tf = R->row[(size_t)lab * C + c] + fa;     /* .cl:585-595 */
        const float *ts = R->row[(size_t)t * C + c] + sa;       /* .cl:591-603 */
        const float *vv = v + bidx + (size_t)n * c;
        float ss = 0.0f;
        for (u32 j = 0; j < L; j++) {
            float s = tf[j] + ts[j];
            ss += s * s;
            cml += s * vv[j];
        }
        if (ss > 0.0) cml = (float)((double)cml - 0.5 * (double)ss); /* .cl:627-630 */
    }
    return cml;
}

/* Best item of one candidate over items [i0, i1), strict-greater in item
 * order starting from `start` (the work-group-size-1 parse scan,
 * .cl:699-706, restricted to a block). */
typedef struct { float best; unsigned long long item; unsigned long long evaluated; int found; } OvBlock;

static OvBlock overlap_block(const float *v, u32 n, const TplRows *R, u32 lab, u32 bidx,
                             const float *Lk, u32 nmax, size_t i0, size_t i1, float start)
{
    const u32 K = R->K, L = R->L;
    const size_t S = 2 * (size_t)nmax + 1;
    OvBlock o = {start, 0, 0, 0};
    for (size_t it = i0; it < i1; it++) {
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
        float ll = overlap_pair_ll(v, n, R, lab, bidx, t, (int)nmax - (int)a, (int)nmax - (int)b);
        o.evaluated++;
        if (ll > o.best) { o.best = ll; o.item = it; o.found = 1; }
    }
    return o;
}

/* overlap_recheck_indices (binary_pursuit.cl:444-654) followed by
 * parse_overlap_recheck_indices (.cl:657-815), with a work-group size of 1:
 * each (a, b, t) work-item is its own group, so the parse kernel's scan over
 * group results (.cl:699-706) is a strict-greater scan over work-items in
 * ascending id, starting from the window's current best likelihood.  The
 * items of a candidate are split into blocks evaluated in parallel; the
 * blocks' results are combined in item order, which gives the same scan. */
static void overlap_recheck(const float *v, u32 n, const TplRows *R, const u32 *cand, u32 ncand,
                            u32 *best_idx, u32 *best_lab, float *best_ll, u32 *ov_idx, u32 *ov_lab,
                            const float *Lk, u32 nmax, const float *thr, u8 *ovr, int nthreads)
{
    const u32 K = R->K, L = R->L;
    const size_t S = 2 * (size_t)nmax + 1;
    const size_t items = S * S * K;
    const size_t blk = 2048;
    const size_t nblk = (items + blk - 1) / blk;
    OvBlock *res = (OvBlock *)malloc((nblk ? nblk : 1) * sizeof(OvBlock));
    for (u32 ci = 0; ci < ncand; ci++) {
        u32 id = cand[ci];
        u32 lab = best_lab[id], bidx = best_idx[id];
        float bll = Lk[(size_t)lab * n + bidx];
        int skip_all = 0;
        if (bll < thr[lab]) skip_all = 1;                    /* .cl:518-522 */
        if (bidx >= n - L) skip_all = 1;                     /* .cl:524-527 */
        float best_group = best_ll[id];                      /* .cl:690-694 */
        size_t best_item = 0;
        unsigned long long evaluated = 0;
        if (!skip_all && res) {
            const float start = best_group;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
            for (long long q = 0; q < (long long)nblk; q++) {
                size_t i0 = (size_t)q * blk, i1 = i0 + blk < items ? i0 + blk : items;
                res[q] = overlap_block(v, n, R, lab, bidx, Lk, nmax, i0, i1, start);
            }
            for (size_t q = 0; q < nblk; q++) {
                evaluated += res[q].evaluated;
                if (res[q].found && res[q].best > best_group) { best_group = res[q].best; best_item = res[q].item; }
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
    free(res);
}

void bpo_overlap_recheck(const float *v, u32 n, u32 C, const float *T, u32 K, u32 L,
                         const u32 *cand, u32 ncand, u32 *best_idx, u32 *best_lab,
                         float *best_ll, u32 *ov_idx, u32 *ov_lab, const float *Lk,
                         u32 nmax, const float *thr, u8 *ovr, int nthreads)
{
    TplRows R;
    if (tpl_rows_init(&R, T, K, C, L, nmax)) return;
    overlap_recheck(v, n, &R, cand, ncand, best_idx, best_lab, best_ll, ov_idx, ov_lab, Lk, nmax, thr, ovr,
                    nthreads);
    tpl_rows_free(&R);
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
    TplRows R;
    memset(&R, 0, sizeof(R));
    if (!Lk || !best_idx || !best_lab || !best_ll || !ov_idx || !ov_lab || !flags ||
        !ovr || !win || !cand || !add_idx || !add_lab) { total = -2; goto done; }
    if (C > 0 && tpl_rows_init(&R, T, K, C, L, nmax)) { total = -2; goto done; }
    u32 nwin = W;
    for (u32 i = 0; i < W; i++) win[i] = i;              /* :418 */
    u32 passes = 0;
    for (;;) {
        passes++;
        g_counters[3]++;
        if (C > 0) full_likelihood(v, n, &R, tss, win, nwin, Lk, nthreads);
        bpo_template_maximum_likelihood(n, L, K, win, nwin, best_idx, best_lab, best_ll,
                                        flags, ovr, ov_idx, ov_lab, Lk);
        u32 ncand = 0;                                   /* :565-569 */
        for (u32 i = 0; i < W; i++) if (ovr[i]) cand[ncand++] = i;
        if (ncand > 0 && do_overlap_recheck) {           /* :570-661 */
            if (C > 0)
                overlap_recheck(v, n, &R, cand, ncand, best_idx, best_lab, best_ll, ov_idx, ov_lab, Lk,
                                nmax, thr, ovr, nthreads);
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
    tpl_rows_free(&R);
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
    TplRows R;
    if (tpl_rows_init(&R, T, K, C, L, nmax)) return;
    for (u32 q = 0; q < count; q++) {
        unsigned long long it = items[q];
        u32 t = (u32)(it % K), a = (u32)((it / K) % S), b = (u32)((it / (S * K)) % S);
        out[q] = overlap_pair_ll(v, n, &R, lab, bidx, t, (int)nmax - (int)a, (int)nmax - (int)b);
    }
    tpl_rows_free(&R);
}
