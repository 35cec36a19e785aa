/*
 * fbp_b200.h -- C ABI of the B200-native Full Binary Pursuit library
 * (libfbp_b200.so, built from spikesorting_fullpursuit_b200/csrc).
 *
 * The reference drives eight OpenCL kernels of
 * spikesorting_fullpursuit/kernels/binary_pursuit.cl from Python through
 * pyopencl (spikesorting_fullpursuit/parallel/binary_pursuit_parallel.py).
 * Each entry point below replaces one kernel, or the whole per-chunk loop,
 * and names the reference code it stands in for.
 *
 * Conventions
 *  - All array arguments are DEVICE pointers unless the name says `host`.
 *  - voltage is channel-major [C][n] float32; templates are [K][C][L]
 *    float32 (the packing described at binary_pursuit.cl:11-29).
 *  - Window `w` covers samples [w*L, (w+1)*L); W = ceil(n / L).
 *  - Per-window state arrays hold at least W + FBP_WINDOW_PAD entries.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *  - Every entry point returns an fbp_status; fbp_last_error() gives text.
 *  - Results are those of the reference kernels executed with a work-group
 *    size of 1, work-items in global-id order: the one schedule under which
 *    the reference is deterministic.
 */
#ifndef FBP_B200_H
#define FBP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FBP_WINDOW_PAD 4

typedef enum fbp_status {
    FBP_OK = 0,
    FBP_ERR_BAD_ARG = 1,     /* invalid size, null pointer, mis-sized workspace */
    FBP_ERR_CUDA = 2,        /* a CUDA runtime call failed                      */
    FBP_ERR_ITER_CAP = 3,    /* the pursuit did not converge within max_passes  */
    FBP_ERR_CAPACITY = 4,    /* the spike output buffer is too small            */
    FBP_ERR_NO_DEVICE = 5,   /* no CUDA device                                  */
    FBP_ERR_OOM = 6,         /* reserved: allocation failure in a caller layer  */
    FBP_ERR_TIMEOUT = 7      /* a bounded wait inside a kernel gave up; the
                                kernel returned and the context stays usable  */
} fbp_status;

/* Arithmetic of the full-pass likelihood (path (a)).  Both modes produce
 * the same spikes.  FBP_PREC_FP32 evaluates every likelihood in the
 * reference's order on the FP32 pipes.  FBP_PREC_BF16_REFINE runs the
 * contraction on the tensor cores (tcgen05, BF16 operands, FP32
 * accumulation), bounds its error, and re-evaluates in the reference's
 * order every entry that could be positive; the others are provably
 * negative, which is all the pursuit reads of them.  Shapes whose templates
 * do not fit in shared memory use the FP32 kernel. */
typedef enum fbp_precision {
    FBP_PREC_FP32 = 0,
    FBP_PREC_BF16_REFINE = 1
} fbp_precision;

/* How the overlap recheck (binary_pursuit.cl:444-815) is evaluated.  Both
 * give the reference's result.  FAST splits each item's likelihood into
 * per-candidate correlations and template-pair prefix sums, bounds the
 * reference's rounding, and re-evaluates exactly (in the reference's order)
 * only the items that can be the maximum; EXACT evaluates every item in the
 * reference's order.  FAST falls back to EXACT for shift ranges above 4L+1. */
typedef enum fbp_overlap_method {
    FBP_OVERLAP_FAST = 0,
    FBP_OVERLAP_EXACT = 1
} fbp_overlap_method;

/* Stages of a pass, for fbp_stage_stats. */
enum {
    FBP_STAGE_LIKELIHOOD = 0,   /* path (a): full-pass likelihood          */
    FBP_STAGE_ARGMAX = 1,       /* per-window argmax over templates        */
    FBP_STAGE_OVERLAP = 2,      /* overlap recheck + parse                 */
    FBP_STAGE_CHECK = 3,        /* check_overlap_reassignments             */
    FBP_STAGE_ACCEPT = 4,       /* accept, flags, spike compaction         */
    FBP_STAGE_RESIDUAL = 5,     /* path (c): residual subtract             */
    FBP_STAGE_LISTS = 6,        /* window/candidate list compaction, resets */
    FBP_STAGE_LIK_REFINE = 7,   /* FBP_PREC_BF16_REFINE: entries whose sign the tensor-core
                                   interval left open, settled exactly             */
    FBP_STAGE_OVERLAP_TABLES = 8, /* FBP_OVERLAP_FAST: per-candidate correlation tables */
    FBP_N_STAGES = 9
};

/* Per-stage counters of one fbp_pursuit_chunk call.  `ms` holds CUDA-event
 * time per stage (filled only when profiling is requested); `launches` the
 * kernels launched per stage; `work` the algorithmic units per stage:
 *  LIKELIHOOD  sample x template likelihoods evaluated
 *  ARGMAX      likelihood values scanned
 *  OVERLAP     (a, b, t) items evaluated after the reference's skip rules
 *  ACCEPT      windows examined
 *  RESIDUAL    spikes subtracted
 *  CHECK       candidate windows */
typedef struct fbp_stage_stats {
    double ms[FBP_N_STAGES];
    uint64_t launches[FBP_N_STAGES];
    uint64_t work[FBP_N_STAGES];
    uint64_t candidates;        /* overlap-recheck candidates over all passes */
    uint64_t refined_items;     /* overlap items re-evaluated exactly because their
                                   interval reached the best one (FBP_OVERLAP_FAST) */
    uint64_t fallback_candidates; /* candidates the fast path handed to the exact kernel */
    uint64_t lik_refined;       /* likelihood entries whose BF16 interval could exceed 0,
                                   re-evaluated exactly (FBP_PREC_BF16_REFINE) */
    uint64_t lik_exact_passes;  /* passes whose refinement list overflowed and were redone
                                   in FP32 */
    uint32_t passes;
    uint32_t spikes;
    uint64_t lik_lazy_refined;  /* likelihood entries left approximate (certainly > 0) and
                                   re-evaluated exactly when a decision needed them
                                   (FBP_PREC_BF16_REFINE) */
    uint64_t lik_seq_refined;   /* entries of lik_refined whose sign a double-precision
                                   interval could not settle, re-evaluated in the
                                   reference's order (FBP_PREC_BF16_REFINE) */
    uint32_t tc_layout;         /* tensor-core likelihood layout the chunk used:
                                   0 none (FP32 path), FBP_TC_LAYOUT_SAMPLES or FBP_TC_LAYOUT_WIDE */
    uint32_t reserved;
} fbp_stage_stats;

/* Library version (major*10000 + minor*100 + patch). */
int fbp_version(void);

/* Text of the last error raised on the calling thread ("" if none). */
const char *fbp_last_error(void);

/* ------------------------------------------------------------------------
 * Whole per-chunk pursuit.
 * Replaces the iterate-until-converged loop of
 * binary_pursuit_parallel.py:386-736 (and the K+6 kernel launches plus the
 * host round trips of each pass) for one chunk that is already resident on
 * the device.
 * ---------------------------------------------------------------------- */

/* Bytes of device workspace fbp_pursuit_chunk needs for these sizes. */
int fbp_pursuit_workspace_bytes(uint32_t n_samples, uint32_t n_chans, uint32_t n_templates,
                                uint32_t template_len, uint32_t n_max_shift, int precision,
                                size_t *bytes_out);

/* Run binary pursuit on one chunk.
 *  voltage      [C][n] float32, turned into the residual in place
 *  templates    [K][C][L] float32
 *  neg_half_ss  [K] float32, float32(-0.5 * template_SS)   (.py:199)
 *  thresholds   [K] float32, float32(neuron_lower_thresholds) (.py:201)
 *  n_max_shift  overlap shift range, S = 2*n_max_shift + 1   (.py:294-298)
 *  overlap_method  fbp_overlap_method
 *  spike_idx/spike_lab  [spike_cap] uint32 outputs: window-relative clip
 *               starts and labels, in pass order and window order inside a
 *               pass (the order the reference's loop concatenates them)
 *  pass_counts  [max_passes] uint32 device array (may be NULL): spikes per pass
 *  n_spikes_host, n_passes_host  host outputs
 *  profile      1: time every stage with CUDA events (into stats->ms)
 *  stats        host fbp_stage_stats (may be NULL)
 * Returns FBP_ERR_CAPACITY if spike_cap is too small (n_spikes_host then
 * holds the number found before the buffer filled), FBP_ERR_ITER_CAP after
 * max_passes passes without convergence. */
int fbp_pursuit_chunk(float *voltage, uint32_t n_samples, uint32_t n_chans,
                      const float *templates, uint32_t n_templates, uint32_t template_len,
                      const float *neg_half_ss, const float *thresholds,
                      uint32_t n_max_shift, int do_overlap_recheck, int precision,
                      int overlap_method, uint32_t max_passes, void *workspace, size_t workspace_bytes,
                      uint32_t *spike_idx, uint32_t *spike_lab, uint32_t spike_cap,
                      uint32_t *pass_counts, uint32_t *n_spikes_host,
                      uint32_t *n_passes_host, int profile, fbp_stage_stats *stats,
                      void *stream);

/* Template group size of the tensor-core likelihood (no counterpart in the
 * reference, whose kernels take one template per work-item).  0 (default):
 * the planner's cost model picks, per chunk, the group size with the least
 * padded MMA work that fits shared memory; 16..256 (multiples of 16): that
 * size when its groups fit, else the cost model.  Applies to the calls the
 * calling thread makes afterwards; set by the tuner
 * (spikesorting_fullpursuit_b200.autotune) from timed trials per shape
 * bucket.  Results do not depend on it. */
int fbp_set_tc_group_size(uint32_t templates_per_group);

/* Layout of the tensor-core likelihood passes (no counterpart in the
 * reference).  FBP_TC_LAYOUT_SAMPLES: tiles of 128 samples, template groups
 * in the MMA's N (fbp_lik_tc.cuh); FBP_TC_LAYOUT_WIDE: tiles of 2048 positions
 * of the pass's window stream, 16 templates x 8 sample shifts in the MMA's M
 * and blocks of 8 samples in N (fbp_lik_tcw.cuh; applies when L >= 16, its
 * shared-memory plan fits -- L up to about 190 -- and the chunk has fewer than
 * 2^31 samples); FBP_TC_LAYOUT_AUTO (default): WIDE where it applies.  Applies to the calls
 * the calling thread makes afterwards.  Results do not depend on it. */
enum { FBP_TC_LAYOUT_AUTO = 0, FBP_TC_LAYOUT_SAMPLES = 1, FBP_TC_LAYOUT_WIDE = 2 };
int fbp_set_tc_layout(int layout);

/* ------------------------------------------------------------------------
 * Testing hooks (no counterpart in the reference).
 * ---------------------------------------------------------------------- */

/* Limits that make rarely taken paths of fbp_pursuit_chunk reachable on
 * small inputs.  Process-wide; they apply to calls made after
 * fbp_set_test_limits returns (do not change them while another thread is
 * inside fbp_pursuit_chunk).  Results are unchanged by the capacities: an
 * overflowing refinement list makes the FP32 kernel redo the pass's windows,
 * an overflowing contender pool hands the candidate to the exact overlap
 * kernel. */
#define FBP_DEFAULT_WAIT_POLLS 16777216u
typedef struct fbp_test_limits {
    uint32_t refine_list_cap;    /* tensor-core refinement list entries (0: workspace capacity) */
    uint32_t contender_pool_cap; /* fast overlap contender pool entries (0: workspace capacity) */
    uint32_t wait_polls;         /* polls after which a pipeline wait of the tensor-core kernel
                                    gives up (FBP_DEFAULT_WAIT_POLLS normally; 0 gives up at
                                    once): the call then returns FBP_ERR_TIMEOUT */
} fbp_test_limits;

/* Set the limits; NULL restores the defaults ({0, 0, FBP_DEFAULT_WAIT_POLLS}). */
int fbp_set_test_limits(const fbp_test_limits *limits);

/* One pass of the tensor-core likelihood (FBP_PREC_BF16_REFINE, path (a))
 * over every window of a chunk, without refinement.  approx[k][s] ([K][n]
 * float32) receives the tensor-core value and bound[k][s] the error bound E
 * the pursuit relies on: |approx - R| <= E for R, the reference's IEEE
 * binary32 likelihood (compute_maximum_likelihood, binary_pursuit.cl:216-252).
 * Entries with s + L >= n hold 0 in both.  workspace: fbp_pursuit_workspace_bytes
 * (..., FBP_PREC_BF16_REFINE) bytes.  FBP_ERR_BAD_ARG when no template group
 * of this shape fits the tensor-core kernel. */
int fbp_tc_likelihood_bounds(const float *voltage, uint32_t n_samples, uint32_t n_chans,
                             const float *templates, uint32_t n_templates, uint32_t template_len,
                             const float *neg_half_ss, void *workspace, size_t workspace_bytes,
                             float *approx, float *bound, void *stream);

/* ------------------------------------------------------------------------
 * Single stages (the reference kernels one by one).
 * ---------------------------------------------------------------------- */

/* compute_residual, binary_pursuit.cl:57-102: voltage[c, idx+i] -= t[lab,c,i]
 * for every listed spike, in list order where spikes overlap.  Labels >= K
 * are skipped, as in the reference.  max_overlap_neighbours bounds how many
 * list positions apart two overlapping spikes can be (a pass's spikes, one
 * per window in window order, need 3 + ceil(2*n_max_shift/L)); spikes
 * farther apart in the list must not overlap. */
int fbp_compute_residual(float *voltage, uint32_t n_samples, uint32_t n_chans,
                         const float *templates, uint32_t n_templates, uint32_t template_len,
                         const uint32_t *spike_idx, const uint32_t *spike_lab,
                         uint32_t n_spikes, uint32_t max_overlap_neighbours, void *stream);

/* get_adjusted_clips, binary_pursuit.cl:1088-1130: clips[s, c*L+i] =
 * voltage[c, idx+i] + t[lab,c,i]; entries past the end of the voltage are
 * left untouched (callers pass zeroed clips, as the reference does). */
int fbp_get_adjusted_clips(const float *voltage, uint32_t n_samples, uint32_t n_chans,
                           const float *templates, uint32_t n_templates, uint32_t template_len,
                           const uint32_t *spike_idx, const uint32_t *spike_lab,
                           uint32_t n_spikes, float *clips, void *stream);

/* compute_full_likelihood, binary_pursuit.cl:255-300: likelihood[k, s] for
 * every sample s of every window in window_list (device count n_windows_dev,
 * a device uint32), 0 where s + L >= n. */
int fbp_compute_full_likelihood(const float *voltage, uint32_t n_samples, uint32_t n_chans,
                                const float *templates, uint32_t n_templates,
                                uint32_t template_len, const float *neg_half_ss,
                                const uint32_t *window_list, const uint32_t *n_windows_dev,
                                uint32_t max_windows, float *likelihood, int precision,
                                void *stream);

/* Per-window state shared by the stage entry points below (all device
 * arrays of W + FBP_WINDOW_PAD entries). */
typedef struct fbp_window_state {
    uint32_t *best_idx;       /* best_spike_indices          */
    uint32_t *best_lab;       /* best_spike_labels           */
    float *best_ll;           /* best_spike_likelihoods      */
    uint32_t *ov_idx;         /* overlap_best_spike_indices  */
    uint32_t *ov_lab;         /* overlap_best_spike_labels   */
    uint8_t *flags;           /* check_window_on_next_pass   */
    uint8_t *overlap_recheck; /* overlap_recheck             */
} fbp_window_state;

/* compute_template_maximum_likelihood, binary_pursuit.cl:350-441, for all
 * K templates in template order (the reference's K launches per pass,
 * binary_pursuit_parallel.py:551-562, fused into one). */
int fbp_window_argmax(uint32_t n_samples, uint32_t template_len, uint32_t n_templates,
                      const uint32_t *window_list, const uint32_t *n_windows_dev,
                      uint32_t max_windows, const fbp_window_state *st,
                      const float *likelihood, void *stream);

/* overlap_recheck_indices + parse_overlap_recheck_indices,
 * binary_pursuit.cl:444-815, for the candidate windows in cand_list (device
 * count n_cand_dev), ascending. */
int fbp_overlap_recheck(const float *voltage, uint32_t n_samples, uint32_t n_chans,
                        const float *templates, uint32_t n_templates, uint32_t template_len,
                        const uint32_t *cand_list, const uint32_t *n_cand_dev,
                        uint32_t max_cand, const fbp_window_state *st,
                        const float *likelihood, uint32_t n_max_shift,
                        const float *thresholds, void *stream);

/* check_overlap_reassignments, binary_pursuit.cl:822-875, for the candidate
 * windows in cand_list.  scratch: W + FBP_WINDOW_PAD bytes. */
int fbp_check_overlap_reassignments(uint32_t n_samples, uint32_t template_len,
                                    const uint32_t *cand_list, const uint32_t *n_cand_dev,
                                    uint32_t max_cand, const fbp_window_state *st,
                                    uint8_t *scratch, void *stream);

/* binary_pursuit kernel, binary_pursuit.cl:918-1063: accept spikes of the
 * windows in window_list, update the flags, append spikes (window order).
 *  active   [W+pad] uint8, 1 for windows in window_list (others 0)
 *  has      [W+pad] uint8 scratch
 *  flags_out[W+pad] uint8: the flags after the kernel (flags in st are read only)
 *  spike_idx/spike_lab/spike_win [>= number of listed windows] outputs
 *  n_spikes_dev  device uint32 count of appended spikes
 *  scan_scratch  fbp_scan_scratch_bytes(W) bytes */
int fbp_binary_pursuit_accept(uint32_t n_samples, uint32_t n_chans, uint32_t template_len,
                              const float *thresholds, const uint32_t *window_list,
                              const uint32_t *n_windows_dev, uint32_t max_windows,
                              const fbp_window_state *st, const uint8_t *active, uint8_t *has,
                              uint8_t *flags_out, uint32_t *spike_idx, uint32_t *spike_lab,
                              uint32_t *spike_win, uint32_t *n_spikes_dev, void *scan_scratch,
                              void *stream);

/* Allocation-free variant of fbp_binary_pursuit_accept (no counterpart in
 * the reference).  For callers that cannot call cudaMalloc: for example a
 * host framework that has reserved the whole device heap for its own pool,
 * or a real-time acquisition loop where an allocation's implicit device
 * synchronisation and unbounded latency are not allowed.  The `has` and
 * `scan_scratch` buffers of fbp_binary_pursuit_accept live instead in one
 * file-scope device array of FBP_NOALLOC_SCRATCH_BYTES (about 4.2 MB), which
 * every GPU that loads the library keeps until the process exits; the
 * caller still passes every input and output.  Limit: at most
 * FBP_NOALLOC_MAX_WINDOWS windows (n_samples <= FBP_NOALLOC_MAX_WINDOWS * L);
 * larger inputs return FBP_ERR_BAD_ARG.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress), so make that first call
 * before any stream capture.  The address is kept for the life of the
 * process: after cudaDeviceReset it is stale, so do not call this entry point
 * after resetting the device.  All calls share the one array: calls whose GPU
 * work overlaps (other streams, other threads) race on it; it is cleared
 * at the start of every call, so its leftover contents do not matter. */
#define FBP_NOALLOC_MAX_WINDOWS 4194300u
#define FBP_NOALLOC_SCRATCH_BYTES (4194304u + 8192u)
int fbp_binary_pursuit_accept_noalloc(uint32_t n_samples, uint32_t n_chans, uint32_t template_len,
                                      const float *thresholds, const uint32_t *window_list,
                                      const uint32_t *n_windows_dev, uint32_t max_windows,
                                      const fbp_window_state *st, const uint8_t *active,
                                      uint8_t *flags_out, uint32_t *spike_idx, uint32_t *spike_lab,
                                      uint32_t *spike_win, uint32_t *n_spikes_dev, void *stream);

/* Scratch bytes the ordered compaction in fbp_binary_pursuit_accept needs. */
size_t fbp_scan_scratch_bytes(uint32_t n_windows);

/* Bytes of a uint8 per-window array that an ordered compaction reads
 * (active, has, flags_out): W + FBP_WINDOW_PAD rounded up to 4096. */
size_t fbp_window_u8_bytes(uint32_t n_windows);

#ifdef __cplusplus
}
#endif
#endif /* FBP_B200_H */
