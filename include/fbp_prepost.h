/*
 * fbp_prepost.h -- C ABI of the steps on either side of the pursuit
 * (libfbp_b200.so, built from spikesorting_fullpursuit_b200/csrc/fbp_prepost.cu).
 *
 * The reference runs these on the host with numpy between the clustering and
 * binary_pursuit() (spikesorting_fullpursuit/full_binary_pursuit.py:299-322,
 * wiener_filter.py, preprocessing.py) and after it (analyze_spike_timing.py,
 * postprocessing.py).  Each entry point names the reference function it
 * stands in for.  Conventions are those of fbp_b200.h: DEVICE pointers,
 * `stream` a cudaStream_t as void*, an fbp_status return, text from
 * fbp_last_error().  Element types: FBP_F32 (float32) and FBP_I16 (int16),
 * the voltage dtypes the reference handles (v_dtype).
 */
#ifndef FBP_PREPOST_H
#define FBP_PREPOST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { FBP_F32 = 0, FBP_I16 = 1, FBP_F64 = 2 };

/* get_clips, parallel/segment_parallel.py:451-503 (the copy loop :491-496):
 * clips[e, k*W + i] = voltage[neighbors[k], events[first + e] + win0 + i]
 * for e < n_events, k < n_neighbors, i < W = win1 - win0.  The caller
 * passes the valid range [first, first + n_events) the reference derives
 * from its sorted events (:463-483).  voltage is [n_chans][n_samples] of
 * dtype (FBP_F32 or FBP_I16); clips has the same dtype. */
int fbp_get_clips(const void *voltage, int dtype, uint64_t n_samples, uint32_t n_chans,
                  const int64_t *neighbors, uint32_t n_neighbors, const int64_t *events,
                  uint32_t first, uint32_t n_events, int32_t win0, int32_t win1, void *clips,
                  void *stream);

/* calculate_robust_template, preprocessing.py:639-659, for many units at
 * once.  clips [n_rows][dim] of dtype, the rows of unit u are
 * [unit_offsets[u], unit_offsets[u+1]).  templates [n_units][dim] of dtype
 * receives, per column, the median of the values within one MAD (median
 * absolute deviation / 0.6745) of the median, or the median when none is;
 * a unit with one row gets that row.  Same arithmetic as numpy: float32
 * medians (mean of the two middle values in float32) for FBP_F32; float64
 * medians truncated to int16 for FBP_I16.  scratch: fbp_robust_scratch_bytes. */
size_t fbp_robust_scratch_bytes(uint32_t n_rows, uint32_t dim, int dtype);
int fbp_robust_templates(const void *clips, int dtype, uint32_t n_rows, uint32_t dim,
                         const uint32_t *unit_offsets, uint32_t n_units, void *templates,
                         void *scratch, size_t scratch_bytes, void *stream);

/* The clip noise covariance of full_binary_pursuit.py:299-322: residual
 * clips (clip - the robust template of its unit, in dtype arithmetic as the
 * reference's `clips - robust_template`), rows `rows` ([n_sel] int64) of
 * them, and per channel c the L x L covariance of columns [c*L, (c+1)*L)
 * with ddof 0 (np.cov(..., rowvar=False, ddof=0)) in float64.
 * clips [n_rows][n_chans*L], row_unit [n_rows] uint32, templates
 * [n_units][n_chans*L]; cov [n_chans][L][L] float64 (overwritten).
 * scratch: fbp_noise_cov_scratch_bytes. */
size_t fbp_noise_cov_scratch_bytes(uint32_t n_chans, uint32_t L);
int fbp_clip_noise_covariance(const void *clips, int dtype, const uint32_t *row_unit, const void *templates,
                              const int64_t *rows, uint32_t n_sel, uint32_t n_chans, uint32_t L,
                              double *cov, void *scratch, size_t scratch_bytes, void *stream);

/* Per-unit duplicate removal of analyze_spike_timing.py over many units at
 * once.  Events of unit u are [unit_offsets[u], unit_offsets[u+1]) (in the
 * order the reference scans them); keep [n_events] uint8 receives 1/0.
 *  mode 0  remove_binary_pursuit_duplicates (:116-157)
 *  mode 1  keep_binary_pursuit_duplicates (:85-113) (clips unused)
 *  mode 2  remove_spike_event_duplicates (:159-184) (bp_bool unused)
 * clips [n_events][dim] float32 and templates [n_units][dim] (float32 or
 * float64, tdtype): the squared error of a clip against its unit's template
 * is summed exactly as numpy's np.sum (pairwise, blocks of 8, leaves of 128
 * elements).  sse [n_events] float64 scratch. */
int fbp_remove_duplicates(int mode, const int64_t *events, const uint8_t *bp_bool, const float *clips,
                          const void *templates, int tdtype, uint32_t dim, const uint32_t *unit_offsets,
                          uint32_t n_units, uint32_t n_events, int64_t tol_inds, double *sse, uint8_t *keep,
                          void *stream);

/* np.mean(clips_of_unit, axis=0) for float32 clips, as numpy computes it
 * (rows added in order in float32, divided by the row count): the unit
 * template postprocessing.py:535-540 passes to remove_binary_pursuit_duplicates. */
int fbp_unit_mean_templates(const float *clips, uint32_t dim, const uint32_t *unit_offsets, uint32_t n_units,
                            float *templates, void *stream);

/* find_overlap_templates, c_cython/sort_cython.pyx:333-458, the search over
 * template sums.  For each listed (test unit, pair) item the kernel scans
 * every (shift1, shift2) in [-n_pre, n_post]^2 (shift1 outer) and keeps the
 * first strictly smallest residual sum of squares
 * sum((test - shift(t1, s1) - shift(t2, s2))**2) in float64 (numpy's
 * pairwise order).  templates [K][n_chans*L] float32; items [n_items][3]
 * uint32 (test, n1, n2); best_ss [n_items] float64, best_shift [n_items][2]
 * int32 outputs; scratch fbp_overlap_template_scratch_bytes.  The pair filters (spike counts, min/max channel
 * amplitudes, :396-423) and the choice across pairs are the caller's (the
 * host restatement in c_cython/sort_cython.py). */
size_t fbp_overlap_template_scratch_bytes(uint32_t n_items, int32_t n_pre, int32_t n_post);
int fbp_overlap_template_search(const float *templates, uint32_t n_templates, uint32_t n_chans, uint32_t L,
                                int32_t n_pre, int32_t n_post, const uint32_t *items, uint32_t n_items,
                                double *best_ss, int32_t *best_shift, void *scratch, size_t scratch_bytes,
                                void *stream);

/* Wiener filter arithmetic of wiener_filter.py:24-72 / :75-121 on device
 * spectra (the FFTs are the caller's), in the spectra's precision dtype
 * (FBP_F32: numpy transforms float32 voltage in single precision; FBP_F64
 * otherwise): power[i] = |spec[i]|^2 (re^2 + im^2) for interleaved complex
 * spec [n_rows][n_bins]; the box-car smoothing of :40-59 with the
 * reference's running sums, per row, when smooth > 1 (scratch: n_rows *
 * n_bins reals); then spec *= S / (S + N + 1e-9) (:124-129). */
int fbp_power_spectrum(const void *spec, int dtype, uint64_t n_rows, uint64_t n_bins, void *power, void *stream);
int fbp_wiener_smooth(void *power, int dtype, uint64_t n_rows, uint64_t n_bins, int64_t smooth, void *scratch,
                      void *stream);
int fbp_wiener_apply(void *spec, const void *S, const void *N, int dtype, uint64_t n_rows, uint64_t n_bins,
                     void *stream);

/* get_noise_sampled_zca_matrix, preprocessing.py:104-169, the data passes:
 * the sample mask (|v| > 0.9 thr dilated by +-cushion, :115-118), and the
 * covariance matrix sigma [C][C] float64 over the samples no channel of the
 * pair masks -- the diagonal as np.var(ddof=1) (:128), off the diagonal the
 * uncentred dot product / (count - 1) (:136-140).  Every unmasked sample is
 * used (the reference subsamples at random above n_samples).  voltage
 * [C][n] of dtype; thresholds [C] float64; mask [C][n] uint8 scratch;
 * scratch: fbp_zca_scratch_bytes. */
size_t fbp_zca_scratch_bytes(uint32_t n_chans);
int fbp_zca_covariance(const void *voltage, int dtype, uint32_t n_chans, uint64_t n_samples,
                       const double *thresholds, int32_t cushion, uint8_t *mask, double *sigma, void *scratch,
                       size_t scratch_bytes, void *stream);

/* (zca_matrix @ voltage).astype(v_dtype), spikesorting_parallel.py:214:
 * out[i, s] = sum_c Z[i, c] * v[c, s] in float64, cast to dtype (rounded
 * for float32, truncated for int16 as numpy's astype). */
int fbp_zca_apply(const double *zca, const void *voltage, int dtype, uint32_t n_chans, uint64_t n_samples,
                  void *out, void *stream);

/* The pursuit's inputs, compute_separability_metrics and set_bp_threshold
 * (neuron_separability.py:88-152, 251-261): per template, template_SS as
 * numpy computes it (ss32: the float32 pairwise sum of squares, from which
 * binary_pursuit() takes float32(-0.5 * SS)) and in float64 (ss64); the
 * likelihood variance sum_c t_c^T cov_c t_c (var, float64); lower_ci =
 * SS/2 - sigma_ci * sqrt(var); thr_raw = -SS/2 + sigma_noise * sqrt(var);
 * thr = max(thr_raw, 0, lower_ci), the neuron_lower_thresholds the pursuit
 * uses.  templates [K][C*L] float32, cov [C][L][L] float64. */
int fbp_separability_metrics(const float *templates, uint32_t n_templates, uint32_t n_chans, uint32_t L,
                             const double *cov, double sigma_noise, double sigma_ci, float *ss32, double *ss64,
                             double *var, double *lower_ci, double *thr_raw, double *thr, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* FBP_PREPOST_H */
