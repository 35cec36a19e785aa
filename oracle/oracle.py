"""ctypes front end of the oracle (TEST INFRASTRUCTURE ONLY).

`binary_pursuit_oracle` restates the reference host driver
spikesorting_fullpursuit/parallel/binary_pursuit_parallel.py:128-845 around
the C restatement of the kernels (bp_oracle.c): same input handling
(:174-201), chunk onsets (:359-368), per-chunk loop (:386-736, in C), output
assembly (:814-845).  The chunk length is passed explicitly instead of being
derived from a device's memory size.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libbp_oracle.so")
_lib = None

u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
U = ctypes.c_uint32


def build():
    subprocess.run(["make", "-s", "-C", HERE, "libbp_oracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.bpo_pursuit_chunk.restype = ctypes.c_longlong
        L.bpo_pursuit_chunk.argtypes = [f32p, U, U, f32p, U, U, f32p, f32p, U, ctypes.c_int,
                                        u32p, u32p, U, ctypes.POINTER(U), u32p, U, ctypes.c_int]
        L.bpo_compute_full_likelihood.argtypes = [f32p, U, U, f32p, U, U, f32p, u32p, U, f32p, ctypes.c_int]
        L.bpo_template_maximum_likelihood.argtypes = [U, U, U, u32p, U, u32p, u32p, f32p, u8p, u8p,
                                                      u32p, u32p, f32p]
        L.bpo_overlap_recheck.argtypes = [f32p, U, U, f32p, U, U, u32p, U, u32p, u32p, f32p, u32p, u32p,
                                          f32p, U, f32p, u8p, ctypes.c_int]
        L.bpo_check_overlap_reassignments.argtypes = [U, U, u32p, U, u32p, u32p, u8p, u32p, u32p, u8p]
        L.bpo_binary_pursuit.restype = U
        L.bpo_binary_pursuit.argtypes = [U, U, U, f32p, u32p, U, u32p, u32p, f32p, u32p, u32p, u8p, u8p]
        L.bpo_compute_residual.argtypes = [f32p, U, U, f32p, U, U, u32p, u32p, U]
        L.bpo_counters.argtypes = [ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int]
        L.bpo_get_adjusted_clips.argtypes = [f32p, U, U, f32p, U, U, u32p, u32p, U, f32p]
        _lib = L
    return _lib


def pursuit_chunk(chunk_v, templates_vec, K, L, tss, thr, n_max_shift, do_overlap,
                  nthreads=None, max_passes=100000):
    """Run the per-chunk loop.  chunk_v: float32 [C, n] (modified in place).
    Returns (indices u32, labels u32, n_passes, spikes-per-pass)."""
    C, n = chunk_v.shape
    if nthreads is None:
        nthreads = os.cpu_count() or 1
    W = (n + L - 1) // L
    cap = max(16, 4 * W + 64)
    while True:
        out_i = np.zeros(cap, np.uint32)
        out_l = np.zeros(cap, np.uint32)
        passes = U(0)
        pc = np.zeros(max_passes, np.uint32)
        work = np.ascontiguousarray(chunk_v, dtype=np.float32)
        r = lib().bpo_pursuit_chunk(work.reshape(-1), n, C, templates_vec, K, L, tss, thr,
                                    int(n_max_shift), int(bool(do_overlap)), out_i, out_l, cap,
                                    ctypes.byref(passes), pc, max_passes, int(nthreads))
        if r == -1:
            cap *= 4
            continue
        if r < 0:
            raise MemoryError("oracle allocation failed")
        chunk_v[...] = work
        return out_i[:r].copy(), out_l[:r].copy(), passes.value, pc[:min(passes.value, max_passes)].copy()


# --- single stages (restated kernels), for stage-level parity tests --------

def stage_full_likelihood(v, T, K, L, tss, win, Lk, nthreads=4):
    C, n = v.shape
    lib().bpo_compute_full_likelihood(np.ascontiguousarray(v, np.float32).reshape(-1), n, C, T, K, L,
                                      tss, np.ascontiguousarray(win, np.uint32), len(win), Lk.reshape(-1),
                                      nthreads)


def stage_template_max(n, L, K, win, st, Lk):
    lib().bpo_template_maximum_likelihood(n, L, K, np.ascontiguousarray(win, np.uint32), len(win),
                                          st["best_idx"], st["best_lab"], st["best_ll"], st["flags"],
                                          st["ovr"], st["ov_idx"], st["ov_lab"], Lk.reshape(-1))


def stage_overlap(v, T, K, L, cand, st, Lk, nmax, thr, nthreads=4):
    C, n = v.shape
    lib().bpo_overlap_recheck(np.ascontiguousarray(v, np.float32).reshape(-1), n, C, T, K, L,
                              np.ascontiguousarray(cand, np.uint32), len(cand), st["best_idx"],
                              st["best_lab"], st["best_ll"], st["ov_idx"], st["ov_lab"], Lk.reshape(-1),
                              nmax, thr, st["ovr"], nthreads)


def stage_check_overlap(n, L, cand, st):
    lib().bpo_check_overlap_reassignments(n, L, np.ascontiguousarray(cand, np.uint32), len(cand),
                                          st["best_idx"], st["best_lab"], st["flags"], st["ov_idx"],
                                          st["ov_lab"], st["ovr"])


def stage_accept(n, C, L, thr, win, st):
    W = len(st["flags"])
    oi = np.zeros(W, np.uint32)
    ol = np.zeros(W, np.uint32)
    cnt = lib().bpo_binary_pursuit(n, C, L, thr, np.ascontiguousarray(win, np.uint32), len(win),
                                   st["best_idx"], st["best_lab"], st["best_ll"], oi, ol, st["ovr"],
                                   st["flags"])
    return oi[:cnt], ol[:cnt]


def stage_residual(v, T, K, L, idx, lab):
    C, n = v.shape
    flat = np.ascontiguousarray(v, np.float32).reshape(-1).copy()
    lib().bpo_compute_residual(flat, n, C, T, K, L, np.ascontiguousarray(idx, np.uint32),
                               np.ascontiguousarray(lab, np.uint32), len(idx))
    return flat.reshape(C, n)


def counters(reset=True):
    """Work counters: likelihood sample*templates, overlap candidates,
    overlap items surviving the skip rules, passes."""
    out = (ctypes.c_ulonglong * 8)()
    lib().bpo_counters(out, int(reset))
    return {"likelihood_st": out[0], "overlap_candidates": out[1],
            "overlap_items": out[2], "passes": out[3]}


def adjusted_clips(resid_v, templates_vec, K, L, idx, lab):
    C, n = resid_v.shape
    clips = np.zeros(idx.size * C * L, np.float32)
    if idx.size:
        lib().bpo_get_adjusted_clips(np.ascontiguousarray(resid_v, np.float32).reshape(-1), n, C,
                                     templates_vec, K, L, np.ascontiguousarray(idx, np.uint32),
                                     np.ascontiguousarray(lab, np.uint32), idx.size, clips)
    return clips.reshape(idx.size, C * L)


def time_window_to_samples(time_window, sampling_rate):
    """Restates segment_parallel.py:82-98."""
    tw = list(time_window)
    if tw[0] > 0:
        tw[0] *= -1
    sw = [min(int(round(tw[0] * sampling_rate)), 0),
          max(int(round(tw[1] * sampling_rate)), 1) + 1]
    return sw, tw


def binary_pursuit_oracle(voltage, v_dtype, sort_info, separability_metrics,
                          n_max_shift_inds=None, chunk_samples=None, nthreads=None,
                          stats=None):
    n_chans = voltage.shape[0]
    n_samples = voltage.shape[1]
    chan_win, _ = time_window_to_samples(sort_info["clip_width"], sort_info["sampling_rate"])
    L = int(sort_info["n_samples_per_chan"])
    templates = separability_metrics["templates"]
    if templates.ndim == 1:
        templates = np.reshape(templates, (1, -1))
    templates = np.float32(templates)
    K = templates.shape[0]
    tvec = np.ascontiguousarray(templates.reshape(templates.size), dtype=np.float32)
    clip_init_samples = int(np.abs(chan_win[0]))
    tss = np.ascontiguousarray(np.float32(-0.5 * separability_metrics["template_SS"]))
    thr = np.ascontiguousarray(np.float32(separability_metrics["neuron_lower_thresholds"]))
    if n_max_shift_inds is None or n_max_shift_inds < 0:
        n_max_shift_inds = L // 2
    n_max_shift_inds = int(np.uint32(n_max_shift_inds))
    if chunk_samples is None:
        # a chunk longer than the recording: one chunk, as on a large device
        chunk_samples = n_samples + 3 * L + 1
    if chunk_samples < 4 * L:
        raise ValueError("Cannot fit enough data on GPU to run binary pursuit. "
                         "Decrease template samples or get a new GPU.")
    onsets = []
    cur = 0
    while cur < n_samples - L:
        onsets.append(cur)
        cur += chunk_samples - 3 * L
    sec_i, sec_l, sec_b, sec_c = [], [], [], []
    for start in onsets:
        stop = min(n_samples, start + chunk_samples)
        cv = np.float32(voltage[:, start:stop]).copy()
        idx, lab, passes, pc = pursuit_chunk(cv, tvec, K, L, tss, thr, n_max_shift_inds,
                                             sort_info["do_overlap_recheck"], nthreads)
        if stats is not None:
            stats.append({"start": start, "stop": stop, "passes": passes,
                          "pass_counts": pc.tolist()})
        if idx.size > 0:
            if sort_info["get_adjusted_clips"]:
                clips = adjusted_clips(cv, tvec, K, L, idx, lab)
            else:
                clips = []
            sec_i.append(idx + start)
            sec_l.append(lab)
            sec_c.append(clips)
            sec_b.append(np.ones(idx.size, dtype=bool))
    if len(sec_i) > 0:
        event_indices = np.int64(np.hstack(sec_i))
        neuron_labels = np.int64(np.hstack(sec_l))
        adjusted = (np.vstack(sec_c)).astype(v_dtype)
        bp_bool = np.hstack(sec_b)
        event_indices += clip_init_samples
    else:
        event_indices, neuron_labels, bp_bool, adjusted = [], [], [], []
    # add_n_spikes (neuron_separability.py:264-273) sizes the array by the
    # dict's templates entry, so 1-D templates give C*L entries.
    nt = separability_metrics["templates"].shape[0]
    separability_metrics["n_spikes"] = np.zeros(nt)
    for k in range(nt):
        separability_metrics["n_spikes"][k] = np.count_nonzero(neuron_labels == k)
    return event_indices, neuron_labels, bp_bool, adjusted
