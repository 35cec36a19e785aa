"""Drop-in `binary_pursuit()` backed by the sm_100a CUDA library.

Mirrors spikesorting_fullpursuit/parallel/binary_pursuit_parallel.py:128-845:
same signature, same inputs read, same 4-tuple return and dtypes, same
`separability_metrics['n_spikes']` side effect, same exceptions for the same
conditions.  The per-chunk pursuit loop runs on the device
(`fbp_pursuit_chunk` in include/fbp_b200.h); this module handles inputs,
chunking and output assembly.
"""
import ctypes

import numpy as np

from .chunking import chunk_onsets, num_indices_per_chunk

_PRECISIONS = {"fp32": 0, "bf16": 1, "bf16_refine": 1}
_TC_LAYOUTS = {"auto": 0, "samples": 1, "wide": 2}   # FBP_TC_LAYOUT_* of include/fbp_b200.h


def time_window_to_samples(time_window, sampling_rate):
    """segment_parallel.time_window_to_samples (segment_parallel.py:82-98)."""
    new_time_window = list(time_window)
    if new_time_window[0] > 0:
        new_time_window[0] *= -1
    sample_window = [0, 0]
    sample_window[0] = min(int(round(new_time_window[0] * sampling_rate)), 0)
    sample_window[1] = max(int(round(new_time_window[1] * sampling_rate)), 1) + 1
    return sample_window, new_time_window


def add_n_spikes(separability_metrics, neuron_labels):
    """neuron_separability.add_n_spikes (neuron_separability.py:264-273)."""
    separability_metrics['n_spikes'] = np.zeros(separability_metrics['templates'].shape[0])
    for n in range(0, separability_metrics['templates'].shape[0]):
        separability_metrics['n_spikes'][n] = np.count_nonzero(neuron_labels == n)
    return None


def _to_device_f32(torch, host_chunk, dev, stream):
    """Upload a [C, n] host chunk in its own dtype and convert to float32 on
    the device (the reference converts on the host, :374; the values are the
    same, round-to-nearest)."""
    a = np.ascontiguousarray(host_chunk)
    t = torch.from_numpy(a)
    with torch.cuda.stream(stream):
        d = t.to(dev, non_blocking=False)
        if d.dtype != torch.float32:
            d = d.to(torch.float32)
    return d


def binary_pursuit(voltage, v_dtype, sort_info, separability_metrics, n_max_shift_inds=None,
                   kernels_path=None, max_gpu_memory=None, *, precision="bf16",
                   chunk_samples=None, device=None, max_passes=1000000, stats=None, profile=False,
                   overlap="fast", tune=False, tc_layout=None):
    """Full Binary Pursuit over `voltage` ([channels, samples], any real dtype).

    Returns (event_indices int64, neuron_labels int64, binary_pursuit_spike_bool
    bool, adjusted_clips v_dtype [n, C*L]) or four empty lists, exactly as
    binary_pursuit_parallel.py:829-845.  `kernels_path` is accepted and
    ignored (there are no OpenCL sources to load).

    Extra keyword-only arguments (not in the reference):
      precision      "bf16" (default: tensor cores with exact refinement) or
                     "fp32" (likelihoods on the FP32 pipes in the reference's
                     order); both give the same spikes.
      chunk_samples  override the chunk length (the reference derives it from
                     device memory, :276-341); needed to reproduce a given
                     chunking exactly.
      device         CUDA device index (default: current device).
      overlap        "fast" (decomposed overlap recheck with exact refinement)
                     or "exact" (every item in the reference's order); both
                     give the reference's result.
      stats          a list; one dict per chunk is appended (passes, spikes,
                     per-stage launches, work and, with profile=True, CUDA-event
                     milliseconds).
      tune           precision "bf16": take the tensor-core plan (layout and
                     template group size) from the tuner's cache for this
                     shape bucket, timing the candidates on a sample of the
                     recording the first time
                     (spikesorting_fullpursuit_b200.autotune); same spikes.
      tc_layout      precision "bf16", for this call: "auto" (wide tiles where
                     they apply), "wide" (2048-position tiles of the pass's
                     window stream, 16 templates x 8 shifts per MMA) or
                     "samples" (128-sample tiles, template groups per MMA);
                     None (default): the calling thread's setting
                     (autotune.apply); same spikes.
    """
    # The CUDA runtime is initialised inside the call, never at import time,
    # so callers may fork worker processes first (reference :166-170).
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("No GPU available")
    from .. import _lib
    lib = _lib.lib()
    if precision not in _PRECISIONS:
        raise ValueError("precision must be one of %s" % sorted(_PRECISIONS))
    prec = _PRECISIONS[precision]
    if overlap not in ("fast", "exact"):
        raise ValueError("overlap must be 'fast' or 'exact'")
    ov_method = _lib.OVERLAP_FAST if overlap == "fast" else _lib.OVERLAP_EXACT
    if tc_layout is not None and tc_layout not in _TC_LAYOUTS:
        raise ValueError("tc_layout must be one of %s" % sorted(_TC_LAYOUTS))

    n_chans = int(voltage.shape[0])
    n_samples = int(voltage.shape[1])
    sampling_rate = sort_info['sampling_rate']
    chan_win, _ = time_window_to_samples(sort_info['clip_width'], sampling_rate)
    template_samples_per_chan = int(sort_info['n_samples_per_chan'])
    L = template_samples_per_chan

    templates = separability_metrics['templates']
    if templates.ndim == 1:
        templates = np.reshape(templates, (1, -1))
    templates = np.float32(templates)
    K = templates.shape[0]
    templates_vector = np.ascontiguousarray(templates.reshape(templates.size), dtype=np.float32)
    clip_init_samples = int(np.abs(chan_win[0]))
    template_sum_squared = np.ascontiguousarray(np.float32(-0.5 * separability_metrics['template_SS']))
    neuron_lower_thresholds = np.ascontiguousarray(np.float32(separability_metrics['neuron_lower_thresholds']))
    if templates_vector.size != K * n_chans * L:
        raise ValueError("templates must have n_channels * n_samples_per_chan columns")

    dev = torch.device("cuda", torch.cuda.current_device() if device is None else int(device))
    if n_max_shift_inds is None or n_max_shift_inds < 0:
        n_max_shift_inds = template_samples_per_chan // 2
    n_max_shift_inds = int(np.uint32(n_max_shift_inds))

    if chunk_samples is None:
        total_mem = torch.cuda.get_device_properties(dev).total_memory
        chunk_samples = num_indices_per_chunk(n_chans, K, L, sampling_rate, total_mem, max_gpu_memory,
                                              n_max_shift=n_max_shift_inds, precision=prec,
                                              v_itemsize=np.dtype(voltage.dtype).itemsize,
                                              adjusted_clips=bool(sort_info['get_adjusted_clips']))
    elif chunk_samples < 4 * L:
        raise ValueError("Cannot fit enough data on GPU to run binary pursuit. "
                         "Decrease template samples or get a new GPU.")
    onsets = chunk_onsets(n_samples, L, chunk_samples)
    if tune and prec == _PRECISIONS["bf16"] and n_samples > 0:
        from .. import autotune
        first = np.ascontiguousarray(voltage[:, :min(n_samples, chunk_samples)], dtype=np.float32)
        plan, _, _ = autotune.tune(first, templates_vector.reshape(K, -1), template_sum_squared, L)
        autotune.apply(plan)
    elif tc_layout is not None:
        _lib.check(lib.fbp_set_tc_layout(_TC_LAYOUTS[tc_layout]))

    stream = torch.cuda.current_stream(dev)
    sp = _lib.stream_ptr(stream)
    T_d = torch.from_numpy(templates_vector).to(dev)
    tss_d = torch.from_numpy(template_sum_squared).to(dev)
    thr_d = torch.from_numpy(neuron_lower_thresholds).to(dev)

    secret_spike_indices, secret_spike_labels, secret_spike_bool, adjusted_spike_clips = [], [], [], []
    for start_index in onsets:
        stop_index = min(n_samples, start_index + chunk_samples)
        n = stop_index - start_index
        W = (n + L - 1) // L
        ws_bytes = ctypes.c_size_t(0)
        _lib.check(lib.fbp_pursuit_workspace_bytes(n, n_chans, K, L, n_max_shift_inds, prec,
                                                   ctypes.byref(ws_bytes)))
        cap = 8 * W + 4096
        while True:
            v_d = _to_device_f32(torch, voltage[:, start_index:stop_index], dev, stream)
            ws = torch.empty(ws_bytes.value, dtype=torch.uint8, device=dev)
            out_i = torch.empty(cap, dtype=torch.int32, device=dev)
            out_l = torch.empty(cap, dtype=torch.int32, device=dev)
            nspk = ctypes.c_uint32(0)
            npass = ctypes.c_uint32(0)
            sst = _lib.StageStats()
            rc = lib.fbp_pursuit_chunk(
                _lib.ptr(v_d), n, n_chans, _lib.ptr(T_d), K, L, _lib.ptr(tss_d), _lib.ptr(thr_d),
                n_max_shift_inds, int(bool(sort_info['do_overlap_recheck'])), prec, ov_method, int(max_passes),
                _lib.ptr(ws), ws.numel(), _lib.ptr(out_i), _lib.ptr(out_l), cap, None,
                ctypes.byref(nspk), ctypes.byref(npass), int(bool(profile)), ctypes.byref(sst), sp)
            if rc == _lib.FBP_ERR_CAPACITY:
                cap *= 4
                continue
            _lib.check(rc)
            break
        m = int(nspk.value)
        if stats is not None:
            d = sst.as_dict()
            d.update({"start": start_index, "stop": stop_index, "n_spikes": m})
            stats.append(d)
        if m > 0:
            idx = out_i[:m].cpu().numpy().view(np.uint32)
            lab = out_l[:m].cpu().numpy().view(np.uint32)
            if sort_info['get_adjusted_clips']:
                clips_d = torch.zeros((m, n_chans * L), dtype=torch.float32, device=dev)
                _lib.check(lib.fbp_get_adjusted_clips(
                    _lib.ptr(v_d), n, n_chans, _lib.ptr(T_d), K, L, _lib.ptr(out_i), _lib.ptr(out_l),
                    m, _lib.ptr(clips_d), sp))
                all_adjusted_clips = clips_d.cpu().numpy()
            else:
                all_adjusted_clips = []
            secret_spike_indices.append(idx + start_index)
            secret_spike_labels.append(lab)
            adjusted_spike_clips.append(all_adjusted_clips)
            secret_spike_bool.append(np.ones(m, dtype="bool"))
        del v_d, ws

    if len(secret_spike_indices) > 0:
        event_indices = np.int64(np.hstack(secret_spike_indices))
        neuron_labels = np.int64(np.hstack(secret_spike_labels))
        adjusted_clips = (np.vstack(adjusted_spike_clips)).astype(v_dtype)
        binary_pursuit_spike_bool = np.hstack(secret_spike_bool)
        event_indices += clip_init_samples
    else:
        event_indices, neuron_labels, binary_pursuit_spike_bool, adjusted_clips = [], [], [], []

    if tune or tc_layout is not None:           # back to the library's own choice
        _lib.check(lib.fbp_set_tc_group_size(0))
        _lib.check(lib.fbp_set_tc_layout(_lib.TC_LAYOUT_AUTO))
    add_n_spikes(separability_metrics, neuron_labels)
    return event_indices, neuron_labels, binary_pursuit_spike_bool, adjusted_clips
