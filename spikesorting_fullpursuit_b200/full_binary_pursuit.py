"""The device glue of spikesorting_fullpursuit/full_binary_pursuit.py that
prepares binary_pursuit()'s inputs (:299-322): the clips of every unit's
spikes on all channels, a robust template per unit, and the per-channel
noise covariance of the clip residuals -- one device-resident pass instead
of a host round trip per unit."""
import numpy as np

from . import _device as D
from . import _lib
from .parallel.binary_pursuit_parallel import time_window_to_samples


def pursuit_templates_and_covariance(voltage, unit_spike_indices, sampling_rate, clip_width, n_cov_samples,
                                     v_dtype=None, cov_sample_inds=None, rng=None):
    """bp_templates and chan_covariance_mats as full_binary_pursuit.py:299-322
    builds them.

    voltage             [channels, samples] (host array or CUDA tensor)
    unit_spike_indices  list of sorted int arrays, one per unit (the
                        units' n['spike_indices'])
    clip_width          the binary pursuit clip width (seconds)
    n_cov_samples       rows of the residual clips used for the covariance;
                        when fewer than all rows, `cov_sample_inds` (or
                        rng.integers, as the reference's np.random.randint)
                        chooses them with replacement
    Returns (bp_templates [units, C*L] of the voltage dtype, list of C
    [L, L] float64 covariance matrices)."""
    v = D.to_dev(voltage)
    dt = np.dtype(str(v.dtype).replace("torch.", "")) if v_dtype is None else np.dtype(v_dtype)
    C, n = int(v.shape[0]), int(v.shape[1])
    window, _ = time_window_to_samples(clip_width, sampling_rate)
    L = window[1] - window[0]
    lib = _lib.lib()
    # clips of every unit, rows unit by unit (get_clips' edge rule per unit)
    from .parallel.segment_parallel import _valid_range
    starts, counts, evs = [], [], []
    for ev in unit_spike_indices:
        ev = np.asarray(ev, dtype=np.int64)
        if ev.size == 0:
            raise ValueError("a unit without spikes has no template")
        _, a, b = _valid_range(ev, window, n, True)
        if a is None:
            raise ValueError("no clip of a unit lies inside the voltage")
        starts.append(a)
        counts.append(b - a + 1)
        evs.append(ev)
    off = np.zeros(len(evs) + 1, np.uint32)
    off[1:] = np.cumsum(counts)
    rows = int(off[-1])
    clips = D.empty((rows, C * L), dt)
    nb = D.to_dev(np.arange(C, dtype=np.int64))
    stream = D.stream()
    keep = []
    for u, ev in enumerate(evs):
        ev_d = D.to_dev(ev)
        keep.append(ev_d)
        view = clips[int(off[u]):int(off[u + 1])]
        _lib.check(lib.fbp_get_clips(_lib.ptr(v), D.code_of(dt), n, C, _lib.ptr(nb), C, _lib.ptr(ev_d),
                                     int(starts[u]), int(counts[u]), int(window[0]), int(window[1]), _lib.ptr(view),
                                     stream))
    from .preprocessing import calculate_robust_templates
    templates = calculate_robust_templates(clips, off, as_tensor=True)
    if n_cov_samples >= rows:
        sel = np.arange(rows, dtype=np.int64)
    elif cov_sample_inds is not None:
        sel = np.ascontiguousarray(cov_sample_inds, dtype=np.int64)
    else:
        rng = np.random.default_rng() if rng is None else rng
        sel = rng.integers(0, rows, int(n_cov_samples)).astype(np.int64)
    row_unit = np.repeat(np.arange(len(evs), dtype=np.uint32), counts)
    ru = D.to_dev(row_unit)
    sel_d = D.to_dev(sel)
    cov = D.empty((C, L, L), np.float64)
    sb = lib.fbp_noise_cov_scratch_bytes(C, L)
    scratch = D.empty((sb,), np.uint8)
    _lib.check(lib.fbp_clip_noise_covariance(_lib.ptr(clips), D.code_of(dt), _lib.ptr(ru), _lib.ptr(templates),
                                             _lib.ptr(sel_d), len(sel), C, L, _lib.ptr(cov), _lib.ptr(scratch), sb,
                                             stream))
    cov_h = D.host(cov)
    return D.host(templates), [cov_h[c] for c in range(C)]
