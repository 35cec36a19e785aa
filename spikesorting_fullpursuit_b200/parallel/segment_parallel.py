"""Clip gathers on the device: spikesorting_fullpursuit/parallel/
segment_parallel.py get_clips (:451-503) and get_singlechannel_clips
(:392-448) with the same arguments, edge handling and return values; the
copy loop runs as one CUDA kernel (fbp_get_clips)."""
import numpy as np

from .. import _device as D
from .. import _lib
from .binary_pursuit_parallel import time_window_to_samples


def _valid_range(event_indices, window, n_samples, strict_end):
    """The reference's scan from both ends of the sorted events (:463-483;
    get_singlechannel_clips tests the end with `>` instead of `>=`).
    Returns (valid bool array, first, stop) or (valid, None, None) when none
    is valid."""
    valid = np.ones(event_indices.shape[0], dtype="bool")
    start = 0
    while event_indices[start] + window[0] < 0:
        valid[start] = False
        start += 1
        if start == event_indices.size:
            valid[:] = False
            return valid, None, None
    stop = event_indices.shape[0] - 1
    past = (lambda x: x + window[1] >= n_samples) if strict_end else (lambda x: x + window[1] > n_samples)
    while past(event_indices[stop]):
        valid[stop] = False
        stop -= 1
        if stop < 0:
            valid[:] = False
            return valid, None, None
    return valid, start, stop


def get_clips(probe_dict, voltage, neighbors, event_indices, clip_width, use_memmap=False, check_valid=True,
              as_tensor=False):
    """segment_parallel.get_clips: clips of every channel in `neighbors`
    (concatenated in that order) around each event; returns (clips,
    valid_event_indices).  `voltage` is a host array or a CUDA tensor
    [channels, samples]; with as_tensor=True the clips stay on the device.
    use_memmap is accepted and ignored (the clips live in device memory)."""
    event_indices = np.asarray(event_indices)
    if event_indices.ndim > 1:
        raise ValueError("Event_indices must be one dimensional array of indices")
    window, clip_width = time_window_to_samples(clip_width, probe_dict['sampling_rate'])
    W = window[1] - window[0]
    neighbors = np.asarray(neighbors, dtype=np.int64).reshape(-1)
    if len(event_indices) == 0:
        return np.zeros((0, W * len(neighbors)), dtype=probe_dict['v_dtype']), np.ones(0, dtype="bool")
    if check_valid:
        valid, start, stop = _valid_range(event_indices, window, probe_dict['n_samples'], True)
        if start is None:
            return None, valid
    else:
        valid, start, stop = np.ones(event_indices.shape[0], dtype="bool"), 0, len(event_indices) - 1
    v = D.to_dev(voltage)
    dt = np.dtype(probe_dict['v_dtype'])
    if np.dtype(str(v.dtype).replace("torch.", "")) != dt:
        raise TypeError("voltage dtype %s differs from v_dtype %s" % (v.dtype, dt))
    count = stop - start + 1
    out = D.empty((count, W * len(neighbors)), dt)
    ev = D.to_dev(np.ascontiguousarray(event_indices, dtype=np.int64))
    nb = D.to_dev(neighbors)
    _lib.check(_lib.lib().fbp_get_clips(_lib.ptr(v), D.code_of(dt), int(v.shape[1]), int(v.shape[0]), _lib.ptr(nb),
                                        len(neighbors), _lib.ptr(ev), int(start), int(count), int(window[0]),
                                        int(window[1]), _lib.ptr(out), D.stream()))
    return (out if as_tensor else D.host(out)), valid


def get_singlechannel_clips(probe_dict, chan_voltage, event_indices, clip_width, use_memmap=False):
    """segment_parallel.get_singlechannel_clips (:392-448)."""
    event_indices = np.asarray(event_indices)
    window, clip_width = time_window_to_samples(clip_width, probe_dict['sampling_rate'])
    valid, start, stop = _valid_range(event_indices, window, probe_dict['n_samples'], False)
    if start is None:
        return None, valid
    chan = D.to_dev(np.asarray(chan_voltage).reshape(1, -1)) if not hasattr(chan_voltage, "is_cuda") \
        else chan_voltage.reshape(1, -1)
    dt = np.dtype(probe_dict['v_dtype'])
    count = stop - start + 1
    W = window[1] - window[0]
    out = D.empty((count, W), dt)
    ev = D.to_dev(np.ascontiguousarray(event_indices, dtype=np.int64))
    nb = D.to_dev(np.zeros(1, np.int64))
    _lib.check(_lib.lib().fbp_get_clips(_lib.ptr(chan), D.code_of(dt), int(chan.shape[1]), 1, _lib.ptr(nb), 1,
                                        _lib.ptr(ev), int(start), int(count), int(window[0]), int(window[1]),
                                        _lib.ptr(out), D.stream()))
    return D.host(out), valid
