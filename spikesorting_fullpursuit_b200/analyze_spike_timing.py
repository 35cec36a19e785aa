"""Duplicate removal of spikesorting_fullpursuit/analyze_spike_timing.py on
the device, many units at once: the squared error of every clip against its
unit's template in one kernel (summed in np.sum's pairwise order, so the
comparisons are the reference's), then the reference's scan of each unit's
events, one thread per unit.  The single-unit functions keep the reference's
signatures; remove_segment_binary_pursuit_duplicates batches the per-unit
loop of postprocessing.py:521-545 (chunk-boundary duplicates of a pursuit
that ran in several chunks are found the same way)."""
import numpy as np

from . import _device as D
from . import _lib

MODE_REMOVE_BP, MODE_KEEP_BP, MODE_REMOVE_EVENTS = 0, 1, 2


def _run(mode, events, bp_bool, clips, templates, offsets, tol_inds):
    events = np.ascontiguousarray(events, dtype=np.int64)
    n = events.size
    if n == 0:
        return np.ones(0, dtype="bool")
    off = np.ascontiguousarray(offsets, dtype=np.uint32)
    ev = D.to_dev(events)
    off_d = D.to_dev(off)
    keep = D.empty((n,), np.uint8)
    bp = D.to_dev(np.ascontiguousarray(bp_bool, dtype=np.uint8)) if bp_bool is not None else None
    cl = tm = sse = None
    dim, tcode = 0, _lib.F32
    if mode != MODE_KEEP_BP:
        cl = D.to_dev(np.ascontiguousarray(clips, dtype=np.float32))
        templates = np.asarray(templates) if not hasattr(templates, "is_cuda") else templates
        tdt = np.dtype(np.float64) if np.dtype(getattr(templates, "dtype", np.float32)) == np.float64 else \
            np.dtype(np.float32)
        tm = D.to_dev(np.ascontiguousarray(templates, dtype=tdt).reshape(len(off) - 1, -1))
        tcode = D.code_of(tdt)
        dim = int(cl.shape[1])
        sse = D.empty((n,), np.float64)
    _lib.check(_lib.lib().fbp_remove_duplicates(mode, _lib.ptr(ev), _lib.ptr(bp), _lib.ptr(cl), _lib.ptr(tm), tcode,
                                                dim, _lib.ptr(off_d), len(off) - 1, n, int(tol_inds), _lib.ptr(sse),
                                                _lib.ptr(keep), D.stream()))
    return D.host(keep).astype(bool)


def keep_binary_pursuit_duplicates(event_indices, binary_pursuit_bool, tol_inds):
    """analyze_spike_timing.keep_binary_pursuit_duplicates (:85-113)."""
    return _run(MODE_KEEP_BP, event_indices, binary_pursuit_bool, None, None, [0, len(event_indices)], tol_inds)


def remove_binary_pursuit_duplicates(event_indices, clips, unit_template, binary_pursuit_bool, tol_inds):
    """analyze_spike_timing.remove_binary_pursuit_duplicates (:116-157)."""
    return _run(MODE_REMOVE_BP, event_indices, binary_pursuit_bool, clips, np.asarray(unit_template)[None, :],
                [0, len(event_indices)], tol_inds)


def remove_spike_event_duplicates(event_indices, clips, unit_template, tol_inds):
    """analyze_spike_timing.remove_spike_event_duplicates (:159-184)."""
    return _run(MODE_REMOVE_EVENTS, event_indices, None, clips, np.asarray(unit_template)[None, :],
                [0, len(event_indices)], tol_inds)


def unit_mean_templates(clips, offsets):
    """np.mean(clips[unit rows], axis=0) per unit for float32 clips, in
    numpy's order (rows added in order in float32, divided by the count)."""
    cl = D.to_dev(np.ascontiguousarray(clips, dtype=np.float32))
    off = np.ascontiguousarray(offsets, dtype=np.uint32)
    out = D.empty((len(off) - 1, int(cl.shape[1])), np.float32)
    off_d = D.to_dev(off)
    _lib.check(_lib.lib().fbp_unit_mean_templates(_lib.ptr(cl), int(cl.shape[1]), _lib.ptr(off_d), len(off) - 1,
                                                  _lib.ptr(out), D.stream()))
    return D.host(out)


def remove_segment_binary_pursuit_duplicates(event_indices, neuron_labels, clips, binary_pursuit_bool, tol_inds):
    """The per-unit loop of postprocessing.WorkItemSummary.
    remove_segment_binary_pursuit_duplicates (postprocessing.py:521-545) for
    one channel and segment: for every label (np.unique order), the unit's
    events in their original order, its template np.mean(clips, axis=0), and
    remove_binary_pursuit_duplicates -- all units in one pass.  Returns the
    keep mask over the inputs."""
    event_indices = np.asarray(event_indices)
    labels = np.asarray(neuron_labels)
    keep = np.ones(event_indices.shape[0], dtype="bool")
    if event_indices.size == 0:
        return keep
    units = np.unique(labels)
    order = np.concatenate([np.nonzero(labels == u)[0] for u in units])
    counts = np.array([np.count_nonzero(labels == u) for u in units])
    off = np.zeros(len(units) + 1, np.uint32)
    off[1:] = np.cumsum(counts)
    cl = np.ascontiguousarray(np.asarray(clips)[order], dtype=np.float32)
    templates = unit_mean_templates(cl, off)
    k = _run(MODE_REMOVE_BP, event_indices[order], np.asarray(binary_pursuit_bool)[order], cl, templates, off, tol_inds)
    keep[order] = k
    return keep
