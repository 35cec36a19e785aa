"""Tuner of the tensor-core likelihood's template group size, per shape
bucket.

The planner in the library picks, per chunk, the group size (templates per
tcgen05 MMA column block) with the least padded MMA work that fits shared
memory: a cost model.  This module times the candidates instead: for a
recording's shape bucket (channels, templates, clip length, template channel
support width) it runs one tensor-core likelihood pass over a sample of the
recording for each group size (fbp_tc_likelihood_bounds, CUDA-event timed
after a warm-up), keeps the fastest, and caches the choice in a JSON file
(FBP_TUNE_CACHE, default ~/.cache/fbp_b200/tc_groups.json).  apply() sets
the chosen size for the calls the calling thread makes afterwards
(fbp_set_tc_group_size).  The spikes do not depend on the group size; only
the time does."""
import ctypes
import json
import os

import numpy as np

from . import _lib

CANDIDATES = (16, 32, 64, 128, 256)


def cache_path():
    return os.environ.get("FBP_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "fbp_b200",
                                                            "tc_groups.json")


def _up(x, m):
    return (int(x) + m - 1) // m * m


def shape_bucket(n_chans, templates, L):
    """The quantities the group plan depends on, rounded: channels up to 8,
    templates up to 16, clip length up to 16, median template support width
    up to 8 channels."""
    T = np.asarray(templates, dtype=np.float32).reshape(-1, n_chans, L)
    K = T.shape[0]
    nz = np.any(T != 0, axis=2)
    widths = [(np.nonzero(r)[0][-1] - np.nonzero(r)[0][0] + 1) if r.any() else 0 for r in nz]
    w = int(np.median(widths)) if widths else n_chans
    return "C%d_K%d_L%d_w%d" % (_up(n_chans, 8), _up(K, 16), _up(L, 16), _up(w, 8))


def candidates_for(n_templates):
    """Group sizes that make distinct plans: up to the template count
    rounded up to 16 (larger sizes give the same single group)."""
    kall = _up(n_templates, 16)
    return tuple(g for g in CANDIDATES if g <= kall) or (16,)


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(table):
    p = cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def time_group_sizes(voltage, templates, neg_half_ss, L, candidates=CANDIDATES, repeats=3):
    """Milliseconds of one tensor-core likelihood pass over `voltage`
    ([C, n] float32, the sample) per candidate group size."""
    import torch
    lib = _lib.lib()
    v = torch.from_numpy(np.ascontiguousarray(voltage, dtype=np.float32)).cuda()
    T = torch.from_numpy(np.ascontiguousarray(templates, dtype=np.float32).reshape(-1)).cuda()
    tss = torch.from_numpy(np.ascontiguousarray(neg_half_ss, dtype=np.float32)).cuda()
    C, n = int(v.shape[0]), int(v.shape[1])
    K = int(tss.numel())
    wsb = ctypes.c_size_t(0)
    _lib.check(lib.fbp_pursuit_workspace_bytes(n, C, K, L, 0, _lib.PREC_BF16_REFINE, ctypes.byref(wsb)))
    ws = torch.empty(wsb.value, dtype=torch.uint8, device="cuda")
    approx = torch.empty((K, n), dtype=torch.float32, device="cuda")
    bound = torch.empty((K, n), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream()
    out = {}
    try:
        for gs in candidates:
            _lib.check(lib.fbp_set_tc_group_size(int(gs)))

            def one():
                _lib.check(lib.fbp_tc_likelihood_bounds(_lib.ptr(v), n, C, _lib.ptr(T), K, L, _lib.ptr(tss),
                                                        _lib.ptr(ws), ws.numel(), _lib.ptr(approx), _lib.ptr(bound),
                                                        _lib.stream_ptr(st)))
            one()                                            # warm-up (and the plan)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(repeats):
                one()
            e1.record(st)
            torch.cuda.synchronize()
            out[int(gs)] = e0.elapsed_time(e1) / repeats
    finally:
        _lib.check(lib.fbp_set_tc_group_size(0))
    return out


def tune(voltage, templates, neg_half_ss, L, sample_samples=120000, force=False):
    """Group size for this recording's shape bucket: from the cache, else
    timed on the first `sample_samples` samples and cached.  Returns
    (group_size, bucket, timings or None)."""
    C = int(np.shape(voltage)[0])
    bucket = shape_bucket(C, templates, L)
    table = _load()
    if not force and bucket in table:
        return int(table[bucket]["group_size"]), bucket, None
    K = int(np.asarray(templates).reshape(-1, C * L).shape[0])
    cands = candidates_for(K)
    if len(cands) == 1:                                      # nothing to choose
        return cands[0], bucket, None
    sample = np.asarray(voltage)[:, :min(int(sample_samples), np.shape(voltage)[1])]
    times = time_group_sizes(sample, templates, neg_half_ss, L, cands)
    best = min(times, key=times.get)
    table[bucket] = {"group_size": int(best), "ms": {str(k): v for k, v in times.items()},
                     "sample_samples": int(sample.shape[1])}
    _store(table)
    return int(best), bucket, times


def apply(group_size):
    """Use `group_size` for the pursuits this thread runs next (0: the cost
    model)."""
    _lib.check(_lib.lib().fbp_set_tc_group_size(int(group_size)))
