"""Tuner of the tensor-core likelihood's plan, per shape bucket.

The library picks, per chunk, a layout for the likelihood passes (wide tiles
of the pass's window stream where they apply, else 128-sample tiles) and,
for the 128-sample tiles and the overlap tables, a template group size with
the least padded MMA work that fits shared memory: a cost model.  This
module times the candidates instead: for a recording's shape bucket
(channels, templates, clip length, template channel support width) it runs
one tensor-core likelihood pass over a sample of the recording per plan
("wide", or "samples:<group size>"; fbp_tc_likelihood_bounds, CUDA-event
timed after a warm-up), keeps the fastest, and caches the choice in a JSON
file (FBP_TUNE_CACHE, default ~/.cache/fbp_b200/tc_plans.json).  apply()
sets the chosen plan for the calls the calling thread makes afterwards
(fbp_set_tc_layout, fbp_set_tc_group_size).  The spikes do not depend on the
plan; only the time does."""
import ctypes
import json
import os

import numpy as np

from . import _lib

CANDIDATES = (16, 32, 64, 128, 256)


def cache_path():
    return os.environ.get("FBP_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "fbp_b200",
                                                            "tc_plans.json")


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


def plans_for(n_templates, L):
    """Plans that time differently: the wide layout (where the clip length
    allows it) and the 128-sample layout with every distinct group size."""
    wide = ("wide",) if 16 <= int(L) <= 1024 else ()
    return wide + tuple("samples:%d" % g for g in candidates_for(n_templates))


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


def apply(plan):
    """Use `plan` ("wide", "samples:<group size>", or a bare group size; 0 or
    None: the library's own choice) for the pursuits this thread runs next."""
    lib = _lib.lib()
    if plan in (None, 0, "auto"):
        layout, gs = _lib.TC_LAYOUT_AUTO, 0
    elif plan == "wide":
        layout, gs = _lib.TC_LAYOUT_WIDE, 0
    elif isinstance(plan, str) and plan.startswith("samples:"):
        layout, gs = _lib.TC_LAYOUT_SAMPLES, int(plan.split(":", 1)[1])
    else:
        layout, gs = _lib.TC_LAYOUT_SAMPLES, int(plan)
    _lib.check(lib.fbp_set_tc_layout(layout))
    _lib.check(lib.fbp_set_tc_group_size(gs))


def time_plans(voltage, templates, neg_half_ss, L, plans, repeats=3):
    """Milliseconds of one tensor-core likelihood pass over `voltage`
    ([C, n] float32, the sample) per plan."""
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
        for plan in plans:
            apply(plan)

            def one():
                _lib.check(lib.fbp_tc_likelihood_bounds(_lib.ptr(v), n, C, _lib.ptr(T), K, L, _lib.ptr(tss),
                                                        _lib.ptr(ws), ws.numel(), _lib.ptr(approx), _lib.ptr(bound),
                                                        _lib.stream_ptr(st)))
            try:
                one()                                        # warm-up (and the plan)
            except ValueError as e:
                if "no tensor-core plan" not in str(e):
                    raise
                continue                                     # the library uses the FP32 kernel here
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(repeats):
                one()
            e1.record(st)
            torch.cuda.synchronize()
            out[plan] = e0.elapsed_time(e1) / repeats
    finally:
        apply(None)
    return out


def tune(voltage, templates, neg_half_ss, L, sample_samples=120000, force=False):
    """Plan for this recording's shape bucket: from the cache, else timed on
    the first `sample_samples` samples and cached.  Returns (plan, bucket,
    timings or None)."""
    C = int(np.shape(voltage)[0])
    bucket = shape_bucket(C, templates, L)
    table = _load()
    if not force and bucket in table and "plan" in table[bucket]:
        return table[bucket]["plan"], bucket, None
    K = int(np.asarray(templates).reshape(-1, C * L).shape[0])
    plans = plans_for(K, L)
    if len(plans) == 1:                                      # nothing to choose
        return plans[0], bucket, None
    sample = np.asarray(voltage)[:, :min(int(sample_samples), np.shape(voltage)[1])]
    times = time_plans(sample, templates, neg_half_ss, L, plans)
    best = min(times, key=times.get) if times else "auto"   # no tensor-core plan: the library's own path
    table[bucket] = {"plan": best, "ms": dict(times), "sample_samples": int(sample.shape[1])}
    _store(table)
    return best, bucket, times
