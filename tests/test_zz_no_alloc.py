"""The allocation-free accept entry point agrees with the regular one.

fbp_binary_pursuit_accept_noalloc exists for callers that cannot allocate
device memory (a host framework that owns the whole device heap, a real-time
loop that must not pay cudaMalloc's synchronisation); its scratch is a fixed
device array inside the library.  This test calls both entry points through
the C ABI on the same inputs, twice in a row with different inputs (the fixed
array keeps the previous call's contents), and requires identical outputs.
This file is collected last so that a failure here cannot hide another test.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from spikesorting_fullpursuit_b200 import _lib  # noqa: E402
from spikesorting_fullpursuit_b200 import build as B  # noqa: E402

pytestmark = pytest.mark.gpu
PAD = 4


def _inputs(seed, W_target=700, L=25, K=6):
    r = np.random.Generator(np.random.PCG64(seed))
    n = W_target * L + int(r.integers(1, L))
    W = (n + L - 1) // L
    thr = np.float32(r.uniform(0.5, 2.0, K))
    win = np.sort(r.choice(W, size=int(W * 0.8), replace=False)).astype(np.uint32)
    st = {
        "best_idx": ((np.arange(W + PAD) * L + r.choice([-L // 2, L // 3, L + 2, -3], size=W + PAD))
                     .clip(0, n - 1)).astype(np.uint32),
        "best_lab": r.integers(0, K, W + PAD).astype(np.uint32),
        "best_ll": r.uniform(0.0, 2.5, W + PAD).astype(np.float32),
        "ov_idx": np.zeros(W + PAD, np.uint32),
        "ov_lab": np.zeros(W + PAD, np.uint32),
        "flags": r.choice([0, 1, 2], size=W + PAD, p=[0.3, 0.6, 0.1]).astype(np.uint8),
        "ovr": np.zeros(W + PAD, np.uint8),
    }
    st["ovr"][win[r.random(len(win)) < 0.05]] = 1
    return n, L, W, thr, win, st


class _Dev:
    def __init__(self):
        self.keep = []

    def t(self, a):
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint32:
            a = a.view(np.int32)
        x = torch.from_numpy(a.copy()).cuda()
        self.keep.append(x)
        return x

    def zeros(self, n, dtype):
        x = torch.zeros(n, dtype=dtype, device="cuda")
        self.keep.append(x)
        return x


def _run(lib, n, L, W, thr, win, st, noalloc):
    d = _Dev()
    C = 3
    ds = {k: d.t(v) for k, v in st.items()}
    ws = _lib.WindowState(*(ctypes.c_void_p(ds[k].data_ptr()) for k in
                            ("best_idx", "best_lab", "best_ll", "ov_idx", "ov_lab", "flags", "ovr")))
    nb = lib.fbp_window_u8_bytes(W)
    active = np.zeros(nb, np.uint8)
    active[win] = 1
    act = d.t(active)
    fout = d.zeros(nb, torch.uint8)
    si, sl, sw = (d.zeros(W + PAD, torch.int32) for _ in range(3))
    ns = d.zeros(1, torch.int32)
    P = lambda x: ctypes.c_void_p(x.data_ptr())
    nw = d.t(np.array([len(win)], np.uint32))
    if noalloc:
        rc = lib.fbp_binary_pursuit_accept_noalloc(n, C, L, P(d.t(thr)), P(d.t(win)), P(nw), W,
                                                   ctypes.byref(ws), P(act), P(fout), P(si), P(sl), P(sw),
                                                   P(ns), None)
    else:
        has = d.zeros(nb, torch.uint8)
        scratch = d.zeros(lib.fbp_scan_scratch_bytes(W), torch.uint8)
        rc = lib.fbp_binary_pursuit_accept(n, C, L, P(d.t(thr)), P(d.t(win)), P(nw), W, ctypes.byref(ws),
                                           P(act), P(has), P(fout), P(si), P(sl), P(sw), P(ns), P(scratch),
                                           None)
    _lib.check(rc)
    torch.cuda.synchronize()
    m = int(ns.cpu().numpy()[0])
    return (m, fout.cpu().numpy()[:W].copy(), si.cpu().numpy()[:m].copy(), sl.cpu().numpy()[:m].copy(),
            sw.cpu().numpy()[:m].copy())


def test_noalloc_accept_matches_allocating_entry_point_on_consecutive_calls():
    B.build()
    lib = _lib.lib()
    # two calls in a row with different inputs: the second must not see the
    # first call's leftovers in the shared fixed scratch
    for seed, Wt in ((41, 700), (42, 1900)):
        inputs = _inputs(seed, W_target=Wt)
        ref = _run(lib, *inputs, noalloc=False)
        got = _run(lib, *inputs, noalloc=True)
        assert ref[0] > 0
        assert got[0] == ref[0]
        for g, e in zip(got[1:], ref[1:]):
            assert np.array_equal(g, e)


def test_noalloc_rejects_more_windows_than_its_scratch_holds():
    B.build()
    lib = _lib.lib()
    L = 2
    n = (_lib.NOALLOC_MAX_WINDOWS + 1) * L
    dummy = ctypes.c_void_p(1)
    ws = _lib.WindowState(*([dummy] * 7))
    rc = lib.fbp_binary_pursuit_accept_noalloc(n, 3, L, dummy, dummy, dummy, 1, ctypes.byref(ws), dummy,
                                               dummy, dummy, dummy, dummy, dummy, None)
    assert rc == _lib.FBP_ERR_BAD_ARG
    assert b"fixed scratch limit" in lib.fbp_last_error()
