"""Parity of the CUDA path with the oracle and the reference's golden vectors.

Whole-pursuit tests compare the drop-in binary_pursuit() with the outputs of
the reference itself (tests/golden) and with the oracle on fresh seeded
recordings.  Stage tests drive each C-ABI stage with randomised window
states and compare every output array with the oracle's restated kernel.
All comparisons are exact: spike indices and labels are integers, and every
floating-point value is produced by the reference's sequence of IEEE binary32
operations.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle as O  # noqa: E402
from spikesorting_fullpursuit_b200 import _lib, synthetic  # noqa: E402
from spikesorting_fullpursuit_b200 import build as B  # noqa: E402
from spikesorting_fullpursuit_b200.parallel import binary_pursuit_parallel as bpp  # noqa: E402
from tests._cases import GoldenCase, assert_same_outputs, golden_paths  # noqa: E402

pytestmark = pytest.mark.gpu
PAD = 4


@pytest.fixture(scope="module")
def lib():
    B.build()
    return _lib.lib()


_KEEP = []


def D(a):
    """numpy -> cuda tensor (uint32 carried as int32 bits).  The tensor is
    kept alive until the test ends: a pointer handed to the C ABI must not
    outlive its tensor (the caching allocator would reuse the block)."""
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    t = torch.from_numpy(a.copy()).cuda()
    _KEEP.append(t)
    return t


@pytest.fixture(autouse=True)
def _release_kept():
    yield
    torch.cuda.synchronize()
    _KEEP.clear()


def H(t, dtype=None):
    a = t.cpu().numpy()
    if dtype is not None:
        a = a.view(dtype)
    return a


def P(t):
    return _lib.ptr(t)


# ----------------------------------------------------------------- whole pursuit

# precision, and for the tensor cores the likelihood layout
MODES = {"fp32": ("fp32", None), "bf16-samples": ("bf16", "samples"), "bf16-wide": ("bf16", "wide")}


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("path", golden_paths(), ids=lambda p: p.split("/")[-1][:-4])
def test_binary_pursuit_matches_reference_golden(lib, path, mode):
    precision, layout = MODES[mode]
    c = GoldenCase(path)
    m = c.metrics()
    out = bpp.binary_pursuit(c.voltage, c.voltage.dtype, c.sort_info, m,
                             n_max_shift_inds=c.n_max_shift_inds, chunk_samples=c.chunk_samples,
                             precision=precision, tc_layout=layout)
    assert_same_outputs(out, c.expected, c.empty)
    assert np.array_equal(m["n_spikes"], c.n_spikes)


LIVE = [
    dict(kind="tetrode", seed=101, L=101, dur=0.5, nmax=100),
    dict(kind="tetrode", seed=102, L=31, dur=1.0, nmax=30, clips=True),
    dict(kind="linear16", seed=103, L=61, dur=0.15, nmax=60, K=32),
    dict(kind="linear16", seed=104, L=101, dur=0.06, nmax=100, K=64),
    dict(kind="hd384", seed=105, L=61, dur=0.1, nmax=30, K=24, C=64, mask=16),
    dict(kind="tetrode", seed=106, L=41, dur=0.5, nmax=20, overlap=False),
    dict(kind="tetrode", seed=107, L=31, dur=0.5, nmax=30, chunk=2000),
]


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("cfg", LIVE, ids=lambda c: "%s-%d" % (c["kind"], c["seed"]))
def test_binary_pursuit_matches_oracle(lib, cfg, mode):
    precision, layout = MODES[mode]
    kw = dict(duration_s=cfg["dur"], seed=cfg["seed"], L=cfg["L"])
    if "K" in cfg:
        kw["n_templates"] = cfg["K"]
    if "C" in cfg:
        kw["n_chans"] = cfg["C"]
        kw["mask_chans"] = cfg["mask"]
    rec = getattr(synthetic, cfg["kind"])(**kw)
    si = rec.sort_info(do_overlap_recheck=cfg.get("overlap", True),
                       get_adjusted_clips=cfg.get("clips", False))
    chunk = cfg.get("chunk")
    exp = O.binary_pursuit_oracle(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(),
                                  n_max_shift_inds=cfg["nmax"], chunk_samples=chunk)
    stats = []
    got = bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(),
                             n_max_shift_inds=cfg["nmax"], chunk_samples=chunk, precision=precision,
                             stats=stats, tc_layout=layout)
    assert_same_outputs(got, tuple(np.asarray(x) for x in exp), isinstance(exp[0], list))
    if precision == "bf16":
        # the tensor-core path ran, in the layout asked for (the 64-channel
        # case as template groups on their channel ranges)
        assert stats[0]["launches"]["lik_refine"] >= 3 * stats[0]["passes"]
        assert all(s["tc_layout"] == layout for s in stats)


@pytest.mark.parametrize("overlap", ["fast", "exact"])
def test_overlap_methods_agree_with_oracle(lib, overlap):
    rec = synthetic.linear16(duration_s=0.08, seed=111, n_templates=24, L=61)
    si = rec.sort_info()
    exp = O.binary_pursuit_oracle(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=60)
    got = bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=60,
                             overlap=overlap)
    assert_same_outputs(got, tuple(np.asarray(x) for x in exp))


def test_fast_overlap_exact_ties_between_duplicate_templates(lib):
    """Two copies of every template: overlap items of twin templates tie
    exactly, so the lowest item id must win, as in the reference."""
    rec = synthetic.tetrode(duration_s=0.5, seed=112, L=41, n_templates=4)
    m = rec.fresh_metrics()
    for key in ("templates", "template_SS", "neuron_lower_thresholds"):
        m[key] = np.concatenate([m[key], m[key]], axis=0)
    m["template_SS_by_chan"] = np.zeros((8, rec.n_chans))
    si = rec.sort_info(get_adjusted_clips=True)
    m2 = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in m.items()}
    exp = O.binary_pursuit_oracle(rec.voltage, rec.voltage.dtype, si, m, n_max_shift_inds=40)
    stats = []
    got = bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, m2, n_max_shift_inds=40, stats=stats,
                             precision="fp32")
    assert_same_outputs(got, tuple(np.asarray(x) for x in exp))
    assert stats[0]["candidates"] > 0


# ----------------------------------------------------------------- stages

def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


@pytest.mark.parametrize("C,n,K,L", [(5, 3000, 7, 37), (20, 2500, 17, 21), (3, 1300, 5, 150)])
def test_stage_likelihood_bit_exact(lib, C, n, K, L):
    r = _rng(C * 1000 + L)
    v = r.standard_normal((C, n)).astype(np.float32)
    T = (r.standard_normal((K, C * L)) * 0.7).astype(np.float32)
    tss = np.float32(-0.5 * np.sum(T.astype(np.float64) ** 2, axis=1))
    W = (n + L - 1) // L
    win = np.sort(r.choice(W, size=max(1, W * 2 // 3), replace=False)).astype(np.uint32)
    Lk0 = r.standard_normal((K, n)).astype(np.float32)
    exp = Lk0.copy()
    O.stage_full_likelihood(v, T.reshape(-1), K, L, tss, win, exp)
    Lk = D(Lk0)
    nwin = D(np.array([len(win)], np.uint32))
    _lib.check(lib.fbp_compute_full_likelihood(P(D(v)), n, C, P(D(T)), K, L, P(D(tss)), P(D(win)),
                                               P(nwin), W, P(Lk), 0, None))
    torch.cuda.synchronize()
    assert np.array_equal(H(Lk).view(np.uint32), exp.view(np.uint32))


def _state(W, r=None):
    z = lambda dt: np.zeros(W + PAD, dt)
    st = {"best_idx": z(np.uint32), "best_lab": z(np.uint32), "best_ll": z(np.float32),
          "ov_idx": z(np.uint32), "ov_lab": z(np.uint32), "flags": z(np.uint8), "ovr": z(np.uint8)}
    return st


def _dev_state(st):
    d = {k: D(v) for k, v in st.items()}
    ws = _lib.WindowState(best_idx=P(d["best_idx"]), best_lab=P(d["best_lab"]), best_ll=P(d["best_ll"]),
                          ov_idx=P(d["ov_idx"]), ov_lab=P(d["ov_lab"]), flags=P(d["flags"]),
                          overlap_recheck=P(d["ovr"]))
    return d, ws


def _compare_state(d, st):
    for k, v in st.items():
        got = H(d[k])
        if v.dtype == np.uint32:
            got = got.view(np.uint32)
        if v.dtype == np.float32:
            assert np.array_equal(got.view(np.uint32), v.view(np.uint32)), k
        else:
            assert np.array_equal(got, v), (k, np.nonzero(got != v)[0][:10])


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_stage_window_argmax_with_ties(lib, seed):
    r = _rng(seed)
    n, L, K = 2000, 23, 9
    W = (n + L - 1) // L
    Lk = r.integers(-6, 4, size=(K, n)).astype(np.float32)       # many exact ties
    st = _state(W)
    st["best_idx"][:W] = r.integers(0, n, W)
    st["best_lab"][:W] = r.integers(0, K, W)
    st["best_ll"][:W] = r.standard_normal(W)
    st["flags"][:W] = r.integers(0, 3, W)
    win = np.sort(r.choice(W, size=W // 2, replace=False)).astype(np.uint32)
    d, ws = _dev_state(st)
    O.stage_template_max(n, L, K, win, st, Lk)
    nwin = D(np.array([len(win)], np.uint32))
    _lib.check(lib.fbp_window_argmax(n, L, K, P(D(win)), P(nwin), W, ctypes.byref(ws), P(D(Lk)), None))
    torch.cuda.synchronize()
    _compare_state(d, st)


@pytest.mark.parametrize("seed,nmax", [(4, 30), (5, 10), (6, 45)])
def test_stage_overlap_recheck(lib, seed, nmax):
    rec = synthetic.linear16(duration_s=0.08, seed=seed, n_templates=10, L=31, n_chans=6)
    v = rec.voltage.astype(np.float32)
    C, n = v.shape
    L, K = 31, 10
    T = rec.templates.reshape(-1)
    tss = np.float32(-0.5 * rec.separability_metrics["template_SS"])
    thr = np.float32(rec.separability_metrics["neuron_lower_thresholds"])
    W = (n + L - 1) // L
    win = np.arange(W, dtype=np.uint32)
    Lk = np.zeros((K, n), np.float32)
    O.stage_full_likelihood(v, T, K, L, tss, win, Lk)
    st = _state(W)
    O.stage_template_max(n, L, K, win, st, Lk)
    cand = np.nonzero(st["ovr"][:W])[0].astype(np.uint32)
    assert len(cand) > 3
    d, ws = _dev_state(st)
    O.stage_overlap(v, T, K, L, cand, st, Lk, nmax, thr)
    nc = D(np.array([len(cand)], np.uint32))
    _lib.check(lib.fbp_overlap_recheck(P(D(v)), n, C, P(D(T)), K, L, P(D(cand)), P(nc), len(cand),
                                       ctypes.byref(ws), P(D(Lk)), nmax, P(D(thr)), None))
    torch.cuda.synchronize()
    _compare_state(d, st)


@pytest.mark.parametrize("seed", [7, 8, 9, 10])
def test_stage_check_overlap_chain(lib, seed):
    r = _rng(seed)
    L, W = 20, 400
    n = W * L
    st = _state(W)
    # candidates: every other window in long runs, so the id-2 chain is exercised
    cand = np.sort(np.unique(np.concatenate([np.arange(2, W - 3, 2)[r.random(len(range(2, W - 3, 2))) < 0.8],
                                             r.integers(2, W - 3, 20)]))).astype(np.uint32)
    st["ovr"][cand] = (r.random(len(cand)) < 0.85).astype(np.uint8)
    st["ov_idx"][:W] = (np.arange(W) * L + r.integers(-L, 2 * L, W)).clip(0, n - 1)
    st["ov_lab"][:W] = r.integers(0, 5, W)
    st["best_idx"][:W] = r.integers(0, n, W)
    st["flags"][:W] = r.integers(0, 2, W)
    d, ws = _dev_state(st)
    O.stage_check_overlap(n, L, cand, st)
    nc = D(np.array([len(cand)], np.uint32))
    scratch = torch.zeros(W + PAD, dtype=torch.uint8, device="cuda")
    _lib.check(lib.fbp_check_overlap_reassignments(n, L, P(D(cand)), P(nc), len(cand), ctypes.byref(ws),
                                                   P(scratch), None))
    torch.cuda.synchronize()
    _compare_state(d, st)


@pytest.mark.parametrize("seed", [11, 12, 13, 14, 15])
def test_stage_accept_flag_chains(lib, seed):
    r = _rng(seed)
    L, W, C = 25, 600, 3
    n = W * L + 7
    W = (n + L - 1) // L
    K = 6
    thr = np.float32(r.uniform(0.5, 2.0, K))
    st = _state(W)
    # long runs of active windows whose best sits in the left neighbour
    win = np.sort(r.choice(W, size=int(W * 0.8), replace=False)).astype(np.uint32)
    off = r.choice([-L // 2, L // 3, L + 2, -3], size=W, p=[0.45, 0.2, 0.2, 0.15])
    st["best_idx"][:W] = (np.arange(W) * L + off).clip(0, n - 1)
    st["best_lab"][:W] = r.integers(0, K, W)
    st["best_ll"][:W] = r.uniform(0.0, 2.5, W)
    st["flags"][:W] = r.choice([0, 1, 2], size=W, p=[0.3, 0.6, 0.1])
    st["ovr"][win[r.random(len(win)) < 0.05]] = 1
    active = np.zeros(_lib.lib().fbp_window_u8_bytes(W), np.uint8)
    active[win] = 1
    F0 = st["flags"].copy()
    d, ws = _dev_state(st)
    exp_i, exp_l = O.stage_accept(n, C, L, thr, win, st)
    nw = D(np.array([len(win)], np.uint32))
    nb = lib.fbp_window_u8_bytes(W)
    has = torch.zeros(nb, dtype=torch.uint8, device="cuda")
    fout = torch.zeros(nb, dtype=torch.uint8, device="cuda")
    si = torch.zeros(W + PAD, dtype=torch.int32, device="cuda")
    sl = torch.zeros(W + PAD, dtype=torch.int32, device="cuda")
    sw = torch.zeros(W + PAD, dtype=torch.int32, device="cuda")
    ns = torch.zeros(1, dtype=torch.int32, device="cuda")
    scratch = torch.zeros(lib.fbp_scan_scratch_bytes(W), dtype=torch.uint8, device="cuda")
    _lib.check(lib.fbp_binary_pursuit_accept(n, C, L, P(D(thr)), P(D(win)), P(nw), W, ctypes.byref(ws),
                                             P(D(active)), P(has), P(fout), P(si), P(sl), P(sw), P(ns),
                                             P(scratch), None))
    torch.cuda.synchronize()
    m = int(H(ns)[0])
    assert m == len(exp_i)
    assert np.array_equal(H(si)[:m].view(np.uint32), exp_i)
    assert np.array_equal(H(sl)[:m].view(np.uint32), exp_l)
    got_flags = H(fout)[:W]
    assert np.array_equal(got_flags, st["flags"][:W]), np.nonzero(got_flags != st["flags"][:W])[0][:10]
    assert np.array_equal(H(d["flags"])[:W], F0[:W])       # input flags untouched


@pytest.mark.parametrize("seed,nmax", [(16, 12), (17, 30), (18, 3)])
def test_stage_residual_overlapping_spikes(lib, seed, nmax):
    r = _rng(seed)
    C, L, K = 4, 31, 5
    W = 300
    n = W * L
    v = r.standard_normal((C, n)).astype(np.float32)
    T = r.standard_normal((K, C * L)).astype(np.float32)
    wins = np.sort(r.choice(np.arange(1, W - 2), size=180, replace=False))
    idx = (wins * L + r.integers(-nmax, L + nmax, len(wins))).clip(0, n - 1).astype(np.uint32)
    lab = r.integers(0, K + 1, len(wins)).astype(np.uint32)     # some labels >= K
    exp = O.stage_residual(v, T.reshape(-1), K, L, idx, lab)
    vd = D(v)
    R = 3 + (2 * nmax + L - 1) // L
    _lib.check(lib.fbp_compute_residual(P(vd), n, C, P(D(T)), K, L, P(D(idx)), P(D(lab)), len(idx), R, None))
    torch.cuda.synchronize()
    assert np.array_equal(H(vd).view(np.uint32), exp.view(np.uint32))


def test_stage_adjusted_clips(lib):
    r = _rng(19)
    C, L, K, n = 3, 17, 4, 500
    v = r.standard_normal((C, n)).astype(np.float32)
    T = r.standard_normal((K, C * L)).astype(np.float32)
    idx = np.array([0, 5, 100, 480, 495, 499], np.uint32)       # the last ones run past n
    lab = np.array([0, 1, 2, 3, 9, 1], np.uint32)
    exp = O.adjusted_clips(v, T.reshape(-1), K, L, idx, lab)
    clips = torch.zeros((len(idx), C * L), dtype=torch.float32, device="cuda")
    _lib.check(lib.fbp_get_adjusted_clips(P(D(v)), n, C, P(D(T)), K, L, P(D(idx)), P(D(lab)), len(idx),
                                          P(clips), None))
    torch.cuda.synchronize()
    assert np.array_equal(H(clips).view(np.uint32), exp.view(np.uint32))


def test_iteration_cap_returns_error_status(lib):
    rec = synthetic.tetrode(duration_s=0.2, seed=20, L=31)
    si = rec.sort_info()
    with pytest.raises(_lib.PursuitError) as e:
        bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=5,
                           max_passes=1, precision="fp32")
    assert e.value.code == _lib.FBP_ERR_ITER_CAP
    # the context is still usable afterwards
    out = bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=5,
                             precision="fp32")
    assert len(out[0]) > 0
