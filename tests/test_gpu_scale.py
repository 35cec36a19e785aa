"""Parity at the structure of the benchmark workloads, the rarely taken
paths, and the tensor-core error bound entry by entry.

* The 384-channel workload at full structure (300 templates on 16-channel
  masks, 61-sample clips, n_max_shift 60, int16 voltage) and the 16-channel
  workload at its full overlap range (64 templates, 101-sample clips,
  n_max_shift 100) against the oracle, in both precisions.
* Longer recordings of both workloads, tensor-core mode with the fast overlap
  recheck against the plain FP32 path with the reference's exhaustive overlap
  recheck, entirely on the GPU.
* Capacities shrunk so the refinement list and the contender pool overflow:
  the FP32 redo and the exact-kernel hand-off still give the oracle's result.
* Every entry of one tensor-core pass: the approximation lies within its
  bound E of the reference's IEEE binary32 value (compute_maximum_likelihood,
  binary_pursuit.cl:216-252); the error against float64 is printed per
  workload.
* The tensor-core kernel's bounded waits made to give up: the call returns
  FBP_ERR_TIMEOUT and the next call on the same context is correct.

Spike comparisons are exact (integer outputs).
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle as O  # noqa: E402
from spikesorting_fullpursuit_b200 import _lib, synthetic  # noqa: E402
from spikesorting_fullpursuit_b200 import build as B  # noqa: E402
from spikesorting_fullpursuit_b200.parallel import binary_pursuit_parallel as bpp  # noqa: E402
from tests._cases import assert_same_outputs  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    B.build()
    return _lib.lib()


@pytest.fixture(autouse=True)
def _default_limits(lib):
    _lib.reset_test_limits()
    yield
    _lib.reset_test_limits()


def _as_tuple(out):
    return tuple(np.asarray(x) for x in out)


def hd384_slice(duration_s, seed):
    """The 384-channel workload's structure on a short recording."""
    return synthetic.hd384(duration_s=duration_s, seed=seed)


def linear16_slice(duration_s, seed):
    return synthetic.linear16(duration_s=duration_s, seed=seed)


# ------------------------------------------------------------ against the oracle

@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_hd384_full_structure_matches_oracle(lib, precision):
    rec = hd384_slice(0.1, seed=301)
    assert rec.n_chans == 384 and rec.n_templates == 300 and rec.n_samples_per_chan == 61
    assert rec.voltage.dtype == np.int16
    si = rec.sort_info()
    exp = O.binary_pursuit_oracle(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=60)
    stats = []
    got = bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=60,
                             precision=precision, stats=stats)
    assert len(exp[0]) > 20
    assert_same_outputs(got, _as_tuple(exp))
    if precision == "bf16":
        assert stats[0]["launches"]["lik_refine"] >= 3 * stats[0]["passes"]


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_linear16_full_overlap_range_matches_oracle(lib, precision):
    rec = linear16_slice(0.25, seed=302)
    assert rec.n_templates == 64 and rec.n_samples_per_chan == 101
    si = rec.sort_info()
    exp = O.binary_pursuit_oracle(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=100)
    got = bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=100,
                             precision=precision)
    assert len(exp[0]) > 100
    assert_same_outputs(got, _as_tuple(exp))


# ------------------------------------------------------------ long recordings, GPU only

@pytest.mark.parametrize("kind,duration_s,nmax", [("linear16", 10.0, 100), ("hd384", 1.0, 60)])
def test_tensor_core_fast_equals_fp32_exhaustive(lib, kind, duration_s, nmax):
    """bf16 + fast overlap against fp32 + the reference's exhaustive overlap
    recheck (the oracle-pinned plain path), every output array equal."""
    rec = linear16_slice(duration_s, 303) if kind == "linear16" else hd384_slice(duration_s, 304)
    si = rec.sort_info()
    s_fast, s_ref = [], []
    fast = bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=nmax,
                              precision="bf16", overlap="fast", stats=s_fast)
    ref = bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=nmax,
                             precision="fp32", overlap="exact", stats=s_ref)
    assert len(ref[0]) > 1000
    assert_same_outputs(fast, _as_tuple(ref))
    print("\n%s %.1f s: %d spikes, %d passes; bf16+fast refined %d likelihood entries (%d in the "
          "reference's order), %d overlap items" % (kind, duration_s, len(ref[0]), s_ref[0]["passes"],
                                                    s_fast[0]["lik_refined"], s_fast[0]["lik_seq_refined"],
                                                    s_fast[0]["refined_items"]))


# ------------------------------------------------------------ overflow paths

@pytest.mark.parametrize("kind,layout", [("linear16", "wide"), ("linear16", "samples"), ("hd384", "wide")])
def test_overflowing_refinement_list_and_pool_match_oracle(lib, kind, layout):
    """A refinement list of 64 entries and a contender pool of 8 overflow on
    almost every pass: the FP32 kernel redoes the likelihood of the pass and
    the candidates go to the exact overlap kernel."""
    if kind == "linear16":
        rec, nmax = linear16_slice(0.1, 305), 100
    else:
        rec, nmax = hd384_slice(0.1, 306), 60
    si = rec.sort_info()
    exp = O.binary_pursuit_oracle(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=nmax)
    _lib.set_test_limits(refine_list_cap=64, contender_pool_cap=8)
    stats = []
    got = bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=nmax,
                             precision="bf16", overlap="fast", stats=stats, tc_layout=layout)
    _lib.reset_test_limits()
    assert_same_outputs(got, _as_tuple(exp))
    assert stats[0]["tc_layout"] == layout
    assert stats[0]["lik_exact_passes"] > 0
    assert stats[0]["fallback_candidates"] > 0


# ------------------------------------------------------------ the bound, entry by entry

BOUND_CASES = {
    "tetrode": (synthetic.tetrode, dict(duration_s=0.2, seed=307)),
    "linear16": (synthetic.linear16, dict(duration_s=0.1, seed=308)),
    "hd384": (synthetic.hd384, dict(duration_s=0.1, seed=309)),
}


def _likelihood_f64(v64, T, tss32, L):
    """float64 likelihood -0.5*SS + sum t*v for every template and every
    sample with s + L < n (over each template's non-zero channels)."""
    C, n = v64.shape
    K = T.shape[0]
    m = n - L
    out = np.zeros((K, n))
    win = np.lib.stride_tricks.sliding_window_view(v64, L, axis=1)[:, :m, :]    # [C][m][L]
    for k in range(K):
        t = T[k].reshape(C, L).astype(np.float64)
        nz = np.nonzero(np.any(t != 0, axis=1))[0]
        out[k, :m] = float(tss32[k]) + np.einsum("cwl,cl->w", win[nz], t[nz])
    return out


@pytest.mark.parametrize("layout", ["samples", "wide"])
@pytest.mark.parametrize("case", sorted(BOUND_CASES))
def test_tensor_core_bound_holds_for_every_entry(lib, case, layout):
    fn, kw = BOUND_CASES[case]
    rec = fn(**kw)
    C, n, K, L = rec.n_chans, rec.n_samples, rec.n_templates, rec.n_samples_per_chan
    m = rec.fresh_metrics()
    T = np.ascontiguousarray(np.float32(m["templates"]).reshape(K, -1))
    tss = np.ascontiguousarray(np.float32(-0.5 * m["template_SS"]))
    v32 = np.ascontiguousarray(rec.voltage.astype(np.float32))
    dev = torch.device("cuda", 0)
    v_d, T_d, tss_d = (torch.from_numpy(x).to(dev) for x in (v32, T.reshape(-1), tss))
    wsb = ctypes.c_size_t(0)
    _lib.check(lib.fbp_pursuit_workspace_bytes(n, C, K, L, 0, _lib.PREC_BF16_REFINE, ctypes.byref(wsb)))
    ws = torch.empty(wsb.value, dtype=torch.uint8, device=dev)
    approx_d = torch.zeros((K, n), dtype=torch.float32, device=dev)
    bound_d = torch.zeros((K, n), dtype=torch.float32, device=dev)
    sp = _lib.stream_ptr(torch.cuda.current_stream(dev))
    _lib.check(lib.fbp_set_tc_layout(_lib.TC_LAYOUT_WIDE if layout == "wide" else _lib.TC_LAYOUT_SAMPLES))
    try:
        _lib.check(lib.fbp_tc_likelihood_bounds(_lib.ptr(v_d), n, C, _lib.ptr(T_d), K, L, _lib.ptr(tss_d),
                                                _lib.ptr(ws), ws.numel(), _lib.ptr(approx_d), _lib.ptr(bound_d),
                                                sp))
    finally:
        _lib.check(lib.fbp_set_tc_layout(_lib.TC_LAYOUT_AUTO))
    torch.cuda.synchronize()
    approx, E = approx_d.cpu().numpy(), bound_d.cpu().numpy()
    # the reference's binary32 values (oracle) and float64 values
    W = (n + L - 1) // L
    ref32 = np.zeros((K, n), np.float32)
    O.stage_full_likelihood(v32, T.reshape(-1), K, L, tss, np.arange(W, dtype=np.uint32), ref32)
    ref64 = _likelihood_f64(v32.astype(np.float64), T, tss, L)
    live = np.zeros((K, n), bool)
    live[:, : n - L] = True                         # s + L < n (.cl:231-234)
    assert np.all(approx[~live] == 0) and np.all(E[~live] == 0)
    assert np.all(E[live] > 0)
    err32 = np.abs(approx.astype(np.float64) - ref32.astype(np.float64))
    assert np.all(err32[live] <= E[live].astype(np.float64)), (
        "bound violated at", np.argwhere(live & (err32 > E))[:5])
    err64 = np.abs(approx.astype(np.float64) - ref64)
    ref_err64 = np.abs(ref32.astype(np.float64) - ref64)
    scale = np.abs(ref64[live]).max()
    print("\nlikelihood error %s, %s layout (C=%d, K=%d, L=%d, %d samples, %d entries): tensor-core vs fp64 "
          "max %.3e (%.2e of max |L|), reference fp32 vs fp64 max %.3e, max |approx - fp32| / E = %.3f, "
          "median E %.3e"
          % (case, layout, C, K, L, n, int(live.sum()), err64[live].max(), err64[live].max() / scale,
             ref_err64[live].max(), float((err32[live] / E[live]).max()), float(np.median(E[live]))))


# ------------------------------------------------------------ bounded waits

@pytest.mark.parametrize("layout", ["samples", "wide"])
def test_bounded_wait_gives_up_and_context_stays_usable(lib, layout):
    rec = synthetic.tetrode(duration_s=0.2, seed=310, L=41)
    si = rec.sort_info()
    _lib.set_test_limits(wait_polls=0)
    with pytest.raises(_lib.PursuitError) as ei:
        bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=40,
                           precision="bf16", tc_layout=layout)
    assert ei.value.code == _lib.FBP_ERR_TIMEOUT
    _lib.reset_test_limits()
    torch.cuda.synchronize()
    exp = O.binary_pursuit_oracle(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=40)
    got = bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=40,
                             precision="bf16")
    assert_same_outputs(got, _as_tuple(exp))


# ------------------------------------------------------------ tuned group size

def test_tuned_plan_gives_the_same_spikes(lib, tmp_path, monkeypatch):
    """The tuner times the candidate plans (wide tiles, 128-sample tiles with
    each template group size) and caches the fastest per shape bucket; a
    pursuit that uses it (and one with every plan forced) returns the
    oracle's spikes."""
    from spikesorting_fullpursuit_b200 import autotune
    monkeypatch.setenv("FBP_TUNE_CACHE", str(tmp_path / "tune.json"))
    rec = linear16_slice(0.1, 311)
    si = rec.sort_info()
    exp = O.binary_pursuit_oracle(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=100)
    got = bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=100,
                             precision="bf16", tune=True)
    assert_same_outputs(got, _as_tuple(exp))
    table = autotune._load()
    assert len(table) == 1
    entry = next(iter(table.values()))
    plans = autotune.plans_for(rec.n_templates, rec.n_samples_per_chan)
    assert entry["plan"] in plans
    assert sorted(entry["ms"]) == sorted(plans)
    for plan in plans:
        autotune.apply(plan)
        try:
            st = []
            got = bpp.binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(), n_max_shift_inds=100,
                                     precision="bf16", stats=st)
        finally:
            autotune.apply(None)
        assert_same_outputs(got, _as_tuple(exp))
        assert st[0]["tc_layout"] == plan.split(":")[0]
