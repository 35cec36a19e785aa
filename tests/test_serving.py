"""Continuous batching: admission under the HBM budget (host logic, CPU) and
results that are the same alone and in the mix (GPU)."""
import threading
import time

import numpy as np
import pytest

from spikesorting_fullpursuit_b200.serving import AdmissionScheduler, latency_summary


class _Tracker:
    """Fake job runner: records the footprint held while jobs run."""

    def __init__(self, budget, hold_s=0.02):
        self.budget = budget
        self.hold_s = hold_s
        self.lock = threading.Lock()
        self.in_use = 0
        self.running = 0
        self.max_in_use = 0
        self.max_running = 0
        self.order = []
        self.solo_violations = 0

    def run(self, job, slot):
        name, fp, fail = job
        with self.lock:
            self.in_use += fp
            self.running += 1
            self.order.append(name)
            self.max_in_use = max(self.max_in_use, self.in_use)
            self.max_running = max(self.max_running, self.running)
            if fp > self.budget and self.running > 1:
                self.solo_violations += 1
        time.sleep(self.hold_s)
        with self.lock:
            self.in_use -= fp
            self.running -= 1
        if fail:
            raise ValueError("job %s failed" % name)
        return name


def test_admission_respects_budget_and_order():
    budget = 100
    tr = _Tracker(budget)
    rng = np.random.default_rng(0)
    fps = [int(x) for x in rng.integers(5, 60, size=40)]
    with AdmissionScheduler(slots=6, budget=budget, run=tr.run) as s:
        futs = [s.submit(("j%d" % i, fp, False), fp, units=fp) for i, fp in enumerate(fps)]
        res = [f.result(timeout=30) for f in futs]
    assert [r.outputs for r in res] == ["j%d" % i for i in range(len(fps))]
    assert tr.order == ["j%d" % i for i in range(len(fps))]          # FIFO starts
    assert tr.max_in_use <= budget
    assert s.max_in_use <= budget
    assert tr.max_running > 1                                        # jobs overlapped
    assert s.max_running <= 6
    for r in res:
        assert r.end_s >= r.start_s >= r.arrival_s
    summ = latency_summary(res, max(r.end_s for r in res) - min(r.arrival_s for r in res))
    assert summ["requests"] == len(fps)
    assert summ["p99_s"] >= summ["p50_s"] > 0
    assert summ["throughput"] > 0


def test_oversized_job_runs_alone():
    budget = 50
    tr = _Tracker(budget)
    fps = [10, 10, 80, 10, 10, 120, 10]
    with AdmissionScheduler(slots=4, budget=budget, run=tr.run) as s:
        futs = [s.submit(("j%d" % i, fp, False), fp) for i, fp in enumerate(fps)]
        assert [f.result(timeout=30).outputs for f in futs] == ["j%d" % i for i in range(len(fps))]
    assert tr.solo_violations == 0


def test_failed_job_reports_and_server_continues():
    tr = _Tracker(100, hold_s=0.005)
    with AdmissionScheduler(slots=2, budget=100, run=tr.run) as s:
        futs = [s.submit(("j%d" % i, 10, i == 3), 10) for i in range(8)]
        for i, f in enumerate(futs):
            if i == 3:
                with pytest.raises(ValueError, match="j3 failed"):
                    f.result(timeout=30)
            else:
                assert f.result(timeout=30).outputs == "j%d" % i
    with pytest.raises(RuntimeError, match="closed"):
        s.submit(("late", 1, False), 1)


def test_cancelled_queued_job_never_runs():
    gate = threading.Event()
    started = threading.Event()
    ran = []

    def run(job, slot):
        if job == "first":
            started.set()
            assert gate.wait(timeout=30)
        ran.append(job)
        return job

    with AdmissionScheduler(slots=1, budget=10, run=run) as s:
        f1 = s.submit("first", 1)
        f2 = s.submit("second", 1)
        f3 = s.submit("third", 1)
        assert started.wait(timeout=30)                # "first" is running, the others wait
        assert f2.cancel()
        assert not f1.cancel()                         # already running
        gate.set()
        assert f1.result(timeout=30).outputs == "first"
        assert f3.result(timeout=30).outputs == "third"
    assert f2.cancelled()
    assert ran == ["first", "third"]


def test_jobs_arriving_while_others_run_are_admitted():
    budget = 30
    tr = _Tracker(budget, hold_s=0.05)
    with AdmissionScheduler(slots=3, budget=budget, run=tr.run) as s:
        first = [s.submit(("a%d" % i, 10, False), 10) for i in range(3)]
        time.sleep(0.01)                                 # the first three hold the whole budget
        late = [s.submit(("b%d" % i, 10, False), 10) for i in range(3)]
        a = [f.result(timeout=30) for f in first]
        b = [f.result(timeout=30) for f in late]
    assert tr.max_in_use <= budget
    # each late job started only after an earlier one released its share
    assert min(r.start_s for r in b) >= min(r.end_s for r in a) - 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16", "fp32"])
def test_results_same_alone_and_in_the_mix(precision):
    torch = pytest.importorskip("torch")
    from spikesorting_fullpursuit_b200 import build as B, synthetic
    from spikesorting_fullpursuit_b200.parallel.binary_pursuit_parallel import binary_pursuit
    from spikesorting_fullpursuit_b200.serving import PursuitServer
    from tests._cases import assert_same_outputs

    B.build()
    recs = [
        (synthetic.tetrode(duration_s=0.5, seed=201, L=61), 60),
        (synthetic.linear16(duration_s=0.15, seed=202, n_templates=32, L=61), 60),
        (synthetic.hd384(duration_s=0.08, seed=203, n_chans=64, mask_chans=16, n_templates=24, L=61), 30),
        (synthetic.tetrode(duration_s=0.3, seed=204, L=31), 30),
        (synthetic.linear16(duration_s=0.1, seed=205, n_templates=16, L=101), 100),
        (synthetic.tetrode(duration_s=0.4, seed=206, L=41), 20),
    ]
    alone = []
    for rec, nmax in recs:
        si = rec.sort_info(do_overlap_recheck=True, get_adjusted_clips=True)
        alone.append(binary_pursuit(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(),
                                    n_max_shift_inds=nmax, precision=precision))
    with PursuitServer(slots=3, precision=precision) as srv:
        futs = []
        for rep in range(2):
            for rec, nmax in recs:
                si = rec.sort_info(do_overlap_recheck=True, get_adjusted_clips=True)
                futs.append(srv.submit(rec.voltage, si, rec.fresh_metrics(), nmax))
        mixed = [f.result(timeout=600) for f in futs]
        assert srv.max_running >= 2
    for i, r in enumerate(mixed):
        exp = tuple(np.asarray(x) for x in alone[i % len(recs)])
        assert_same_outputs(r.outputs, exp, isinstance(alone[i % len(recs)][0], list))
    torch.cuda.synchronize()


def test_request_footprint_counts_workspace_and_buffers():
    """The admission footprint is the library's workspace for the request's
    largest chunk plus its voltage, spike buffers and templates; it grows
    with the segment and the bf16 path's extra buffers are counted."""
    import ctypes
    from spikesorting_fullpursuit_b200 import _lib, synthetic
    from spikesorting_fullpursuit_b200.serving import request_footprint
    rec = synthetic.tetrode(duration_s=0.2, seed=1)
    si = rec.sort_info()
    C, n = rec.voltage.shape
    L = rec.n_samples_per_chan
    K = rec.templates.shape[0]
    ws = ctypes.c_size_t(0)
    _lib.check(_lib.lib().fbp_pursuit_workspace_bytes(n, C, K, L, 100, 0, ctypes.byref(ws)))
    W = (n + L - 1) // L
    fp32 = request_footprint(rec.voltage, si, rec.fresh_metrics(), 100, precision="fp32", total_mem=180e9)
    assert fp32 == ws.value + 4 * C * n + 8 * (8 * W + 4096) + 4 * K * C * L + 8 * K
    bf16 = request_footprint(rec.voltage, si, rec.fresh_metrics(), 100, precision="bf16", total_mem=180e9)
    assert bf16 > fp32
    # a chunk length caps what one request holds at a time
    capped = request_footprint(rec.voltage, si, rec.fresh_metrics(), 100, precision="fp32", chunk_samples=2000)
    assert capped < fp32
    longer = synthetic.tetrode(duration_s=0.4, seed=1)
    assert request_footprint(longer.voltage, longer.sort_info(), longer.fresh_metrics(), 100,
                             precision="fp32", total_mem=180e9) > fp32


def test_batch_and_serve_mixes_follow_the_stated_ranges():
    from spikesorting_fullpursuit_b200 import synthetic
    b = synthetic.batch_mix(256, seed=3, time_scale=1.0)
    assert len(b) == 256 and len({s.seed for s in b}) == 256
    assert all(4 <= s.n_chans <= 32 and 2 <= s.n_templates <= 40 and 61 <= s.L <= 101 for s in b)
    assert all(1.0 <= s.duration_s <= 60.0 and s.fs == 40000.0 for s in b)
    r = synthetic.serve_mix(500, seed=4, time_scale=1.0)
    assert all(4 <= s.n_chans <= 384 and 2.0 <= s.duration_s <= 120.0 for s in r)
    assert all((s.model == "tetrode") == (s.n_chans <= 32) for s in r)
    assert all(s.fs == (40000.0 if s.model == "tetrode" else 30000.0) for s in r)
    assert all(4 <= s.n_templates <= (40 if s.model == "tetrode" else 300) for s in r)
    small = synthetic.batch_mix(3, seed=3, time_scale=0.001)[0]
    rec = small.make()
    assert rec.voltage.shape == (small.n_chans, int(round(small.duration_s * small.fs)))
    assert rec.templates.shape == (small.n_templates, small.n_chans * small.L)
