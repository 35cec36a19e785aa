"""The oracle (oracle/bp_oracle.c + oracle/oracle.py) pinned to the reference.

1. Against the golden vectors in tests/golden/, which the reference's own
   host code and kernels produced (tests/golden/make_golden.py).
2. Where the reference tree is present, live against the reference on fresh
   seeded inputs.
"""
import numpy as np
import pytest

from tests._cases import GoldenCase, assert_same_outputs, golden_paths
from oracle import oracle as O
from oracle import reference_harness as R
from spikesorting_fullpursuit_b200 import synthetic


@pytest.mark.parametrize("path", golden_paths(), ids=lambda p: p.split("/")[-1][:-4])
def test_oracle_reproduces_golden(path):
    c = GoldenCase(path)
    m = c.metrics()
    out = O.binary_pursuit_oracle(c.voltage, c.voltage.dtype, c.sort_info, m,
                                  n_max_shift_inds=c.n_max_shift_inds,
                                  chunk_samples=c.chunk_samples, nthreads=4)
    assert_same_outputs(out, c.expected, c.empty)
    assert np.array_equal(m["n_spikes"], c.n_spikes)


LIVE = [
    dict(kind="tetrode", seed=21, L=31, dur=0.25, nmax=30, overlap=True),
    dict(kind="tetrode", seed=22, L=61, dur=0.25, nmax=20, overlap=True),
    dict(kind="linear16", seed=23, L=31, dur=0.08, nmax=30, overlap=True, K=16),
    dict(kind="hd384", seed=24, L=21, dur=0.1, nmax=10, overlap=True, K=12, C=48, mask=8),
    dict(kind="tetrode", seed=25, L=41, dur=0.25, nmax=40, overlap=False),
    # the 384-channel workload's template structure: 16-channel masks, L = 61, 30 kHz, int16
    dict(kind="hd384", seed=26, L=61, dur=0.05, nmax=10, overlap=True, K=24, C=64, mask=16),
]


@pytest.mark.skipif(not R.available(), reason="reference tree not present")
@pytest.mark.parametrize("cfg", LIVE, ids=lambda c: "%s-%d" % (c["kind"], c["seed"]))
def test_oracle_matches_reference_live(cfg):
    kw = dict(duration_s=cfg["dur"], seed=cfg["seed"], L=cfg["L"])
    if "K" in cfg:
        kw["n_templates"] = cfg["K"]
    if "C" in cfg:
        kw["n_chans"] = cfg["C"]
        kw["mask_chans"] = cfg["mask"]
    rec = getattr(synthetic, cfg["kind"])(**kw)
    si = rec.sort_info(do_overlap_recheck=cfg["overlap"], get_adjusted_clips=True)
    ref, _ = R.run_reference(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(),
                             n_max_shift_inds=cfg["nmax"])
    got = O.binary_pursuit_oracle(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(),
                                  n_max_shift_inds=cfg["nmax"], nthreads=4)
    assert_same_outputs(got, tuple(np.asarray(x) for x in ref), isinstance(ref[0], list))


@pytest.mark.skipif(not R.available(), reason="reference tree not present")
def test_reference_chunk_formula_matches_reference_log():
    """reference_chunk_samples restates binary_pursuit_parallel.py:276-341."""
    rec = synthetic.tetrode(duration_s=0.5, seed=3, L=31)
    si = rec.sort_info()
    (_, _, _, _), log = R.run_reference(rec.voltage, rec.voltage.dtype, si, rec.fresh_metrics(),
                                        n_max_shift_inds=10, max_gpu_memory=2.0e6)
    cs = R.reference_chunk_samples(rec.n_chans, rec.n_templates, 31, rec.sampling_rate, 10,
                                   16 * 1024 ** 3, 2.0e6)
    starts = [l for l in log.splitlines() if l.startswith("Starting chunk")]
    assert "from 0 to %d samples" % cs in starts[0]
