"""Host-side logic of the drop-in binary_pursuit() (no GPU needed)."""
import numpy as np
import pytest

from spikesorting_fullpursuit_b200.parallel import binary_pursuit_parallel as bpp
from spikesorting_fullpursuit_b200.parallel import chunking
from oracle import reference_harness as R


@pytest.mark.parametrize("tw,fs", [([-0.001, 0.0015], 40000.0), ([0.0008, 0.0012], 30000.0),
                                   ([-1e-6, 1e-6], 40000.0), ([-0.00033, 0.00047], 30000.0)])
def test_time_window_to_samples(tw, fs):
    got = bpp.time_window_to_samples(tw, fs)
    if R.available():
        R._import()
        from spikesorting_fullpursuit.parallel import segment_parallel
        assert got == segment_parallel.time_window_to_samples(list(tw), fs)
    assert got[0][1] - got[0][0] >= 2


def test_chunk_onsets_match_reference_rule():
    # binary_pursuit_parallel.py:363-367
    assert chunking.chunk_onsets(1000, 31, 500) == [0, 407, 814]
    assert chunking.chunk_onsets(31, 31, 500) == []
    assert chunking.chunk_onsets(32, 31, 500) == [0]


def test_chunk_too_small_raises_value_error():
    with pytest.raises(ValueError, match="Cannot fit enough data on GPU"):
        chunking.num_indices_per_chunk(384, 300, 61, 30000.0, 8 * 1024 ** 3, max_gpu_memory=1e5)


B200_BYTES = 183_359 * 1024 ** 2          # total memory a B200 reports


# (channels, templates, L, n_max_shift, voltage itemsize, samples of the segment)
PLAN_CASES = {
    "tetrode_30s": (4, 8, 101, 100, 4, 1_200_000),
    "linear16_10min": (16, 64, 101, 100, 4, 24_000_000),
    "hd384_5min": (384, 300, 61, 60, 2, 9_000_000),
    "hd384_60min": (384, 300, 61, 60, 2, 108_000_000),
}


@pytest.mark.parametrize("precision", [0, 1], ids=["fp32", "bf16"])
@pytest.mark.parametrize("case", sorted(PLAN_CASES))
def test_planned_chunk_fits_usable_memory(case, precision):
    """The planner sizes chunks with the library's own workspace: the chunk it
    picks, with its workspace, voltage and spike buffers, fits the usable
    memory, and one sample more would not."""
    C, K, L, nmax, isz, n_seg = PLAN_CASES[case]
    usable = chunking.usable_bytes(B200_BYTES)
    n = chunking.num_indices_per_chunk(C, K, L, 30000.0, B200_BYTES, n_max_shift=nmax, precision=precision,
                                       v_itemsize=isz)
    need = chunking.chunk_footprint_bytes(n, C, K, L, nmax, precision, isz)
    assert need <= usable
    if n < chunking.MAX_CHUNK_SAMPLES:
        assert chunking.chunk_footprint_bytes(n + 1, C, K, L, nmax, precision, isz) > usable
    # the footprint counts the library's workspace, which is most of it
    assert need > chunking.workspace_bytes(n, C, K, L, nmax, precision) > 4 * C * n
    # the chunk of a segment is at most the segment; every chunk of it fits
    cs, onsets = chunking.plan_chunks(n_seg, C, K, L, B200_BYTES, n_max_shift=nmax, precision=precision,
                                      v_itemsize=isz)
    for o in onsets:
        m = min(n_seg, o + cs) - o
        assert chunking.chunk_footprint_bytes(m, C, K, L, nmax, precision, isz) <= usable


def test_ten_minute_linear16_segment_is_one_chunk():
    n = chunking.num_indices_per_chunk(16, 64, 101, 40000.0, B200_BYTES, n_max_shift=100, precision=1)
    assert n >= 24_000_000


def test_max_gpu_memory_caps_the_chunk():
    big = chunking.num_indices_per_chunk(16, 64, 101, 40000.0, B200_BYTES, n_max_shift=100)
    capped = chunking.num_indices_per_chunk(16, 64, 101, 40000.0, B200_BYTES, max_gpu_memory=2 * 1024 ** 3,
                                            n_max_shift=100)
    assert capped < big
    assert chunking.chunk_footprint_bytes(capped, 16, 64, 101, 100) <= 2 * 1024 ** 3


def test_add_n_spikes_semantics():
    m = {"templates": np.zeros((3, 10))}
    bpp.add_n_spikes(m, np.array([0, 2, 2]))
    assert m["n_spikes"].tolist() == [1.0, 0.0, 2.0]
    m = {"templates": np.zeros(10)}          # 1-D templates: sized by shape[0]
    bpp.add_n_spikes(m, [])
    assert m["n_spikes"].shape == (10,)


def test_no_gpu_raises_runtime_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="No GPU available"):
        bpp.binary_pursuit(np.zeros((2, 100), np.float32), np.float32,
                           {"sampling_rate": 1000.0, "clip_width": [-0.002, 0.002],
                            "n_samples_per_chan": 5, "do_overlap_recheck": True,
                            "get_adjusted_clips": False},
                           {"templates": np.zeros((1, 10)), "template_SS": np.zeros(1),
                            "neuron_lower_thresholds": np.zeros(1)})


def test_tuner_bucket_and_cache(tmp_path, monkeypatch):
    """The tuner's shape bucket and its JSON cache (no GPU: a cached bucket
    is answered without timing)."""
    from spikesorting_fullpursuit_b200 import autotune, synthetic
    monkeypatch.setenv("FBP_TUNE_CACHE", str(tmp_path / "t.json"))
    rec = synthetic.hd384(duration_s=0.01, seed=2)
    T = rec.fresh_metrics()["templates"]
    b = autotune.shape_bucket(rec.n_chans, T, rec.n_samples_per_chan)
    assert b == "C384_K304_L64_w16"
    assert autotune.candidates_for(300) == autotune.CANDIDATES
    assert autotune.candidates_for(20) == (16, 32)
    assert autotune.plans_for(20, 61) == ("wide", "samples:16", "samples:32")
    assert autotune.plans_for(20, 8) == ("samples:16", "samples:32")
    autotune._store({b: {"plan": "samples:32", "ms": {"wide": 2.0, "samples:32": 1.0}}})
    plan, bucket, times = autotune.tune(rec.voltage, T, -0.5 * rec.fresh_metrics()["template_SS"],
                                        rec.n_samples_per_chan)
    assert (plan, bucket, times) == ("samples:32", b, None)
