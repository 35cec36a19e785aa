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


def test_chunk_fits_memory():
    n = chunking.num_indices_per_chunk(16, 64, 101, 40000.0, 180 * 1024 ** 3)
    assert n * chunking.device_bytes_per_sample(16, 64, 101) < 180 * 1024 ** 3
    assert n >= 24_000_000            # a 10-minute 16-channel segment is one chunk


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
