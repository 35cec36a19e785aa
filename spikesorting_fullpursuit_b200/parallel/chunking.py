"""Chunk planning for binary_pursuit().

The reference splits a segment into chunks that fit the device
(binary_pursuit_parallel.py:276-344) and starts a new chunk every
`chunk - 3L` samples so consecutive chunks overlap by three template widths
(:359-368).  The same rules are kept here; the per-sample footprint is this
implementation's own (voltage, likelihood, per-window state), since it does
not allocate the reference's per-work-group overlap buffers.
"""
import numpy as np


def device_bytes_per_sample(n_chans, n_templates, L):
    per = 4 * n_chans + 4 * n_templates          # voltage + likelihood
    per += (4 * 12 + 8) / float(L)               # per-window state
    return per


def num_indices_per_chunk(n_chans, n_templates, L, sampling_rate, gpu_total_bytes,
                          max_gpu_memory=None):
    """Samples per chunk (reference :276-341 with this implementation's
    footprint).  Raises ValueError like the reference (:343-344)."""
    usable = max(gpu_total_bytes * 0.5, gpu_total_bytes - (1024 * 1024 * 1024))
    if max_gpu_memory is not None:
        usable = min(usable, max_gpu_memory)
    assert usable > 0
    const = n_templates * n_chans * L * 4 + n_templates * 8 + (1 << 20)
    per_sample = device_bytes_per_sample(n_chans, n_templates, L)
    n = int(np.floor((usable - const) / per_sample))
    # 32-bit sample indices on the device
    n = min(n, (1 << 32) - 1)
    if n < 4 * L:
        raise ValueError("Cannot fit enough data on GPU to run binary pursuit. "
                         "Decrease template samples or get a new GPU.")
    return n


def chunk_onsets(n_samples, L, chunk_samples):
    """Chunk start indices, binary_pursuit_parallel.py:363-367."""
    onsets = []
    cur = 0
    while cur < n_samples - L:
        onsets.append(cur)
        cur += chunk_samples - 3 * L
    return onsets
