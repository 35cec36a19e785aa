"""Chunk planning for binary_pursuit().

The reference splits a segment into chunks that fit the device
(binary_pursuit_parallel.py:276-344) and starts a new chunk every
`chunk - 3L` samples so consecutive chunks overlap by three template widths
(:359-368).  The same rules are kept here.  The bytes a chunk holds are this
implementation's own: the library's workspace for the chunk
(`fbp_pursuit_workspace_bytes`, which depends on the precision mode and the
overlap shift range), the voltage on the device, the spike outputs and, when
adjusted clips are requested, their buffer.  The chunk is the longest one
whose bytes fit the usable memory.
"""
import ctypes

# 32-bit sample indices on the device
MAX_CHUNK_SAMPLES = (1 << 32) - 1


def spike_capacity(n, L):
    """Initial spike buffer length binary_pursuit() allocates for a chunk."""
    W = (n + L - 1) // L
    return 8 * W + 4096


def workspace_bytes(n, n_chans, n_templates, L, n_max_shift, precision=0):
    """Device workspace of fbp_pursuit_chunk for a chunk of n samples (from
    the library; a host-side computation, no device needed)."""
    from .. import _lib
    out = ctypes.c_size_t(0)
    _lib.check(_lib.lib().fbp_pursuit_workspace_bytes(int(n), int(n_chans), int(n_templates), int(L),
                                                      int(n_max_shift), int(precision), ctypes.byref(out)))
    return int(out.value)


def chunk_footprint_bytes(n, n_chans, n_templates, L, n_max_shift, precision=0, v_itemsize=4,
                          adjusted_clips=False):
    """Device bytes binary_pursuit() holds while it pursues a chunk of n
    samples: the workspace, the float32 voltage (plus its upload in the
    caller's dtype while it is converted), the spike outputs, the templates
    and thresholds, and -- with adjusted clips -- a clip buffer sized for
    one spike per window."""
    C, K = int(n_chans), int(n_templates)
    W = (n + L - 1) // L
    total = workspace_bytes(n, C, K, L, n_max_shift, precision)
    total += 4 * C * n
    if v_itemsize != 4:
        total += int(v_itemsize) * C * n
    total += 2 * 4 * spike_capacity(n, L)
    total += 4 * K * C * L + 8 * K
    if adjusted_clips:
        total += 4 * W * C * L
    return total


def device_bytes_per_sample(n_chans, n_templates, L, n_max_shift=None, precision=0, n=1 << 22):
    """Average device bytes per sample of a chunk of n samples."""
    if n_max_shift is None:
        n_max_shift = L // 2
    return chunk_footprint_bytes(n, n_chans, n_templates, L, n_max_shift, precision) / float(n)


def usable_bytes(gpu_total_bytes, max_gpu_memory=None):
    """Memory a chunk may use: half the device or all but 1 GiB, whichever is
    more, capped by max_gpu_memory (binary_pursuit_parallel.py:276-291)."""
    usable = max(gpu_total_bytes * 0.5, gpu_total_bytes - (1024 * 1024 * 1024))
    if max_gpu_memory is not None:
        usable = min(usable, max_gpu_memory)
    assert usable > 0
    return usable


def num_indices_per_chunk(n_chans, n_templates, L, sampling_rate, gpu_total_bytes,
                          max_gpu_memory=None, *, n_max_shift=None, precision=0, v_itemsize=4,
                          adjusted_clips=False):
    """Samples per chunk: the longest chunk whose device bytes
    (chunk_footprint_bytes) fit the usable memory (reference :276-341, with
    this implementation's footprint).  Raises ValueError like the reference
    when fewer than 4L samples fit (:343-344)."""
    del sampling_rate                      # the reference converts to seconds and back; samples suffice
    usable = usable_bytes(gpu_total_bytes, max_gpu_memory)
    if n_max_shift is None:
        n_max_shift = L // 2

    def fits(n):
        return chunk_footprint_bytes(n, n_chans, n_templates, L, n_max_shift, precision, v_itemsize,
                                     adjusted_clips) <= usable

    lo = 4 * L
    if not fits(lo):
        raise ValueError("Cannot fit enough data on GPU to run binary pursuit. "
                         "Decrease template samples or get a new GPU.")
    hi = MAX_CHUNK_SAMPLES
    if fits(hi):
        return hi
    # the footprint grows with n: largest n that fits
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if fits(mid):
            lo = mid
        else:
            hi = mid
    return lo


def chunk_onsets(n_samples, L, chunk_samples):
    """Chunk start indices, binary_pursuit_parallel.py:363-367."""
    onsets = []
    cur = 0
    while cur < n_samples - L:
        onsets.append(cur)
        cur += chunk_samples - 3 * L
    return onsets


def plan_chunks(n_samples, n_chans, n_templates, L, gpu_total_bytes, max_gpu_memory=None, **kw):
    """(chunk_samples, onsets) for a segment of n_samples."""
    cs = num_indices_per_chunk(n_chans, n_templates, L, None, gpu_total_bytes, max_gpu_memory, **kw)
    return cs, chunk_onsets(n_samples, L, cs)


__all__ = ["chunk_footprint_bytes", "chunk_onsets", "device_bytes_per_sample", "num_indices_per_chunk",
           "plan_chunks", "spike_capacity", "usable_bytes", "workspace_bytes"]
