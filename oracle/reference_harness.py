"""Run the reference's own host code on the CPU (TEST INFRASTRUCTURE ONLY).

Imports spikesorting_fullpursuit.parallel.binary_pursuit_parallel from the
staged, unmodified reference package (baseline/_ref, made by
oracle/install_reference.sh) with the stand-in pyopencl of
oracle/fake_modules, whose kernels are the reference's binary_pursuit.cl
compiled as C (oracle/_ref/libbp_ref.so, `make -C oracle ref`).  Available
where the staged package and the compiled kernels exist (both are built in a
container that has the reference tree, and travel with the repository).
"""
import contextlib
import io
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF_STAGED = os.path.join(REPO, "baseline", "_ref")
REF_LIB = os.path.join(HERE, "_ref", "libbp_ref.so")


def reference_tree():
    """Root of the reference checkout: $FBP_REFERENCE_TREE, else a checkout
    named `reference` beside this repository."""
    return os.environ.get("FBP_REFERENCE_TREE") or os.path.normpath(os.path.join(REPO, "..", "reference"))


REF_TREE = reference_tree()
# the kernel source as the reference's host code opens it: from the staged
# package (it travels with the repository), else from the reference tree
_CL_STAGED = os.path.join(REF_STAGED, "spikesorting_fullpursuit", "kernels", "binary_pursuit.cl")
CL_PATH = _CL_STAGED if os.path.exists(_CL_STAGED) else os.path.join(
    REF_TREE, "spikesorting_fullpursuit", "kernels", "binary_pursuit.cl")


def available():
    return (os.path.isdir(os.path.join(REF_STAGED, "spikesorting_fullpursuit"))
            and os.path.exists(REF_LIB) and os.path.exists(CL_PATH))


def _import():
    fake = os.path.join(HERE, "fake_modules")
    for p in (fake, REF_STAGED):
        if p not in sys.path:
            sys.path.insert(0, p)
    import pyopencl  # the stand-in
    assert os.path.abspath(pyopencl.__file__).startswith(fake), pyopencl.__file__
    from spikesorting_fullpursuit.parallel import binary_pursuit_parallel as bpp
    return pyopencl, bpp


def run_reference(voltage, v_dtype, sort_info, separability_metrics, n_max_shift_inds=None,
                  max_gpu_memory=None, global_mem_bytes=16 * 1024 ** 3, quiet=True):
    """Call the reference binary_pursuit() unchanged.  Returns (outputs, log)."""
    cl, bpp = _import()
    cl.GLOBAL_MEM_SIZE_BYTES = int(global_mem_bytes)
    cl.launch_counts.clear()
    buf = io.StringIO()
    ctx = contextlib.redirect_stdout(buf) if quiet else contextlib.nullcontext()
    with ctx:
        out = bpp.binary_pursuit(voltage, v_dtype, sort_info, separability_metrics,
                                 n_max_shift_inds=n_max_shift_inds, kernels_path=CL_PATH,
                                 max_gpu_memory=max_gpu_memory)
    return out, buf.getvalue()


def reference_chunk_samples(n_chans, n_templates, L, sampling_rate, n_max_shift_inds,
                            global_mem_bytes, max_gpu_memory=None, overlap_lws=1):
    """num_indices_per_chunk as binary_pursuit_parallel.py:276-341 computes it
    for the stand-in device (work-group size 1, 64 address bits)."""
    import numpy as np
    gpu = max(global_mem_bytes * 0.5, global_mem_bytes - (1024 ** 3))
    if max_gpu_memory is not None:
        gpu = min(gpu, max_gpu_memory)
    if n_max_shift_inds is None or n_max_shift_inds < 0:
        n_max_shift_inds = L // 2
    nm = np.uint32(n_max_shift_inds)
    items = np.int64((2 * nm + 1) * (2 * nm + 1) * n_templates)
    n_local_ID = np.int64(((items - 1) / overlap_lws) + 1)
    const = n_templates * n_chans * L * 4 + n_templates * 4
    per_s = n_chans * sampling_rate * 4
    per_s += n_templates * sampling_rate * 4
    per_s += (sampling_rate / L) * (4 * 5 + (n_local_ID / 3) * 4 + (n_local_ID / 3) * 4)
    secs = (gpu - const) / per_s
    max_addr = (((1 << 64) - 1) / (4 * sampling_rate * n_chans))
    secs = min(secs, np.floor(max_addr))
    return int(np.floor(secs * sampling_rate))
