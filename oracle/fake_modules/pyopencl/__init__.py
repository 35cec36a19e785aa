"""Minimal stand-in for pyopencl (TEST INFRASTRUCTURE ONLY).

It implements exactly the surface that the reference's host driver
spikesorting_fullpursuit/parallel/binary_pursuit_parallel.py:128-845 touches,
so that the reference's own `binary_pursuit()` runs unchanged on this CPU.
Kernels dispatch to the reference's binary_pursuit.cl compiled as C
(oracle/_ref/libbp_ref.so).  Every kernel reports a WORK_GROUP_SIZE of 1.
Work-items run one after another in global-id order, except those of the
kernels whose work-items write disjoint outputs (compute_full_likelihood,
overlap_recheck_indices, get_adjusted_clips), which run on THREADS host threads
(default: all; FBP_REF_THREADS overrides) with private local memory.  Buffers
are host numpy arrays, padded by 64 bytes for the reference's known
out-of-range reads.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.environ.get(
    "FBP_REF_LIB", os.path.join(_HERE, "..", "..", "_ref", "libbp_ref.so"))
_lib = None

# Configurable device description (tests set these before calling).
GLOBAL_MEM_SIZE_BYTES = 16 * 1024 ** 3
ADDRESS_BITS_VALUE = 64
MAX_COMPUTE_UNITS = 8

# Host threads for the kernels whose work-items are independent.
THREADS = int(os.environ.get("FBP_REF_THREADS", "0")) or (os.cpu_count() or 1)

# Counters the tests read back (number of kernel launches by name).
launch_counts = {}

_KERNEL_IDS = {
    "compute_residual": 0,
    "compute_full_likelihood": 1,
    "compute_template_maximum_likelihood": 2,
    "overlap_recheck_indices": 3,
    "parse_overlap_recheck_indices": 4,
    "check_overlap_reassignments": 5,
    "binary_pursuit": 6,
    "get_adjusted_clips": 7,
}
_NARGS = [9, 10, 14, 17, 15, 10, 15, 10]


def _load():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(os.path.abspath(_LIB_PATH))
        _lib.bpref_launch.restype = ctypes.c_int
        _lib.bpref_launch.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64,
                                      ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]
        _lib.bpref_launch_mt.restype = ctypes.c_int
        _lib.bpref_launch_mt.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                         ctypes.POINTER(ctypes.c_uint64), ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]
    return _lib


class device_type:
    GPU = 4
    CPU = 2


class device_info:
    GLOBAL_MEM_SIZE = "GLOBAL_MEM_SIZE"
    ADDRESS_BITS = "ADDRESS_BITS"
    MAX_WORK_GROUP_SIZE = "MAX_WORK_GROUP_SIZE"


class kernel_work_group_info:
    WORK_GROUP_SIZE = "WORK_GROUP_SIZE"


class mem_flags:
    READ_ONLY = 1
    WRITE_ONLY = 2
    READ_WRITE = 4
    COPY_HOST_PTR = 8


class _Device:
    name = "fbp-oracle-cpu"

    @property
    def max_compute_units(self):
        return MAX_COMPUTE_UNITS

    def get_info(self, key):
        if key == device_info.GLOBAL_MEM_SIZE:
            return GLOBAL_MEM_SIZE_BYTES
        if key == device_info.ADDRESS_BITS:
            return ADDRESS_BITS_VALUE
        if key == device_info.MAX_WORK_GROUP_SIZE:
            return 1
        raise KeyError(key)


class _Platform:
    def get_devices(self, dtype=None):
        return [_Device()]


def get_platforms():
    return [_Platform()]


class Context:
    def __init__(self, devices):
        self.devices = devices


class CommandQueue:
    def __init__(self, ctx):
        self.ctx = ctx

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def finish(self):
        return None


class Buffer:
    _PAD = 64

    def __init__(self, ctx, flags, size=None, hostbuf=None):
        if hostbuf is not None:
            src = np.ascontiguousarray(hostbuf)
            nbytes = src.nbytes
        else:
            src = None
            nbytes = int(size)
        self._raw = np.zeros(nbytes + self._PAD, dtype=np.uint8)
        if src is not None and nbytes:
            self._raw[:nbytes] = src.view(np.uint8).reshape(-1)
        self.nbytes = nbytes

    @property
    def address(self):
        return self._raw.ctypes.data

    def release(self):
        self._raw = None


class LocalMemory:
    def __init__(self, nbytes):
        self.nbytes = int(nbytes)
        self._raw = np.zeros(int(nbytes) + 64, dtype=np.uint8)

    @property
    def address(self):
        return self._raw.ctypes.data


class _Event:
    pass


class Kernel:
    def __init__(self, name):
        self.name = name
        self.kid = _KERNEL_IDS[name]
        self.args = [None] * _NARGS[self.kid]

    def set_arg(self, i, value):
        self.args[i] = value

    def get_work_group_info(self, key, device):
        return 1

    def _local_sizes(self):
        words = (ctypes.c_uint64 * len(self.args))()
        for i, a in enumerate(self.args):
            words[i] = a.nbytes if isinstance(a, LocalMemory) else 0
        return words

    def _pack(self):
        words = (ctypes.c_uint64 * len(self.args))()
        for i, a in enumerate(self.args):
            if isinstance(a, (Buffer, LocalMemory)):
                words[i] = a.address
            elif a is None:
                words[i] = 0
            else:
                words[i] = int(a) & 0xFFFFFFFFFFFFFFFF
        return words


class Program:
    def __init__(self, ctx, src):
        self.src = src

    def build(self, *args, **kwargs):
        return self

    def __getattr__(self, name):
        if name in _KERNEL_IDS:
            k = Kernel(name)
            self.__dict__[name] = k
            return k
        raise AttributeError(name)


def enqueue_nd_range_kernel(queue, kernel, global_size, local_size, global_work_offset=None,
                            wait_for=None):
    off = 0 if global_work_offset is None else int(global_work_offset[0])
    gsz = int(global_size[0])
    lsz = int(local_size[0]) if local_size is not None else 1
    rc = _load().bpref_launch_mt(kernel.kid, off, gsz, lsz, kernel._pack(), len(kernel.args),
                                 kernel._local_sizes(), THREADS)
    if rc != 0:
        raise RuntimeError("fake pyopencl launch failed: %d" % rc)
    launch_counts[kernel.name] = launch_counts.get(kernel.name, 0) + 1
    return _Event()


def enqueue_copy(queue, dest, src, wait_for=None, is_blocking=True):
    if isinstance(dest, Buffer) and isinstance(src, np.ndarray):
        s = np.ascontiguousarray(src).view(np.uint8).reshape(-1)
        dest._raw[:s.size] = s
    elif isinstance(src, Buffer) and isinstance(dest, np.ndarray):
        d = dest.view(np.uint8).reshape(-1)
        d[:] = src._raw[:d.size]
    else:
        raise TypeError("unsupported enqueue_copy")
    return _Event()
