"""Device plumbing shared by the modules that mirror the reference's
numpy steps: host arrays in, device buffers (owned by PyTorch) for the C ABI
of include/fbp_prepost.h, host arrays out.  No CPU fallback: without a CUDA
device these raise RuntimeError("No GPU available"), as binary_pursuit() does."""
import numpy as np

from . import _lib

_DT = {np.dtype(np.float32): _lib.F32, np.dtype(np.int16): _lib.I16, np.dtype(np.float64): _lib.F64}


def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("No GPU available")
    return torch


def code_of(dtype):
    dt = np.dtype(dtype)
    if dt not in _DT:
        raise TypeError("unsupported dtype %s (float32 and int16 voltages, float64 templates)" % dt)
    return _DT[dt]


def device():
    torch = torch_cuda()
    return torch.device("cuda", torch.cuda.current_device())


def to_dev(a, dtype=None):
    """Host array (or CUDA tensor) -> contiguous CUDA tensor."""
    torch = torch_cuda()
    if isinstance(a, torch.Tensor):
        t = a if a.is_cuda else a.to(device())
        return t.contiguous()
    arr = np.ascontiguousarray(a if dtype is None else np.asarray(a, dtype=dtype))
    if arr.dtype == np.uint32:
        arr = arr.view(np.int32)
    return torch.from_numpy(arr).to(device())


def empty(shape, dtype):
    torch = torch_cuda()
    tdt = {np.dtype(np.float32): torch.float32, np.dtype(np.int16): torch.int16,
           np.dtype(np.float64): torch.float64, np.dtype(np.uint8): torch.uint8,
           np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64}[np.dtype(dtype)]
    return torch.empty(shape, dtype=tdt, device=device())


def stream():
    torch = torch_cuda()
    return _lib.stream_ptr(torch.cuda.current_stream())


def host(t):
    return t.cpu().numpy()
