"""The Wiener filter of spikesorting_fullpursuit/wiener_filter.py on the
device: wiener (:24-72, one filter per channel) and wiener_all (:75-121, one
filter for all channels), same arguments and result.  The FFTs are cuFFT's
(torch.fft, float64 as numpy's pocketfft); the power spectra, the box-car
smoothing with the reference's running sums and the filter are this
library's kernels (fbp_power_spectrum, fbp_wiener_smooth, fbp_wiener_apply).
Precision follows numpy's: float32 voltage is transformed and filtered in
single precision (complex64 spectra, float32 result), other dtypes in
double."""
import numpy as np

from . import _device as D
from . import _lib


def wiener_optimal_filter(signal_power, noise_power, epsilon=1e-9):
    """wiener_filter.wiener_optimal_filter (:124-129)."""
    return (signal_power) / (signal_power + noise_power + epsilon)


def _real_dtype(a):
    """numpy's FFT precision for the voltage dtype."""
    return np.float32 if np.asarray(a).dtype == np.float32 else np.float64


def _filter_rows(torch, ov, sv, nv, smooth, rdt):
    """ov, sv, nv: CUDA tensors [rows, n] of the real dtype rdt; returns the
    filtered rows in rdt."""
    lib = _lib.lib()
    code = D.code_of(rdt)
    n = int(ov.shape[1])
    rows = int(ov.shape[0])
    st = D.stream()
    spec = torch.fft.rfft(ov, dim=1).contiguous()
    nb = int(spec.shape[1])
    S = D.empty((rows, nb), rdt)
    N = D.empty((rows, nb), rdt)
    tmp = torch.fft.rfft(sv, dim=1).contiguous()
    _lib.check(lib.fbp_power_spectrum(_lib.ptr(torch.view_as_real(tmp)), code, rows, nb, _lib.ptr(S), st))
    tmp = torch.fft.rfft(nv, dim=1).contiguous()
    _lib.check(lib.fbp_power_spectrum(_lib.ptr(torch.view_as_real(tmp)), code, rows, nb, _lib.ptr(N), st))
    del tmp
    smooth = int(smooth)
    if smooth > 1:
        scratch = D.empty((rows, nb), rdt)
        _lib.check(lib.fbp_wiener_smooth(_lib.ptr(S), code, rows, nb, smooth, _lib.ptr(scratch), st))
        _lib.check(lib.fbp_wiener_smooth(_lib.ptr(N), code, rows, nb, smooth, _lib.ptr(scratch), st))
    _lib.check(lib.fbp_wiener_apply(_lib.ptr(torch.view_as_real(spec)), _lib.ptr(S), _lib.ptr(N), code, rows, nb,
                                    st))
    return torch.fft.irfft(spec, n=n, dim=1)


def wiener(original_voltage, signal_voltage, noise_voltage, smooth=1):
    """wiener_filter.wiener (:24-72): per channel, the input's spectrum times
    S / (S + N + 1e-9) of the (optionally box-car smoothed) signal and noise
    power spectra; returns [channels, samples] on the host (float32 for
    float32 voltage, else float64)."""
    torch = D.torch_cuda()
    ov, sv, nv = (np.asarray(x) for x in (original_voltage, signal_voltage, noise_voltage))
    if ov.ndim == 1:
        ov, sv, nv = ov[None, :], sv[None, :], nv[None, :]
    assert (sv.shape == ov.shape) and (nv.shape == ov.shape)
    rdt = _real_dtype(ov)
    t = [D.to_dev(np.ascontiguousarray(x, dtype=rdt)) for x in (ov, sv, nv)]
    return D.host(_filter_rows(torch, *t, smooth, rdt))


def wiener_all(original_voltage, signal_voltage, noise_voltage, smooth=1):
    """wiener_filter.wiener_all (:75-121): one filter from all channels'
    samples taken as a single row (C order)."""
    torch = D.torch_cuda()
    ov, sv, nv = (np.asarray(x) for x in (original_voltage, signal_voltage, noise_voltage))
    assert (sv.shape == ov.shape) and (nv.shape == ov.shape)
    rdt = _real_dtype(ov)
    t = [D.to_dev(np.ascontiguousarray(x, dtype=rdt).reshape(1, -1)) for x in (ov, sv, nv)]
    return D.host(_filter_rows(torch, *t, smooth, rdt)).reshape(ov.shape)
