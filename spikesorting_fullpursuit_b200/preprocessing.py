"""Device versions of the numpy steps of spikesorting_fullpursuit/
preprocessing.py that feed the pursuit: calculate_robust_template
(:639-659, many units in one launch) and the ZCA whitening of
get_noise_sampled_zca_matrix (:104-169) with its application
(spikesorting_parallel.py:214).  Same arguments and return values as the
reference functions."""
import numpy as np

from . import _device as D
from . import _lib


def calculate_robust_templates(clips, unit_offsets, as_tensor=False):
    """calculate_robust_template for many units at once: `clips` [rows, dim]
    (float32 or int16, host array or CUDA tensor), the rows of unit u are
    unit_offsets[u]:unit_offsets[u+1].  Returns [n_units, dim] of the clips'
    dtype, each row what calculate_robust_template returns for that unit's
    clips."""
    c = D.to_dev(clips)
    dt = np.dtype(str(c.dtype).replace("torch.", ""))
    n_rows, dim = int(c.shape[0]), int(c.shape[1])
    off = np.ascontiguousarray(unit_offsets, dtype=np.uint32)
    n_units = len(off) - 1
    out = D.empty((n_units, dim), dt)
    lib = _lib.lib()
    sb = lib.fbp_robust_scratch_bytes(n_rows, dim, D.code_of(dt))
    scratch = D.empty((max(1, sb),), np.uint8)
    off_d = D.to_dev(off)
    _lib.check(lib.fbp_robust_templates(_lib.ptr(c), D.code_of(dt), n_rows, dim, _lib.ptr(off_d), n_units,
                                        _lib.ptr(out), _lib.ptr(scratch), sb, D.stream()))
    return out if as_tensor else D.host(out)


def calculate_robust_template(clips):
    """preprocessing.calculate_robust_template (:639-659): per sample, the
    median of the clips within one MAD (median absolute deviation / 0.6745)
    of the median (the median itself when none is); a single clip is
    returned squeezed, as the reference does."""
    clips = np.asarray(clips)
    if clips.shape[0] == 1 or clips.ndim == 1:
        return np.squeeze(clips)
    return calculate_robust_templates(clips, [0, clips.shape[0]])[0]


def _thresholds_f64(thresholds):
    return np.ascontiguousarray(np.asarray(thresholds, dtype=np.float64))


def zca_covariance(voltage_data, thresholds, thresh_cushion):
    """The covariance matrix get_noise_sampled_zca_matrix builds (:104-141)
    from every sample that no channel of a pair masks (the reference draws
    n_samples of them at random when more are available; here all are used,
    which is the reference's own choice whenever n_samples >= the valid
    samples).  Returns sigma [C, C] float64 on the host."""
    v = D.to_dev(voltage_data)
    dt = np.dtype(str(v.dtype).replace("torch.", ""))
    C, n = int(v.shape[0]), int(v.shape[1])
    lib = _lib.lib()
    thr = D.to_dev(_thresholds_f64(thresholds))
    mask = D.empty((C, n), np.uint8)
    sigma = D.empty((C, C), np.float64)
    sb = lib.fbp_zca_scratch_bytes(C)
    scratch = D.empty((sb,), np.uint8)
    _lib.check(lib.fbp_zca_covariance(_lib.ptr(v), D.code_of(dt), C, n, _lib.ptr(thr), int(thresh_cushion),
                                      _lib.ptr(mask), _lib.ptr(sigma), _lib.ptr(scratch), sb, D.stream()))
    return D.host(sigma)


def get_noise_sampled_zca_matrix(voltage_data, thresholds, sigma, thresh_cushion, n_samples=1e6):
    """preprocessing.get_noise_sampled_zca_matrix (:104-169): the covariance
    on the device (zca_covariance), then the reference's own
    U diag(1/sqrt(S + 1e-9)) U^T from the SVD of the C x C matrix on the
    host, rows scaled by the diagonal.  `sigma` (the threshold multiple) and
    n_samples are accepted as in the reference; every valid sample is used."""
    from scipy import linalg
    if np.ndim(voltage_data) == 1:
        return 1.
    cov = zca_covariance(voltage_data, thresholds, thresh_cushion)
    U, S, _ = linalg.svd(cov)
    zca_matrix = U @ np.diag(1.0 / np.sqrt(S + 1e-9)) @ U.T
    zca_matrix = zca_matrix / np.diag(zca_matrix)[:, None]
    return zca_matrix


def zca_apply(zca_matrix, voltage, as_tensor=False):
    """(zca_matrix @ voltage).astype(voltage.dtype) as
    spikesorting_parallel.py:214 computes it: float64 sums over channels,
    rounded to float32 or truncated to int16."""
    v = D.to_dev(voltage)
    dt = np.dtype(str(v.dtype).replace("torch.", ""))
    C, n = int(v.shape[0]), int(v.shape[1])
    Z = D.to_dev(np.ascontiguousarray(zca_matrix, dtype=np.float64))
    out = D.empty((C, n), dt)
    _lib.check(_lib.lib().fbp_zca_apply(_lib.ptr(Z), _lib.ptr(v), D.code_of(dt), C, n, _lib.ptr(out), D.stream()))
    return out if as_tensor else D.host(out)
