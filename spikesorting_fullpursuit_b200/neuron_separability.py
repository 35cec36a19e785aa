"""The pursuit's inputs from spikesorting_fullpursuit/neuron_separability.py
on the device: compute_separability_metrics (:88-152) and set_bp_threshold
(:251-261), same arguments and dictionary.  The per-template sums --
template_SS (numpy's float32 pairwise sum, bit for bit, plus the float64
sum), the likelihood variance and both bounds in float64 -- come from one
kernel (fbp_separability_metrics); the per-channel noise fractions, peak
channels and contamination are the reference's host arithmetic."""
import numpy as np

from . import _device as D
from . import _lib


def separability_sums(templates, channel_covariance_mats, sigma_bp_noise, sigma_bp_CI):
    """Device sums per template: dict of ss32 (float32), ss64, var, lower_ci,
    thr_raw and thr (float64), thr = max(thr_raw, 0, lower_ci)."""
    T = np.ascontiguousarray(np.vstack(templates), dtype=np.float32)
    K = T.shape[0]
    cov = np.ascontiguousarray(np.stack([np.asarray(c, dtype=np.float64) for c in channel_covariance_mats]))
    C, L = cov.shape[0], cov.shape[1]
    if T.shape[1] != C * L:
        raise ValueError("templates must have n_channels * n_samples_per_chan columns")
    T_d, cov_d = D.to_dev(T), D.to_dev(cov)
    ss32 = D.empty((K,), np.float32)
    outs = [D.empty((K,), np.float64) for _ in range(5)]
    _lib.check(_lib.lib().fbp_separability_metrics(_lib.ptr(T_d), K, C, L, _lib.ptr(cov_d), float(sigma_bp_noise),
                                                   float(sigma_bp_CI), _lib.ptr(ss32),
                                                   *[_lib.ptr(o) for o in outs], D.stream()))
    res = {"ss32": D.host(ss32)}
    for name, o in zip(("ss64", "var", "lower_ci", "thr_raw", "thr"), outs):
        res[name] = D.host(o)
    return res


def compute_separability_metrics(templates, channel_covariance_mats, sort_info):
    """neuron_separability.compute_separability_metrics (:88-152)."""
    from scipy.stats import norm
    n_chans = sort_info['n_channels']
    n_templates = len(templates)
    L = sort_info['n_samples_per_chan']
    sums = separability_sums(templates, channel_covariance_mats, sort_info['sigma_bp_noise'],
                             sort_info['sigma_bp_CI'])
    m = {}
    m['bp_n_samples_per_chan'] = L
    m['templates'] = np.vstack(templates)
    m['template_SS'] = sums["ss32"]
    m['template_SS_by_chan'] = np.zeros((n_templates, n_chans))
    m['channel_covariance_mats'] = channel_covariance_mats
    m['contamination'] = np.zeros(n_templates)
    m['peak_channel'] = np.zeros(n_templates, dtype=np.int64)
    m['channel_p_noise'] = np.zeros(n_chans)
    for chan in range(0, n_chans):
        m['channel_p_noise'][chan] = ((sort_info['n_samples'] - sort_info['n_threshold_crossings'][chan])
                                      / sort_info['n_samples'])
    m['neuron_variances'] = sums["var"]
    m['neuron_lower_thresholds'] = sums["thr_raw"].copy()
    m['neuron_lower_CI'] = sums["lower_ci"]
    for n in range(0, n_templates):
        expectation = 0.5 * m['template_SS'][n]
        m['peak_channel'][n] = np.argmax(np.abs(m['templates'][n, :])) // L
        m['contamination'][n] = norm.sf(m['neuron_lower_thresholds'][n], -expectation,
                                        np.sqrt(m['neuron_variances'][n]))
    return m


def set_bp_threshold(separability_metrics):
    """neuron_separability.set_bp_threshold (:251-261)."""
    for n in range(0, separability_metrics['neuron_lower_CI'].shape[0]):
        separability_metrics['neuron_lower_thresholds'][n] = max(
            separability_metrics['neuron_lower_thresholds'][n], 0)
        separability_metrics['neuron_lower_thresholds'][n] = max(
            separability_metrics['neuron_lower_thresholds'][n], separability_metrics['neuron_lower_CI'][n])
    return separability_metrics
