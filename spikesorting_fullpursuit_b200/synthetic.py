"""Seeded synthetic recordings for Full Binary Pursuit.

The reference has no public dataset for this path; its own test generator
(spikesorting_fullpursuit/test/gen_dataset.py) builds band-limited Gaussian
noise (:182-205), Poisson spike trains with a refractory period (:148-171) and
adds templates at the spike times (:219-293).  This module restates that
recipe in vectorised form, with every draw taken from one
``numpy.random.Generator(PCG64(seed))`` so a seed fixes the recording:

* noise: i.i.d. N(0, 1) per channel, band-passed by zeroing FFT bins outside
  [f_lo, f_hi], rescaled to unit standard deviation;
* templates: biphasic waveforms (a trough at the alignment sample followed by
  a slower rebound), peak amplitude in noise SD, times a per-channel gain;
* spike trains: exponential inter-spike intervals at the requested rate plus
  a refractory period, optionally with a fraction of spikes moved onto
  another unit's spike (temporal overlap);
* thresholds: the reference's separability formulas
  (neuron_separability.py:103, 126-142, 251-261) with the per-channel noise
  covariance taken as the Toeplitz matrix of the noise autocovariance.

Outputs follow the reference's layouts: voltage ``[C, N]``, templates
``[K, C*L]`` (channel-major inside a template), as consumed by
``binary_pursuit()``.
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np


@dataclasses.dataclass
class Recording:
    voltage: np.ndarray              # [C, N], float32 or int16
    templates: np.ndarray            # [K, C*L], float32
    sampling_rate: float
    clip_width: list                 # seconds, [-pre, post]
    n_samples_per_chan: int          # L
    spike_times: list                # per unit, alignment-sample indices
    noise_sd: float                  # in voltage units
    chan_covariance: np.ndarray      # [L, L] noise covariance (voltage units^2)
    separability_metrics: dict
    seed: int
    name: str = ""

    @property
    def n_chans(self):
        return self.voltage.shape[0]

    @property
    def n_samples(self):
        return self.voltage.shape[1]

    @property
    def n_templates(self):
        return self.templates.shape[0]

    def sort_info(self, **overrides):
        info = {
            "sampling_rate": self.sampling_rate,
            "clip_width": list(self.clip_width),
            "n_samples_per_chan": self.n_samples_per_chan,
            "n_channels": self.n_chans,
            "n_samples": self.n_samples,
            "do_overlap_recheck": True,
            "get_adjusted_clips": False,
            "sigma_bp_noise": 1.645,
            "sigma_bp_CI": 4.0,
        }
        info.update(overrides)
        return info

    def fresh_metrics(self):
        """A copy of the separability metrics (binary_pursuit() adds a key)."""
        return {k: (v.copy() if isinstance(v, np.ndarray) else v)
                for k, v in self.separability_metrics.items()}


def clip_width_for(L: int, pre_fraction: float, fs: float):
    """Clip window in seconds giving exactly L samples with the reference's
    time_window_to_samples rounding (segment_parallel.py:82-98)."""
    pre = int(round(pre_fraction * (L - 1)))
    post = L - 1 - pre
    return [-pre / fs, post / fs]


def bandlimited_noise(rng, n_chans, n, fs, f_lo=300.0, f_hi=8000.0, dtype=np.float32,
                      batch=16):
    import scipy.fft as sfft
    out = np.empty((n_chans, n), dtype=dtype)
    freqs = np.fft.rfftfreq(n, 1.0 / fs)
    drop = ~((freqs >= f_lo) & (freqs <= f_hi))
    for c0 in range(0, n_chans, batch):
        c1 = min(n_chans, c0 + batch)
        x = rng.standard_normal((c1 - c0, n), dtype=np.float32)
        X = sfft.rfft(x, axis=1, workers=-1)
        del x
        X[:, drop] = 0
        y = sfft.irfft(X, n, axis=1, workers=-1)
        del X
        y /= np.std(y, axis=1, keepdims=True)
        out[c0:c1] = y.astype(dtype)
    return out


def noise_autocov(noise, L):
    """Autocovariance at lags 0..L-1, averaged over channels, via FFT."""
    C, n = noise.shape
    nfft = 1 << int(np.ceil(np.log2(2 * n)))
    acc = np.zeros(L)
    for c in range(C):
        X = np.fft.rfft(noise[c].astype(np.float64), nfft)
        r = np.fft.irfft(np.abs(X) ** 2, nfft)[:L] / n
        acc += r
    return acc / C


def biphasic_waveform(rng, L, align):
    """One unit-peak biphasic spike shape of L samples, trough at `align`."""
    x = np.arange(L, dtype=np.float64)
    w1 = rng.uniform(0.035, 0.07) * L          # trough width
    w2 = rng.uniform(0.08, 0.18) * L           # rebound width
    d = rng.uniform(0.08, 0.2) * L             # rebound delay
    r = rng.uniform(0.25, 0.6)                 # rebound ratio
    pre = rng.uniform(0.0, 0.3)                # small positive pre-peak
    y = (-np.exp(-0.5 * ((x - align) / w1) ** 2)
         + r * np.exp(-0.5 * ((x - align - d) / w2) ** 2)
         + pre * np.exp(-0.5 * ((x - align + 0.6 * d) / (0.6 * w1)) ** 2))
    y -= np.linspace(y[0], y[-1], L) * 0.5     # soften the edges
    if rng.random() < 0.5:
        y = -y
    return y / np.max(np.abs(y))


def poisson_train(rng, rate, n, fs, refractory_s=1.5e-3, edge_s=5e-3):
    if rate <= 0:
        return np.zeros(0, dtype=np.int64)
    ref = refractory_s
    adj = rate / max(1e-9, (1.0 - rate * ref))   # rate adjusted for refractoriness
    dur = n / fs
    est = int(dur * rate * 1.3) + 16
    isi = ref + rng.exponential(1.0 / adj, size=est)
    t = np.cumsum(isi)
    while t[-1] < dur:
        more = ref + rng.exponential(1.0 / adj, size=est)
        t = np.concatenate([t, t[-1] + np.cumsum(more)])
    t = t[(t >= edge_s) & (t < dur - edge_s)]
    return np.unique(np.round(t * fs).astype(np.int64))


def _refractory(s, ref):
    """Drop the later spike of every pair closer than `ref` samples."""
    while s.size > 1:
        bad = np.nonzero(np.diff(s) <= ref)[0]
        if bad.size == 0:
            break
        s = np.delete(s, bad + 1)
    return s


def _insert_spikes(volt, templates, spikes, align, L, n):
    """volt[c, t_k + i - align] += templates[k, c, i] for every spike; spikes
    whose clip would leave the recording are dropped.  Uses torch's
    index_add_ on the CPU, which accumulates duplicates one by one."""
    import torch
    C = volt.shape[0]
    V = torch.from_numpy(volt)
    offs = torch.arange(L, dtype=torch.int64)
    for k in range(len(spikes)):
        s = spikes[k]
        if s.size == 0:
            continue
        starts = s - align
        ok = (starts >= 0) & (starts + L <= n)
        spikes[k] = s[ok]
        st = torch.from_numpy(starts[ok].astype(np.int64))
        if st.numel() == 0:
            continue
        flat = (st[:, None] + offs[None, :]).reshape(-1)
        tk = templates[k].reshape(C, L)
        for c in np.nonzero(np.any(tk != 0, axis=1))[0]:
            src = torch.from_numpy(np.ascontiguousarray(tk[c], dtype=volt.dtype)).repeat(st.numel())
            V[c].index_add_(0, flat, src)


def separability(templates, chan_cov, n_chans, L, sigma_bp_noise=1.645, sigma_bp_CI=4.0):
    """template_SS, variances and thresholds as neuron_separability.py:103,
    126-142 compute them, followed by set_bp_threshold (:251-261)."""
    K = templates.shape[0]
    SS = np.sum(templates.astype(np.float64) ** 2, axis=1)
    var = np.zeros(K)
    for k in range(K):
        for c in range(n_chans):
            tc = templates[k, c * L:(c + 1) * L].astype(np.float64)
            var[k] += tc @ chan_cov @ tc
    lower = -0.5 * SS + sigma_bp_noise * np.sqrt(var)
    lower_ci = 0.5 * SS - sigma_bp_CI * np.sqrt(var)
    thr = np.maximum(np.maximum(lower, 0.0), lower_ci)
    return {
        "bp_n_samples_per_chan": L,
        "templates": templates,
        "template_SS": SS,
        "template_SS_by_chan": np.zeros((K, n_chans)),
        "neuron_variances": var,
        "neuron_lower_CI": lower_ci,
        "neuron_lower_thresholds": thr,
    }


def make_recording(*, n_chans, duration_s, fs, n_templates, L, pre_fraction,
                   amp_range=(3.0, 10.0), amp_lognormal_median=None,
                   rate_range=(5.0, 50.0), gain="uniform", mask_chans=None,
                   overlap_fraction=0.0, overlap_window_s=1e-3,
                   int16_scale=None, autocov_chans=None, seed=0, name="") -> Recording:
    rng = np.random.Generator(np.random.PCG64(seed))
    n = int(round(duration_s * fs))
    C, K = n_chans, n_templates
    clip_width = clip_width_for(L, pre_fraction, fs)
    align = int(round(pre_fraction * (L - 1)))

    noise = bandlimited_noise(rng, C, n, fs)
    # the noise is i.i.d. across channels: autocov_chans (None = all) bounds
    # the channels the average is taken over
    acov = noise_autocov(noise[: (C if autocov_chans is None else min(C, autocov_chans)), : min(n, 400000)], L)
    idx = np.abs(np.subtract.outer(np.arange(L), np.arange(L)))
    cov = acov[idx]

    templates = np.zeros((K, C * L), dtype=np.float64)
    for k in range(K):
        shape = biphasic_waveform(rng, L, align)
        if amp_lognormal_median is not None:
            amp = amp_lognormal_median * np.exp(0.35 * rng.standard_normal())
        else:
            amp = rng.uniform(*amp_range)
        if gain == "uniform":
            g = rng.uniform(0.15, 1.0, size=C)
            g[rng.integers(C)] = 1.0
            chans = np.arange(C)
        elif gain == "exp_distance":
            centre = rng.integers(C)
            g = np.exp(-np.abs(np.arange(C) - centre) / 2.0)
            chans = np.arange(C)
        elif gain == "mask":
            m = int(mask_chans)
            lo = int(rng.integers(0, C - m + 1))
            chans = np.arange(lo, lo + m)
            centre = lo + rng.integers(m)
            g = np.zeros(C)
            g[chans] = np.exp(-np.abs(chans - centre) / 4.0)
        else:
            raise ValueError(gain)
        for c in chans:
            if g[c] <= 0:
                continue
            # small per-channel shape jitter so channels are not collinear
            jitter = 1.0 + 0.1 * rng.standard_normal(L) * np.exp(-0.5 * ((np.arange(L) - align) / (0.3 * L)) ** 2)
            templates[k, c * L:(c + 1) * L] = amp * g[c] * shape * jitter

    spikes = []
    for k in range(K):
        rate = rng.uniform(*rate_range)
        spikes.append(poisson_train(rng, rate, n, fs))
    if overlap_fraction > 0 and K > 1:
        win = max(1, int(round(overlap_window_s * fs)))
        for k in range(K):
            s = spikes[k]
            if s.size == 0:
                continue
            nmove = int(round(overlap_fraction * s.size))
            pick = rng.choice(s.size, size=nmove, replace=False)
            others = rng.integers(0, K - 1, size=nmove)
            others = others + (others >= k)
            jit = rng.integers(-win, win + 1, size=nmove)
            for o in np.unique(others):
                sel = np.nonzero(others == o)[0]
                if spikes[o].size:
                    anchors = spikes[o][rng.integers(0, spikes[o].size, size=sel.size)]
                    s[pick[sel]] = anchors + jit[sel]
            spikes[k] = _refractory(np.unique(np.clip(s, L, n - L)), int(1.5e-3 * fs))

    volt = noise.astype(np.float64) if int16_scale else noise
    _insert_spikes(volt, templates, spikes, align, L, n)

    if int16_scale:
        q = np.clip(np.round(volt * int16_scale), -32768, 32767).astype(np.int16)
        voltage = q
        templates = templates * int16_scale
        cov = cov * int16_scale ** 2
        noise_sd = float(int16_scale)
    else:
        voltage = volt.astype(np.float32)
        noise_sd = 1.0
    templates32 = templates.astype(np.float32)
    metrics = separability(templates32, cov, C, L)
    return Recording(voltage=voltage, templates=templates32, sampling_rate=float(fs),
                     clip_width=clip_width, n_samples_per_chan=L, spike_times=spikes,
                     noise_sd=noise_sd, chan_covariance=cov,
                     separability_metrics=metrics, seed=seed, name=name)


# --- the workloads used by the tests and the benchmark ---------------------

def tetrode(duration_s=30.0, seed=0, **kw):
    """4 channels at 40 kHz, 8 units, 101-sample clips (-1.0/+1.5 ms),
    peaks 3-10 SD, Poisson 5-50 Hz."""
    args = dict(n_chans=4, duration_s=duration_s, fs=40000.0, n_templates=8, L=101,
                pre_fraction=0.4, amp_range=(3.0, 10.0), rate_range=(5.0, 50.0),
                gain="uniform", seed=seed, name="tetrode_4ch")
    args.update(kw)
    return make_recording(**args)


def linear16(duration_s=600.0, seed=1, **kw):
    """16-channel linear probe at 40 kHz, 64 units on all channels with gain
    exp(-d/2) from a centre channel, 101-sample clips, Poisson 1-80 Hz, 15% of
    spikes moved into overlaps within 1 ms."""
    args = dict(n_chans=16, duration_s=duration_s, fs=40000.0, n_templates=64, L=101,
                pre_fraction=0.4, amp_range=(3.0, 10.0), rate_range=(1.0, 80.0),
                gain="exp_distance", overlap_fraction=0.15, seed=seed,
                name="linear16_64u")
    args.update(kw)
    return make_recording(**args)


def hd384(duration_s=300.0, seed=2, **kw):
    """384-channel high-density probe at 30 kHz, int16 voltage, 300 units on
    16-channel masks, 61-sample clips (-0.8/+1.2 ms), lognormal amplitude
    (median 6 SD), Poisson 0.5-100 Hz."""
    args = dict(n_chans=384, duration_s=duration_s, fs=30000.0, n_templates=300, L=61,
                pre_fraction=0.4, amp_lognormal_median=6.0, rate_range=(0.5, 100.0),
                gain="mask", mask_chans=16, int16_scale=16.0, seed=seed,
                name="hd384_300u")
    args.update(kw)
    return make_recording(**args)


# --- request mixes for batched sorting and serving -------------------------

class SegmentSpec:
    """Shape of one request segment; `make()` generates it from its seed."""

    __slots__ = ("seed", "model", "n_chans", "duration_s", "fs", "n_templates", "L")

    def __init__(self, seed, model, n_chans, duration_s, fs, n_templates, L):
        self.seed, self.model, self.n_chans = int(seed), model, int(n_chans)
        self.duration_s, self.fs = float(duration_s), float(fs)
        self.n_templates, self.L = int(n_templates), int(L)

    @property
    def units(self):
        """samples x templates of the segment."""
        return int(round(self.duration_s * self.fs)) * self.n_templates

    def make(self):
        common = dict(n_chans=self.n_chans, duration_s=self.duration_s, fs=self.fs,
                      n_templates=self.n_templates, L=self.L, seed=self.seed, autocov_chans=16)
        if self.model == "tetrode":
            return make_recording(pre_fraction=0.4, amp_range=(3.0, 10.0), rate_range=(5.0, 50.0),
                                  gain="uniform", name="seg_tetrode", **common)
        return make_recording(pre_fraction=0.4, amp_lognormal_median=6.0, rate_range=(0.5, 100.0),
                              gain="mask", mask_chans=16, name="seg_hd", **common)

    def as_dict(self):
        return {k: getattr(self, k) for k in self.__slots__}


def batch_mix(n_segments=256, seed=3, time_scale=1.0):
    """Uneven segments of the batched-sorting workload: durations uniform
    1-60 s (times `time_scale`) at 40 kHz, 4-32 channels, 2-40 templates,
    61-101-sample clips; the tetrode generative model."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(n_segments):
        out.append(SegmentSpec(seed * 1000003 + i, "tetrode", rng.integers(4, 33),
                               rng.uniform(1.0, 60.0) * time_scale, 40000.0, rng.integers(2, 41),
                               rng.integers(61, 102)))
    return out


def serve_mix(n_requests, seed=4, time_scale=1.0):
    """Requests of the serving workload, each with its own seed: 4-384
    channels, 2-120 s (times `time_scale`) at 30 or 40 kHz float32, 4-300
    templates.  Up to 32 channels the tetrode model (templates on all
    channels, at most 40 of them, 40 kHz); above, the high-density model
    (16-channel masks, 61-sample clips, 30 kHz)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(n_requests):
        C = int(rng.integers(4, 385))
        dur = rng.uniform(2.0, 120.0) * time_scale
        if C <= 32:
            spec = SegmentSpec(seed * 1000003 + i, "tetrode", C, dur, 40000.0, rng.integers(4, 41),
                               rng.integers(61, 102))
        else:
            spec = SegmentSpec(seed * 1000003 + i, "hd", C, dur, 30000.0, rng.integers(4, 301), 61)
        out.append(spec)
    return out
