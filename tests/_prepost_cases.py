"""Seeded inputs of the pre- and post-pursuit parity cases.  The reference's
outputs for them are stored in tests/golden/prepost/prepost.npz
(tests/golden/make_prepost_golden.py); the inputs are regenerated here from
their seeds (numpy PCG64), so the fixtures hold outputs only."""
import numpy as np

FS = 40000.0


def rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def clips_case(seed, dtype):
    r = rng(seed)
    C, n = 8, 4000
    if dtype == np.int16:
        v = np.round(r.standard_normal((C, n)) * 60).astype(np.int16)
    else:
        v = (r.standard_normal((C, n)) * 3).astype(np.float32)
    ev = np.sort(np.concatenate([r.integers(-12, 15, 4), r.integers(0, n, 50), r.integers(n - 15, n + 12, 4)]))
    neighbors = np.array([3, 1, 6, 0], dtype=np.int64)
    clip_width = [-0.0005, 0.00075]
    probe = {"sampling_rate": FS, "n_samples": n, "v_dtype": np.dtype(dtype)}
    return probe, v, neighbors, ev.astype(np.int64), clip_width


ROBUST_SIZES = (1, 2, 3, 8, 101, 1000, 2048)


def robust_case(seed, dtype):
    r = rng(seed)
    dim = 4 * 31
    out = []
    for m in ROBUST_SIZES:
        if dtype == np.int16:
            c = np.round(r.standard_normal((m, dim)) * 40 + r.standard_normal(dim) * 100).astype(np.int16)
        else:
            c = (r.standard_normal((m, dim)) * 2 + r.standard_normal(dim) * 5).astype(np.float32)
            if m > 8:                        # exact ties
                c[m // 3: m // 3 + 4] = c[0]
        out.append(c)
    return out


def glue_case(seed):
    from spikesorting_fullpursuit_b200 import synthetic
    rec = synthetic.tetrode(duration_s=0.5, seed=seed, L=41, n_templates=5)
    units = [np.asarray(s, dtype=np.int64) for s in rec.spike_times]
    clip_width = list(rec.clip_width)
    return rec, units, clip_width


def dup_case(seed, n_units=6):
    r = rng(seed)
    dim = 3 * 21
    events, labels, clips, bp = [], [], [], []
    for u in range(n_units):
        m = int(r.integers(5, 60))
        e = np.sort(r.integers(0, 3000, m))
        e[1::4] = e[0::4][: len(e[1::4])] + r.integers(0, 12, len(e[1::4]))   # pairs within the tolerance
        e = np.sort(e)
        events.append(e)
        labels.append(np.full(m, u))
        clips.append((r.standard_normal((m, dim)) + r.standard_normal(dim) * 3).astype(np.float32))
        bp.append(r.random(m) < 0.7)
    order = np.argsort(np.concatenate(events), kind="stable")
    return (np.concatenate(events)[order].astype(np.int64), np.concatenate(labels)[order],
            np.vstack(clips)[order], np.concatenate(bp)[order], 10)


def overlap_tpl_case(seed):
    r = rng(seed)
    C, L, K = 4, 31, 9
    x = np.arange(L)
    T = np.zeros((K, C * L), np.float32)
    for k in range(6):
        centre = r.uniform(10, 20)
        shape = -np.exp(-0.5 * ((x - centre) / r.uniform(1.5, 3)) ** 2) + 0.4 * np.exp(
            -0.5 * ((x - centre - 5) / 3) ** 2)
        g = r.uniform(0.2, 1.0, C)
        T[k] = (np.outer(g, shape) * r.uniform(4, 9)).reshape(-1)

    def shifted(t, s):
        out = np.zeros_like(t)
        for c in range(C):
            ct = t[c * L:(c + 1) * L]
            if s > 0:
                out[c * L + s:(c + 1) * L] = ct[:-s]
            else:
                out[c * L:(c + 1) * L + s] = ct[-s:]
        return out
    T[6] = shifted(T[0], 2) + shifted(T[1], -3)
    T[7] = shifted(T[2], -1) + shifted(T[4], 4) + (r.standard_normal(C * L) * 0.05).astype(np.float32)
    T[8] = T[3] * 0.9
    n_spikes = np.array([900, 800, 1000, 700, 950, 850, 50, 60, 40], dtype=np.int64)
    return T, L, C, 6, 8, n_spikes


def wiener_case(seed):
    r = rng(seed)
    C, n = 3, 6000
    noise = r.standard_normal((C, n))
    signal = np.zeros((C, n))
    shape = -np.exp(-0.5 * ((np.arange(31) - 12) / 2.0) ** 2)
    for s in r.integers(0, n - 31, 60):
        signal[:, s:s + 31] += shape * r.uniform(3, 6)
    original = (signal + noise).astype(np.float32)
    return original, signal.astype(np.float32), (original - signal).astype(np.float32)


def zca_case(seed):
    r = rng(seed)
    C, n = 6, 40000
    mix = np.eye(C) + 0.3 * r.standard_normal((C, C))
    v = mix @ r.standard_normal((C, n))
    shape = -np.exp(-0.5 * ((np.arange(21) - 8) / 2.0) ** 2)
    for s in r.integers(0, n - 21, 80):
        v[:, s:s + 21] += np.outer(r.uniform(2, 8, C), shape)
    v = v.astype(np.float32)
    thresholds = 4.0 * np.median(np.abs(v), axis=1) / 0.6745
    return v, thresholds, 4.0, 10


def separability_case(seed):
    r = rng(seed)
    C, L, K = 4, 31, 7
    x = np.arange(L)
    T = []
    for k in range(K):
        shape = -np.exp(-0.5 * ((x - r.uniform(8, 20)) / r.uniform(1.5, 3)) ** 2)
        T.append((np.outer(r.uniform(0.1, 1.0, C), shape) * r.uniform(2, 9)).reshape(-1).astype(np.float32))
    covs = []
    for c in range(C):
        a = r.standard_normal((L, 3 * L))
        covs.append(a @ a.T / (3 * L))
    sort_info = {"n_channels": C, "n_samples_per_chan": L, "sigma": 4.0, "sigma_bp_noise": 2.326,
                 "sigma_bp_CI": 12.0, "n_samples": 100000, "n_threshold_crossings": r.integers(10, 500, C)}
    return T, covs, sort_info
