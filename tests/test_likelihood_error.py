"""Likelihood error against a float64 NumPy evaluation, per workload.

(1) The FP32 likelihood (the oracle's restatement of compute_full_likelihood,
bit-identical to the reference and to the FP32 GPU path) lies within the
recursive-sum bound gamma * (sum|t v| + |SS/2|) of the float64 value.
(2) A NumPy model of the tensor-core operands -- voltage and templates scaled
by powers of two and rounded to fp16 as the kernel does, products summed in
float64 -- lies within the product-rounding part of the kernel's error bound
(2^-10 + 2^-22 per unit of ||t|| ||window||, plus the fp16 subnormal terms).
The accumulation part of the bound (FP32 sums in the tensor core) is not
modelled here; the GPU parity tests cover the whole bound through the
pursuit's results.

Run with -s to see the per-workload figures.
"""
import numpy as np
import pytest

from oracle import oracle as O
from spikesorting_fullpursuit_b200 import synthetic

CASES = [
    ("tetrode (config 0)", lambda: synthetic.tetrode(duration_s=0.1, seed=11)),
    ("linear16 (config 1)", lambda: synthetic.linear16(duration_s=0.05, seed=12)),
    ("hd384 (config 2)", lambda: synthetic.hd384(duration_s=0.02, seed=13)),
]


def _scale_exp(mx):
    """The kernels' power-of-two scale: magnitudes below 2^14 after scaling."""
    if mx <= 0:
        return 0
    _, e = np.frexp(np.float32(mx))
    return int(max(-126, min(126, 14 - int(e))))


def _corr(x, k, m):
    """sum_j x[s + j] * k[j] for s = 0 .. m - 1, float64."""
    return np.correlate(x, k, mode="valid")[:m]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0].split()[0] for c in CASES])
def test_likelihood_error_vs_float64(name, make):
    rec = make()
    v32 = np.ascontiguousarray(rec.voltage, dtype=np.float32)        # as binary_pursuit() casts it
    C, n = v32.shape
    L = rec.n_samples_per_chan
    T32 = np.ascontiguousarray(rec.templates, dtype=np.float32)
    K = T32.shape[0]
    SS = rec.separability_metrics["template_SS"].astype(np.float64)
    tss = np.float32(-0.5 * SS)
    W = (n + L - 1) // L
    Lk = np.zeros((K, n), np.float32)
    O.stage_full_likelihood(v32, T32.reshape(-1), K, L, tss, np.arange(W, dtype=np.uint32), Lk)

    v64 = v32.astype(np.float64)
    T3 = T32.astype(np.float64).reshape(K, C, L)
    ns = n - L - 1                              # last sample with s + L < n (.cl:231-234)
    u, u_h = 2.0 ** -24, 2.0 ** -11
    # fp16 operand model: voltage tiles of 128 samples, one scale per tile
    kexp = np.array([_scale_exp(np.abs(v32[:, s0:s0 + 128 + L]).max()) for s0 in range(0, ns, 128)])
    worst32 = worst16 = 0.0
    rel32 = []
    nz_max = 0
    for t in range(K):
        sup = np.nonzero(np.any(T3[t] != 0, axis=1))[0]
        nz_max = max(nz_max, len(sup))
        texp = _scale_exp(np.abs(T32[t]).max())
        th = (T3[t][sup] * 2.0 ** texp).astype(np.float16).astype(np.float64)
        dot = np.zeros(ns + 1)
        adot = np.zeros(ns + 1)
        wsq = np.zeros(ns + 1)
        wab = np.zeros(ns + 1)
        dot16 = np.zeros(ns + 1)
        ones = np.ones(L)
        for j, c in enumerate(sup):
            dot += _corr(v64[c], T3[t, c], ns + 1)
            adot += _corr(np.abs(v64[c]), np.abs(T3[t, c]), ns + 1)
            wsq += _corr(v64[c] ** 2, ones, ns + 1)
            wab += _corr(np.abs(v64[c]), ones, ns + 1)
        # the fp16 model, tile by tile (each tile's own voltage scale)
        for i, s0 in enumerate(range(0, ns + 1, 128)):
            s1 = min(ns + 1, s0 + 128)
            ke = kexp[min(i, len(kexp) - 1)]
            seg = v64[sup, s0:s1 + L - 1]
            vh = (seg * 2.0 ** ke).astype(np.float16).astype(np.float64)
            acc = np.zeros(s1 - s0)
            for j in range(len(sup)):
                acc += _corr(vh[j], th[j], s1 - s0)
            dot16[s0:s1] = acc * 2.0 ** (-ke - texp)
        lik64 = dot - 0.5 * SS[t]
        lik32 = Lk[t, :ns + 1].astype(np.float64)
        scale = adot + 0.5 * SS[t]
        err32 = np.abs(lik32 - lik64)
        rel32.append(float(np.max(err32 / scale)))
        # kernel bound, product-rounding part
        tn = np.sqrt(np.sum(T3[t] ** 2))
        t1 = np.sum(np.abs(T3[t]))
        kex = np.repeat(kexp, 128)[:ns + 1]
        E16 = ((2 * (2.0 ** -11) + 2.0 ** -22) * tn * np.sqrt(wsq)
               + 2.0 ** -25 * 1.001 * (wab * 2.0 ** -texp + t1 * 2.0 ** -kex.astype(np.float64)))
        err16 = np.abs(dot16 - dot)
        worst16 = max(worst16, float(np.max(err16 / np.maximum(E16, 1e-300))))
        worst32 = max(worst32, rel32[-1])
    n_ref = nz_max * L + 1
    gamma = n_ref * u / (1 - n_ref * u)
    print("\n%s: C=%d K=%d L=%d n=%d | FP32 (reference) vs float64: max |err| / (sum|tv| + |SS/2|) = %.3g "
          "(bound gamma = %.3g) | fp16-operand model: max err / its bound = %.3f"
          % (name, C, K, L, n, worst32, gamma, worst16))
    assert worst32 <= gamma
    assert worst16 <= 1.0
