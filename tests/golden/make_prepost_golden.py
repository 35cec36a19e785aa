"""Generate tests/golden/prepost/prepost.npz: outputs of the REFERENCE's own numpy
functions (its package staged unmodified under baseline/_ref by
oracle/install_reference.sh) on the seeded inputs of tests/_prepost_cases.py.
Run where the reference is staged:  python tests/golden/make_prepost_golden.py"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle", "fake_modules"))     # mkl stand-in for the package import
sys.path.insert(0, os.path.join(REPO, "baseline", "_ref"))

from spikesorting_fullpursuit import analyze_spike_timing as AST  # noqa: E402
from spikesorting_fullpursuit import neuron_separability as NS  # noqa: E402
from spikesorting_fullpursuit import preprocessing as PRE  # noqa: E402
from spikesorting_fullpursuit import wiener_filter as WF  # noqa: E402
from spikesorting_fullpursuit.c_cython import sort_cython  # noqa: E402
from spikesorting_fullpursuit.parallel import segment_parallel as SP  # noqa: E402
from tests import _prepost_cases as P  # noqa: E402


def main():
    out = {}
    for tag, dt in (("f32", np.float32), ("i16", np.int16)):
        probe, v, nb, ev, cw = P.clips_case(11, dt)
        clips, valid = SP.get_clips(probe, v, nb, ev, cw)
        out["clips_%s" % tag] = clips
        out["clips_valid_%s" % tag] = valid
        ch, cvalid = SP.get_singlechannel_clips(probe, v[2], ev, cw)
        out["sclips_%s" % tag] = ch
        out["sclips_valid_%s" % tag] = cvalid
        for i, c in enumerate(P.robust_case(12, dt)):
            out["robust_%s_%d" % (tag, i)] = PRE.calculate_robust_template(c)
    # the glue of full_binary_pursuit.py:299-322 with every residual row
    rec, units, cw = P.glue_case(13)
    probe = {"sampling_rate": rec.sampling_rate, "n_samples": rec.n_samples, "v_dtype": rec.voltage.dtype}
    chans = np.arange(rec.n_chans)
    bp_templates, resid = [], []
    for ev in units:
        clips, _ = SP.get_clips(probe, rec.voltage, chans, ev, cw)
        t = PRE.calculate_robust_template(clips)
        bp_templates.append(t)
        resid.append(clips - t)
    resid = np.vstack(resid)
    L = rec.n_samples_per_chan
    cov = [np.cov(resid[:, c * L:(c + 1) * L], rowvar=False, ddof=0) for c in range(rec.n_chans)]
    out["glue_templates"] = np.vstack(bp_templates)
    out["glue_cov"] = np.stack(cov)
    # duplicates
    ev, lab, clips, bp, tol = P.dup_case(14)
    for u in np.unique(lab):
        s = lab == u
        tmpl = np.mean(clips[s], axis=0)
        out["dup_rm_bp_%d" % u] = AST.remove_binary_pursuit_duplicates(ev[s], clips[s], tmpl, bp[s], tol)
        out["dup_keep_bp_%d" % u] = AST.keep_binary_pursuit_duplicates(ev[s], bp[s], tol)
        out["dup_rm_ev_%d" % u] = AST.remove_spike_event_duplicates(ev[s], clips[s], tmpl, tol)
        out["dup_tmpl_%d" % u] = tmpl
    # find_overlap_templates
    T, L, C, pre, post, nsp = P.overlap_tpl_case(15)
    res = sort_cython.find_overlap_templates(T, L, C, np.int64(pre), np.int64(post), nsp)
    out["ovt_units"] = np.array([r[0] for r in res], dtype=np.int64)
    out["ovt_pairs"] = np.array([r[2] for r in res], dtype=np.int64).reshape(-1, 2)
    out["ovt_templates"] = np.array([r[1] for r in res]).reshape(len(res), -1)
    # Wiener
    o, s, nz = P.wiener_case(16)
    for sm in (0, 1, 25):
        out["wiener_%d" % sm] = WF.wiener(o, s, nz, sm)
        out["wiener_all_%d" % sm] = WF.wiener_all(o, s, nz, sm)
    # ZCA (n_samples above the sample count: every valid sample is used)
    v, thr, sigma, cushion = P.zca_case(17)
    out["zca"] = PRE.get_noise_sampled_zca_matrix(v, thr, sigma, cushion, n_samples=1e7)
    # pursuit inputs: separability metrics and the pursuit thresholds
    T, covs, si = P.separability_case(18)
    m = NS.compute_separability_metrics(T, covs, si)
    for k in ("template_SS", "neuron_variances", "neuron_lower_CI", "neuron_lower_thresholds", "peak_channel",
              "contamination", "channel_p_noise"):
        out["sep_" + k] = np.array(m[k], copy=True)       # set_bp_threshold changes some in place
    m = NS.set_bp_threshold(m)
    out["sep_bp_thresholds"] = np.asarray(m["neuron_lower_thresholds"])
    np.savez_compressed(os.path.join(HERE, "prepost", "prepost.npz"), **out)
    print("wrote", os.path.join(HERE, "prepost", "prepost.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()
