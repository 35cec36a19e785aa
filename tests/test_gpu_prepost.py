"""The steps on either side of the pursuit on the GPU against the
reference's own numpy functions (outputs stored in tests/golden/prepost/
prepost.npz by tests/golden/make_prepost_golden.py; inputs regenerated from
their seeds by tests/_prepost_cases.py).

Exact: clip gathers, robust templates (float32 and int16), duplicate keep
masks, the template-sum search.  Within a stated tolerance: the clip noise
covariance (float64 sums in another order: 1e-9 of its largest entry), the
Wiener filter (float32 throughout as numpy does it, cuFFT against numpy's
pocketfft transform: 1e-5 of the largest output) and the ZCA matrix (the
reference sums the covariance in float32, this library in float64: 1e-5 of
the largest entry)."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from spikesorting_fullpursuit_b200 import analyze_spike_timing as AST  # noqa: E402
from spikesorting_fullpursuit_b200 import build as B  # noqa: E402
from spikesorting_fullpursuit_b200 import full_binary_pursuit as FBP  # noqa: E402
from spikesorting_fullpursuit_b200 import neuron_separability as NS  # noqa: E402
from spikesorting_fullpursuit_b200 import preprocessing as PRE  # noqa: E402
from spikesorting_fullpursuit_b200 import wiener_filter as WF  # noqa: E402
from spikesorting_fullpursuit_b200.c_cython import sort_cython  # noqa: E402
from spikesorting_fullpursuit_b200.parallel import segment_parallel as SP  # noqa: E402
from tests import _prepost_cases as P  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "prepost", "prepost.npz"))


@pytest.fixture(scope="module", autouse=True)
def lib():
    B.build()


@pytest.mark.parametrize("tag,dt", [("f32", np.float32), ("i16", np.int16)])
def test_get_clips_match_reference(tag, dt):
    probe, v, nb, ev, cw = P.clips_case(11, dt)
    clips, valid = SP.get_clips(probe, v, nb, ev, cw)
    assert clips.dtype == GOLD["clips_%s" % tag].dtype
    assert np.array_equal(clips, GOLD["clips_%s" % tag])
    assert np.array_equal(valid, GOLD["clips_valid_%s" % tag])
    sc, sv = SP.get_singlechannel_clips(probe, v[2], ev, cw)
    assert np.array_equal(sc, GOLD["sclips_%s" % tag])
    assert np.array_equal(sv, GOLD["sclips_valid_%s" % tag])


@pytest.mark.parametrize("tag,dt", [("f32", np.float32), ("i16", np.int16)])
def test_robust_templates_match_reference(tag, dt):
    units = P.robust_case(12, dt)
    for i, c in enumerate(units):
        got = PRE.calculate_robust_template(c)
        exp = GOLD["robust_%s_%d" % (tag, i)]
        assert got.dtype == exp.dtype and got.shape == exp.shape
        assert np.array_equal(got, exp), (tag, i, np.nonzero(got != exp)[0][:5])
    # all units in one launch
    off = np.concatenate([[0], np.cumsum([c.shape[0] for c in units])])
    batch = PRE.calculate_robust_templates(np.vstack(units), off)
    for i in range(len(units)):
        assert np.array_equal(batch[i], np.atleast_1d(GOLD["robust_%s_%d" % (tag, i)]).reshape(-1))


def test_pursuit_templates_and_noise_covariance_match_reference():
    rec, units, cw = P.glue_case(13)
    tmpl, cov = FBP.pursuit_templates_and_covariance(rec.voltage, units, rec.sampling_rate, cw,
                                                     n_cov_samples=10 ** 9)
    assert np.array_equal(tmpl, GOLD["glue_templates"])
    ref = GOLD["glue_cov"]
    err = np.abs(np.stack(cov) - ref).max() / np.abs(ref).max()
    assert err < 1e-9, err


def test_duplicate_removal_matches_reference():
    ev, lab, clips, bp, tol = P.dup_case(14)
    for u in np.unique(lab):
        s = lab == u
        tm = AST.unit_mean_templates(clips[s], [0, int(s.sum())])[0]
        assert np.array_equal(tm, GOLD["dup_tmpl_%d" % u])
        assert np.array_equal(AST.remove_binary_pursuit_duplicates(ev[s], clips[s], tm, bp[s], tol),
                              GOLD["dup_rm_bp_%d" % u])
        assert np.array_equal(AST.keep_binary_pursuit_duplicates(ev[s], bp[s], tol), GOLD["dup_keep_bp_%d" % u])
        assert np.array_equal(AST.remove_spike_event_duplicates(ev[s], clips[s], tm, tol), GOLD["dup_rm_ev_%d" % u])
    # every unit of the segment in one pass (postprocessing.py:521-545)
    keep = AST.remove_segment_binary_pursuit_duplicates(ev, lab, clips, bp, tol)
    for u in np.unique(lab):
        assert np.array_equal(keep[lab == u], GOLD["dup_rm_bp_%d" % u])


def test_find_overlap_templates_matches_reference():
    T, L, C, pre, post, nsp = P.overlap_tpl_case(15)
    res = sort_cython.find_overlap_templates(T, L, C, pre, post, nsp)
    assert [r[0] for r in res] == GOLD["ovt_units"].tolist()
    assert [list(r[2]) for r in res] == GOLD["ovt_pairs"].tolist()
    assert np.array_equal(np.array([r[1] for r in res]), GOLD["ovt_templates"])


@pytest.mark.parametrize("smooth", [0, 1, 25])
def test_wiener_filter_matches_reference(smooth):
    o, s, nz = P.wiener_case(16)
    for fn, key in ((WF.wiener, "wiener_%d"), (WF.wiener_all, "wiener_all_%d")):
        got = fn(o, s, nz, smooth)
        ref = GOLD[key % smooth]
        assert got.shape == ref.shape and got.dtype == ref.dtype
        err = np.abs(got.astype(np.float64) - ref).max() / np.abs(ref).max()
        print("\n%s smooth=%d: max difference %.2e of the largest output" % (key % smooth, smooth, err))
        assert err < 1e-5, (key, err)


def test_zca_matrix_and_whitening_match_reference():
    v, thr, sigma, cushion = P.zca_case(17)
    Z = PRE.get_noise_sampled_zca_matrix(v, thr, sigma, cushion, n_samples=1e7)
    ref = GOLD["zca"]
    err = np.abs(Z - ref).max() / np.abs(ref).max()
    print("\nZCA matrix: max difference %.2e of the largest entry" % err)
    assert err < 1e-5, err
    # the whitening itself against numpy's float64 product, rounded to float32
    out = PRE.zca_apply(ref, v)
    exp = (ref @ v).astype(np.float32)
    ulp = np.abs(out.astype(np.float64) - exp) / np.spacing(np.abs(exp).astype(np.float32)).astype(np.float64)
    assert ulp.max() <= 1.0, ulp.max()


def test_separability_metrics_and_thresholds_match_reference():
    """template_SS bit for bit (numpy's float32 pairwise sum); variances and
    bounds in float64 within 1e-12 relative; the float32 thresholds the
    pursuit uses identical."""
    T, covs, si = P.separability_case(18)
    m = NS.compute_separability_metrics(T, covs, si)
    assert m["template_SS"].dtype == GOLD["sep_template_SS"].dtype
    assert np.array_equal(m["template_SS"], GOLD["sep_template_SS"])
    for k in ("neuron_variances", "neuron_lower_CI", "neuron_lower_thresholds", "contamination"):
        ref = GOLD["sep_" + k]
        assert np.allclose(m[k], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max()), k
    assert np.array_equal(m["peak_channel"], GOLD["sep_peak_channel"])
    assert np.array_equal(m["channel_p_noise"], GOLD["sep_channel_p_noise"])
    m = NS.set_bp_threshold(m)
    assert np.array_equal(np.float32(m["neuron_lower_thresholds"]), np.float32(GOLD["sep_bp_thresholds"]))
    sums = NS.separability_sums(T, covs, si["sigma_bp_noise"], si["sigma_bp_CI"])
    assert np.array_equal(np.float32(sums["thr"]), np.float32(GOLD["sep_bp_thresholds"]))
    assert np.allclose(sums["ss64"], np.sum(np.vstack(T).astype(np.float64) ** 2, axis=1), rtol=1e-14)
