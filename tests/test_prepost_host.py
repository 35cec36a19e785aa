"""Host logic of the pre/post-pursuit drop-ins, without a GPU: the device
calls are replaced by numpy restatements of their C-ABI contracts, and the
results are compared with the reference's outputs (tests/golden/prepost)."""
import os

import numpy as np

from spikesorting_fullpursuit_b200.c_cython import sort_cython
from spikesorting_fullpursuit_b200.parallel import segment_parallel as SP
from tests import _prepost_cases as P

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "prepost", "prepost.npz"))


def _search_items(T, C, L, n_pre, n_post, items):
    """fbp_overlap_template_search's contract: per item, the first strictly
    smallest sum((test - shift(t1, s1) - shift(t2, s2))**2), shift1 outer."""
    out_ss, out_sh = [], []
    shifted = {}

    def sh(k, s):
        if (k, s) not in shifted:
            shifted[(k, s)] = sort_cython.get_shifted_template(T[k], s, C, L).astype(np.float64)
        return shifted[(k, s)]
    for test, n1, n2 in items:
        best, arg = np.inf, (0, 0)
        for s1 in range(-n_pre, n_post + 1):
            for s2 in range(-n_pre, n_post + 1):
                r = np.sum((T[test] - (sh(n1, s1) + sh(n2, s2))) ** 2)
                if r < best:
                    best, arg = r, (s1, s2)
        out_ss.append(best)
        out_sh.append(arg)
    return np.array(out_ss), np.array(out_sh, dtype=np.int32)


def test_find_overlap_templates_host_logic(monkeypatch):
    """Pair filters, unit order and the choice across pairs on the host,
    with the per-item device search restated in numpy."""
    T, L, C, pre, post, nsp = P.overlap_tpl_case(15)

    class FakeLib:
        def fbp_overlap_template_scratch_bytes(self, n_items, n_pre, n_post):
            return 8

        def fbp_overlap_template_search(self, Tp, K, C_, L_, n_pre, n_post, items, n_items, ss, shift, scratch,
                                        sb, st):
            a, b = _search_items(T, C, L, n_pre, n_post, np.asarray(items).reshape(-1, 3).tolist())
            ss[...] = a
            shift[...] = b
            return 0
    monkeypatch.setattr(sort_cython._lib, "lib", lambda: FakeLib())
    monkeypatch.setattr(sort_cython._lib, "check", lambda rc: None)
    monkeypatch.setattr(sort_cython._lib, "ptr", lambda t: t)
    monkeypatch.setattr(sort_cython.D, "to_dev", lambda x, dtype=None: np.asarray(x))
    monkeypatch.setattr(sort_cython.D, "empty", lambda shape, dtype: np.zeros(shape, dtype))
    monkeypatch.setattr(sort_cython.D, "stream", lambda: None)
    monkeypatch.setattr(sort_cython.D, "host", lambda x: x)
    res = sort_cython.find_overlap_templates(T, L, C, pre, post, nsp)
    assert [r[0] for r in res] == GOLD["ovt_units"].tolist()
    assert [list(r[2]) for r in res] == GOLD["ovt_pairs"].tolist()
    assert np.array_equal(np.array([r[1] for r in res]), GOLD["ovt_templates"])


def test_clip_valid_range_matches_reference():
    for tag, dt in (("f32", np.float32), ("i16", np.int16)):
        probe, v, nb, ev, cw = P.clips_case(11, dt)
        window, _ = SP.time_window_to_samples(cw, probe["sampling_rate"])
        valid, a, b = SP._valid_range(ev, window, probe["n_samples"], True)
        assert np.array_equal(valid, GOLD["clips_valid_%s" % tag])
        # the copy itself, restated
        W = window[1] - window[0]
        clips = np.stack([np.concatenate([v[c, e + window[0]:e + window[1]] for c in nb]) for e in ev[a:b + 1]])
        assert clips.shape[1] == W * len(nb)
        assert np.array_equal(clips, GOLD["clips_%s" % tag])
        valid, a, b = SP._valid_range(ev, window, probe["n_samples"], False)
        assert np.array_equal(valid, GOLD["sclips_valid_%s" % tag])
