"""Shared helpers: golden cases and result comparison."""
import glob
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN_DIR = os.path.join(HERE, "golden")


def golden_paths():
    return sorted(glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))


class GoldenCase:
    def __init__(self, path):
        z = np.load(path, allow_pickle=False)
        self.name = os.path.splitext(os.path.basename(path))[0]
        self.voltage = z["voltage"]
        self.templates = z["templates"]
        self.template_SS = z["template_SS"]
        self.thresholds = z["neuron_lower_thresholds"]
        self.ss_by_chan = z["template_SS_by_chan"]
        self.n_spikes = z["n_spikes"]
        self.sort_info = {
            "sampling_rate": float(z["sampling_rate"]),
            "clip_width": [float(x) for x in z["clip_width"]],
            "n_samples_per_chan": int(z["n_samples_per_chan"]),
            "do_overlap_recheck": bool(z["do_overlap_recheck"]),
            "get_adjusted_clips": bool(z["get_adjusted_clips"]),
        }
        nm = int(z["n_max_shift_inds"])
        self.n_max_shift_inds = None if nm < 0 else nm
        cs = int(z["chunk_samples"])
        self.chunk_samples = None if cs < 0 else cs
        self.empty = bool(z["empty"])
        self.expected = (z["out_event_indices"], z["out_neuron_labels"], z["out_bp_bool"],
                         z["out_adjusted_clips"])

    def metrics(self):
        return {"templates": self.templates.copy(), "template_SS": self.template_SS.copy(),
                "template_SS_by_chan": self.ss_by_chan.copy(),
                "neuron_lower_thresholds": self.thresholds.copy()}


def assert_same_outputs(got, expected, empty_expected=False):
    """The 4-tuple must match element for element (values, dtypes, shapes)."""
    if empty_expected:
        for g in got:
            assert isinstance(g, list) and len(g) == 0, type(g)
        return
    names = ("event_indices", "neuron_labels", "bp_bool", "adjusted_clips")
    for nm, g, e in zip(names, got, expected):
        g = np.asarray(g)
        assert g.dtype == e.dtype, (nm, g.dtype, e.dtype)
        assert g.shape == e.shape, (nm, g.shape, e.shape)
        assert np.array_equal(g, e), (nm, "mismatch at", np.nonzero(g != e)[0][:10])


def as_expected_tuple(out):
    return tuple(np.asarray(o) for o in out)
