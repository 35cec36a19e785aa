"""find_overlap_templates of spikesorting_fullpursuit/c_cython/
sort_cython.pyx:333-458 with the search on the device.

The reference tests, for every unit in descending order of its template's
sum of squares, every pair of other units (with enough spikes and
amplitudes able to account for the unit's minimum and maximum) at every
pair of shifts, and keeps the pair and shifts whose sum best explains the
template.  Here the order of units and the pair filters are restated on the
host in the reference's float32 arithmetic; every (unit, pair) item's
shift search runs on the GPU (fbp_overlap_template_search), in the
reference's float64 arithmetic and summation order, so the minima and
their positions are the reference's."""
import numpy as np

from .. import _device as D
from .. import _lib


def get_shifted_template(template, shift, n_chans, n_samples_per_chan):
    """get_shifted_template of sort_cython.pyx:338-349."""
    L = n_samples_per_chan
    out = np.zeros_like(template)
    for chan in range(0, n_chans):
        chan_temp = template[chan * L:(chan + 1) * L]
        if shift > 0:
            out[chan * L + shift:(chan + 1) * L] = chan_temp[:-shift]
        else:
            out[chan * L:(chan + 1) * L + shift] = chan_temp[-shift:]
    return out


def find_overlap_templates(templates, n_samples_per_chan, n_chans, n_pre_inds, n_post_inds, n_template_spikes):
    """Same arguments and result as the reference: a list of
    [test_unit, best_shifted_template (float64), [n1, n2]]."""
    templates = np.ascontiguousarray(templates, dtype=np.float32)
    K = templates.shape[0]
    L = int(n_samples_per_chan)
    C = int(n_chans)
    n_pre, n_post = int(n_pre_inds), int(n_post_inds)
    n_template_spikes = np.asarray(n_template_spikes, dtype=np.int64)
    templates_to_check = []
    if K < 3:
        return templates_to_check
    templates_SS = np.sum(templates ** 2, axis=1)
    order = np.argsort(templates_SS)[-1::-1]
    per_chan = templates.reshape(K, C, L)
    items, owner = [], []
    for test_unit in order:
        test = templates[test_unit, :]
        cmin = int(np.argmin(test) // L)
        cmax = int(np.argmax(test) // L)
        ok = (n_template_spikes >= 4 * n_template_spikes[test_unit])
        ok[test_unit] = False
        mins = per_chan[:, cmin, :].min(axis=1)          # np.amin over the channel's samples
        maxs = per_chan[:, cmax, :].max(axis=1)
        testmin = test[cmin * L:(cmin + 1) * L].min()
        testmax = test[cmax * L:(cmax + 1) * L].max()
        lim_min = np.float32(0.75) * testmin
        lim_max = np.float32(0.75) * testmax
        for n1 in range(K):
            if not ok[n1]:
                continue
            n2 = np.arange(n1 + 1, K)
            sel = ok[n2] & ~((mins[n1] + mins[n2]) > lim_min) & ~((maxs[n1] + maxs[n2]) < lim_max)
            for b in n2[sel]:
                items.append((int(test_unit), n1, int(b)))
                owner.append(int(test_unit))
    best_ss = np.zeros(0)
    best_shift = np.zeros((0, 2), np.int32)
    if items:
        lib = _lib.lib()
        it = np.ascontiguousarray(np.array(items, dtype=np.uint32))
        T_d = D.to_dev(templates)
        it_d = D.to_dev(it)
        ss_d = D.empty((len(items),), np.float64)
        sh_d = D.empty((len(items), 2), np.int32)
        sb = lib.fbp_overlap_template_scratch_bytes(len(items), n_pre, n_post)
        scratch = D.empty((sb,), np.uint8)
        _lib.check(lib.fbp_overlap_template_search(_lib.ptr(T_d), K, C, L, n_pre, n_post, _lib.ptr(it_d), len(items),
                                                   _lib.ptr(ss_d), _lib.ptr(sh_d), _lib.ptr(scratch), sb,
                                                   D.stream()))
        best_ss, best_shift = D.host(ss_d), D.host(sh_d)
    # the first strictly smallest residual over pairs in the reference's order
    q = 0
    for test_unit in order:
        best, pick = np.inf, None
        while q < len(items) and owner[q] == int(test_unit):
            if best_ss[q] < best:
                best, pick = best_ss[q], q
            q += 1
        if pick is not None:
            _, n1, n2 = items[pick]
            s1, s2 = int(best_shift[pick][0]), int(best_shift[pick][1])
            t = (get_shifted_template(templates[n1], s1, C, L).astype(np.float64)
                 + get_shifted_template(templates[n2], s2, C, L).astype(np.float64))
            templates_to_check.append([int(test_unit), t, [n1, n2]])
    return templates_to_check
