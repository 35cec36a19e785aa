"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own host code (spikesorting_fullpursuit/parallel/
binary_pursuit_parallel.py, unmodified, staged by oracle/install_reference.sh)
with the stand-in pyopencl whose kernels are the reference's own
binary_pursuit.cl compiled for the CPU (oracle/_ref/libbp_ref.so).  Needs the
reference tree; run from the repository root:

    bash oracle/install_reference.sh && make -C oracle ref
    python tests/golden/make_golden.py

Each case is stored as an .npz holding the inputs (voltage, templates,
template_SS, thresholds, sort settings) and the reference's four outputs.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from spikesorting_fullpursuit_b200 import synthetic  # noqa: E402
from oracle import reference_harness as R  # noqa: E402

GLOBAL_MEM = 16 * 1024 ** 3


def cases():
    yield "tetrode_L31_overlap", synthetic.tetrode(duration_s=0.5, seed=3, L=31), \
        dict(nmax=30, overlap=True, clips=True)
    yield "tetrode_L31_no_overlap", synthetic.tetrode(duration_s=0.5, seed=3, L=31), \
        dict(nmax=30, overlap=False, clips=False)
    yield "tetrode_L101_nmax12", synthetic.tetrode(duration_s=0.3, seed=5), \
        dict(nmax=12, overlap=True, clips=True)
    yield "tetrode_L31_4chunks", synthetic.tetrode(duration_s=0.5, seed=3, L=31), \
        dict(nmax=10, overlap=True, clips=True, max_gpu_memory=2.0e6)
    yield "linear16_L41_dense", synthetic.linear16(duration_s=0.1, seed=7, n_templates=12, L=41), \
        dict(nmax=40, overlap=True, clips=False)
    yield "hd32_int16_masked", synthetic.hd384(duration_s=0.2, seed=11, n_chans=32, n_templates=10,
                                               L=21, mask_chans=8), \
        dict(nmax=20, overlap=True, clips=True)
    yield "single_template_1d", synthetic.tetrode(duration_s=0.3, seed=13, L=31, n_templates=1), \
        dict(nmax=None, overlap=True, clips=False, one_d=True)
    yield "noise_only_no_overlap", synthetic.tetrode(duration_s=0.2, seed=17, L=31,
                                                     rate_range=(0.0, 0.0)), \
        dict(nmax=15, overlap=False, clips=False, thr_scale=50.0)
    yield "zero_voltage_empty", synthetic.tetrode(duration_s=0.1, seed=1, L=31), \
        dict(nmax=5, overlap=False, clips=False, zero_voltage=True)


def main():
    manifest = {}
    for name, rec, opt in cases():
        metrics = rec.fresh_metrics()
        if opt.get("thr_scale"):
            metrics["neuron_lower_thresholds"] = metrics["neuron_lower_thresholds"] * opt["thr_scale"] + 1e4
        if opt.get("one_d"):
            metrics["templates"] = metrics["templates"].reshape(-1)
        if opt.get("zero_voltage"):
            rec.voltage = np.zeros_like(rec.voltage)
        si = rec.sort_info(do_overlap_recheck=opt["overlap"], get_adjusted_clips=opt["clips"])
        maxmem = opt.get("max_gpu_memory")
        (ei, nl, bb, cl), log = R.run_reference(rec.voltage, rec.voltage.dtype, si, metrics,
                                                n_max_shift_inds=opt["nmax"], max_gpu_memory=maxmem,
                                                global_mem_bytes=GLOBAL_MEM)
        L = rec.n_samples_per_chan
        chunk = None
        if maxmem is not None:
            chunk = R.reference_chunk_samples(rec.n_chans, rec.n_templates, L, rec.sampling_rate,
                                              opt["nmax"], GLOBAL_MEM, maxmem)
        empty = isinstance(ei, list)
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"),
            voltage=rec.voltage, templates=np.asarray(metrics["templates"]),
            template_SS=metrics["template_SS"],
            neuron_lower_thresholds=metrics["neuron_lower_thresholds"],
            template_SS_by_chan=metrics["template_SS_by_chan"],
            n_spikes=metrics["n_spikes"],
            sampling_rate=rec.sampling_rate, clip_width=np.asarray(rec.clip_width),
            n_samples_per_chan=L,
            do_overlap_recheck=opt["overlap"], get_adjusted_clips=opt["clips"],
            n_max_shift_inds=-1 if opt["nmax"] is None else opt["nmax"],
            chunk_samples=-1 if chunk is None else chunk,
            empty=empty,
            out_event_indices=np.asarray(ei), out_neuron_labels=np.asarray(nl),
            out_bp_bool=np.asarray(bb), out_adjusted_clips=np.asarray(cl))
        manifest[name] = {"n_spikes": 0 if empty else int(len(ei)),
                          "chunks": sum(1 for l in log.splitlines() if l.startswith("Starting chunk")),
                          "passes": sum(1 for l in log.splitlines() if "secret spikes" in l and l.startswith("Added"))}
        print(name, manifest[name])
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
