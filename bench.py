"""Benchmark: pursuit sample*template/s of Full Binary Pursuit on B200.

One step = one complete binary pursuit (all passes until convergence,
overlap recheck and residuals included) of one synthetic recording segment.
Default workload: the 384-channel high-density probe, 5 min at 30 kHz (9M
samples per channel, int16), 300 templates of 61 samples on 16-channel masks,
Poisson 0.5-100 Hz, n_max_shift_inds = L-1 (the production setting,
full_binary_pursuit.py:145).  The headline value is the tensor-core mode
(bf16 + exact refinement); the same line carries the plain FP32 path on the
same recording (fp32_value, bf16_over_fp32) and whether the two spike trains
are identical.  Inputs are seeded synthetic data: the voltage (13.8 GB as
float32) and the likelihood buffer (10.8 GB) are far larger than L2.
`--workload linear16` runs the 16-channel, 10-minute, 64-template workload.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun, one process per GPU; each rank pursues its own
segment (segments are independent units; no data-path collective), and the
reported value is the total over ranks divided by the slowest rank's time.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "pursuit sample*template/s"
UNIT = "sample*template/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["hd384", "linear16", "tetrode"], default="hd384")
    ap.add_argument("--duration", type=float, default=None,
                    help="override the segment length in seconds (development only)")
    ap.add_argument("--precision", choices=["fp32", "bf16"], default="bf16",
                    help="bf16: 16-bit tensor-core likelihood and overlap tables with exact fp32 refinement "
                         "(results identical to fp32); fp32: exact fp32 pipes only")
    ap.add_argument("--overlap", choices=["fast", "exact"], default="fast")
    ap.add_argument("--tc-layout", choices=["auto", "wide", "samples"], default="auto",
                    help="tensor-core likelihood layout (same spikes): wide tiles of the window stream, "
                         "128-sample tiles, or the library's choice")
    ap.add_argument("--cpu-sample-s", type=float, default=0.05,
                    help="seconds of recording timed on the CPU baseline")
    ap.add_argument("--ref-windows", type=int, default=None,
                    help="windows (of L samples) per step of the reference arm (default: 3 for 384 channels, "
                         "16 otherwise); each step pursues the next slice of the recording")
    ap.add_argument("--fp32-steps", type=int, default=1,
                    help="timed steps of the plain FP32 path reported beside the headline (0: skip)")
    ap.add_argument("--fp32-warmup", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=3, help="steps of the end-to-end measurement")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--mode", choices=["pursuit", "batch", "serve"], default="pursuit",
                    help="pursuit: one segment per step (the headline line); batch: many uneven segments "
                         "sorted concurrently; serve: Poisson request arrivals, p50/p99 latency")
    ap.add_argument("--segments", type=int, default=None,
                    help="batch: segments (default 256); serve: requests (default 48)")
    ap.add_argument("--time-scale", type=float, default=0.05,
                    help="batch/serve: factor on the segment durations of the workload")
    ap.add_argument("--slots", type=int, default=4, help="batch/serve: concurrent requests on the GPU")
    ap.add_argument("--tune", action="store_true",
                    help="batch/serve: tensor-core plan per shape bucket from the tuner (buckets tuned "
                         "before the timed runs, untimed)")
    ap.add_argument("--fp32-segments", type=int, default=0,
                    help="batch/serve: run the plain-FP32 comparison on the first N requests only "
                         "(saturated, no Poisson sweep); 0: all of them")
    ap.add_argument("--rates", default="0.5,0.8,0.95",
                    help="serve: arrival rates as fractions of the measured saturated request rate")
    return ap.parse_args()


def workload(name, duration, seed):
    from spikesorting_fullpursuit_b200 import synthetic
    fn = {"linear16": synthetic.linear16, "tetrode": synthetic.tetrode, "hd384": synthetic.hd384}[name]
    kw = {"seed": seed}
    if duration is not None:
        kw["duration_s"] = duration
    return fn(**kw)


def template_channels(templates, C, L):
    """Mean number of channels a template is non-zero on (C_t)."""
    t = templates.reshape(templates.shape[0], C, L)
    return float(np.mean(np.sum(np.any(t != 0, axis=2), axis=1)))


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        loaded = [x for x in sm if x > 0.5 * (max(mx) if mx else 1)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(rows)}


# DRAM bytes (read + write) per unit of algorithmic work of the tensor-core
# likelihood kernel of each layout, from one ncu capture of pass 1 of a 10 s
# slice of each workload (every window listed; dram__bytes_read.sum +
# dram__bytes_write.sum over sample x templates of the pass); see the
# k_lik_tc* summaries in profiles/.
LIK_TC_DRAM_BYTES_PER_ST = {("hd384_300u", "wide"): 12.23, ("linear16_64u", "wide"): None,
                            ("hd384_300u", "samples"): 11.5, ("linear16_64u", "samples"): None}
LIK_KERNEL = {"wide": "k_lik_tcw", "samples": "k_lik_tc<0>"}


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], d["bf16_tflops"], d["bf16_tflops_sustained"], "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


# ---------------------------------------------------------------- reference arm

def searched_samples(n, L):
    """Samples of the windows the reference searches in a chunk of n samples:
    compute_template_maximum_likelihood skips a window whose end is at or
    past n - L (binary_pursuit.cl:380-383)."""
    W = (n + L - 1) // L
    return sum(min((w + 1) * L, n) - w * L for w in range(W) if (w + 1) * L < n - L)


def run_reference_arm(args, rank, world):
    """The reference's CPU implementation of the path on the host cores: its
    own binary_pursuit() host code (staged unmodified) driving its
    binary_pursuit.cl kernels compiled for the CPU, the kernels whose
    work-items write disjoint outputs (full likelihood, overlap recheck,
    adjusted clips) on all host threads.  Same workload, metric and config as
    our arm; each step pursues the next slice of `--ref-windows` windows of a
    recording of that workload, and its units are the samples of the windows
    the reference searches in the slice (the last two are not searched,
    .cl:380-383) times the templates.  Where the staged package or the
    compiled kernels are missing, the oracle (the reference restated in C)
    stands in, on all host threads."""
    if rank != 0:
        return
    from oracle import oracle as O
    from oracle import reference_harness as RH
    use_ref = RH.available()
    probe = workload(args.workload, 0.01, seed=1)
    L, fs, C, K = probe.n_samples_per_chan, probe.sampling_rate, probe.n_chans, probe.n_templates
    full = workload(args.workload, args.duration, seed=1) if args.duration is not None and args.duration < 5 else None
    full_n = int(round((args.duration if args.duration is not None else
                        {"hd384": 300.0, "linear16": 600.0, "tetrode": 30.0}[args.workload]) * fs))
    nwin = args.ref_windows or (3 if C >= 128 else 16)
    slice_n = nwin * L
    nsteps = args.warmup + args.steps
    # one recording holding every step's slice (same generative model, sizes and seed as our arm)
    # slices start 10 ms in: the synthetic spike trains leave the first and
    # last 5 ms of a recording empty
    lead = int(round(0.01 * fs))
    rec = full if full is not None else workload(args.workload, (lead + nsteps * slice_n) / fs + 0.006, seed=1)
    si = rec.sort_info()
    threads = os.cpu_count() or 1
    note = None
    crashes = [0]

    def one(i, use):
        a = (lead + i * slice_n) % max(1, rec.n_samples - slice_n + 1)
        sl = np.ascontiguousarray(rec.voltage[:, a:a + slice_n])
        if use:
            try:
                RH.run_reference(sl, sl.dtype, si, rec.fresh_metrics(), n_max_shift_inds=L - 1)
            except UnboundLocalError as e:
                # the reference's own failure on a chunk without any overlap
                # candidate: it raises while releasing its buffers, after the
                # pursuit of the chunk has finished (binary_pursuit_parallel.py:750-752)
                if "overlap_group" not in str(e):
                    raise
                crashes[0] += 1
        else:
            O.binary_pursuit_oracle(sl, sl.dtype, si, rec.fresh_metrics(), n_max_shift_inds=L - 1,
                                    nthreads=threads)
        return sl.shape[1]

    if use_ref:
        try:
            one(0, True)
        except Exception as e:           # the staged reference does not run here: the oracle instead
            note = "reference harness failed (%s: %s); oracle port timed instead" % (type(e).__name__, e)
            use_ref = False
    times, units = [], 0
    for i in range(nsteps):
        t0 = time.perf_counter()
        m = one(i, use_ref)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
            units += searched_samples(m, L) * K
    sec = float(sum(times))
    value = units / sec
    sample = ("%d steps, each the next %d-window slice (%d samples, %d of them in windows the reference "
              "searches) of a %s recording (%d ch, %d templates, L=%d, n_max_shift=L-1), all passes; units "
              "= searched samples x templates; %s"
              % (args.steps, nwin, slice_n, searched_samples(slice_n, L), args.workload, C, K, L,
                 "the reference's own binary_pursuit() and binary_pursuit.cl compiled for the CPU, "
                 "independent work-items on %d threads" % threads
                 if use_ref else "the oracle (C restatement of the reference) on %d threads" % threads))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3 / max(1, len(times)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": probe.name, "n_chans": C, "n_samples": full_n, "n_templates": K,
                       "template_len": L, "n_max_shift": L - 1},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                             "kind": "reference" if use_ref else "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if crashes[0]:
        line["reference_cleanup_errors"] = ("%d slices ended with the reference's UnboundLocalError at buffer "
                                            "release (no overlap candidate in the chunk), after their pursuit "
                                            "finished; their time is counted" % crashes[0])
    if note:
        line["note"] = note
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- batch / serve

def _make_segment(spec_dict):
    from spikesorting_fullpursuit_b200 import synthetic
    rec = synthetic.SegmentSpec(**spec_dict).make()
    return (np.ascontiguousarray(rec.voltage), rec.sort_info(), rec.fresh_metrics(),
            rec.n_samples_per_chan - 1)


def make_segments(specs):
    """Generate the segments on the host cores (spawned workers, before any
    CUDA call of this process)."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    workers = max(1, min(len(specs), os.cpu_count() or 1))
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_make_segment, [sp.as_dict() for sp in specs], chunksize=1))


def _same(a, b):
    if isinstance(a[0], list) or isinstance(b[0], list):
        return len(a[0]) == len(b[0]) == 0
    return np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def run_mix(args):
    """Batched sorting (uneven segments, all submitted at once) or serving
    (Poisson arrivals at rates swept up to the saturated rate) through the
    continuous-batching server; bf16+refine and plain fp32 side by side.
    Every request's spikes are compared across precisions and runs."""
    from spikesorting_fullpursuit_b200 import synthetic
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        # one server per GPU; several GPUs take shares of the segments with
        # parallel.distributed instead
        if rank == 0:
            print(json.dumps({"mode": args.mode, "unavailable": "batch and serve modes run on one GPU"}),
                  flush=True)
        return
    serve = args.mode == "serve"
    nseg = args.segments or (48 if serve else 256)
    specs = (synthetic.serve_mix(nseg, seed=4 + rank, time_scale=args.time_scale) if serve else
             synthetic.batch_mix(nseg, seed=3 + rank, time_scale=args.time_scale))
    t_gen = time.perf_counter()
    segs = make_segments(specs)
    t_gen = time.perf_counter() - t_gen

    import torch
    from spikesorting_fullpursuit_b200 import build as B
    from spikesorting_fullpursuit_b200.serving import PursuitServer, drive, latency_summary, poisson_arrivals
    if B.needs_build():
        B.build()
    torch.cuda.set_device(local)
    units = float(sum(sp.units for sp in specs))
    tuned = None
    if args.tune:
        # one timed trial per shape bucket, before (and outside) the timed runs
        from spikesorting_fullpursuit_b200 import autotune
        t_tune = time.perf_counter()
        seen = {}
        for (v, si, m, nmax) in segs:
            L = int(si["n_samples_per_chan"])
            b = autotune.shape_bucket(v.shape[0], m["templates"], L)
            if b not in seen:
                seen[b] = autotune.tune(v, m["templates"], np.float32(-0.5 * m["template_SS"]), L)[0]
        tuned = {"buckets": len(seen), "plans": seen, "tuning_s": time.perf_counter() - t_tune}
    clocks = ClockSampler(local)
    out = {}
    reference_outputs = None
    identical = True
    clocks.start()
    for prec in ("bf16", "fp32"):
        # the plain-FP32 comparison may run on the first --fp32-segments
        # requests only (a bounded call); its spikes are checked against the
        # same requests of the bf16 run
        run_segs = segs if (prec == "bf16" or not args.fp32_segments) else segs[: args.fp32_segments]
        with PursuitServer(slots=args.slots, precision=prec, overlap=args.overlap,
                           tune=bool(args.tune) and prec == "bf16") as srv:
            drive(srv, run_segs[: 2 * args.slots])                    # warm-up (untimed)
            torch.cuda.synchronize()
            res, wall = drive(srv, run_segs)                            # saturated: all at once
            torch.cuda.synchronize()
            summ = latency_summary(res, wall)
            summ.update({"wall_s": wall, "requests_per_s": len(res) / wall, "max_running": srv.max_running,
                         "max_hbm_in_use_gb": srv.max_in_use / 1e9, "hbm_budget_gb": srv.hbm_budget / 1e9})
            outs = [r.outputs for r in res]
            if reference_outputs is None:
                reference_outputs = outs
            identical &= all(_same(a, b) for a, b in zip(outs, reference_outputs))
            entry = {"saturated": summ}
            if prec == "bf16" and args.fp32_segments:
                # the same subset the FP32 run takes, for a like-for-like ratio
                rs, ws_ = drive(srv, segs[: args.fp32_segments])
                torch.cuda.synchronize()
                entry["saturated_fp32_subset"] = latency_summary(rs, ws_)
            if serve and (prec == "bf16" or not args.fp32_segments):
                sweep = []
                cap = len(res) / wall
                for j, frac in enumerate(float(x) for x in args.rates.split(",")):
                    arr = poisson_arrivals(frac * cap, len(run_segs), seed=100 + j)
                    r2, w2 = drive(srv, run_segs, arr)
                    torch.cuda.synchronize()
                    s2 = latency_summary(r2, w2)
                    s2.update({"rate_fraction": frac, "rate_per_s": frac * cap, "max_running": srv.max_running})
                    identical &= all(_same(a.outputs, b) for a, b in zip(r2, reference_outputs))
                    sweep.append(s2)
                entry["poisson"] = sweep
            out[prec] = entry
    clock_info = clocks.stop()
    bf, fp = out["bf16"]["saturated"], out["fp32"]["saturated"]
    line = {"metric": ("serving p50/p99 segment latency vs pursuit sample*template/s" if serve
                       else "batched pursuit sample*template/s"),
            "value": bf["throughput"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
            "fp32_value": fp["throughput"],
            "bf16_over_fp32": (out["bf16"].get("saturated_fp32_subset", bf)["throughput"] / fp["throughput"]),
            "fp32_requests": fp["requests"], "tuned": tuned,
            "spikes_identical_bf16_fp32_and_across_runs": bool(identical),
            "data": "synthetic (seeded per request)",
            "config": {"workload": "serve_mix" if serve else "batch_mix", "requests": nseg,
                       "time_scale": args.time_scale, "slots": args.slots, "overlap": args.overlap,
                       "n_max_shift": "L-1", "units": units,
                       "channels": [min(sp.n_chans for sp in specs), max(sp.n_chans for sp in specs)],
                       "templates": [min(sp.n_templates for sp in specs), max(sp.n_templates for sp in specs)],
                       "durations_s": [min(sp.duration_s for sp in specs), max(sp.duration_s for sp in specs)],
                       "generation_s": t_gen,
                       "timing": "wall clock from first arrival to last completion, GPU synchronised; "
                                 "host voltage copied to the device inside each request"},
            "bf16": out["bf16"], "fp32": out["fp32"], "clocks": clock_info}
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm

def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.mode != "pursuit":
        run_mix(args)
        return

    import torch
    import torch.distributed as dist
    from spikesorting_fullpursuit_b200 import _lib, binary_pursuit
    from spikesorting_fullpursuit_b200 import build as B
    from spikesorting_fullpursuit_b200.parallel.distributed import max_over_ranks

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=dev)
    lib = _lib.lib() if not B.needs_build() else (B.build(), _lib.lib())[1]
    # every pursuit this thread runs (timed steps, fp32 arm, end to end)
    _lib.check(lib.fbp_set_tc_layout({"auto": _lib.TC_LAYOUT_AUTO, "wide": _lib.TC_LAYOUT_WIDE,
                                      "samples": _lib.TC_LAYOUT_SAMPLES}[args.tc_layout]))

    t_gen = time.perf_counter()
    rec = workload(args.workload, args.duration, seed=1 + rank)
    t_gen = time.perf_counter() - t_gen
    C, n, K, L = rec.n_chans, rec.n_samples, rec.n_templates, rec.n_samples_per_chan
    nmax = L - 1
    prec = 0 if args.precision == "fp32" else 1
    metrics = rec.fresh_metrics()
    T = np.ascontiguousarray(np.float32(metrics["templates"]).reshape(-1))
    tss = np.ascontiguousarray(np.float32(-0.5 * metrics["template_SS"]))
    thr = np.ascontiguousarray(np.float32(metrics["neuron_lower_thresholds"]))
    stream = torch.cuda.current_stream(dev)
    sp = _lib.stream_ptr(stream)
    pristine = torch.from_numpy(np.ascontiguousarray(rec.voltage)).to(dev).to(torch.float32)
    v = torch.empty_like(pristine)
    T_d, tss_d, thr_d = (torch.from_numpy(x).to(dev) for x in (T, tss, thr))
    W = (n + L - 1) // L
    cap = 16 * W + 4096
    out_i = torch.empty(cap, dtype=torch.int32, device=dev)
    out_l = torch.empty(cap, dtype=torch.int32, device=dev)
    last = {}

    def workspace(p):
        wsb = ctypes.c_size_t(0)
        _lib.check(lib.fbp_pursuit_workspace_bytes(n, C, K, L, nmax, p, ctypes.byref(wsb)))
        return torch.empty(wsb.value, dtype=torch.uint8, device=dev)

    def step(profile, p, ws):
        v.copy_(pristine)
        nspk, npass = ctypes.c_uint32(0), ctypes.c_uint32(0)
        st = _lib.StageStats()
        _lib.check(lib.fbp_pursuit_chunk(
            _lib.ptr(v), n, C, _lib.ptr(T_d), K, L, _lib.ptr(tss_d), _lib.ptr(thr_d), nmax, 1, p,
            0 if args.overlap == "fast" else 1, 1000000, _lib.ptr(ws), ws.numel(), _lib.ptr(out_i),
            _lib.ptr(out_l), cap, None, ctypes.byref(nspk), ctypes.byref(npass), int(profile), ctypes.byref(st),
            sp))
        last["n"] = int(nspk.value)
        return st

    def spikes_of_last_step():
        m = last["n"]
        return out_i[:m].cpu().numpy().copy(), out_l[:m].cpu().numpy().copy()

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(p, ws, warmup, steps, sampler=None):
        """Device time per step (max over ranks) of `steps` graph-mode steps after `warmup`."""
        for _ in range(warmup):
            step(False, p, ws)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            step(False, p, ws)
        ev1.record(stream)
        torch.cuda.synchronize()
        info = sampler.stop() if sampler else None
        barrier()
        return max_over_ranks(ev0.elapsed_time(ev1), device=dev) / steps, info

    # ---- headline: the requested precision, W warm-up and K timed steps
    ws = workspace(prec)
    clocks = ClockSampler(local)
    ms_step, clock_info = timed(prec, ws, args.warmup, args.steps, clocks)
    units_per_step = world * n * K
    value = units_per_step / (ms_step / 1e3)
    spikes_main = spikes_of_last_step()

    # one more step with CUDA events around every stage (outside the timed
    # region): the per-stage times, work and launches of a step
    st_prof = step(True, prec, ws)
    torch.cuda.synchronize()
    stage_ms = np.array(st_prof.ms[:])
    work = np.array(st_prof.work[:], dtype=np.float64)
    launches = np.array(st_prof.launches[:], dtype=np.float64)
    Ct = template_channels(T.reshape(K, -1), C, L)
    S_sh = 2 * nmax + 1
    hbm, tf_burst, tf_sust, peak_src = measured_peaks()
    cands = float(st_prof.candidates)
    # stage: (bound, algorithmic flops or bytes of the stage per step)
    alg_of = {
        0: ("tensor", work[0] * 2.0 * Ct * L),          # likelihood: 2*C_t*L flops per sample*template
        8: ("tensor", cands * 2.0 * Ct * L * K * S_sh),  # overlap tables: C_t*L MACs per (template, shift)
        1: ("hbm", work[1] / 3.0 * 4.0),                # argmax: each likelihood entry of a listed window once
        2: ("hbm", cands * 8.0 * K * S_sh),             # overlap search: tables and likelihood signs per candidate
        5: ("hbm", work[5] * 8.0 * Ct * L),             # residual: read and write C_t*L fp32 per spike
    }
    per_stage = {}
    for i, (bound, alg) in alg_of.items():
        secs = stage_ms[i] / 1e3
        if secs <= 0 or alg <= 0:
            continue
        if bound == "tensor":
            ach, peak, unit = alg / secs / 1e12, tf_sust, "TFLOP/s"
        else:
            ach, peak, unit = alg / secs / 1e9, hbm, "GB/s"
        per_stage[_lib.STAGE_NAMES[i]] = {"bound": bound, "achieved": ach, "peak": peak, "unit": unit,
                                          "frac": ach / peak if peak else None, "ms": stage_ms[i]}
        if i == 1:
            # the argmax reads only the templates whose per-window upper bound
            # reaches the window's best lower bound: its bytes here are the
            # reference's (every entry once), so the ratio to the HBM peak is
            # not a bandwidth fraction
            per_stage[_lib.STAGE_NAMES[i]].update({"frac": None, "achieved_kind": "reference-equivalent bytes"})
        if i == 2:
            # the reference's own work unit for the overlap recheck: 5*C_t*L
            # flops per (a, b, t) item that survives its skip rules
            per_stage["overlap"]["surviving_items"] = float(work[2])
            per_stage["overlap"]["reference_equivalent_tflops"] = work[2] * 5.0 * Ct * L / secs / 1e12
    dom = max((k for k in per_stage if per_stage[k]["frac"] is not None), key=lambda k: per_stage[k]["ms"])
    d = per_stage[dom]
    traffic = None
    layout = {1: "samples", 2: "wide"}.get(int(st_prof.tc_layout))
    per_st = LIK_TC_DRAM_BYTES_PER_ST.get((rec.name, layout))
    if dom == "likelihood" and prec == 1 and per_st:
        # algorithmic: every listed sample's voltage read once (4 C bytes,
        # shared by the K templates) and 4 + 1 bytes written per entry
        traffic = {"bytes_per_step": per_st * float(work[0]),
                   "algorithmic_bytes_per_step": float(work[0]) * (5.0 + 4.0 * C / K),
                   "source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of %s, pass 1 of a 10 s "
                             "slice (every window), per sample*template, times the step's sample*templates"
                             % LIK_KERNEL[layout]}
    roofline = {"bound": d["bound"], "achieved": d["achieved"], "peak": d["peak"], "unit": d["unit"],
                "frac": d["frac"], "traffic": traffic, "kernel": dom,
                "peak_source": peak_src + (" sustained" if d["bound"] == "tensor" else ""),
                "stages": per_stage,
                "stage_ms_per_step": {_lib.STAGE_NAMES[i]: stage_ms[i] for i in range(_lib.N_STAGES)}}
    gpu_launches = int(launches.sum()) * args.steps

    # ---- the plain FP32 path on the same recording (the north star's
    # denominator): its throughput and whether its spike train is the same
    fp32 = None
    if prec != 0 and args.fp32_steps > 0:
        del ws
        torch.cuda.empty_cache()
        ws32 = workspace(0)
        ms32, _ = timed(0, ws32, args.fp32_warmup, args.fp32_steps)
        spikes32 = spikes_of_last_step()
        del ws32
        torch.cuda.empty_cache()
        same = (spikes32[0].shape == spikes_main[0].shape and np.array_equal(spikes32[0], spikes_main[0])
                and np.array_equal(spikes32[1], spikes_main[1]))
        same = bool(max_over_ranks(0.0 if same else 1.0, device=dev) == 0.0)
        fp32 = {"value": units_per_step / (ms32 / 1e3), "ms_per_step": ms32, "steps": args.fp32_steps,
                "warmup": args.fp32_warmup, "spikes": int(spikes32[0].size)}
        ws = workspace(prec)

    # end to end through the public API: host voltage (pinned) -> spikes on the host
    e2e = None
    if not args.no_e2e:
        pinned = torch.empty(rec.voltage.shape, dtype=torch.from_numpy(rec.voltage[:1, :1]).dtype).pin_memory()
        pinned.numpy()[...] = rec.voltage
        host_v = pinned.numpy()
        si = rec.sort_info()
        del ws, v
        torch.cuda.empty_cache()
        binary_pursuit(host_v, host_v.dtype, si, rec.fresh_metrics(), n_max_shift_inds=nmax,
                       precision=args.precision, overlap=args.overlap)
        barrier()
        e_times = []
        d2h = 0
        nsteps_e2e = max(1, min(args.steps, args.e2e_steps))
        for _ in range(nsteps_e2e):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = binary_pursuit(host_v, host_v.dtype, si, rec.fresh_metrics(), n_max_shift_inds=nmax,
                                 precision=args.precision, overlap=args.overlap)
            e_times.append(time.perf_counter() - t0)
            d2h = 8 * len(out[0])
        te = max_over_ranks(float(np.mean(e_times)), device=dev)
        e2e = {"value": units_per_step / te, "unit": UNIT,
               "h2d_bytes_per_step": int(host_v.nbytes + T.nbytes + tss.nbytes + thr.nbytes),
               "d2h_bytes_per_step": int(d2h), "steps": nsteps_e2e,
               "timing": "host clock around binary_pursuit() from pinned host voltage to int64 spike "
                         "arrays on the host, GPU synchronised"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as O
        sample_s = args.cpu_sample_s
        m = int(round(sample_s * rec.sampling_rate))
        sl = np.ascontiguousarray(rec.voltage[:, :m])
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        O.binary_pursuit_oracle(sl, sl.dtype, rec.sort_info(), rec.fresh_metrics(), n_max_shift_inds=nmax,
                                nthreads=threads)
        dt = time.perf_counter() - t0
        cpu = {"value": m * K / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": "first %.3f s (%d samples) of the same recording, all passes, the oracle (the "
                         "reference restated in C, zero template rows skipped) on %d threads"
                         % (sample_s, m, threads)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if args.precision == "fp32" else "f16-tc+f32",
                "data": "synthetic (seeded; one independent segment per rank)",
                "config": {"workload": rec.name, "n_chans": C, "n_samples": n, "n_templates": K,
                           "template_len": L, "n_max_shift": nmax, "precision": args.precision,
                           "overlap": args.overlap, "voltage_dtype": str(rec.voltage.dtype),
                           "tc_layout": {1: "samples", 2: "wide"}.get(int(st_prof.tc_layout)),
                           "l2": "inputs larger than L2 (voltage %.2f GB, likelihood %.2f GB)"
                                 % (C * n * 4 / 1e9, K * n * 4 / 1e9),
                           "passes": int(st_prof.passes), "spikes": int(st_prof.spikes),
                           "overlap_candidates": int(st_prof.candidates),
                           "overlap_surviving_items": int(st_prof.work[2]),
                           "overlap_refined_items": int(st_prof.refined_items),
                           "overlap_fallback_candidates": int(st_prof.fallback_candidates),
                           "likelihood_refined": int(st_prof.lik_refined),
                           "likelihood_lazy_refined": int(st_prof.lik_lazy_refined),
                           "likelihood_seq_refined": int(st_prof.lik_seq_refined),
                           "likelihood_exact_passes": int(st_prof.lik_exact_passes),
                           "generation_s": t_gen,
                           "parallelism": "segment-parallel x%d" % world},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": gpu_launches,
                "clocks": clock_info}
        if fp32 is not None:
            line["fp32_value"] = fp32["value"]
            line["fp32"] = fp32
            line["bf16_over_fp32"] = value / fp32["value"]
            line["spikes_identical"] = same
            # every decision reads the reference's binary32 value or an
            # interval that cannot cross the threshold: the margin band is empty
            line["margin_band"] = {
                "epsilon": 0.0, "in_band_events": 0,
                "entries_in_tensor_core_band": int(st_prof.lik_refined),
                "note": "likelihood entries whose tensor-core interval contained 0 were re-evaluated "
                        "(double interval, else the reference's own sum) before any decision read them"}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
