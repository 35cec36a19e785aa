"""Continuous-batching pursuit server on one GPU (segment-sorting requests).

Requests arrive at any time; each is one recording segment with its own
channels, length and templates, pursued exactly as `binary_pursuit()` does
(same result alone or in the mix: the kernels are deterministic and a
request's buffers are its own).  The server runs up to `slots` requests at
once, each on its own CUDA stream and host thread, so their kernels overlap
on the device while every request's residual, window state and spike lists
stay resident in HBM across its pursuit passes.  A request is admitted, in
arrival order, when a slot is free and its HBM footprint (voltage chunk,
pursuit workspace, spike buffers, templates) fits in what the running
requests leave of the budget; a request larger than the whole budget runs
alone.

    server = PursuitServer(slots=4)
    fut = server.submit(voltage, sort_info, separability_metrics, n_max_shift_inds=L - 1)
    result = fut.result()        # Completed: .outputs (the 4-tuple), .latency_s, ...
    server.close()

`sort_batch()` sorts a list of segments through the same server and returns
the results in input order.
"""
import collections
import concurrent.futures
import threading
import time

import numpy as np

from .parallel.binary_pursuit_parallel import binary_pursuit
from .parallel.chunking import chunk_footprint_bytes, num_indices_per_chunk


class Completed:
    """One finished request: the pursuit outputs and its timing."""

    __slots__ = ("outputs", "arrival_s", "start_s", "end_s", "footprint", "units", "slot")

    def __init__(self, outputs, arrival_s, start_s, end_s, footprint, units, slot):
        self.outputs = outputs          # (indices, labels, bp_bool, clips) as binary_pursuit()
        self.arrival_s = arrival_s      # perf_counter() times
        self.start_s = start_s
        self.end_s = end_s
        self.footprint = footprint      # admitted HBM bytes
        self.units = units              # samples x templates of the segment
        self.slot = slot

    @property
    def latency_s(self):
        """Arrival to completion (queueing included)."""
        return self.end_s - self.arrival_s

    @property
    def service_s(self):
        return self.end_s - self.start_s


class _Request:
    __slots__ = ("args", "footprint", "units", "arrival_s", "future")

    def __init__(self, args, footprint, units, arrival_s):
        self.args = args
        self.footprint = footprint
        self.units = units
        self.arrival_s = arrival_s
        self.future = concurrent.futures.Future()


def request_footprint(voltage, sort_info, separability_metrics, n_max_shift_inds=None, precision="bf16",
                      overlap="fast", chunk_samples=None, total_mem=None, max_gpu_memory=None):
    """HBM bytes one request holds while it runs (its largest chunk), as the
    chunk planner counts them (parallel.chunking.chunk_footprint_bytes): the
    library's workspace (`fbp_pursuit_workspace_bytes`), the voltage chunk,
    the spike buffers sized as `binary_pursuit()` sizes them, the templates
    and thresholds."""
    C, n_total = int(voltage.shape[0]), int(voltage.shape[1])
    L = int(sort_info['n_samples_per_chan'])
    templates = np.asarray(separability_metrics['templates'])
    K = 1 if templates.ndim == 1 else int(templates.shape[0])
    if n_max_shift_inds is None or n_max_shift_inds < 0:
        n_max_shift_inds = L // 2
    prec = 0 if precision == "fp32" else 1
    if chunk_samples is None:
        if total_mem is None:
            import torch
            total_mem = torch.cuda.get_device_properties(torch.cuda.current_device()).total_memory
        chunk_samples = num_indices_per_chunk(C, K, L, sort_info['sampling_rate'], total_mem, max_gpu_memory,
                                              n_max_shift=int(n_max_shift_inds), precision=prec,
                                              v_itemsize=np.dtype(voltage.dtype).itemsize,
                                              adjusted_clips=bool(sort_info['get_adjusted_clips']))
    n = min(n_total, int(chunk_samples))
    return chunk_footprint_bytes(n, C, K, L, int(n_max_shift_inds), prec, np.dtype(voltage.dtype).itemsize,
                                 bool(sort_info['get_adjusted_clips']))


class AdmissionScheduler:
    """FIFO admission of jobs into `slots` worker threads under a byte budget.

    `run(job, slot)` does one job on the calling worker thread; `worker_init(slot)`
    runs once per worker before its first job (the GPU server makes the
    worker's CUDA stream there).  The head job starts when a worker is free
    and its footprint fits in what the running jobs leave of `budget`, or
    when nothing runs (a job larger than the budget runs alone).  Jobs
    start in submission order."""

    def __init__(self, slots, budget, run, worker_init=None):
        if slots < 1:
            raise ValueError("slots must be >= 1")
        self.budget = int(budget)
        self._run = run
        self._init = worker_init
        self._cv = threading.Condition()
        self._queue = collections.deque()
        self._in_use = 0
        self._running = 0
        self._closed = False
        self.max_running = 0            # largest number of jobs seen running at once
        self.max_in_use = 0             # largest admitted footprint at once
        self._workers = [threading.Thread(target=self._work, args=(i,), daemon=True) for i in range(slots)]
        for t in self._workers:
            t.start()

    def submit(self, job, footprint, units=0):
        """Queue `job`; returns a Future of `Completed` (its `outputs` are what
        `run` returned) or of the exception `run` raised.  Cancelling the
        future before the job starts removes it from the queue."""
        req = _Request(job, int(footprint), int(units), time.perf_counter())
        with self._cv:
            if self._closed:
                raise RuntimeError("server is closed")
            self._queue.append(req)
            self._cv.notify_all()
        return req.future

    def close(self, wait=True):
        """Stop accepting jobs; the queued ones still run."""
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        if wait:
            for t in self._workers:
                t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _admissible(self):
        # a request cancelled while it waited (Future.cancel()) leaves the queue unrun
        while self._queue and self._queue[0].future.cancelled():
            self._queue.popleft()
        if not self._queue:
            return False
        head = self._queue[0]
        return self._running == 0 or self._in_use + head.footprint <= self.budget

    def _work(self, slot):
        if self._init is not None:
            self._init(slot)
        while True:
            with self._cv:
                while not self._admissible():
                    if self._closed and not self._queue:
                        return
                    self._cv.wait()
                req = self._queue.popleft()
                if not req.future.set_running_or_notify_cancel():
                    continue                    # cancelled between the check and now
                self._in_use += req.footprint
                self._running += 1
                self.max_running = max(self.max_running, self._running)
                self.max_in_use = max(self.max_in_use, self._in_use)
            start = time.perf_counter()
            try:
                out = self._run(req.args, slot)
                end = time.perf_counter()
                req.future.set_result(Completed(out, req.arrival_s, start, end, req.footprint, req.units, slot))
            except BaseException as e:          # the job fails, the workers keep serving
                req.future.set_exception(e)
            finally:
                with self._cv:
                    self._in_use -= req.footprint
                    self._running -= 1
                    self._cv.notify_all()


class PursuitServer:
    """Admits pursuit requests by HBM footprint into `slots` concurrent CUDA
    streams.  `hbm_budget` defaults to 80 % of the device's free memory when
    the server starts."""

    def __init__(self, slots=4, hbm_budget=None, device=None, precision="bf16", overlap="fast", tune=False):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("No GPU available")
        self.device = torch.cuda.current_device() if device is None else int(device)
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(0.8 * free)
        self.precision = precision
        self.overlap = overlap
        self.tune = tune                # tensor-core group size from the tuner's cache per shape bucket
        self.total_mem = torch.cuda.get_device_properties(self.device).total_memory
        self._streams = [None] * slots
        self._sched = AdmissionScheduler(slots, hbm_budget, self._run, self._init_worker)

    @property
    def hbm_budget(self):
        return self._sched.budget

    @property
    def max_running(self):
        return self._sched.max_running

    @property
    def max_in_use(self):
        return self._sched.max_in_use

    def submit(self, voltage, sort_info, separability_metrics, n_max_shift_inds=None, **kwargs):
        """Queue one segment; returns a Future of `Completed` whose `outputs`
        is `binary_pursuit()`'s 4-tuple.  Keyword arguments are those of
        `binary_pursuit()` (precision and overlap default to the server's).
        Like `binary_pursuit()`, the call adds 'n_spikes' to
        `separability_metrics`: give concurrent requests their own dicts."""
        kwargs.setdefault("precision", self.precision)
        kwargs.setdefault("overlap", self.overlap)
        kwargs.setdefault("device", self.device)
        kwargs.setdefault("tune", self.tune)
        fp = request_footprint(voltage, sort_info, separability_metrics, n_max_shift_inds,
                               kwargs["precision"], kwargs["overlap"], kwargs.get("chunk_samples"),
                               self.total_mem, kwargs.get("max_gpu_memory"))
        templates = np.asarray(separability_metrics['templates'])
        K = 1 if templates.ndim == 1 else int(templates.shape[0])
        job = ((voltage, voltage.dtype, sort_info, separability_metrics),
               dict(kwargs, n_max_shift_inds=n_max_shift_inds))
        return self._sched.submit(job, fp, int(voltage.shape[1]) * K)

    def close(self, wait=True):
        self._sched.close(wait)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _init_worker(self, slot):
        import torch
        torch.cuda.set_device(self.device)
        self._streams[slot] = torch.cuda.Stream(self.device)

    def _run(self, job, slot):
        import torch
        args, kwargs = job
        stream = self._streams[slot]
        with torch.cuda.stream(stream):
            out = binary_pursuit(*args, **kwargs)
        stream.synchronize()
        return out


def sort_batch(segments, slots=4, **kwargs):
    """Pursue many segments concurrently (all submitted at once).

    `segments` is a list of (voltage, sort_info, separability_metrics,
    n_max_shift_inds) tuples; returns the `Completed` results in input order."""
    with PursuitServer(slots=slots, **{k: kwargs.pop(k) for k in ("hbm_budget", "device", "precision", "overlap")
                                       if k in kwargs}) as srv:
        futs = [srv.submit(v, si, m, nmax, **kwargs) for (v, si, m, nmax) in segments]
        return [f.result() for f in futs]


def latency_summary(results, wall_s):
    """p50 / p99 latency (s) and whole-run throughput (sample*template/s)."""
    lat = np.array([r.latency_s for r in results])
    units = float(sum(r.units for r in results))
    return {"requests": len(results), "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
            "throughput": units / wall_s if wall_s > 0 else 0.0}


def poisson_arrivals(rate_per_s, n, seed=0):
    """Arrival offsets (s) of `n` requests of a Poisson process."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.cumsum(rng.exponential(1.0 / rate_per_s, size=n))


def drive(server, requests, arrivals=None):
    """Submit `requests` ((voltage, sort_info, separability_metrics,
    n_max_shift_inds) tuples) to `server` at the offsets `arrivals` (s from
    now; None submits all at once) and wait for all of them.  Returns the
    `Completed` results in request order and the wall time from the first
    arrival to the last completion."""
    t0 = time.perf_counter()
    futs = []
    for i, (v, si, m, nmax) in enumerate(requests):
        if arrivals is not None:
            delay = t0 + float(arrivals[i]) - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
        futs.append(server.submit(v, si, dict(m), nmax))
    res = [f.result() for f in futs]
    first = min(r.arrival_s for r in res)
    last = max(r.end_s for r in res)
    return res, last - first
