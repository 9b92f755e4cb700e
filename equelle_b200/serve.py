"""Many simulator instances on one GPU: batched runs and a serving loop.

Each request is one generated-style simulation: an implicit heat case or a
2D fully implicit two-phase case, with its own grid, inputs and number of
time steps.  A request runs on its own runtime, whose kernels go to its own
CUDA stream, driven by its own host thread (the simulator call releases the
interpreter lock), so requests that are on the GPU at the same time overlap
there: the small grids of the mix leave most of the B200 idle when run one
at a time.  Results do not depend on what else runs: every kernel is
deterministic, so a request's fields are bit-identical alone and in a mix.

Admission: a request that has arrived starts when a slot (host thread) is
free and its estimated device memory fits under the cap, in arrival order.
"""
import concurrent.futures as cf
import math
import os
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import cases, simrun

# Device bytes per cell, measured peaks with margin (2D two-phase: 2
# unknowns with 2x2 blocks and a multigrid hierarchy; heat: 1 unknown), and
# a fixed cost per runtime (grid, caches, graphs).
BYTES_PER_CELL = {"twophase": 6000, "heateq": 2500}
BYTES_PER_RUNTIME = 64 << 20


@dataclass
class Request:
    rid: int
    program: str           # "heateq" or "twophase"
    nx: int
    ny: int
    steps: int
    seed: int
    arrival: float = 0.0   # seconds after the start of the run
    args: list = field(default_factory=list)
    workdir: str = ""

    @property
    def cells(self):
        return self.nx * self.ny

    def estimate_bytes(self):
        return BYTES_PER_RUNTIME + BYTES_PER_CELL[self.program] * self.cells


@dataclass
class Record:
    rid: int
    program: str
    cells: int
    steps: int
    arrival: float
    start: float
    finish: float
    error: str = ""
    device_bytes_peak: int = 0

    @property
    def latency(self):
        return self.finish - self.arrival

    @property
    def wait(self):
        return self.start - self.arrival


def make_requests(count, seed=0, rate=None, programs=("heateq", "twophase"), side=(64, 1024),
                  steps=(10, 100)):
    """Seeded requests: program chosen uniformly from `programs`, square
    grids with a side log-uniform in `side`, steps uniform in `steps`
    (inclusive), Poisson arrivals at `rate` per second (all at 0 when rate
    is None)."""
    rng = np.random.default_rng(seed)
    arrivals = np.random.default_rng([seed, 1])  # the same requests at every rate
    out = []
    t = 0.0
    for i in range(count):
        prog = programs[int(rng.integers(0, len(programs)))]
        s = int(round(math.exp(rng.uniform(math.log(side[0]), math.log(side[1])))))
        k = int(rng.integers(steps[0], steps[1] + 1))
        if rate:
            t += float(arrivals.exponential(1.0 / rate))
        out.append(Request(rid=i, program=prog, nx=s, ny=s, steps=k, seed=int(rng.integers(0, 2**31)),
                           arrival=t if rate else 0.0))
    return out


def prepare(req, root, extra=()):
    """Writes the request's input files under `root` and sets its args."""
    d = os.path.join(root, "req%05d" % req.rid)
    if req.program == "twophase":
        args = cases.two_phase(d, req.nx, req.ny, None, steps=req.steps, seed=req.seed, corr_len=4.0)
        args += ["abs_res_tol=1e-8", "linsolver_residual_tolerance=1e-8", "linsolver_max_iterations=5000"]
    else:
        args = cases.heat(d, req.nx, req.ny, steps=req.steps, seed=req.seed)
    req.args = args + list(extra)
    req.workdir = d
    return req


class Server:
    """Runs requests with at most `slots` at once and their estimated device
    memory under `memory_cap` bytes."""

    def __init__(self, slots=16, memory_cap=150 << 30, host_threads=None, output_values="none"):
        self.slots = slots
        self.memory_cap = memory_cap
        ncpu = os.cpu_count() or 1
        self.host_threads = host_threads or max(1, ncpu // max(slots, 1))
        self.output_values = output_values

    def _run_one(self, req, t0):
        start = time.perf_counter() - t0
        args = req.args + ["output_values=%s" % self.output_values, "host_threads=%d" % self.host_threads]
        if self.output_values == "last":
            args.append("output_dir=%s/" % req.workdir)
        err = ""
        peak = 0
        try:
            rep = simrun.run(req.program, args, allow_failure=True)
            err = rep.error.decode()
            peak = rep.stats.device_bytes_peak
        except Exception as e:  # a failed request is reported, the others go on
            err = str(e)
        return Record(req.rid, req.program, req.cells, req.steps, req.arrival, start,
                      time.perf_counter() - t0, err, peak)

    def run(self, requests, realtime=True):
        """Runs every request; with `realtime`, requests become eligible at
        their arrival times.  Returns the records in completion order and
        the wall time."""
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        in_use = 0
        running = {}
        records = []
        cond = threading.Condition()
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(max_workers=self.slots) as pool:
            while pending or running:
                now = time.perf_counter() - t0
                # admit in arrival order while a slot and memory are free
                while pending and len(running) < self.slots:
                    req = pending[0]
                    if realtime and req.arrival > now:
                        break
                    need = req.estimate_bytes()
                    if running and in_use + need > self.memory_cap:
                        break
                    pending.pop(0)
                    in_use += need
                    fut = pool.submit(self._run_one, req, t0)
                    fut.add_done_callback(lambda _f: _notify(cond))
                    running[fut] = need
                done = [f for f in running if f.done()]
                for f in done:
                    in_use -= running.pop(f)
                    records.append(f.result())
                if done:
                    continue
                wait = None
                if pending and realtime and len(running) < self.slots:
                    wait = max(0.0, pending[0].arrival - (time.perf_counter() - t0))
                with cond:
                    if not any(f.done() for f in running):
                        cond.wait(timeout=wait if wait is not None else 0.05)
        return records, time.perf_counter() - t0


def _notify(cond):
    with cond:
        cond.notify_all()


def percentile(values, q):
    if not values:
        return float("nan")
    return float(np.percentile(np.asarray(values), q))


def last_fields(req):
    """The final fields a request wrote with output_values=last."""
    tags = ("pressure", "saturation") if req.program == "twophase" else ("u",)
    out = []
    for tag in tags:
        path = os.path.join(req.workdir, "%s-last.output" % tag)
        out.append(np.loadtxt(path) if os.path.exists(path) else None)
    return out
