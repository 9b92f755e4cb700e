"""Many instances on one GPU (equelle_b200/serve.py): the scheduler's
admission rules on the CPU with a stand-in runner, and on the GPU that
every request's fields are the same alone and in a concurrent mix."""
import threading
import time

import numpy as np
import pytest

from equelle_b200 import serve


class _Recorder(serve.Server):
    """Runs no simulator: sleeps in proportion to the steps and records how
    many requests and how many estimated bytes were running at once."""

    def __init__(self, *a, **k):
        super().__init__(*a, **k)
        self.lock = threading.Lock()
        self.now = 0
        self.now_bytes = 0
        self.max_running = 0
        self.max_bytes = 0

    def _run_one(self, req, t0):
        with self.lock:
            self.now += 1
            self.now_bytes += req.estimate_bytes()
            self.max_running = max(self.max_running, self.now)
            self.max_bytes = max(self.max_bytes, self.now_bytes)
        start = time.perf_counter() - t0
        time.sleep(0.004 * req.steps)
        with self.lock:
            self.now -= 1
            self.now_bytes -= req.estimate_bytes()
        return serve.Record(req.rid, req.program, req.cells, req.steps, req.arrival, start, time.perf_counter() - t0)


def test_scheduler_respects_arrivals_slots_and_memory():
    reqs = serve.make_requests(20, seed=3, rate=400.0, side=(32, 96), steps=(2, 6))
    srv = _Recorder(slots=3, memory_cap=1 << 40)
    recs, wall = srv.run(reqs, realtime=True)
    assert sorted(r.rid for r in recs) == list(range(20))
    assert all(r.start >= r.arrival - 1e-6 for r in recs)
    assert srv.max_running <= 3
    # a cap of about two requests' memory keeps at most two running
    cap = 2 * max(r.estimate_bytes() for r in reqs)
    srv = _Recorder(slots=8, memory_cap=cap)
    recs, _ = srv.run(reqs, realtime=False)
    assert len(recs) == 20 and srv.max_bytes <= cap
    # arrivals are Poisson: increasing, mean gap near 1/rate
    arr = np.array([r.arrival for r in serve.make_requests(400, seed=4, rate=100.0)])
    assert np.all(np.diff(arr) >= 0) and 0.007 < np.mean(np.diff(arr)) < 0.013


@pytest.mark.gpu
def test_requests_identical_alone_and_in_a_mix(gpu_lib, tmp_path):
    """Small heat and two-phase requests, one at a time and all at once
    (own runtimes and streams): bit-identical final fields."""
    def batch(root, slots):
        reqs = serve.make_requests(6, seed=5, side=(24, 48), steps=(3, 5))
        for r in reqs:
            serve.prepare(r, str(root / ("r%d" % r.rid)))
        recs, _ = serve.Server(slots=slots, output_values="last").run(reqs, realtime=False)
        assert all(not r.error for r in recs), [r.error for r in recs]
        return {r.rid: serve.last_fields(r) for r in reqs}

    alone = batch(tmp_path / "alone", 1)
    mix = batch(tmp_path / "mix", 6)
    assert {len(v) for v in alone.values()} >= {1}
    for rid, fields in alone.items():
        for a, b in zip(fields, mix[rid]):
            assert a is not None and b is not None
            assert np.array_equal(a, b), rid
