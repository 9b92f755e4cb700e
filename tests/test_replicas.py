"""Several GPUs run independent replicas (equelle_b200/replicas.py): the
timing plumbing bench.py uses with NCCL, run here with gloo, two ranks on
the CPU, each rank running the oracle's heat simulator."""
import json
import os
import socket
import subprocess
import sys
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WORKER = os.path.join(ROOT, "tests", "replica_worker.py")


@pytest.fixture(scope="module")
def oracle_sims():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torchrun(args, nproc=2, timeout=240):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=%d" % nproc,
           "--master-addr", "127.0.0.1", "--master-port", str(_port())] + args
    env = dict(os.environ, OMP_NUM_THREADS="1")
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout)


def test_two_replicas_time_is_the_max_over_ranks(oracle_sims, tmp_path):
    r = _torchrun([WORKER, "--out", str(tmp_path), "--steps", "4", "--warmup", "1"])
    assert r.returncode == 0, r.stderr[-2000:]
    recs = [json.load(open(tmp_path / ("rank%d.json" % k))) for k in range(2)]
    assert [x["rank"] for x in recs] == [0, 1]
    assert all(x["world"] == 2 and x["backend"] == "gloo" and x["solves"] == 5 for x in recs)
    mx = max(x["ms"] for x in recs)
    for x in recs:
        assert x["max_ms"] == mx
        assert x["value"] == pytest.approx(2 * 4 / (mx / 1000.0), rel=1e-12)
    # the replicas share nothing on the data path: same case, same fields
    for tag in ("u",):
        a = np.loadtxt(tmp_path / "out_r0" / ("%s-last.output" % tag))
        b = np.loadtxt(tmp_path / "out_r1" / ("%s-last.output" % tag))
        assert np.array_equal(a, b)


def test_reference_arm_prints_one_line_from_rank0(oracle_sims):
    r = _torchrun(["bench.py", "--impl", "reference", "--workload", "heat", "--nx", "24", "--ny", "24",
                   "--steps", "2", "--warmup", "1", "--gpus", "2"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"


def test_rank_that_leaves_ends_the_others_wait(oracle_sims, tmp_path):
    """Rank 1 exits after the group is up; rank 0's barrier ends with an
    error inside the group's timeout (rank processes started by hand, so
    nothing but the group itself tells rank 0)."""
    port = _port()
    procs = []
    t0 = time.perf_counter()
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), OMP_NUM_THREADS="1")
        procs.append(subprocess.Popen([sys.executable, WORKER, "--out", str(tmp_path), "--fail-rank", "1",
                                       "--timeout", "15"], cwd=ROOT, env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    rcs = [p.wait(timeout=120) for p in procs]
    wall = time.perf_counter() - t0
    assert rcs[1] != 0 and rcs[0] == 3, (rcs, procs[0].stderr.read()[-2000:])
    rec = json.load(open(tmp_path / "rank0.json"))
    assert rec["error"] and rec["waited_s"] < 60
    assert wall < 110
