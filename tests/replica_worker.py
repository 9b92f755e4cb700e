"""One rank of a CPU replica run (launched by torchrun or by hand with
RANK / WORLD_SIZE / MASTER_* set): each rank runs the oracle's heat
simulator on the same seeded case through equelle_b200.replicas over gloo,
exactly as bench.py's ranks run the device simulator over NCCL, and writes
what it saw to <out>/rank<r>.json.

--fail-rank R makes rank R raise after the group is up, before the barrier
that opens the timed region; the other ranks must end with an error from
that barrier, inside the group's timeout, instead of waiting for good."""
import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from equelle_b200 import cases, simrun  # noqa: E402
from equelle_b200.replicas import Replicas  # noqa: E402
from bench import timed_window  # noqa: E402

ORACLE_SIM = os.path.join(ROOT, "oracle", "_build", "libsim_heateq_oracle.so")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--fail-rank", type=int, default=-1)
    ap.add_argument("--timeout", type=float, default=20.0)
    a = ap.parse_args()
    rp = Replicas("gloo", timeout_s=a.timeout)
    rec = {"rank": rp.rank, "world": rp.world, "backend": rp.backend}
    path = os.path.join(a.out, "rank%d.json" % rp.rank)
    if rp.rank == a.fail_rank:
        raise SystemExit("rank %d leaves before the timed region" % rp.rank)
    t0 = time.perf_counter()
    try:
        rp.barrier()
        d = os.path.join(a.out, "in_r%d" % rp.rank)
        o = os.path.join(a.out, "out_r%d" % rp.rank)
        os.makedirs(o, exist_ok=True)
        W, K = a.warmup, a.steps
        args = cases.heat(d, 24, 20, steps=W + K, seed=7) + ["output_values=last", "output_dir=%s/" % o]
        rep = simrun.run("heateq", args, path=ORACLE_SIM)
        ms = timed_window(rep, W, K)
        mx = rp.max(ms)
        rec.update(ms=ms, max_ms=mx, value=rp.throughput(K, mx), solves=rep.solves)
        rp.close()
    except Exception as e:  # the peer left: report how long the wait lasted
        rec.update(error="%s: %s" % (type(e).__name__, e), waited_s=time.perf_counter() - t0)
        with open(path, "w") as f:
            json.dump(rec, f)
        raise SystemExit(3)
    with open(path, "w") as f:
        json.dump(rec, f)


if __name__ == "__main__":
    main()
