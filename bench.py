#!/usr/bin/env python
"""Benchmark: implicit Newton time steps of a generated-style simulator.

Default workload: the fully implicit oil-water case on a 128x128x64
Cartesian grid (2 unknowns per cell, 2,097,152 unknowns), seeded
log-normal permeability, 1-day steps; each "step" is one time step = one
newtonSolveSystem with BiCGStab + ILU(0) inner solves, run through the
generated-style C++ simulator equelle_b200/sims/twophase.cpp linked to
libeqg.so and called in this process.

    python bench.py [--gpus N] [--steps K] [--warmup W]
                    [--impl ours|reference] [--precision double|mixed|refine]
                    [--workload twophase3d|twophase2d|heat] [--nx --ny --nz]

`value` (time steps/s) is timed on the device clock between the runtime's
solve marks of steps W .. W+K-1 (inputs resident in HBM); `e2e` re-runs the
whole program through its public entry point with host input files and
host outputs every step, timed on the host clock.  --impl reference times
the CPU oracle (the restated reference serial backend) on a bounded sample
of the same workload on the host cores.  Under torchrun each rank runs an
independent replica (no collective on the data path); rank 0 prints one
JSON line with the max time over ranks.
"""
import argparse
import csv
import io
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SPMV_KERNEL = "bicg_spmv_omega"
# DRAM bytes (read + write) that ncu measured for one launch of a kernel
# against its algorithmic bytes, on the FP64 2 x 2 block layout of the
# two-phase 128x128x48 case (profiles/solver_kernels_twophase_128x128x48.md,
# profiles/bilu_upper_kernel_twophase_128x128x48.md).
# Both scale with the number of blocks, so a launch of the same layout on
# another grid moves this ratio times its algorithmic bytes.
TRAFFIC_RATIO = {
    "bicg_spmv_omega": 242.5 / 237.0,
    "mg_residual": 245.5 / 237.0,
    "bilu_lower": 114.8 / 118.5,
    "bilu_upper": 116.6 / 118.5,
}

# Kernels of one BiCGStab iteration (its V-cycles, SpMVs and vector steps),
# of the preconditioner set-up per linear solve; every other kernel belongs
# to residual and Jacobian assembly.
KRYLOV_KERNELS = {"bicg_p", "bicg_spmv_alpha", "bicg_s", "bicg_spmv_omega", "bicg_xr", "bilu_lower", "bilu_upper",
                  "mg_residual", "mg_restrict", "mg_correct", "mg_prolong", "mg_tail", "mg_dense_apply",
                  "residual", "add_float", "sumsq"}
SETUP_KERNELS = {"bicg_init", "gather_values", "mg_galerkin", "mg_ap_values", "bilu_factor", "mg_dense_inverse",
                 "to_float", "permute", "unpermute"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["double", "mixed", "refine"], default="double")
    ap.add_argument("--ordering", choices=["multicolor", "natural"], default="multicolor")
    ap.add_argument("--workload", choices=["twophase3d", "twophase2d", "heat", "swe", "batched", "serve"],
                    default="twophase3d")
    ap.add_argument("--instances", type=int, default=64, help="batched: number of instances")
    ap.add_argument("--requests", type=int, default=48, help="serve: requests per arrival rate")
    ap.add_argument("--rates", default="50,200,1000,2000", help="serve: Poisson arrival rates (req/s)")
    ap.add_argument("--slots", type=int, default=32, help="batched/serve: instances on the GPU at once")
    ap.add_argument("--seq-sample", type=int, default=128,
                    help="batched: instances of the sequential FP64 arm (the first ones of the same seeded set)")
    ap.add_argument("--side-max", type=int, default=None, help="batched/serve: largest grid side")
    ap.add_argument("--max-steps", type=int, default=None, help="serve: most time steps of a request")
    ap.add_argument("--host-threads", type=int, default=None,
                    help="batched/serve: OpenMP threads of each runtime's solver analysis (default: cores / slots)")
    ap.add_argument("--nx", type=int)
    ap.add_argument("--ny", type=int)
    ap.add_argument("--nz", type=int)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="two-phase: skip the mixed and refine runs that the line compares with FP64")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--extra", action="append", default=[],
                    help="extra key=value runtime parameter (repeatable)")
    ap.add_argument("--kernel-profile", action="store_true",
                    help="time every kernel launch with CUDA events and print the per-kernel totals")
    ap.add_argument("--cpu-sample-krylov", type=int, default=12,
                    help="Krylov iterations in the CPU oracle sample")
    return ap.parse_args()


# ---------------------------------------------------------------------------
def workload(a):
    from equelle_b200 import cases
    if a.workload == "twophase3d":
        nx, ny, nz = a.nx or 128, a.ny or 128, a.nz or 64
        name, key = "twophase", "twophase_%dx%dx%d" % (nx, ny, nz)
        desc = "two-phase oil-water fully implicit %dx%dx%d, 2 unknowns/cell" % (nx, ny, nz)
        cells = nx * ny * nz

        def write(d, steps):
            return cases.two_phase(d, nx, ny, nz, steps=steps)
        tol = ["abs_res_tol=1e-8", "linsolver_residual_tolerance=1e-8", "linsolver_max_iterations=5000"]
    elif a.workload == "twophase2d":
        nx, ny = a.nx or 512, a.ny or 512
        name, key = "twophase", "twophase_%dx%d" % (nx, ny)
        desc = "two-phase oil-water fully implicit %dx%d, 2 unknowns/cell" % (nx, ny)
        cells = nx * ny

        def write(d, steps):
            return cases.two_phase(d, nx, ny, None, steps=steps, corr_len=4.0)
        tol = ["abs_res_tol=1e-8", "linsolver_residual_tolerance=1e-8", "linsolver_max_iterations=5000"]
    elif a.workload == "swe":
        nx, ny = a.nx or 4096, a.ny or 4096
        name, key = "swe", "swe_%dx%d" % (nx, ny)
        desc = "explicit shallow water %dx%d, first-order Rusanov flux, Heun steps, CFL 0.45" % (nx, ny)
        cells = nx * ny

        def write(d, steps):
            return cases.swe(d, nx, ny, steps=steps)
        tol = []
    else:
        nx, ny = a.nx or 64, a.ny or 64
        name, key = "heateq", "heat_%dx%d" % (nx, ny)
        desc = "implicit heat equation %dx%d" % (nx, ny)
        cells = nx * ny

        def write(d, steps):
            return cases.heat(d, nx, ny, steps=steps)
        tol = []
    return name, key, desc, cells, write, tol


def input_dir(key, steps, rank):
    d = os.path.join(tempfile.gettempdir(), "eqg_bench", "%s_s%d_r%d" % (key, steps, rank))
    os.makedirs(d, exist_ok=True)
    return d


def dir_bytes(d, exclude=("timesteps.txt",)):
    """Bytes of numeric input the run uploads (8 B per value read)."""
    n = 0
    for f in os.listdir(d):
        if f in exclude or not f.endswith(".txt"):
            continue
        with open(os.path.join(d, f)) as fh:
            n += 8 * len(fh.read().split())
    return n


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.proc:
            self.proc.terminate()
            out, _ = self.proc.communicate(timeout=10)
            for r in csv.reader(io.StringIO(out)):
                if len(r) >= 9:
                    self.rows.append([x.strip() for x in r])
        return False

    def summary(self):
        rows = getattr(self, "rows", [])
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi samples"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        loaded = [s for s in sm if s > 0.5 * smax] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        power = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        return {"sm_mhz": loaded[len(loaded) // 2], "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows), "power_w_max": max(power) if power else None}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def timed_window(rep, w, k):
    """Device ms from the start of solve w to the end of solve w+k-1."""
    ms = sum(rep.gap_ms[i] for i in range(w, w + k - 1)) + rep.solve_ms[w + k - 1]
    return ms


# ---------------------------------------------------------------------------
def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_sample(name, args, sample_krylov, per_step, threads=1):
    """Times the CPU oracle on a bounded sample of the same workload: the
    first Newton iteration of time step 1 (residual + Jacobian assembly,
    ILU(0) factorization, `sample_krylov` BiCGStab iterations), then scales
    the measured phase times by the oracle's own per-step counts `per_step`
    (residual evaluations, factorizations, Krylov iterations of its
    natural-order ILU(0) BiCGStab, measured once to convergence on the full
    grid: equelle_b200/bench_counts.json).  threads > 1 runs the OpenMP
    build of the oracle (the same code with its Krylov solve parallel: SpMV,
    dots, vector updates, wavefront-ordered triangular solves) on that many
    threads.  Returns (steps/s, description, ms per step)."""
    from equelle_b200 import simrun
    lib = "libsim_%s_oracle.so" % name if threads == 1 else "libsim_%s_oracle_omp.so" % name
    path = os.path.join(ROOT, "oracle", "_build", lib)
    sargs = [a for a in args if not a.startswith(("linsolver_max_iterations", "max_iter"))]
    sargs += ["max_iter=1", "linsolver_max_iterations=%d" % sample_krylov]
    old = os.environ.get("OMP_NUM_THREADS")
    os.environ["OMP_NUM_THREADS"] = str(threads)
    try:
        t0 = time.perf_counter()
        rep = simrun.run(name, sargs, path=path, allow_failure=True)
        wall = time.perf_counter() - t0
    finally:
        if old is None:
            os.environ.pop("OMP_NUM_THREADS", None)
        else:
            os.environ["OMP_NUM_THREADS"] = old
    st = rep.stats
    t_res = st.residual_ms / max(st.residual_evaluations, 1)
    t_fac = st.factor_ms / max(st.linear_solves, 1)
    t_kry = st.krylov_ms / max(st.krylov_iterations, 1)
    ms_step = per_step["residuals"] * t_res + per_step["solves"] * t_fac + per_step["krylov"] * t_kry
    desc = ("oracle (C++ restatement of the reference serial backend; BiCGStab with natural-order ILU(0)), %s: "
            "first Newton iteration of step 1 on the full grid (%d residual evals %.0f ms each, ILU(0) %.0f ms, "
            "%d BiCGStab its %.1f ms each; %.1f s wall), projected to the oracle's own counts per step measured to "
            "convergence on the full grid (%.1f residuals, %.1f factorizations, %.0f Krylov its)"
            % ("1 thread" if threads == 1 else "OpenMP build, %d threads" % threads, st.residual_evaluations, t_res,
               t_fac, st.krylov_iterations, t_kry, wall, per_step["residuals"], per_step["solves"],
               per_step["krylov"]))
    return 1000.0 / ms_step, desc, ms_step


# ---------------------------------------------------------------------------
def main():
    a = parse()
    from equelle_b200.replicas import Replicas
    # the reference arm runs on rank 0's host cores alone: no group
    rp = Replicas("nccl", group=a.impl != "reference")
    rank, local_rank, world = rp.rank, rp.local_rank, rp.world

    if a.workload in ("batched", "serve"):
        return main_many(a, rp)
    name, key, desc, cells, write, tol = workload(a)
    W, K = a.warmup, a.steps
    if name == "swe":
        return main_explicit(a, rp, name, key, desc, cells, write)
    metric = "Newton-steps/s"
    unit = "steps/s"

    if a.impl == "reference":
        if rank != 0:
            return
        d = input_dir(key, 1, rank)
        args = write(d, 1) + tol + ["output_values=none"]
        per = reference_counts(a)
        threads = host_threads()
        times = []
        descs = None
        # each step: one sample of the OpenMP oracle on every host thread
        for _ in range(W + K):
            v, descs, ms = cpu_sample(name, args, a.cpu_sample_krylov, per, threads=threads)
            times.append(ms)
        ms_step = sum(times[W:]) / K
        val = 1000.0 / ms_step
        sval, sdesc, sms = cpu_sample(name, args, a.cpu_sample_krylov, per, threads=1)
        line = {
            "impl": "reference", "metric": metric, "value": val, "unit": unit, "n_gpus": a.gpus, "steps": K,
            "warmup": W, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": config(a, desc, cells),
            "solver": "Newton + BiCGStab with natural-order ILU(0) (the oracle's restatement of the reference "
                      "serial backend; projected per step from a sample, see cpu_baseline.sample)",
            "cpu_baseline": {"value": val, "unit": unit, "cores": threads, "kind": "port", "sample": descs},
            "serial": {"value": sval, "unit": unit, "cores": 1, "ms_per_step": sms, "sample": sdesc},
            "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return

    # ---- our arm ----------------------------------------------------------
    from equelle_b200 import simrun
    import equelle_b200
    equelle_b200.load_library()
    d = input_dir(key, W + K, rank)
    args = write(d, W + K) + tol + [
        "output_values=none", "device=%d" % local_rank,
        "linsolver_precision=" + a.precision, "linsolver_ordering=" + a.ordering]
    args += a.extra
    if a.kernel_profile:
        args.append("time_kernel=*")
    flushed = a.workload in FLUSHED
    if flushed:
        args.append("flush_l2=256")
    rp.barrier()
    with ClockSampler(local_rank) as clk:
        rep = simrun.run(name, args)
    if rep.solves < W + K:
        raise SystemExit("simulator ran %d solves, expected %d" % (rep.solves, W + K))
    if flushed:
        ms = rp.max(sum(rep.solve_ms[i] for i in range(W, W + K)))
    else:
        ms = rp.max(timed_window(rep, W, K))
    infos = window_counts(rep, W, K)
    value = rp.throughput(K, ms)
    st = rep.stats
    n_rows, nnz = st.last_matrix_rows, st.last_matrix_nnz
    bsz, nblk = max(st.last_block_size, 1), st.last_matrix_blocks or st.last_matrix_nnz

    # Per-kernel profile: a second, short run of the same workload with every
    # launch bracketed by CUDA events on the runtime stream (which turns the
    # CUDA graphs of the timed run off), each launch with its algorithmic
    # bytes (the library's accounting of the data its operation must move).
    if a.kernel_profile:
        prep = rep
    else:
        d3 = input_dir(key, 2, rank)
        prep = simrun.run(name, write(d3, 2) + tol + [
            "output_values=none", "device=%d" % local_rank, "time_kernel=*",
            "linsolver_precision=" + a.precision, "linsolver_ordering=" + a.ordering] + a.extra)
    prof = json.loads(prep.profile.decode() or "{}")
    peak, peak_kind = peaks()
    per_step = {"residuals": infos["residuals"] / K, "solves": infos["solves"] / K, "krylov": infos["krylov"] / K}
    roofline = roofline_entry(a, prof, prep.stats, per_step, ms / K, infos, K, peak, peak_kind, bsz)

    line = {
        "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if a.precision == "double" else "f64+f32",
        "data": "synthetic (seeded Gaussian-random-field log-permeability, corner wells)",
        "config": config(a, desc, cells),
        "solver": "Newton + BiCGStab, V-cycle with %dx%d block ILU(0) smoothers (%s ordering)" % (bsz, bsz, a.ordering),
        "newton_iterations_per_step": infos["newton"] / K,
        "krylov_iterations_per_step": infos["krylov"] / K,
        "cell_updates_per_s": world * K * cells / (ms / 1000.0),
        "gpu_launches": infos["launches"],
        "phase_ms_per_step": {k: infos[k + "_ms"] / K for k in ("residual", "factor", "krylov")},
        "roofline": roofline,
        "clocks": clk.summary(),
    }

    # the reduced-precision forms of the same workload against this FP64 run:
    # throughput, and the saturation field after the last step relative to
    # the FP64 run's (both written with precision 17)
    if name == "twophase" and a.precision == "double" and not a.no_forms:
        def last_sw(rdir, precision):
            args4 = write(d, W + K) + tol + ["output_values=last", "output_dir=%s/" % rdir, "device=%d" % local_rank,
                                             "linsolver_precision=" + precision, "linsolver_ordering=" + a.ordering]
            os.makedirs(rdir, exist_ok=True)
            r = simrun.run(name, args4 + a.extra)
            import numpy as np
            return r, np.loadtxt(os.path.join(rdir, "saturation-last.output"))

        base_dir = os.path.join(tempfile.gettempdir(), "eqg_bench", "forms_r%d" % rank)
        _, sw64 = last_sw(os.path.join(base_dir, "double"), "double")
        # the comparison is of the last step's saturation: water has entered
        if not sw64.max() > 0.2 + 1e-3:
            raise SystemExit("precision forms: the FP64 run's last saturation output is the initial state")
        forms = {"sw_max_after_last_step": float(sw64.max())}
        for form in ("mixed", "refine"):
            r, sw = last_sw(os.path.join(base_dir, form), form)
            ms_f = rp.max(timed_window(r, W, K))
            forms[form] = {"value": world * K / (ms_f / 1000.0), "ms_per_step": ms_f / K,
                           "speedup_vs_fp64": ms / ms_f,
                           "krylov_iterations_per_step": window_counts(r, W, K)["krylov"] / K,
                           "sw_max_rel_err_vs_fp64": float(abs(sw - sw64).max() / abs(sw64).max())}
        line["precision_forms"] = forms
        if a.workload == "twophase3d":
            line["precision_forms"]["vs_oracle"] = forms_vs_oracle(local_rank, a)

    # end to end through the public entry point: host input files in, host
    # outputs out every step, host wall clock
    if not a.no_e2e:
        d2 = input_dir(key, K, rank)
        args2 = write(d2, K) + tol + ["output_values=none", "device=%d" % local_rank,
                                      "linsolver_precision=" + a.precision, "linsolver_ordering=" + a.ordering]
        rp.barrier()
        t0 = time.perf_counter()
        rep2 = simrun.run(name, args2)
        wall = rp.max(time.perf_counter() - t0)
        nfields = 2 if name == "twophase" else 1
        line["e2e"] = {"value": world * K / wall, "unit": unit,
                       "h2d_bytes_per_step": dir_bytes(d2) / K,
                       "d2h_bytes_per_step": nfields * 8 * cells * (K + 1) / K,
                       "what": "whole program run (grid build, input files, %d steps, output copies) on the "
                               "host clock" % K, "solves": rep2.solves}

    if rank == 0 and world == 1 and not a.no_cpu:
        cargs = write(input_dir(key, 1, rank), 1) + tol + ["output_values=none"]
        per = reference_counts(a)
        val, sdesc, _ = cpu_sample(name, cargs, a.cpu_sample_krylov, per)
        line["cpu_baseline"] = {"value": val, "unit": unit, "cores": 1, "kind": "port", "sample": sdesc}
        threads = host_threads()
        oval, odesc, _ = cpu_sample(name, cargs, a.cpu_sample_krylov, per, threads=threads)
        line["cpu_baseline_openmp"] = {"value": oval, "unit": unit, "cores": threads, "kind": "port", "sample": odesc}

    if a.kernel_profile:
        line["kernel_profile"] = kernel_table(prof, peak)
    if rank == 0:
        print(json.dumps(line))
    rp.close()


def kernel_table(prof, peak, top=None):
    """Per kernel name: launches, device ms, share of the profiled time,
    algorithmic bytes per launch and the bandwidth they imply."""
    total = sum(v[1] for v in prof.values()) or 1.0
    out = {}
    for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])[:top]:
        launches, ms_k = v[0], v[1]
        nbytes = v[2] if len(v) > 2 and v[3] == launches else None
        e = {"launches": launches, "ms": round(ms_k, 3), "share": round(ms_k / total, 4)}
        if nbytes is not None and ms_k > 0:
            e["bytes_per_launch"] = nbytes / launches
            e["gbs"] = round(nbytes / (ms_k / 1000.0) / 1e9, 1)
            e["frac"] = round(nbytes / (ms_k / 1000.0) / 1e9 / peak, 3)
        out[k] = e
    return out


def roofline_entry(a, prof, pstats, per_step, ms_step, infos, K, peak, peak_kind, bsz):
    """The `roofline` object of the line.

    Dominant kernel: the kernel name with the largest device time in the
    profile run; achieved = its algorithmic bytes per launch / its mean
    CUDA-event launch duration.  `step`: the algorithmic bytes of one time
    step (per Krylov iteration, per linear solve and per residual evaluation,
    summed over the profile run's kernels and divided by its counts, times
    the timed window's counts per step) over the timed ms per step; `krylov`
    the same for the Krylov phase alone over its device time per step.
    `spmv`: the BiCGStab SpMV t = A s (with its two dots), for continuity."""
    def gbs(nbytes, ms_):
        return nbytes / (ms_ / 1000.0) / 1e9 if ms_ > 0 else 0.0

    stated = {k: v for k, v in prof.items() if len(v) > 2 and v[3] == v[0] and v[0] > 0}
    dom = max(prof.items(), key=lambda kv: kv[1][1])[0] if prof else SPMV_KERNEL
    dl, dt = prof.get(dom, [0, 0.0])[:2]
    dbytes = stated[dom][2] / dl if dom in stated else None
    ach = gbs(dbytes, dt / dl) if dbytes and dl else 0.0
    # a layout the committed ncu capture measured: 3D two-phase, FP64 2 x 2
    # blocks (FP32 preconditioner matrices in `mixed` change the V-cycle's)
    captured = (a.workload == "twophase3d" and bsz == 2 and a.precision == "double" and dom in TRAFFIC_RATIO)
    entry = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
             "frac": ach / peak, "peak_source": peak_kind,
             "traffic": TRAFFIC_RATIO[dom] * dbytes if captured else None,
             "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of a launch of the same kernel on "
                                "the 128x128x48 case, as a ratio to its algorithmic bytes, times this mean launch's "
                                "algorithmic bytes" if captured else "not captured for this kernel and layout"),
             "algorithmic_bytes_per_launch": dbytes, "launches": dl, "avg_launch_ms": dt / dl if dl else None,
             "share_of_profiled_time": dt / (sum(v[1] for v in prof.values()) or 1.0)}
    # per-phase bytes in the profile run, scaled to the timed window's counts
    kry = sum(v[2] for k, v in stated.items() if k in KRYLOV_KERNELS)
    setup = sum(v[2] for k, v in stated.items() if k in SETUP_KERNELS)
    asm = sum(v[2] for k, v in stated.items() if k not in KRYLOV_KERNELS and k not in SETUP_KERNELS)
    unstated_ms = sum(v[1] for k, v in prof.items() if k not in stated)
    p_kry = max(pstats.krylov_iterations, 1)
    p_solves = max(pstats.linear_solves, 1)
    p_res = max(pstats.residual_evaluations, 1)
    step_bytes = (kry / p_kry * per_step["krylov"] + setup / p_solves * per_step["solves"]
                  + asm / p_res * per_step["residuals"])
    kry_ms = infos["krylov_ms"] / K
    entry["step"] = {"achieved": gbs(step_bytes, ms_step), "frac": gbs(step_bytes, ms_step) / peak,
                     "algorithmic_bytes_per_step": step_bytes,
                     "bytes_per_krylov_iteration": kry / p_kry, "bytes_per_linear_solve_setup": setup / p_solves,
                     "bytes_per_residual_evaluation": asm / p_res,
                     "profiled_ms_without_stated_bytes": unstated_ms}
    entry["krylov"] = {"achieved": gbs(kry / p_kry * per_step["krylov"], kry_ms),
                       "frac": gbs(kry / p_kry * per_step["krylov"], kry_ms) / peak, "ms_per_step": kry_ms}
    sl, st = prof.get(SPMV_KERNEL, [0, 0.0])[:2]
    if sl and SPMV_KERNEL in stated:
        sb = stated[SPMV_KERNEL][2] / sl
        sa = gbs(sb, st / sl)
        entry["spmv"] = {"kernel": SPMV_KERNEL, "achieved": sa, "frac": sa / peak, "algorithmic_bytes_per_launch": sb,
                         "avg_launch_ms": st / sl, "launches": sl}
    return entry


def forms_vs_oracle(local_rank, a, n=(32, 32, 32), steps=3):
    """Each precision form's saturation against the FP64 CPU oracle on a case
    the oracle finishes in seconds: 32x32x32 cells, 3 steps (65,536
    unknowns: the V-cycle's top level above the A P threshold, the rest in
    the fused cluster kernel).  Max relative difference per cell over every
    step's output."""
    import numpy as np
    from equelle_b200 import cases, simrun
    root = os.path.join(tempfile.gettempdir(), "eqg_bench", "forms_vs_oracle")
    args = cases.two_phase(os.path.join(root, "in"), *n, steps=steps) + [
        "abs_res_tol=1e-8", "linsolver_residual_tolerance=1e-8", "linsolver_max_iterations=50000",
        "output_to_file=true"]

    def run(tag, path, extra):
        out = os.path.join(root, tag)
        os.makedirs(out, exist_ok=True)
        simrun.run("twophase", args + extra + ["output_dir=%s/" % out], path=path)
        return [np.loadtxt(os.path.join(out, "saturation-%05d.output" % k)) for k in range(steps + 1)]

    oracle = run("oracle", os.path.join(ROOT, "oracle", "_build", "libsim_twophase_oracle.so"), [])
    res = {"case": "two-phase %dx%dx%d, %d steps, FP64 oracle (natural-order ILU(0))" % (n + (steps,)),
           "metric": "max over steps and cells of |Sw - Sw_oracle| / |Sw_oracle|"}
    for form in ("double", "mixed", "refine"):
        sw = run(form, None, ["device=%d" % local_rank, "linsolver_precision=" + form,
                              "linsolver_ordering=" + a.ordering] + a.extra)
        res[form] = float(max(np.max(np.abs(x - y) / np.abs(y)) for x, y in zip(sw, oracle)))
    return res


# Workloads whose working set fits in the 126 MB L2: 256 MB are written
# before each time step's start mark (runtime parameter flush_l2), and each
# step is timed between its own marks, which exclude that write.
FLUSHED = ("heat",)


def config(a, desc, cells):
    """The workload, the same in both arms (each line names its solver
    outside the config)."""
    l2 = ("working set smaller than L2: 256 MB written before each time step, each step timed between its own "
          "marks (the write excluded)" if a.workload in FLUSHED else
          "working set larger than L2 (126 MB), no flush")
    return {"workload": desc, "cells": cells, "precision": a.precision,
            "dt": "1 day" if a.workload != "heat" else "0.5", "l2": l2, "parallelism": "replicas"}


def main_many(a, rp):
    """Many independent instances on the GPU (equelle_b200/serve.py):
    `batched` runs a seeded set of 2D two-phase instances all at once;
    `serve` feeds requests (heat or 2D two-phase) at Poisson arrival rates.
    Both compare against the same requests run one at a time in plain FP64.
    Times are host wall clock around runs that end with their results on
    the host."""
    from equelle_b200 import serve
    import equelle_b200
    equelle_b200.load_library()
    rank, world = rp.rank, rp.world
    root = os.path.join(tempfile.gettempdir(), "eqg_bench", "%s_r%d" % (a.workload, rank))
    if a.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched or serving mode; "
                              "its arm for these workloads is the one-at-a-time FP64 line of our bench"}))
        return
    rp.barrier()

    def prepared(reqs, precision):
        for r in reqs:
            serve.prepare(r, os.path.join(root, "%s_%d_%d_%d" % (r.program, r.nx, r.steps, r.seed)),
                          ["linsolver_precision=" + precision, "device=%d" % rp.local_rank]
                          + a.extra)
        return reqs

    def summary(recs, wall):
        steps = sum(r.steps for r in recs)
        lat = [r.latency for r in recs]
        return {"requests": len(recs), "instance_steps": steps, "wall_s": wall,
                "instance_steps_per_s": steps / wall, "requests_per_s": len(recs) / wall,
                "latency_p50_s": serve.percentile(lat, 50), "latency_p99_s": serve.percentile(lat, 99),
                "errors": sum(1 for r in recs if r.error),
                "error_samples": ["%s %d cells: %s" % (r.program, r.cells, r.error[:160]) for r in recs if r.error][:4]}

    if a.workload == "batched":
        side_max = a.side_max or 512
        reqs = serve.make_requests(a.instances, seed=1, programs=("twophase",), side=(32, side_max),
                                   steps=(a.steps, a.steps))
        # the sequential plain-FP64 arm on the first seq_sample instances of
        # the same seeded set (instance-steps/s)
        seq_reqs = serve.make_requests(min(a.seq_sample, a.instances), seed=1, programs=("twophase",),
                                       side=(32, side_max), steps=(a.steps, a.steps))
        seq = summary(*serve.Server(slots=1).run(prepared(seq_reqs, "double"), realtime=False))
        bat64 = summary(*serve.Server(slots=a.slots, host_threads=a.host_threads).run(prepared(reqs, "double"), realtime=False))
        with ClockSampler(rp.local_rank) as clk:
            bat = summary(*serve.Server(slots=a.slots, host_threads=a.host_threads).run(prepared(reqs, "mixed"), realtime=False))
        value = rp.throughput(bat["instance_steps"], 1000.0 * rp.max(bat["wall_s"]))
        line = {"metric": "instance-steps/s", "value": value, "unit": "instance-steps/s", "n_gpus": world,
                "steps": a.steps, "warmup": 0, "ms_per_step": 1000.0 * bat["wall_s"] / bat["instance_steps"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
                "data": "synthetic (seeded log-permeability per instance, corner wells)",
                "config": {"workload": "%d 2D two-phase instances, sides log-uniform in [32, %d], %d steps each, "
                                       "%d on the GPU at once (own runtime, stream and host thread each)"
                                       % (a.instances, side_max, a.steps, a.slots),
                           "precision": "mixed (batched), double (sequential and batched_fp64)",
                           "sequential_sample": "the first %d of the same instances" % len(seq_reqs),
                           "l2": "no flush: whole runs on the host clock; a small instance run alone keeps its "
                                 "data in L2 between steps, instances run together share it",
                           "parallelism": "replicas"},
                "batched": bat, "batched_fp64": bat64, "sequential_fp64": seq,
                "speedup_vs_sequential": bat["instance_steps_per_s"] / seq["instance_steps_per_s"],
                "speedup_vs_sequential_same_precision": bat64["instance_steps_per_s"] / seq["instance_steps_per_s"],
                "clocks": clk.summary()}
    else:
        rates = [float(x) for x in a.rates.split(",")]
        per_rate = {}
        side_max, max_steps = a.side_max or 1024, a.max_steps or 100
        base = serve.make_requests(a.requests, seed=2, side=(64, side_max), steps=(10, max_steps))
        seq = summary(*serve.Server(slots=1).run(prepared(base, "double"), realtime=False))
        for lam in rates:
            reqs = serve.make_requests(a.requests, seed=2, rate=lam, side=(64, side_max), steps=(10, max_steps))
            recs, wall = serve.Server(slots=a.slots, host_threads=a.host_threads).run(prepared(reqs, "mixed"), realtime=True)
            per_rate["%g" % lam] = summary(recs, wall)
        top = per_rate["%g" % rates[-1]]
        line = {"metric": "requests/s", "value": rp.throughput(top["requests"], 1000.0 * rp.max(top["wall_s"])),
                "unit": "requests/s",
                "n_gpus": world, "steps": a.requests, "warmup": 0, "ms_per_step": 1000.0 / top["requests_per_s"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
                "data": "synthetic (seeded requests: heat or 2D two-phase, sides log-uniform in [64, %d], "
                        "10-%d steps)" % (side_max, max_steps),
                "config": {"workload": "serving loop, Poisson arrivals at %s req/s, %d requests per rate, up to %d on "
                                       "the GPU at once, admission under 150 GB" % (a.rates, a.requests, a.slots),
                           "l2": "no flush: whole requests on the host clock; a small request run alone keeps "
                                 "its data in L2 between steps, requests run together share it",
                           "parallelism": "replicas"},
                "per_rate": per_rate, "one_at_a_time_fp64": seq,
                "throughput_vs_one_at_a_time": top["requests_per_s"] / seq["requests_per_s"]}
    if rank == 0:
        print(json.dumps(line))
    rp.close()


# Bytes one time step of the shallow-water case must move at least (two
# stages, each reading the state (24 B) and the bottom (8 B) and writing the
# state (24 B) per cell, the CFL maximum fused in): the fused-stencil
# roofline the step time is compared with.
SWE_BYTES_PER_CELL = 112


def main_explicit(a, rp, name, key, desc, cells, write):
    """The explicit shallow-water workload: steps are the intervals between
    the program's outputs (device clock marks); the metric is cell updates
    per second."""
    from equelle_b200 import simrun
    rank, local_rank, world = rp.rank, rp.local_rank, rp.world
    W, K = a.warmup, a.steps
    metric = unit = "cell-updates/s"
    oracle = os.path.join(ROOT, "oracle", "_build", "libsim_%s_oracle.so" % name)

    # CPU sample: one step of the same case on at most 1024 x 1024 cells (the
    # oracle's cost per cell is nearly independent of the grid size; a full
    # 4096 x 4096 step takes it minutes)
    from equelle_b200 import cases
    sx, sy = min(a.nx or 4096, 1024), min(a.ny or 4096, 1024)
    scells = sx * sy

    def cpu_step():
        d = input_dir("swe_%dx%d" % (sx, sy), 1, rank)
        t0 = time.perf_counter()
        r = simrun.run(name, cases.swe(d, sx, sy, steps=1) + ["output_values=off"], path=oracle)
        wall = time.perf_counter() - t0
        ms = r.solve_ms[0]
        return scells / (ms / 1000.0), ms, wall

    sample = ("oracle (serial C++ restatement of the reference backend), 1 thread: one time step of the same "
              "case on %dx%d cells, host clock between the program's outputs" % (sx, sy))
    if a.impl == "reference":
        if rank != 0:
            return
        times = [cpu_step()[1] for _ in range(W + K)]
        ms_step = sum(times[W:]) / K
        val = cells / (ms_step / 1000.0)
        print(json.dumps({
            "impl": "reference", "metric": metric, "value": val, "unit": unit, "n_gpus": a.gpus, "steps": K,
            "warmup": W, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": {"workload": desc, "cells": cells},
            "cpu_baseline": {"value": val, "unit": unit, "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    import equelle_b200
    equelle_b200.load_library()
    d = input_dir(key, W + K, rank)
    args = write(d, W + K) + ["output_values=off", "device=%d" % local_rank] + a.extra
    if a.kernel_profile:
        args.append("time_kernel=*")
    rp.barrier()
    with ClockSampler(local_rank) as clk:
        rep = simrun.run(name, args)
    if rep.solves < W + K:
        raise SystemExit("simulator ran %d steps, expected %d" % (rep.solves, W + K))
    ms = rp.max(timed_window(rep, W, K))
    value = rp.throughput(K * cells, ms)
    peak, peak_kind = peaks()
    step_s = ms / K / 1000.0
    achieved = SWE_BYTES_PER_CELL * cells / step_s / 1e9
    st = rep.stats
    line = {
        "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded Gaussian bumps, sinusoidal bottom)",
        "config": {"workload": desc, "cells": cells, "l2": "working set larger than L2 (126 MB), no flush",
                   "parallelism": "replicas",
                   "execution": ("fused steps matched from the deferred operations (fuse=1): %d fused evaluations"
                                 % st.fused_evaluations) if st.fused_evaluations else
                                "one kernel per runtime operation"},
        "gpu_launches": int(st.kernel_launches * K / max(rep.solves, 1)),
        "roofline": {"kernel": "one time step (all its kernels)", "bound": "hbm", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": None, "algorithmic_bytes_per_step": SWE_BYTES_PER_CELL * cells,
                     "note": "algorithmic bytes of a fused stencil step (112 B per cell); the fused kernels read "
                             "five bottom arrays per stage (200 B per cell), the per-operation path moves more"},
        "clocks": clk.summary(),
    }
    if not a.no_e2e:
        d2 = input_dir(key, K, rank)
        args2 = write(d2, K) + ["output_values=none", "device=%d" % local_rank]
        rp.barrier()
        t0 = time.perf_counter()
        rep2 = simrun.run(name, args2)
        wall = rp.max(time.perf_counter() - t0)
        inbytes = sum(os.path.getsize(os.path.join(d2, f)) for f in os.listdir(d2) if f.endswith(".f64"))
        line["e2e"] = {"value": world * K * cells / wall, "unit": unit, "h2d_bytes_per_step": inbytes / K,
                       "d2h_bytes_per_step": 3 * 8 * cells * (K + 1) / K,
                       "what": "whole program run (grid build, input files, %d steps, output copies of the three "
                               "fields every step) on the host clock" % K, "steps": rep2.solves}
    if rank == 0 and world == 1 and not a.no_cpu:
        val, ms_cpu, wall = cpu_step()
        line["cpu_baseline"] = {"value": val, "unit": unit, "cores": 1, "kind": "port",
                                "sample": sample + " (%.1f s step, %.1f s with set-up)" % (ms_cpu / 1000.0, wall)}
    if a.kernel_profile:
        line["kernel_profile"] = kernel_table(json.loads(rep.profile.decode() or "{}"), peak, top=20)
    if rank == 0:
        print(json.dumps(line))
    rp.close()


def window_counts(rep, w, k):
    """Counters summed over the timed solves w .. w+k-1."""
    sel = [rep.info[i] for i in range(w, w + k)]
    newton = sum(s.newton_iterations for s in sel)
    return {"newton": newton, "krylov": sum(s.krylov_iterations for s in sel),
            "launches": sum(s.kernel_launches for s in sel),
            "residual_ms": sum(s.residual_ms for s in sel), "factor_ms": sum(s.factor_ms for s in sel),
            "krylov_ms": sum(s.krylov_ms for s in sel),
            "residuals": newton + k, "solves": newton,
            "unconverged_steps": sum(1 for s in sel if not s.converged)}


def reference_counts(a):
    """The CPU oracle's own counts per time step (residual evaluations,
    linear solves, Krylov iterations of its natural-order ILU(0) BiCGStab),
    measured once with solves run to convergence on the full grid
    (equelle_b200/bench_counts.json); they scale its sampled phase times."""
    path = os.path.join(ROOT, "equelle_b200", "bench_counts.json")
    with open(path) as f:
        d = json.load(f)
    if a.workload not in d:
        raise SystemExit("no oracle counts for workload %s in %s" % (a.workload, path))
    return {k: float(d[a.workload][k]) for k in ("residuals", "solves", "krylov")}


if __name__ == "__main__":
    main()
