#!/usr/bin/env python
"""Benchmark: converged LM fits per second of the period scan on B200.

Workload (the production-size sparse search): a seeded synthetic asteroid
with 600 sparse calibrated points over 10 years plus 2 dense relative
lightcurves of 80 points (N = 760), fit with lmax = mmax = 6 (49 Laplace
coefficients) on nrows = 10 (800 facets), 50 LM iterations per fit, trial
periods 2-100 h at the reference step rule with step coefficient 2.15
(39 153 trial periods), 10 initial poles each.  A step is one batch of
consecutive trial periods (x 10 poles); ranks take disjoint batches
(weak scaling, no collective on the data path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

value      fits/s over the K timed steps, inputs resident in HBM, timed with
           CUDA events on the launching stream, L2 flushed between steps
e2e        the same through the public C ABI from host buffers (open from
           host arrays, upload, scan, records back to host, close)
roofline   algorithmic FLOPs (2 N F C + N mfit (mfit + 1) per evaluation,
           51 evaluations per 50-iteration fit) per launch over the launch time
cpu_baseline  the CPU oracle (the restatement pinned bit-exact to the
           reference build) on the host cores, a bounded sample of the same fits
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

# what the line measures: LM fits (trial period x initial pole, each run to
# the reference's stop rule) per second; the form that produced `value` is
# config.form, and `forms` holds the other forms timed on the same batch
METRIC = "converged LM fits/sec on 1 B200 (reference stop rule)"
WORKLOAD = ("c2 production sparse search: N=760 (600 sparse + 2x80 dense), lmax=mmax=6 (C=49), nrows=10 (F=800), "
            "50 LM iterations/fit, 2-100 h at step coef 2.15 (39153 periods) x 10 poles")


WORKLOAD_C5 = ("c5 large shape: N=20000 (40x100 dense + 16000 sparse), true lmax=10, fit lmax=mmax=8 (C=81), "
               "nrows=16 (F=2048), 50 LM iterations/fit, 2000 trial periods x 10 poles; explicit J in HBM")


def make_input(directory: str, config: str = "c2") -> str:
    from periodsearch_b200 import synth

    if config == "c5":
        w = synth.make_workload("c5_lmax8_n20000_f2048", 5, dense_lcs=40, dense_pts=100, sparse_pts=16000,
                                years=10, true_lmax=10, fit_lmax=8, nrows=16, noise=0.03, n_periods=2000)
        return synth.write_input(w, directory)
    w = synth._c2()
    return synth.write_input(w, directory)


def flop_per_eval(n_points, F, C, mfit):
    return 2.0 * n_points * F * C + n_points * mfit * (mfit + 1)


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = tempfile.mktemp(prefix="psclk", suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [l.split(",") for l in open(self.path) if l.strip()]
        except Exception:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        smax = float(rows[0][2])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": reasons, "samples": len(rows)}


def _oracle_worker(args):
    path, conw_r, fits = args
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pso

    o = pso.Oracle(path)
    o.set_conw_r(conw_r)
    for n, pole in fits:
        o.fit(o.freq(n), pole)
    return len(fits)


def _oracle_eval_worker(args):
    path, conw_r, n, pole = args
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pso

    o = pso.Oracle(path)
    o.set_conw_r(conw_r)
    a = o.initial_parameters(o.freq(n), pole)
    t0 = time.perf_counter()
    o.mrqcof(a)
    return time.perf_counter() - t0


def cpu_eval_sample(path, conw_r, n_first, evals_per_fit):
    """For workloads whose fits take minutes on a CPU core: time one model
    evaluation (mrqcof: model, Jacobian, alpha, beta) of the CPU oracle per
    host core and convert with the evaluations of one fit (the LM solve is
    negligible beside them on a CPU).  Returns (fits/s, cores, evals, s)."""
    import multiprocessing as mp

    cores = os.cpu_count() or 1
    jobs = [(path, conw_r, n_first + c // 10, c % 10 + 1) for c in range(cores)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        ts = pool.map(_oracle_eval_worker, jobs)
    t_eval = statistics.mean(ts)
    return cores / (t_eval * evals_per_fit), cores, cores, max(ts)


def cpu_sample(path, conw_r, n_first, fits_per_core=2):
    """Time the CPU oracle on cores x fits_per_core fits of the workload,
    one process per host core (the reference is single-threaded)."""
    import multiprocessing as mp

    cores = os.cpu_count() or 1
    jobs = []
    k = 0
    for c in range(cores):
        fl = []
        for _ in range(fits_per_core):
            fl.append((n_first + k // 10, k % 10 + 1))
            k += 1
        jobs.append((path, conw_r, fl))
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        pool.map(_oracle_worker, [(path, conw_r, [(1, 1)])] * cores)  # load + warm
        t0 = time.perf_counter()
        done = sum(pool.map(_oracle_worker, jobs))
        dt = time.perf_counter() - t0
    return done / dt, cores, done, dt


REF_EXE = os.path.join(REPO, "oracle", "_ref", "period_search_ref")


def ref_cpu_sample(path, n_first, periods_per_proc=1):
    """Time the reference's own CPU application (oracle/_ref, built from the
    reference sources) on the host cores: one process per core, each on its
    own slice of `periods_per_proc` consecutive trial periods (10 fits each)
    of the same input, started through the reference's checkpoint file
    (period_search_state = first period - 1).  The convexity-weight line is
    raised to 10 so that the application skips its pre-pass (it runs while
    conw_r escl^2 < 10, period_search_BOINC.cpp:489); the fits themselves
    (points, facets, coefficients, 50 iterations) are unchanged.  Returns
    (fits/s, cores, fits, seconds) or None when the reference is not built."""
    if not os.path.exists(REF_EXE):
        return None
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pso

    o = pso.Oracle(path)
    o.set_conw_r(o.conw_r)  # sets up the trial-period grid
    o.refresh()
    df = o.freq(1) - o.freq(2)
    lines = open(path).read().split("\n")
    p_start, coef = lines[0].split()[:2]
    ia = lines[0].split()[3]
    cores = os.cpu_count() or 1
    root = tempfile.mkdtemp(prefix="psref")
    procs = []
    for c in range(cores):
        n0 = n_first + c * periods_per_proc
        f_end = o.freq(n0) - (periods_per_proc - 0.5) * df
        d = os.path.join(root, "p%03d" % c)
        os.makedirs(d)
        text = list(lines)
        text[0] = "%s %s %.17g %s" % (p_start, coef, 1.0 / f_end, ia)
        text[3] = "10\tconvexity weight"
        open(os.path.join(d, "period_search_in"), "w").write("\n".join(text))
        open(os.path.join(d, "period_search_state"), "w").write("%d" % (n0 - 1))
        procs.append(d)
    t0 = time.perf_counter()
    running = [subprocess.Popen([REF_EXE], cwd=d, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
               for d in procs]
    rcs = [p.wait() for p in running]
    dt = time.perf_counter() - t0
    done = 0
    for d, rc in zip(procs, rcs):
        out = os.path.join(d, "period_search_out")
        n = len(open(out).read().splitlines()) if os.path.exists(out) else 0
        if rc != 0 or n != periods_per_proc:
            raise RuntimeError(f"reference run in {d} ended with {rc}, {n} records")
        done += 10 * n
    return done / dt, cores, done, dt


# The reference application keeps its data in static arrays
# (constants.h: MAX_N_FAC = 1000 facets, MAX_N_OBS = 20000 points); a
# workload beyond them (the lmax = 8, 2048-facet, 20 000-point one) cannot run
# there, and the CPU leg times the restatement instead.
REF_LIMITS = {"facets": 1000, "points": 20000}


def ref_cpu_sample_or_none(path, n_first):
    """ref_cpu_sample, or (None, reason) when the reference application is
    not built or the workload exceeds its static array sizes."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pso

    o = pso.Oracle(path)
    o.set_conw_r(o.conw_r)  # builds the shape model (facet count)
    if o.numfac > REF_LIMITS["facets"] or o.n_points > REF_LIMITS["points"]:
        return None, (f"the reference application holds at most {REF_LIMITS['facets']} facets and "
                      f"{REF_LIMITS['points']} points (MAX_N_FAC, MAX_N_OBS); this workload has "
                      f"{o.numfac} facets, {o.n_points} points")
    r = ref_cpu_sample(path, n_first)
    return r, None if r is not None else "the reference application is not built"


def run_reference(args, path, rank):
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pso

    o = pso.Oracle(path)
    conw_r = o.conw_r  # the pre-pass value is not needed for timing a fit
    o.set_conw_r(conw_r)  # builds the shape model (facet count)
    fits_ref = o.numfac <= REF_LIMITS["facets"] and o.n_points <= REF_LIMITS["points"]
    kind = "reference" if os.path.exists(REF_EXE) and fits_ref else "port"
    vals = []
    for s in range(args.warmup + args.steps):
        if kind == "reference":
            v, cores, done, dt = ref_cpu_sample(path, 1 + 37 * s)
        elif args.config == "c5":
            v, cores, done, dt = cpu_eval_sample(path, conw_r, 1 + 37 * s, 51)
            done, dt = v * dt, dt  # fits-equivalent of the timed evaluations
        else:
            v, cores, done, dt = cpu_sample(path, conw_r, 1 + 37 * s, fits_per_core=1)
        if s >= args.warmup:
            vals.append((v, done, dt))
    value = sum(d for _, d, _ in vals) / sum(t for _, _, t in vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "fits/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * statistics.mean(t for _, _, t in vals),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_C5 if args.config == "c5" else WORKLOAD,
                   "form": "reference CPU application (oracle/_ref, -O3)" if kind == "reference"
                   else "cpu oracle (reference restated, bit-exact)"},
        "cpu_baseline": {"value": value, "unit": "fits/s", "cores": cores, "kind": kind,
                         "sample": (f"{cores} processes x 1 trial period (10 fits) per step, pre-pass skipped"
                                    if kind == "reference" else
                                    f"{cores} processes x 1 model evaluation per step, converted at 51 "
                                    f"evaluations per fit; the reference application's static arrays hold at most "
                                    f"{REF_LIMITS['facets']} facets" if args.config == "c5" else
                                    f"{cores} processes x 1 fit per step (consecutive periods x poles)")},
        "e2e": {"value": value, "unit": "fits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _c4_worker(args):
    i, directory = args
    sys.path.insert(0, REPO)
    from periodsearch_b200 import synth

    w, width = synth.c4_asteroid(i)
    return synth.write_input(w, os.path.join(directory, "a%04d" % i)), w.n_points


def run_c4(args, local):
    print(json.dumps(c4_measure(args, local)), flush=True)


def c4_measure(args, local):
    """Uneven multi-asteroid batch: many asteroids, point counts
    log-uniform in 100-5000, dense/sparse mix, lmax = 6, nrows = 10,
    per-fit convergence, all in one persistent launch replayed from a CUDA
    graph.  A step scans `periods` consecutive trial periods of every
    asteroid.  The convexity pre-pass is not part of the timed steps (each
    asteroid uses conw / escl^2, the pre-pass start value)."""
    import multiprocessing as mp

    import numpy as np
    import torch

    import periodsearch_b200 as ps

    workdir = tempfile.mkdtemp(prefix="psc4")
    with mp.get_context("spawn").Pool(min(os.cpu_count() or 1, 16)) as pool:
        made = pool.map(_c4_worker, [(i, workdir) for i in range(args.asteroids)])
    torch.cuda.set_device(local)
    form = {"fp64": ps.PS_FORM_FP64, "fast": ps.PS_FORM_FAST, "mixed": ps.PS_FORM_MIXED}[args.form]
    # per-asteroid host setup + uploads: on host threads (the product's
    # open_many), timed; one asteroid on one thread for comparison
    t0 = time.perf_counter()
    ctxs = ps.open_many([p for p, _ in made], device=local, form=form, conw_r="start")
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    ps.open_many([made[0][0]], device=local, form=form, conw_r="start", threads=1)[0].close()
    setup_one_s = time.perf_counter() - t0
    P = args.c4_periods
    n_per = np.array([c.n_periods for c in ctxs])
    tiles = None
    if not args.no_autotune and args.form != "mixed":  # the mixed form has fixed tiles
        a0 = np.ones(len(ctxs), dtype=np.int32)
        tiles, _ = ps.PeriodSearchBatch.autotune(ctxs, a0, np.minimum(a0 + P - 1, n_per).astype(np.int32))
    batch = ps.PeriodSearchBatch(ctxs)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    total_periods = int(len(ctxs) * P)
    d_rec = torch.zeros(total_periods * 6, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def ranges(step):
        a = 1 + (step * P) % np.maximum(n_per - P + 1, 1)
        return a, np.minimum(a + P - 1, n_per)

    for s in range(args.warmup):
        a, b = ranges(s)
        batch.scan_device(a, b, d_rec.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    launches0 = ps.load_library().ps_kernel_launches()
    times, fits, busy, done = [], 0, None, None
    with ClockSampler(local) as clk:
        for s in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            a, b = ranges(args.warmup + s)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            batch.scan_device(a, b, d_rec.data_ptr(), stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1000.0)
            fits += int(10 * (b - a + 1).sum())
            busy, done = batch.fit_times()
    launches = ps.load_library().ps_kernel_launches() - launches0
    clocks = clk.summary()
    value = fits / sum(times)
    line = {
        "metric": METRIC + " (uneven batch)", "value": value, "unit": "fits/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * sum(times) / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"c4 uneven batch: {len(ctxs)} asteroids, N log-uniform 100-5000 "
                               f"(mean {np.mean([m for _, m in made]):.0f}), lmax=mmax=6, nrows=10, "
                               f"stop_condition 1e-4 / n_iter_min 5, {P} periods x 10 poles per asteroid per step",
                   "form": args.form, "graph": "persistent fit kernel + reduction replayed from a CUDA graph",
                   "tiles": ({"fch": tiles[0], "rt": tiles[1], "sortseg": tiles[2],
                              "chosen_by": "PeriodSearchBatch.autotune (ps_autotune on the work-weighted "
                                           "median asteroid, checked against the defaults on one batch scan)"}
                             if tiles else "defaults"),
                   "l2": "flushed (256 MB write) between timed steps",
                   "setup": {"seconds": setup_s, "asteroids": len(ctxs), "threads": min(len(made), os.cpu_count() or 1, 32),
                             "one_asteroid_s": setup_one_s,
                             "what": "host setup + uploads of every asteroid (ps.open_many), not in the timed steps"}},
        "per_asteroid_ms": {"p50": float(np.percentile(done, 50)), "p99": float(np.percentile(done, 99)),
                            "max": float(np.max(done)),
                            "what": "wall latency of one asteroid in the last timed step: from the start of the "
                                    "step's first fit to the end of the asteroid's last fit (GPU global timer)",
                            "busy_p50": float(np.percentile(busy, 50)), "busy_p99": float(np.percentile(busy, 99)),
                            "busy_what": "summed duration of the asteroid's fits (fits run in parallel)"},
        "gpu_launches": int(launches), "clocks": clocks,
    }
    batch.close()
    for c in ctxs:
        c.close()
    # end to end through the public API: open every asteroid from its input
    # file (host setup and uploads on host threads), open the batch, scan the
    # step's periods into host records, close everything
    e2e_times, phases = [], {"open_many": [], "batch_open": [], "scan": [], "close": []}
    h2d = sum(os.path.getsize(p) for p, _ in made)
    for s in range(0 if getattr(args, "no_e2e", False) else 1):
        a, b = ranges(args.warmup + s)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cs = ps.open_many([p for p, _ in made], device=local, form=form, conw_r="start")
        if tiles:  # the tile shapes the timed steps ran with
            for c in cs:
                c.set_tiles(*tiles)
        t1 = time.perf_counter()
        bt = ps.PeriodSearchBatch(cs)
        t2 = time.perf_counter()
        recs = bt.scan(a, b)
        t3 = time.perf_counter()
        bt.close()
        for c in cs:
            c.close()
        t4 = time.perf_counter()
        e2e_times.append(t4 - t0)
        for k, dt in zip(phases, (t1 - t0, t2 - t1, t3 - t2, t4 - t3)):
            phases[k].append(dt)
    if e2e_times:
        n_rec = sum(len(r) for r in recs)
        line["e2e"] = {"value": fits / args.steps * len(e2e_times) / sum(e2e_times), "unit": "fits/s",
                       "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(n_rec * 48),
                       "what": "per step: open all asteroids from their input files, open the batch (graph "
                               "capture), scan, records to host, close",
                       "step_ms": [round(1000 * t, 1) for t in e2e_times],
                       "phase_ms": {k: round(1000 * statistics.median(v), 1) for k, v in phases.items() if v}}
    return line


def extra_workloads(args, local):
    """The uneven 512-asteroid batch (c4) and the 20 000-point lmax 8 shape
    (c5), each one warm-up and one timed step with the default tiles, so that
    every bench run records them beside the headline."""
    import types

    import torch

    import periodsearch_b200 as ps

    out = {}
    try:
        a = types.SimpleNamespace(form=args.form if args.form in ("fp64", "fast") else "fast", asteroids=512,
                                  c4_periods=4, steps=1, warmup=1, no_autotune=True, no_e2e=True)
        line = c4_measure(a, local)
        out["c4"] = {k: line[k] for k in ("value", "unit", "ms_per_step", "per_asteroid_ms", "gpu_launches")}
        out["c4"]["workload"] = line["config"]["workload"]
        out["c4"]["setup_s"] = line["config"]["setup"]["seconds"]
    except Exception as e:  # recorded, not fatal: the headline line still prints
        out["c4"] = {"error": repr(e)[:300]}
    try:
        path = make_input(tempfile.mkdtemp(prefix="psc5"), "c5")
        g = ps.PeriodSearch(path, device=local, form=ps.PS_FORM_FAST)
        g.set_conw_r(g.conw_r)
        B = 14
        d = torch.zeros(B * 6, dtype=torch.float64, device="cuda")
        stream = torch.cuda.Stream()
        g.scan_device(1, B, d.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.scan_device(1 + B, 2 * B, d.data_ptr(), stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1000.0
        fl = 10 * B * 51 * flop_per_eval(g.n_points, g.numfac, g.ncoef, g.mfit)
        out["c5"] = {"value": 10 * B / t, "unit": "fits/s", "ms_per_step": 1000 * t, "tflops": fl / t / 1e12,
                     "frac_of_fp64_peak": fl / t / 1e12 / ps.fp64_tensor_peak(local), "workload": WORKLOAD_C5,
                     "fits_per_step": 10 * B}
        g.close()
    except Exception as e:
        out["c5"] = {"error": repr(e)[:300]}
    return out


def initial_parameters(g, freq, pole):
    """cg at the start of fit (freq, pole), period_search_BOINC.cpp:819-844,
    from the context's own host tables."""
    import numpy as np

    beta_pole = [0, 0, 0, 0, 60, 60, 60, -60, -60, -60]
    lambda_pole = [0, 90, 180, 270, 60, 180, 300, 60, 180, 300]
    C = g.ncoef
    a = np.zeros(g.ma)
    a[:C] = g.array("cg_first")
    a[C] = np.radians(90.0 - beta_pole[pole - 1])
    a[C + 1] = np.radians(lambda_pole[pole - 1])
    a[C + 2] = 24 * 2 * np.pi * freq
    return a


def run_adjoint(args, path, local):
    """Matrix-free Gauss-Newton products J^T W (J v) (ps_gn_product) at the
    workload's size: products per second through the C ABI (parameters and
    direction uploaded, result read back per call), with the FLOP count of
    one product, 4 N F C (two passes over the (point, facet) pairs, two F x C
    contractions)."""
    import numpy as np
    import torch

    import periodsearch_b200 as ps

    torch.cuda.set_device(local)
    g = ps.PeriodSearch(path, device=local, form=ps.PS_FORM_FAST)
    g.set_conw_r(g.conw_r)
    lines = open(path).read().split("\n")
    par = [float(lines[k].split()[0]) for k in (6, 7, 8)]
    cl = float(lines[9].split()[0])
    a = initial_parameters(g, g.freq_start, 1)
    a[g.ncoef + 3:g.ncoef + 6] = par
    a[g.ncoef + 6] = np.log(cl)
    a[g.ncoef + 7] = 1.0
    v = np.random.default_rng(0).standard_normal(g.mfit)
    n = 3 if args.profile else 20
    for _ in range(3):
        g.gn_product(a, v)
    torch.cuda.synchronize()
    launches0 = ps.load_library().ps_kernel_launches()
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps * n):
            out = g.gn_product(a, v)
        dt = time.perf_counter() - t0
    launches = ps.load_library().ps_kernel_launches() - launches0
    assert np.all(np.isfinite(out))
    N, F, C = g.n_points, g.numfac, g.ncoef
    flop = 4.0 * N * F * C
    rate = args.steps * n / dt
    fp64_peak = ps.fp64_tensor_peak(local)
    line = {"metric": "matrix-free Gauss-Newton products/sec on 1 B200", "value": rate, "unit": "products/s",
            "n_gpus": 1, "steps": args.steps, "warmup": 3, "ms_per_step": 1000 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": (WORKLOAD_C5 if args.config == "c5" else WORKLOAD), "form": "adjoint (ps_gn_product)",
                       "products_per_step": n},
            "roofline": {"bound": "tensor", "achieved": flop * rate / 1e12, "peak": fp64_peak, "unit": "TFLOP/s",
                         "frac": flop * rate / 1e12 / fp64_peak, "flop_rule": "4 N F C per product",
                         "peak_source": "FP64 tensor-core throughput measured live on this GPU"},
            "gpu_launches": int(launches), "clocks": clk.summary(),
            "e2e": {"value": rate, "unit": "products/s", "h2d_bytes_per_step": int(n * 8 * (g.ma + g.ma)),
                    "d2h_bytes_per_step": int(n * 8 * (g.mfit + 1))}}
    if not args.profile:
        # one whole LM fit driven by these kernels alone (ps_fit_jfree)
        t0 = time.perf_counter()
        rj = g.fit_jfree(g.freq_start, 1)
        tj = time.perf_counter() - t0
        line["jfree_fit"] = {"fits_per_s": 1.0 / tj, "seconds": tj, "niter": int(rj["niter"]),
                             "what": "one Jacobian-free LM fit (ps_fit_jfree, period 1, pole 1): per accepted step "
                                     "alpha from mfit Gauss-Newton products plus the gradient pass, per trial "
                                     "point the gradient pass, each over the whole GPU; the solve on the host"}
    g.close()
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--periods-per-step", type=int, default=592)
    ap.add_argument("--form", default="fast", choices=["fp64", "fast", "mixed", "adjoint"],
                    help="fast: FP64 with the shape block on FP64 tensor cores (the headline); fp64: reference operation order")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip timing the other numerical forms on one batch")
    ap.add_argument("--no-extra", action="store_true", help="skip the one-step c4 and c5 measurements")
    ap.add_argument("--config", default="c2", choices=["c2", "c4", "c5"],
                    help="c2: production sparse search (the headline); c4: uneven multi-asteroid batch; "
                         "c5: lmax 8 / 2048 facets / 20000 points (14 periods per step, no pre-pass)")
    ap.add_argument("--asteroids", type=int, default=512)
    ap.add_argument("--no-autotune", action="store_true", help="keep the default tile shapes")
    ap.add_argument("--c4-periods", type=int, default=4)
    ap.add_argument("--profile", action="store_true",
                    help="small case for ncu: 30 periods (300 fits, about one wave) per step, no pre-pass, no e2e/cpu legs")
    args = ap.parse_args()
    if args.config == "c5":
        # 140 fits: one wave at one fit (CTA) per SM; the pre-pass is skipped
        args.periods_per_step = min(args.periods_per_step, 14)
    if args.profile:
        args.periods_per_step = 30
        args.no_cpu = args.no_e2e = args.no_forms = args.no_extra = True

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.config == "c4" and args.impl == "b200":
        if args.form == "adjoint":
            ap.error("the batched scan runs the fp64, fast and mixed forms")
        run_c4(args, local)
        return
    workdir = tempfile.mkdtemp(prefix="psbench")
    path = make_input(workdir, args.config)

    if args.impl == "reference":
        run_reference(args, path, rank)
        return
    if args.form == "adjoint":
        run_adjoint(args, path, local)
        return

    import numpy as np
    import torch

    import periodsearch_b200 as ps

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    form = {"fp64": ps.PS_FORM_FP64, "fast": ps.PS_FORM_FAST, "mixed": ps.PS_FORM_MIXED}[args.form]
    g = ps.PeriodSearch(path, device=local, form=form)
    # convexity-weight pre-pass (100 fits per round), timed on its own
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    if args.profile or args.config == "c5":
        conw_r = g.conw_r
        g.set_conw_r(conw_r)
    else:
        conw_r = g.precalc()
    torch.cuda.synchronize()
    prepass_s = time.perf_counter() - t0
    tiles = None
    if not args.no_autotune and not args.profile and args.form in ("fp64", "fast"):
        tiles, _ = g.autotune(60)
    n_total = g.n_periods
    B = args.periods_per_step
    fits_per_step = 10 * B
    # a dedicated stream: the C ABI treats a NULL stream as "the library's own
    # stream", and torch's default stream has handle 0
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    d_rec = torch.zeros(B * 6, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    # the product's period partition (periodsearch_b200.shard): blocks of B
    # consecutive trial periods dealt round-robin over the ranks; a rank's
    # steps walk through its own full blocks (and start over on a long run),
    # so ranks never scan the same periods
    from periodsearch_b200.shard import period_blocks

    blocks = [blk for blk in period_blocks(n_total, world, rank, B) if blk[1] - blk[0] + 1 == B]
    if not blocks:
        raise SystemExit(f"fewer than {B * world} trial periods for {world} ranks")

    def batch(step):
        return blocks[step % len(blocks)]

    for s in range(args.warmup):
        a, b = batch(s)
        g.scan_device(a, b, d_rec.data_ptr(), stream.cuda_stream)
    barrier()
    launches0 = ps.load_library().ps_kernel_launches()
    times = []
    with ClockSampler(local) as clk:
        for s in range(args.steps):
            flush.zero_()
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            a, b = batch(args.warmup + s)
            e0.record(stream)
            g.scan_device(a, b, d_rec.data_ptr(), stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1000.0)
    launches = ps.load_library().ps_kernel_launches() - launches0
    t_rank = torch.tensor([sum(times)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t_rank, op=dist.ReduceOp.MAX)
    t_max = float(t_rank.item())
    value = world * fits_per_step * args.steps / t_max
    clocks = clk.summary()

    # e2e through the public API from host buffers: per step, open a context
    # from the caller's host arrays (host setup, uploads), set conw_r, scan
    # the step's periods into host records, close.  The timed e2e steps scan
    # the same period batches as the first device-timed steps, so the two
    # can be compared batch for batch; one untimed e2e call on a warm-up
    # batch comes first.
    rec_host = np.zeros(B, dtype=ps.RECORD_DTYPE)
    desc = _desc_from(g, path)
    h2d = sum(np.asarray(v).nbytes for v in desc.values() if isinstance(v, np.ndarray))
    n_e2e = 0 if args.no_e2e else min(args.steps, 5)
    e2e_times, phases = [], {"open": [], "set_conw_r": [], "scan": [], "close": []}
    for s in range(-1, n_e2e):
        a, b = batch(args.warmup + s)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h = ps.PeriodSearch(desc=desc, device=local, form=form)
        t1 = time.perf_counter()
        h.set_conw_r(conw_r)
        t2 = time.perf_counter()
        rec_host = h.scan(a, b)
        t3 = time.perf_counter()
        h.close()
        t4 = time.perf_counter()
        if s >= 0:
            e2e_times.append(t4 - t0)
            for k, dt in zip(phases, (t1 - t0, t2 - t1, t3 - t2, t4 - t3)):
                phases[k].append(dt)
    e2e_sum = sum(e2e_times)
    if dist and e2e_times:
        t_e2e = torch.tensor([e2e_sum], dtype=torch.float64, device="cuda")
        dist.all_reduce(t_e2e, op=dist.ReduceOp.MAX)  # the slowest rank, as for the device time
        e2e_sum = float(t_e2e.item())
    e2e_value = world * fits_per_step * len(e2e_times) / e2e_sum if e2e_times else None
    same = times[:len(e2e_times)]
    e2e_extra = {"device_same_batches": world * fits_per_step * len(same) / sum(same) if same else None,
                 "phase_ms_median": {k: 1000 * statistics.median(v) for k, v in phases.items() if v},
                 "step_ms": [round(1000 * t, 1) for t in e2e_times],
                 "device_step_ms": [round(1000 * t, 1) for t in same],
                 "steps": len(e2e_times)}

    # the other numerical forms on the first timed batch (same periods, same
    # L2 flush, device-resident), with their per-period chi2 difference to
    # this run's records of that batch
    forms = {}
    if not args.no_forms and world == 1:
        a0, b0 = batch(args.warmup)
        g.scan_device(a0, b0, d_rec.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        base = d_rec.view(B, 6).cpu().numpy().copy()
        own_s = times[0]
        for other in [f for f in ("fp64", "fast", "mixed") if f != args.form]:
            if other == "mixed" and g.ncoef > 64:
                forms[other] = {"unavailable": "the mixed form holds at most 64 shape coefficients"}
                continue
            h = ps.PeriodSearch(path, device=local, form={"fp64": ps.PS_FORM_FP64, "fast": ps.PS_FORM_FAST,
                                                           "mixed": ps.PS_FORM_MIXED}[other])
            h.set_conw_r(conw_r)
            h.scan_device(a0, a0 + 29, d_rec.data_ptr(), stream.cuda_stream)  # warm-up
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            h.scan_device(a0, b0, d_rec.data_ptr(), stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            t_o = e0.elapsed_time(e1) / 1000.0
            rec_o = d_rec.view(B, 6).cpu().numpy()
            rel = np.abs(rec_o[:, 2] - base[:, 2]) / np.abs(base[:, 2])
            top = lambda r, k: list(np.argsort(r[:, 2], kind="stable")[:k])
            forms[other] = {"fits_per_s": fits_per_step / t_o, "ratio_of_this_form_to_it": t_o / own_s,
                            "chi2_rel_diff_to_this_form": {"median": float(np.median(rel)),
                                                           "p90": float(np.quantile(rel, 0.9)),
                                                           "max": float(rel.max())},
                            "same_top1_10_20": [top(rec_o, k) == top(base, k) for k in (1, 10, 20)]}
            h.close()

    # check a few records of the last timed batch against the same call again
    got = d_rec.view(B, 6).cpu().numpy()
    assert np.all(np.isfinite(got)), "non-finite records"

    F, C, mfit, N = g.numfac, g.ncoef, g.mfit, g.n_points
    fe = flop_per_eval(N, F, C, mfit)
    flop_launch = fits_per_step * 51 * fe
    t_launch = statistics.mean(times)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    bf16 = peaks.get("bf16_tflops_sustained")
    bf16_src = "of measured (bf16 sustained)" if bf16 else "of fallback (1400 TFLOP/s)"
    bf16 = bf16 or 1400.0
    # the fits compute in FP64: the bound is the FP64 tensor pipe (equal to the
    # FP64 SIMT rate on B200), measured live on this GPU
    fp64_peak = ps.fp64_tensor_peak(local)
    achieved = flop_launch / t_launch / 1e12
    # nominal FP64 tensor rate: SMs x 64 FMA/clk (m8n8k4 DMMA) x 2 FLOP x the
    # maximum SM clock
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    theo = sms * 64 * 2 * (clocks.get("sm_max_mhz") or 1965.0) * 1e6 / 1e12
    roofline = {"bound": "tensor", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak, "peak_theoretical": theo, "frac_of_theoretical": achieved / theo,
                "peak_source": "FP64 tensor-core throughput (m8n8k4 MMA) measured live on this GPU; "
                               "the measured-peaks file holds bf16 and HBM figures only",
                "traffic": None,
                "bf16_peak_tflops": bf16, "frac_of_bf16": achieved / bf16, "bf16_peak_source": bf16_src,
                "kernel": {"fp64": f"fit_kernel<{g.ncb},false> (FP64 SIMT, reference operation order, no FMA)",
                           "fast": f"fit_kernel<{g.ncb},true> (shape block on FP64 tensor cores, FP64 SIMT per pair)",
                           "mixed": "mixed_fit_kernel (FP64/FP32 SIMT + tcgen05 split-BF16 shape block)"}[args.form],
                "flop_per_launch": flop_launch,
                "flop_rule": "per evaluation 2 N F C + N mfit (mfit + 1), 51 evaluations per fit"}
    # DRAM bytes per fit from ncu (dram__bytes_read.sum + dram__bytes_write.sum)
    # on the 300-fit profile launch of the c2 workload (bench.py --profile),
    # scaled to this launch's fits: mostly the per-CTA J scratch (356 KB),
    # written back from L2 at two fits per SM
    per_fit = {"fast": 2.50e7, "fp64": 1.83e7}.get(args.form) if args.config == "c2" else None
    if per_fit:
        roofline["traffic"] = per_fit * fits_per_step
        roofline["traffic_source"] = ("ncu dram bytes of the 300-fit c2 profile launch of this form, "
                                      "scaled by fits per launch")
    line = {
        "metric": METRIC, "value": value, "unit": "fits/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32+bf16x3" if args.form == "mixed" else "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD_C5 if args.config == "c5" else WORKLOAD, "form": {"fp64": "fp64 (drop-in, reference operation order)", "fast": "fast fp64 (rearranged, fused; rounding-level differences)", "mixed": "mixed (FP64 model/solve, FP32 derivatives, tcgen05 split-BF16 shape block)"}[args.form], "periods_per_step": B,
                   "fits_per_step": fits_per_step, "l2": "flushed (256 MB write) between timed steps",
                   "prepass": {"fits": getattr(g, "prepass_fits", 0), "seconds": prepass_s, "conw_r": conw_r,
                               "fits_per_s": (getattr(g, "prepass_fits", 0) / prepass_s) if prepass_s else None},
                   "tiles": {"fch": tiles[0], "rt": tiles[1], "sortseg": tiles[2], "chosen_by": "ps_autotune"}
                   if tiles else "defaults (40, 32, 1024)",
                   "parallelism": f"period shards x{world}"},
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": "fits/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(rec_host.nbytes), **e2e_extra},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "forms": forms or None,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        r, why = ref_cpu_sample_or_none(path, 1)
        if r is not None:
            v, cores, done, dt = r
            line["cpu_baseline"] = {"value": v, "unit": "fits/s", "cores": cores, "kind": "reference",
                                    "sample": f"{done} fits: {cores} processes of the reference CPU application x 1 "
                                              f"trial period, pre-pass skipped, {dt:.1f} s"}
        else:
            if args.config == "c5":
                v, cores, done, dt = cpu_eval_sample(path, conw_r, 1, 51)
                sample = (f"{done} model evaluations (one per process) of the CPU oracle, {dt:.1f} s, "
                          f"converted at 51 evaluations per 50-iteration fit")
            else:
                v, cores, done, dt = cpu_sample(path, conw_r, 1)
                sample = f"{done} fits ({cores} processes x 2) of the same workload, {dt:.1f} s"
            line["cpu_baseline"] = {"value": v, "unit": "fits/s", "cores": cores, "kind": "port",
                                    "sample": sample + (f"; {why}" if why else "")}
    g.close()
    if rank == 0 and world == 1 and not args.no_extra and args.config == "c2":
        line["other_workloads"] = extra_workloads(args, local)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def _desc_from(g, path):
    """Host arrays of the workload as ps_open takes them (what a caller of
    the C ABI owns), taken from the library's own host parse."""
    import numpy as np

    lines = open(path).read().splitlines()
    hdr = lines[0].split()
    vals = [l.split() for l in lines[1:14]]
    nlc = int(lines[14].split()[0])
    i = 15
    lc_points, lc_rel, jd = [], [], []
    for _ in range(nlc):
        n, flag = (int(x) for x in lines[i].split()[:2])
        lc_points.append(n)
        lc_rel.append(1 - flag)
        jd.extend(float(lines[i + 1 + k].split()[0]) for k in range(n))
        i += n + 1
    N = g.n_points
    return {
        "lc_points": np.array(lc_points, np.int32), "lc_relative": np.array(lc_rel, np.int32),
        "tim": g.array("tim"), "ee": g.array("ee"), "ee0": g.array("ee0"),
        "brightness": g.array("brightness")[:N], "sig": g.array("sig")[:N], "weight": g.array("weight")[:N],
        "per_start": float(hdr[0]), "per_step_coef": float(hdr[1]), "per_end": float(hdr[2]),
        "ia_prd": int(hdr[3]), "phi0_rad": float(vals[1][0]) * (np.pi / 180), "conw": float(vals[2][0]),
        "lmax": int(vals[3][0]), "mmax": int(vals[3][1]), "nrows": int(vals[4][0]),
        "par": [float(vals[5][0]), float(vals[6][0]), float(vals[7][0])],
        "ia_par": [int(vals[5][1]), int(vals[6][1]), int(vals[7][1])], "cl": float(vals[8][0]),
        "ia_cl": int(vals[8][1]), "stop_condition": float(vals[9][0]), "n_iter_min": int(vals[10][0]),
        "alamda_incr": float(vals[11][0]), "alamda_start": float(vals[12][0]), "jd_min": min(jd),
        "jd_max": max(jd), "escl": g.escl,
    }


if __name__ == "__main__":
    main()
