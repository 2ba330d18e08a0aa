#!/usr/bin/env python
"""Benchmark: exact Matern log-likelihood evaluations per second on B200.

One step = one evaluation of the hot path (generate Sigma(theta) -> tiled
Cholesky with fused log-det and solve -> log-likelihood) for the N = 100,000
univariate Matern field (317 x 317 jittered unit-square grid truncated to
1e5 points, theta = (1.0, 0.05, 0.5), z = L e from the reference's
generator).  Three legs are timed: plain FP64; the reduced-precision path
that gives the headline value (default: FP64 tiles with INT8-sliced trailing
updates on the tensor cores; its |dl|/|l| against the FP64 leg is in the
line); and, as a reported sub-result, the reference's banded mixed-precision
scheme (FP32 off-band tiles, TF32 tensor cores).  The covariance (20-40 GB of
tiles) is far larger than L2, so no explicit L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--n N] [--impl ours|reference]

With N > 1 GPUs (torchrun) every rank evaluates its own replica field (the
single-field path does not shard); value = all ranks' evaluations / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("exact Matern log-likelihood evaluations per second, N=100000, 1 B200: reduced-precision tensor-core "
          "path (FP64 tiles, INT8-sliced trailing updates) vs plain FP64")
UNIT = "loglik-evals/s"
THETA = [1.0, 0.05, 0.5]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--n", type=int, default=100000)
    ap.add_argument("--ts", type=int, default=512)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mle", action="store_true", help="skip the time-to-MLE block (N = 40000) of the default line")
    ap.add_argument("--no-mixed-leg", action="store_true", help="skip the TF32 banded mixed-precision sub-result")
    ap.add_argument("--band", type=int, default=2, help="FP64 band width in tiles (mixed leg)")
    ap.add_argument("--mode", choices=["evals", "bands", "mle", "batch", "grad", "predict", "assess"], default="evals",
                    help="evals: the default bench line; bands: accuracy/time per band width; "
                         "mle: time-to-MLE of the drivers; batch: batched regional fields; grad: gradient cost; "
                         "predict: kriging; assess: Fisher information and MLOE / MMOM")
    ap.add_argument("--bands", default="1,2,4,8,16")
    ap.add_argument("--no-sliced-row", dest="sliced_row", action="store_false",
                    help="bands mode: skip the INT8-sliced row")
    ap.add_argument("--fields", type=int, default=512)
    ap.add_argument("--nmiss", type=int, default=1000, help="predict and assess modes: held-out points")
    ap.add_argument("--fisher-n", type=int, default=20000, help="assess mode: locations of the Fisher matrix")
    ap.add_argument("--assess-n", type=int, default=40000, help="assess mode: locations for MLOE / MMOM")
    ap.add_argument("--stage1-ftol", type=float, default=1e-3, help="mle mode, two_stage: first-stage tolerance")
    ap.add_argument("--stage1-maxeval", type=int, default=400, help="mle mode, two_stage: first-stage cap")
    ap.add_argument("--theta0", default="1.0,0.1,0.5", help="mle mode: parameters of the synthetic field")
    ap.add_argument("--drivers", default="bobyqa_fp64,bobyqa_sliced,lbfgsb_grad_fp64,lbfgsb_grad_sliced,"
                    "lbfgsb_sliced_polish",
                    help="mle mode: comma list of bobyqa_fp64, bobyqa_sliced, bobyqa_mixed, lbfgsb_grad_fp64, "
                         "lbfgsb_grad_sliced, lbfgsb_sliced_polish, bobyqa_sliced_polish, two_stage, tr_fp64, "
                         "tr_sliced")
    ap.add_argument("--passes", type=int, default=3, help="TF32 passes of the off-band update (1 or 3)")
    ap.add_argument("--scheme", choices=["mixed", "sliced"], default="sliced",
                    help="reduced-precision leg: mixed = FP32 off-band tiles on TF32 tensor cores; "
                         "sliced = FP64 tiles with INT8-sliced off-band updates")
    return ap.parse_args()


def workload(n):
    side = 1
    while side * side < n:
        side += 1
    return "univariate Matern exact loglik, N=%d (%dx%d jittered grid truncated), theta=(%g, %g, %g), FP64" % (
        n, side, side, *THETA)


# ---------------------------------------------------------------- clocks ----
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------- CPU (oracle) leg ----
C2_N = 40000  # the 200 x 200 grid of the plain-FP64 GPU configuration


def cpu_eval(n, seed=0, theta=THETA):
    """One full oracle log-likelihood evaluation (the C restatement of the
    reference CPU path: generation, tile Cholesky, log-det, solve) of the
    GenerateXYLoc(n, seed) field on all host threads; z ~ N(0,1).  Returns
    (seconds, (generation, factorisation, solve) seconds)."""
    import numpy as np

    import oracle

    oracle.build()
    oracle.set_threads(os.cpu_count() or 1)
    x, y = oracle.generate_xy_loc(n, seed)
    z = np.random.default_rng(seed).standard_normal(n)
    t0 = time.perf_counter()
    _, _, _, phases = oracle.dmle(x, y, z, theta)
    return time.perf_counter() - t0, phases


def scaled_to(n_target, n, phases):
    """Seconds of one evaluation at n_target from the phases measured at n:
    generation and solve scale by N^2, the Cholesky by N^3."""
    s = n_target / n
    tg, tc, tsv = phases
    return tg * s * s + tc * s ** 3 + tsv * s * s


def cpu_baseline_from(n_target, n, wall, phases, label):
    threads = os.cpu_count() or 1
    t_full = scaled_to(n_target, n, phases)
    return {"value": 1.0 / t_full, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "%s: one full oracle evaluation at N=%d measured (%.2f s: gen %.2f, chol %.2f, solve %.2f) on "
                      "%d threads, extrapolated to N=%d by N^2 (gen, solve) and N^3 (chol)" % (
                          label, n, wall, phases[0], phases[1], phases[2], threads, n_target),
            "measured_n": n, "measured_seconds_per_eval": wall, "extrapolated": n_target != n,
            "seconds_per_eval_extrapolated": t_full}


def run_reference(args):
    """The reference arm: the oracle port of the reference CPU path on all
    host threads.  A full evaluation at N = 1e5 needs an 80 GB dense array and
    ~10 minutes of CPU per step, so every timed step is one full evaluation of
    the C2-sized field (N = 40 000, the same generator and theta) and the
    value is extrapolated from it to N = 1e5 (N^3 factorisation, N^2 rest),
    labelled as such.  Warm-up steps evaluate a small field."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n_s = min(args.n, C2_N)
    for _ in range(args.warmup):
        cpu_eval(2000, args.seed)
    walls, phases = [], []
    # each step is a full N = 40 000 evaluation (about 30-60 s on 16 host
    # cores); at most three are run so the arm ends within a few minutes
    steps_run = min(args.steps, 3)
    for _ in range(steps_run):
        w, ph = cpu_eval(n_s, args.seed)
        walls.append(w)
        phases.append(ph)
    med = sorted(range(len(walls)), key=lambda i: walls[i])[len(walls) // 2]
    cb = cpu_baseline_from(args.n, n_s, walls[med], phases[med], "reference arm step")
    value = cb["value"]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload(args.n), "sample": cb["sample"],
                       "measured_seconds_per_step": walls, "measured_n": n_s, "steps_run": steps_run,
                       "value_is": "extrapolated from the measured N=%d evaluations" % n_s if n_s != args.n
                       else "measured"},
            "cpu_baseline": cb, "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------- our arm -----
def measured_dgemm_tflops(torch):
    """cuBLAS DGEMM (torch.matmul, float64, 8192^3) best of 5 -- the FP64
    tensor-core denominator (MEASURED_PEAKS.json has no FP64 entry)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = torch.empty_like(a)
    best = 0.0
    for _ in range(6):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b, out=c)
        e.record()
        e.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b, c
    torch.cuda.empty_cache()
    return best


def peak_bf16_tflops():
    """Measured dense bf16 peak from MEASURED_PEAKS.json, if present."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["bf16_tflops"]), float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), "MEASURED_PEAKS.json"
    except (OSError, KeyError, ValueError):
        return 1590.0, 1400.0, "fallback"


def timed_leg(sess, theta, steps, warmup, barrier):
    for _ in range(warmup):
        sess.loglik(theta)
    sess.set_profiling(True)
    barrier()
    lls = [sess.loglik(theta) for _ in range(steps)]
    barrier()
    prof = sess.profile()
    sess.set_profiling(False)
    return lls, prof


def mode_bands(args):
    """|dl|/|l| and time per evaluation for each FP64 band width (mixed path)
    against the FP64 path on the same field."""
    os.environ.setdefault("EXAGEOSTAT_B200_SILENT", "1")
    import exageostat_b200 as xg
    from exageostat_b200.synthetic import dlarnv

    xg.init(args.ts)
    x, y = xg.generate_xy_loc(args.n, args.seed)
    sess = xg.Session(x, y, dts=args.ts)
    sess.zvg(THETA, dlarnv(args.seed, args.n))

    def timed(k):
        t0 = time.perf_counter()
        v = [sess.loglik(THETA) for _ in range(k)]
        return v[-1], (time.perf_counter() - t0) / k

    sess.loglik(THETA)
    ll64, t64 = timed(2)
    rows = []
    for band in [int(b) for b in args.bands.split(",") if b]:
        sess.set_mixed(band=band, passes=args.passes)
        sess.loglik(THETA)
        ll, t = timed(2)
        rows.append({"scheme": "fp32-offband-tf32x%d" % args.passes, "band": band, "seconds": t,
                     "speedup_vs_fp64": t64 / t, "loglik": ll, "rel_err_vs_fp64": abs(ll - ll64) / abs(ll64)})
        sess.set_fp64()
    if args.sliced_row:
        sess.set_sliced()
        sess.loglik(THETA)
        ll, t = timed(2)
        rows.append({"scheme": "fp64-int8-sliced", "band": None, "seconds": t, "speedup_vs_fp64": t64 / t,
                     "loglik": ll, "rel_err_vs_fp64": abs(ll - ll64) / abs(ll64)})
        sess.set_fp64()
    sess.close()
    print(json.dumps({"mode": "bands", "workload": workload(args.n), "tile": args.ts, "fp64_seconds": t64,
                      "loglik_fp64": ll64, "rows": rows}), flush=True)


def mode_mle(args):
    """Time-to-MLE of the reference driver's maximiser (derivative-free, start
    at the lower bounds, examples/examples.c:263-264, tolerance 1e-9) on the
    plain FP64 objective and on the reduced-precision objectives, and of
    L-BFGS-B with the adjoint gradient (FP64, or sliced with an optional FP64
    polish from its optimum; start at the box centre); bounds [0.01, 5]^3.
    theta-hat and loglik(theta-hat) are compared with the FP64 derivative-free
    run."""
    os.environ.setdefault("EXAGEOSTAT_B200_SILENT", "1")
    import numpy as np

    import exageostat_b200 as xg
    from exageostat_b200.autograd import fit_lbfgsb
    from exageostat_b200.synthetic import dlarnv

    xg.init(args.ts)
    theta0 = [float(v) for v in args.theta0.split(",")]
    x, y = xg.generate_xy_loc(args.n, args.seed)
    sess = xg.Session(x, y, dts=args.ts)
    sess.zvg(theta0, dlarnv(args.seed, args.n))
    lb, ub = [0.01] * 3, [5.0] * 3
    runs = {}

    def bobyqa(name, **extra):
        t0 = time.perf_counter()
        th, ll, ev = sess.fit_bobyqa(lb, ub, ftol_abs=1e-9)
        runs[name] = dict({"seconds": time.perf_counter() - t0, "evals": ev, "theta": th.tolist(), "loglik": ll},
                          **extra)
        progress("%s: %s" % (name, runs[name]))

    t_start = time.perf_counter()

    def progress(msg):
        print("[mle %.1f s] %s" % (time.perf_counter() - t_start, msg), file=sys.stderr, flush=True)

    drivers = args.drivers.split(",")
    if "bobyqa_fp64" in drivers:
        bobyqa("bobyqa_fp64")
    if "bobyqa_sliced" in drivers:
        sess.set_sliced()
        bobyqa("bobyqa_sliced")
        sess.set_fp64()
    if "bobyqa_sliced_polish" in drivers:
        # the reference driver on the sliced objective, then FP64 gradient steps from its optimum
        sess.set_sliced()
        t0 = time.perf_counter()
        th, ll, ev = sess.fit_bobyqa(lb, ub, ftol_abs=1e-9)
        sess.set_fp64()
        th2, ll2, ev2 = fit_lbfgsb(sess, lb, ub, x0=th)
        runs["bobyqa_sliced_polish"] = {"seconds": time.perf_counter() - t0, "evals": ev, "evals_fp64": ev2,
                                        "theta": th2.tolist(), "loglik": ll2, "theta_sliced": th.tolist()}
    if "two_stage" in drivers:
        # exageostat_b200.mle.fit_two_stage: derivative-free on the sliced objective, FP64 Newton polish
        from exageostat_b200.mle import fit_two_stage

        t0 = time.perf_counter()
        th, ll, ev1, ev2, th1 = fit_two_stage(sess, lb, ub, ftol_abs=args.stage1_ftol, maxeval=args.stage1_maxeval,
                                              log=progress)
        runs["two_stage"] = {"seconds": time.perf_counter() - t0, "evals": ev1, "grad_evals_fp64": ev2,
                             "theta": th.tolist(), "loglik": ll, "theta_sliced": th1.tolist()}
    if "bobyqa_mixed" in drivers:
        sess.set_mixed(band=args.band, passes=args.passes)
        bobyqa("bobyqa_mixed", band=args.band)
        sess.set_fp64()
    if "lbfgsb_grad_sliced" in drivers or "lbfgsb_sliced_polish" in drivers:
        sess.set_sliced()
        t0 = time.perf_counter()
        th, ll, ev = fit_lbfgsb(sess, lb, ub, x0=[0.5, 0.5, 0.5])
        t_sl = time.perf_counter() - t0
        sess.set_fp64()
        if "lbfgsb_grad_sliced" in drivers:
            runs["lbfgsb_grad_sliced"] = {"seconds": t_sl, "evals": ev, "theta": th.tolist(), "loglik": ll}
        if "lbfgsb_sliced_polish" in drivers:
            # the sliced optimum refined by FP64 gradient steps
            t0 = time.perf_counter()
            th2, ll2, ev2 = fit_lbfgsb(sess, lb, ub, x0=th)
            runs["lbfgsb_sliced_polish"] = {"seconds": t_sl + time.perf_counter() - t0, "evals": ev,
                                            "evals_fp64": ev2, "theta": th2.tolist(), "loglik": ll2}
    if "tr_sliced" in drivers:
        # mixed-precision adjoint-gradient MLE (exageostat_b200.mle.fit_mixed): start point, trust region on the
        # sliced objective and gradient, ridge search with sliced values
        from exageostat_b200.mle import fit_mixed

        t0 = time.perf_counter()
        th, ll, ev1, ev2, th1 = fit_mixed(sess, lb, ub, log=progress)
        runs["tr_sliced"] = {"seconds": time.perf_counter() - t0, "grad_evals": ev1, "loglik_evals": ev2,
                             "theta": th.tolist(), "loglik": ll, "theta_gradient_stage": th1.tolist()}
        progress("tr_sliced: %s" % runs["tr_sliced"])
    if "tr_fp64" in drivers:
        # the same driver in plain FP64 (exageostat_b200.mle.fit_fp64)
        from exageostat_b200.mle import fit_fp64

        t0 = time.perf_counter()
        th, ll, ev, ne = fit_fp64(sess, lb, ub, log=progress)
        runs["tr_fp64"] = {"seconds": time.perf_counter() - t0, "grad_evals": ev, "loglik_evals": ne,
                           "theta": th.tolist(), "loglik": ll}
        progress("tr_fp64: %s" % runs["tr_fp64"])
    if "lbfgsb_grad_fp64" in drivers:
        t0 = time.perf_counter()
        th, ll, ev = fit_lbfgsb(sess, lb, ub, x0=[0.5, 0.5, 0.5])
        runs["lbfgsb_grad_fp64"] = {"seconds": time.perf_counter() - t0, "evals": ev, "theta": th.tolist(),
                                    "loglik": ll}
    refname = next((r for r in ("bobyqa_fp64", "tr_fp64", "lbfgsb_grad_fp64") if r in runs), None)
    if refname:
        ref = np.array(runs[refname]["theta"])
        llref = runs[refname]["loglik"]
        for name, r in runs.items():
            r["theta_rel_diff_vs_ref"] = float(np.max(np.abs(np.array(r["theta"]) - ref) / np.abs(ref)))
            r["speedup_vs_" + refname] = runs[refname]["seconds"] / r["seconds"]
            # the objective of every run evaluated in FP64 at its own optimum
            r["loglik_fp64_at_theta"] = sess.loglik(r["theta"])
            r["loglik_rel_diff_vs_ref"] = abs(r["loglik_fp64_at_theta"] - llref) / abs(llref)
    sess.close()
    print(json.dumps({"mode": "mle", "n": args.n, "theta0": theta0, "reference_run": refname, "runs": runs}),
          flush=True)


def mode_grad(args):
    """Seconds per log-likelihood + gradient evaluation, plain FP64 and
    sliced, and the difference of the two gradients."""
    os.environ.setdefault("EXAGEOSTAT_B200_SILENT", "1")
    import numpy as np

    import exageostat_b200 as xg
    from exageostat_b200.synthetic import dlarnv

    xg.init(args.ts)
    x, y = xg.generate_xy_loc(args.n, args.seed)
    sess = xg.Session(x, y, dts=args.ts)
    sess.zvg(THETA, dlarnv(args.seed, args.n))
    out = {"mode": "grad", "workload": workload(args.n), "tile": args.ts}
    for name in (["fp64"] if args.n > 120000 else []) + ["fp64", "sliced"]:
        if name == "sliced":
            sess.set_sliced()
        sess.loglik(THETA, grad=True)
        t0 = time.perf_counter()
        ll, g = sess.loglik(THETA, grad=True)
        dt = time.perf_counter() - t0
        t0 = time.perf_counter()
        sess.loglik(THETA)
        dl = time.perf_counter() - t0
        out[name] = {"seconds_loglik_grad": dt, "seconds_loglik": dl, "ratio": dt / dl, "loglik": ll,
                     "grad": list(np.asarray(g, dtype=float))}
    g64, gsl = np.array(out["fp64"]["grad"]), np.array(out["sliced"]["grad"])
    out["grad_max_rel_diff"] = float(np.max(np.abs(gsl - g64)) / max(np.max(np.abs(g64)), 1.0))
    out["speedup_grad"] = out["fp64"]["seconds_loglik_grad"] / out["sliced"]["seconds_loglik_grad"]
    sess.close()
    print(json.dumps(out), flush=True)


def mode_predict(args):
    """Kriging (EXAGEOSTAT_dmle_Predict_Tile, MLE_dexact.c:688-874): a seeded
    uniform hold-out of --nmiss points of the field, prediction from the rest
    at theta0 through the C ABI (host arrays, copies included), wall clock;
    the CPU oracle on a bounded sample (N_s observed points) scaled by N^3."""
    os.environ.setdefault("EXAGEOSTAT_B200_SILENT", "1")
    import numpy as np

    import exageostat_b200 as xg
    from exageostat_b200.synthetic import dlarnv

    xg.init(args.ts)
    theta0 = [float(v) for v in args.theta0.split(",")]
    N, nmiss = args.n, args.nmiss
    x, y = xg.generate_xy_loc(N, args.seed)
    sess = xg.Session(x, y, dts=args.ts)
    sess.zvg(theta0, dlarnv(args.seed, N))
    z = sess.z()
    rng = np.random.default_rng(args.seed)
    miss = np.zeros(N, dtype=bool)
    miss[rng.choice(N, nmiss, replace=False)] = True
    xm, ym, zact, xo, yo, zo = x[miss], y[miss], z[miss], x[~miss], y[~miss], z[~miss]
    sess.predict(theta0, xm, ym, xo, yo, zo, zact)  # warm-up (allocates the kriging descriptors)
    times = []
    for _ in range(max(1, args.steps)):
        t0 = time.perf_counter()
        mse, zmiss = sess.predict(theta0, xm, ym, xo, yo, zo, zact)
        times.append(time.perf_counter() - t0)
    sess.close()
    out = {"mode": "predict", "n": N, "n_obs": int(N - nmiss), "n_miss": nmiss, "theta0": theta0,
           "seconds": min(times), "mse": mse, "var_z_actual": float(np.var(zact))}
    if not args.no_cpu_baseline:
        import oracle

        oracle.set_threads(os.cpu_count() or 1)
        ns = min(N, 8000)
        t0 = time.perf_counter()
        oracle.dpredict(xm[:min(nmiss, 200)], ym[:min(nmiss, 200)], xo[:ns], yo[:ns], zo[:ns], None, theta0)
        tc = time.perf_counter() - t0
        out["cpu_baseline"] = {"seconds_sample": tc, "sample_n_obs": ns, "cores": os.cpu_count(), "kind": "port",
                               "seconds_extrapolated": tc * ((N - nmiss) / ns) ** 3}
    print(json.dumps(out), flush=True)


def mode_assess(args):
    """Assessment of a fit: the Fisher information (EXAGEOSTAT_Fisher_Tile,
    MLE_dexact.c:1777-1934) of --fisher-n locations at theta0, and MLOE / MMOM
    (EXAGEOSTAT_dmle_mloe_mmom_Tile, MLE_dexact.c:1109-1434) of kriging --nmiss
    held-out points of --assess-n locations with a perturbed estimate, both
    through the C ABI on host arrays (wall clock, plus the library's device
    times).  CPU: the oracle on bounded samples, scaled by the reference
    algorithm's operation counts."""
    os.environ.setdefault("EXAGEOSTAT_B200_SILENT", "1")
    import numpy as np

    import exageostat_b200 as xg

    xg.init(0)
    theta0 = [float(v) for v in args.theta0.split(",")]
    est = [theta0[0] * 0.9, theta0[1] * 1.2, theta0[2] * 1.1]
    out = {"mode": "assess", "theta0": theta0, "estimated_theta": est}
    # Fisher information
    nf = args.fisher_n
    x, y = xg.generate_xy_loc(nf, args.seed)
    xg.fisher_host(x[:2048], y[:2048], theta0)  # warm-up (kernel load)
    t0 = time.perf_counter()
    F = xg.fisher_host(x, y, theta0, ts=args.ts)
    tf = time.perf_counter() - t0
    Np = -(-nf // 512) * 512
    out["fisher"] = {"n": nf, "seconds": tf, "F": F.tolist(), "inverse_diag": np.diag(np.linalg.inv(F)).tolist(),
                     "dense_gemm_tflops": 3 * 2.0 * Np ** 3 / tf / 1e12,
                     "check_F00_vs_N_over_2sigma4": float(F[0, 0] / (nf / (2 * theta0[0] ** 2)) - 1)}
    # MLOE / MMOM
    n, nmiss = args.assess_n, args.nmiss
    x, y = xg.generate_xy_loc(n, args.seed)
    rng = np.random.default_rng(args.seed)
    miss = np.zeros(n, dtype=bool)
    miss[rng.choice(n, nmiss, replace=False)] = True
    xm, ym, xo, yo = x[miss], y[miss], x[~miss], y[~miss]
    xg.mloe_mmom_host(xm[:16], ym[:16], xo[:2048], yo[:2048], theta0, est)  # warm-up
    t0 = time.perf_counter()
    mloe, mmom, _, dev = xg.mloe_mmom_host(xm, ym, xo, yo, theta0, est, ts=args.ts)
    tm = time.perf_counter() - t0
    out["mloe_mmom"] = {"n_obs": int(n - nmiss), "n_miss": nmiss, "seconds": tm, "mloe": mloe, "mmom": mmom,
                        "device_seconds": {"generation": dev[0], "factorisations": dev[1], "solves": dev[2],
                                           "total": dev[3]}}
    if not args.no_cpu_baseline:
        import oracle

        oracle.set_threads(os.cpu_count() or 1)
        ns = min(nf, 1500)
        t0 = time.perf_counter()
        oracle.fisher(x[:ns], y[:ns], theta0)
        tc = time.perf_counter() - t0
        # the reference: N^3/3 factorisation + per (j, k) two N x N TRSMs (and
        # per j two more) and one GEMM: 3 * 2 N^3 + 6 * (2 N^3 + 2 N^3) = 30 N^3
        out["fisher"]["cpu_baseline"] = {"seconds_sample": tc, "sample_n": ns, "cores": os.cpu_count(),
                                         "kind": "port", "seconds_extrapolated": tc * (nf / ns) ** 3}
        no_s, nm_s = min(n - nmiss, 4000), min(nmiss, 100)
        t0 = time.perf_counter()
        oracle.mloe_mmom(xm[:nm_s], ym[:nm_s], xo[:no_s], yo[:no_s], theta0, est)
        tc = time.perf_counter() - t0
        cost = lambda no, nm: 2.0 * no ** 3 / 3 + 5.0 * nm * no ** 2
        out["mloe_mmom"]["cpu_baseline"] = {
            "seconds_sample": tc, "sample_n_obs": no_s, "sample_n_miss": nm_s, "cores": os.cpu_count(),
            "kind": "port", "seconds_extrapolated": tc * cost(n - nmiss, nmiss) / cost(no_s, nm_s)}
    print(json.dumps(out), flush=True)


def mode_batch(args):
    """Batched regional fields (the batch workload: sizes U[500, 6000],
    locations uniform in each region's unit square, sigma^2 ~ U(0.5, 2), beta ~
    U(0.02, 0.3), nu ~ U(0.3, 2.5), z_i = L_i e_i from the library's MLE_zvg):
    seconds per evaluation of every field's loglik (one persistent launch
    under a CUDA graph), and of loglik + gradient, against looping the
    single-field FP64 path over every field (measured, wall clock)."""
    os.environ.setdefault("EXAGEOSTAT_B200_SILENT", "1")
    import numpy as np
    import torch

    import exageostat_b200 as xg

    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        return mode_batch_sharded(args)
    xg.init(0)
    rng = np.random.default_rng(args.seed)
    xs, ys, zs, th = [], [], [], []
    for f in range(args.fields):
        n = int(rng.integers(500, 6001))
        x, y = rng.random(n), rng.random(n)
        t = [rng.uniform(0.5, 2.0), rng.uniform(0.02, 0.3), rng.uniform(0.3, 2.5)]
        with xg.Session(x, y, dts=256) as s:
            s.zvg(t, rng.standard_normal(n))
            z = s.z()
        xs.append(x), ys.append(y), zs.append(z), th.append(t)
    th = np.array(th)
    with xg.Batch(xs, ys, zs, ts=256) as b:
        b.loglik(th)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            out = b.loglik(th)
        tb = (time.perf_counter() - t0) / args.steps
        b.loglik(th, grad=True)
        t0 = time.perf_counter()
        _, gb = b.loglik(th, grad=True)
        tbg = time.perf_counter() - t0
    t0 = time.perf_counter()
    loop = np.array([xg.dmle_host(x, y, z, t, ts=256)[0] for x, y, z, t in zip(xs, ys, zs, th)])
    tl = time.perf_counter() - t0
    # single fields of the workload's sizes: plain FP64 vs INT8-sliced (CUDA events of the library)
    per_field = []
    for n in (1000, 3000, 6000):
        i = int(np.argmin([abs(len(x) - n) for x in xs]))
        row = {"n": len(xs[i])}
        with xg.Session(xs[i], ys[i], dts=256) as s:
            s.set_data(z=zs[i])
            for name in ("fp64", "sliced"):
                if name == "sliced":
                    s.set_sliced()
                try:
                    for _ in range(2):
                        s.loglik(th[i])
                    s.set_profiling(True)
                    for _ in range(5):
                        s.loglik(th[i])
                    p = s.profile()
                    row[name + "_seconds"] = p["t_total"] / p["evals"]
                except xg.XgError as exc:
                    # a strongly correlated field can lose positive definiteness
                    # under the sliced update: recorded, not timed
                    row[name + "_seconds"] = None
                    row[name + "_error"] = str(exc)
                s.set_profiling(False)
        per_field.append(row)
    ok = np.isfinite(loop) & np.isfinite(out)
    err = float(np.max(np.abs(loop[ok] - out[ok]) / np.abs(loop[ok])))
    sizes = np.array([len(x) for x in xs])
    print(json.dumps({"mode": "batch", "fields": args.fields, "sizes": [int(sizes.min()), int(sizes.max())],
                      "flops": float(np.sum(sizes.astype(float) ** 3) / 3), "batched_seconds": tb,
                      "fields_per_s_batched": args.fields / tb, "batched_tflops": float(
                          np.sum(sizes.astype(float) ** 3) / 3) / tb / 1e12,
                      "batched_grad_seconds": tbg, "looped_seconds": tl,
                      "fields_per_s_looped": args.fields / tl, "speedup": tl / tb,
                      "fields_not_spd": int(np.sum(~np.isfinite(out))),
                      "single_field_sliced_vs_fp64": per_field,
                      "max_rel_diff_batched_vs_looped": err}), flush=True)


def c2_pair(xg, seed, ts):
    """Measured at the C2 size (N = 40 000, 200 x 200 grid, the headline's
    theta): evaluations per second of the GPU's plain FP64 and INT8-sliced
    paths (CUDA events, 3 timed after 2 warm-up) and of the CPU oracle (one
    full evaluation, all host threads) on the same z, with the log-likelihoods
    of all three."""
    from exageostat_b200.synthetic import dlarnv

    n = C2_N
    x, y = xg.generate_xy_loc(n, seed)
    sess = xg.Session(x, y, dts=ts)
    sess.zvg(THETA, dlarnv(seed, n))
    z = sess.z()
    out = {"n": n, "theta": THETA, "tile": ts}
    for name in ("fp64", "sliced"):
        if name == "sliced":
            sess.set_sliced()
        for _ in range(2):
            sess.loglik(THETA)
        sess.set_profiling(True)
        lls = [sess.loglik(THETA) for _ in range(3)]
        p = sess.profile()
        sess.set_profiling(False)
        out["gpu_" + name] = {"evals_per_s": p["evals"] / p["t_total"], "loglik": lls[-1]}
    sess.close()
    import oracle

    oracle.build()
    oracle.set_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    ll, _, _, phases = oracle.dmle(x, y, z, THETA)
    wall = time.perf_counter() - t0
    out["cpu_seconds_per_eval"] = wall
    out["cpu_phases"] = list(phases)
    out["cpu_cores"] = os.cpu_count()
    out["cpu_evals_per_s"] = 1.0 / wall
    out["cpu_loglik"] = ll
    out["gpu_fp64_rel_diff_vs_cpu"] = abs(out["gpu_fp64"]["loglik"] - ll) / abs(ll)
    out["gpu_sliced_rel_diff_vs_cpu"] = abs(out["gpu_sliced"]["loglik"] - ll) / abs(ll)
    out["speedup_fp64_vs_cpu"] = out["gpu_fp64"]["evals_per_s"] * wall
    out["speedup_sliced_vs_cpu"] = out["gpu_sliced"]["evals_per_s"] * wall
    return out


def mle_block(xg, seed, ts, n=C2_N, theta0=(1.0, 0.1, 0.5)):
    """Time-to-MLE at the C2 size (N = 40 000, a field z = L e generated at
    theta0), bounds [0.01, 5]^3, through the library's gradient drivers: the
    mixed-precision driver (exageostat_b200.mle.fit_mixed: INT8-sliced
    objective, sliced adjoint gradient, value-based Newton polish) against
    the same driver in plain FP64 (fit_fp64).  Wall clock of each fit; theta-hat
    compared with the FP64 one, and both optima evaluated in FP64."""
    import numpy as np

    from exageostat_b200.mle import fit_fp64, fit_mixed
    from exageostat_b200.synthetic import dlarnv

    x, y = xg.generate_xy_loc(n, seed)
    lb, ub = [0.01] * 3, [5.0] * 3
    out = {"n": n, "theta0": list(theta0), "bounds": [lb, ub]}
    with xg.Session(x, y, dts=ts) as s:
        s.zvg(list(theta0), dlarnv(seed, n))
        s.loglik(list(theta0))  # warm-up of the FP64 path
        t0 = time.perf_counter()
        th64, _, ev64, ne64 = fit_fp64(s, lb, ub)
        t64 = time.perf_counter() - t0
        s.set_sliced()
        s.loglik(list(theta0))  # warm-up of the sliced path
        t0 = time.perf_counter()
        thmx, _, evmx, nemx, _ = fit_mixed(s, lb, ub)
        tmx = time.perf_counter() - t0
        s.set_fp64()
        l64 = s.loglik(list(th64))
        lmx = s.loglik(list(thmx))
    out["fp64"] = {"seconds": t64, "grad_evals": ev64, "loglik_evals": ne64, "theta": list(th64), "loglik": l64}
    out["mixed"] = {"seconds": tmx, "grad_evals": evmx, "loglik_evals": nemx, "theta": list(thmx),
                    "loglik_fp64_at_theta": lmx}
    out["speedup"] = t64 / tmx
    out["theta_max_rel_diff"] = float(np.max(np.abs(np.array(thmx) - np.array(th64)) / np.abs(np.array(th64))))
    out["loglik_rel_diff"] = abs(lmx - l64) / abs(l64)
    return out


def ncu_traffic(kernel):
    """DRAM bytes per algorithmic operation of `kernel` from an ncu capture
    (profiles/ncu_traffic.json, written from the capture's raw CSV by
    profiles' recipe; holds the command that made it), or None."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)[kernel]
        return float(d["dram_bytes_per_op"]), d
    except (OSError, KeyError, ValueError, TypeError):
        return None, None


def mode_batch_sharded(args):
    """The batch workload sharded over the ranks of torchrun (NCCL): each
    rank evaluates its LPT share of the fields (exageostat_b200.sharding.
    ShardedBatch) and one all_gather hands every rank all log-likelihoods and
    gradients.  Timed on the device between barriers, max over ranks; value =
    all fields / that time."""
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    import exageostat_b200 as xg
    from exageostat_b200.sharding import ShardedBatch

    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    xg.init(0)
    rng = np.random.default_rng(args.seed)
    xs, ys, zs, th = [], [], [], []
    for f in range(args.fields):
        n = int(rng.integers(500, 6001))
        x, y = rng.random(n), rng.random(n)
        t = [rng.uniform(0.5, 2.0), rng.uniform(0.02, 0.3), rng.uniform(0.3, 2.5)]
        e = rng.standard_normal(n)
        xs.append(x), ys.append(y), th.append(t), zs.append(e)
    th = np.array(th)
    # z_i = L_i e_i for this rank's fields only (the others are never read here)
    sb = ShardedBatch(xs, ys, zs, ts=256)
    for i in sb.mine:
        with xg.Session(xs[i], ys[i], dts=256) as s:
            s.zvg(th[i], zs[i])
            zs[i] = s.z()
    sb.close()
    sb = ShardedBatch(xs, ys, zs, ts=256)
    out = {}
    for grad in (False, True):
        for _ in range(max(args.warmup, 1)):
            sb.loglik(th, grad=grad)
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            res = sb.loglik(th, grad=grad)
        torch.cuda.synchronize()
        dt = torch.tensor([(time.perf_counter() - t0) / args.steps], device="cuda", dtype=torch.float64)
        dist.all_reduce(dt, op=dist.ReduceOp.MAX)
        out["grad" if grad else "loglik"] = float(dt.item())
    ll = res[0]
    sb.close()
    if rank == 0:
        sizes = np.array([len(x) for x in xs])
        print(json.dumps({"mode": "batch", "n_gpus": world, "fields": args.fields, "scaling": "strong",
                          "sizes": [int(sizes.min()), int(sizes.max())],
                          "batched_seconds": out["loglik"], "fields_per_s_batched": args.fields / out["loglik"],
                          "batched_grad_seconds": out["grad"], "fields_not_spd": int(np.sum(~np.isfinite(ll))),
                          "fields_per_rank": [len(p) for p in sb.parts]}), flush=True)
    dist.barrier()
    dist.destroy_process_group()


def ingest_ncu(path, case, command, out_path=None):
    """Writes profiles/ncu_traffic.json from the raw page of an ncu capture
    (``ncu -i <rep> --page raw --csv``): per captured kernel, DRAM bytes
    (dram__bytes_read.sum + dram__bytes_write.sum, scaled by the unit row of
    the CSV) per algorithmic operation, the operations counted by the same
    capture -- INT8 tensor ops (sm__ops_path_tensor_op_utcimma_src_int8*.sum)
    or FP64 DMMA flops.  The DMMA instruction counter counts 8 x 8 x 4
    operations (512 flops each): the last sub-block GEMM of a 512 tile, one
    128^3 block of 4.19e6 flops, counts 8192."""
    import csv

    with open(path, newline="") as f:
        rows = list(csv.reader(f))
    head, units = rows[0], rows[1]
    col = {name: i for i, name in enumerate(head)}
    scale = {"": 1.0, "byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "Tbyte": 1e12, "inst": 1.0}

    def num(r, name):
        if name not in col:
            return None
        v = r[col[name]].replace(",", "")
        try:
            return float(v) * scale.get(units[col[name]].strip(), 1.0)
        except ValueError:
            return None

    i8_name = next((n for n in ("sm__ops_path_tensor_op_utcimma_src_int8.sum",
                                "sm__ops_path_tensor_op_utcimma_src_int8_sparsity_off.sum") if n in col), None)
    per = {}
    for r in rows[2:]:
        if len(r) != len(head):
            continue
        name = r[col["Kernel Name"]].split("(")[0].split("<")[0].strip()
        name = name[5:] if name.startswith("void ") else name
        rd, wr = num(r, "dram__bytes_read.sum"), num(r, "dram__bytes_write.sum")
        i8 = num(r, i8_name) if i8_name else None
        dm = num(r, "sm__inst_executed_pipe_tensor_subpipe_dmma.sum")
        ops = i8 if i8 else (512.0 * dm if dm else None)
        if rd is None or wr is None or not ops:
            continue
        per.setdefault(name, []).append((rd + wr, ops))
    out_path = out_path or os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(out_path) as f:
            out = json.load(f)
    except (OSError, ValueError):
        out = {}
    for name, v in per.items():
        b = sum(x[0] for x in v)
        o = sum(x[1] for x in v)
        out[name] = {"dram_bytes_per_op": b / o, "launches": len(v), "dram_bytes": b, "ops": o, "case": case,
                     "command": command}
    with open(out_path, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "--ingest-ncu":
        ingest_ncu(sys.argv[2], sys.argv[3], sys.argv[4])
        return
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.mode != "evals":
        {"bands": mode_bands, "mle": mode_mle, "batch": mode_batch, "grad": mode_grad,
         "predict": mode_predict, "assess": mode_assess}[args.mode](args)
        return
    import numpy as np
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    os.environ.setdefault("EXAGEOSTAT_B200_SILENT", "1")
    import exageostat_b200 as xg
    from exageostat_b200 import build as xgbuild
    from exageostat_b200.synthetic import dlarnv

    if not os.path.exists(xg.LIB_PATH):
        xgbuild.build()
    fp64_peak = measured_dgemm_tflops(torch)
    bf16_peak, bf16_sust, bf16_src = peak_bf16_tflops()
    tf32_peak = bf16_peak / 2.0  # dense TF32 runs at half the BF16 rate on B200
    xg.init(args.ts)
    N = args.n
    x, y = xg.generate_xy_loc(N, args.seed)
    e = dlarnv(args.seed, N)
    sess = xg.Session(x, y, dts=args.ts)
    sess.zvg(THETA, e)
    z = sess.z()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- plain FP64 leg ----
    lls64, p64 = timed_leg(sess, THETA, args.steps, args.warmup, barrier)
    t64 = max_over_ranks(p64["t_total"])
    fp64_value = world * args.steps / t64
    ach64 = p64["gemm_flops"] / p64["t_gemm"] / 1e12

    # ---- banded reduced-precision leg (the headline) ----
    sliced = args.scheme == "sliced"
    if sliced:
        sess.set_sliced()
    else:
        sess.set_mixed(band=args.band, passes=args.passes)
    clk = ClockSampler(local)
    for _ in range(args.warmup):
        sess.loglik(THETA)
    sess.set_profiling(True)
    barrier()
    clk.start()
    t0 = time.perf_counter()
    llsmx = [sess.loglik(THETA) for _ in range(args.steps)]
    wall = time.perf_counter() - t0
    barrier()
    clocks = clk.stop()
    pmx = sess.profile()
    sess.set_profiling(False)
    tmx = max_over_ranks(pmx["t_total"])
    value = world * args.steps / tmx
    rel_err = abs(llsmx[-1] - lls64[-1]) / abs(lls64[-1])

    # ---- end to end: C ABI from pinned host buffers (reduced-precision path) ----
    px = torch.from_numpy(x).pin_memory()
    py = torch.from_numpy(y).pin_memory()
    pz = torch.from_numpy(z).pin_memory()
    e2e_steps = max(1, min(args.steps, 2))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sess.set_data(px.numpy(), py.numpy(), pz.numpy())
        ll_e2e = sess.mle_alg(THETA)
    e2e_wall = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": world * e2e_steps / e2e_wall, "unit": UNIT, "h2d_bytes_per_step": 3 * N * 8,
           "d2h_bytes_per_step": 5 * 8,
           "path": "exageostat_b200_set_data + MLE_alg (C ABI, precision %d), wall clock" % (3 if sliced else 2)}

    passes = args.passes
    t_off = pmx["t_offband"]
    if sliced:
        # ten 8-bit digit-pair products per FP64 product; dense INT8 runs at twice the BF16 rate.
        # t_offband / offband_flops: the split column updates on the main stream (nt - 2 launches per
        # evaluation, nearly all the work); t_band / band_flops: the last-chunk updates on the panel stream
        mult, peak, kname, unit = 10, 2.0 * bf16_sust, "xg_sliced_left_kernel (tcgen05 kind::i8, 10 digit " \
            "pairs, S32 TMEM levels, FP64 epilogue)", "TOP/s"
        psrc = "dense INT8 = 2 x sustained bf16 (the kernel runs inside a seconds-long step), bf16 from %s " \
            "(of measured); burst: %.1f TOP/s" % (bf16_src, 2.0 * bf16_peak)
        launches = max(pmx["nt"] - 2, 1)
    else:
        mult, peak, kname, unit = passes, bf16_sust / 2.0, "xg_offband_gemm_kernel (tcgen05 kind::tf32, %d " \
            "pass%s, TMEM)" % (passes, "es" if passes > 1 else ""), "TFLOP/s"
        psrc = "dense TF32 = sustained bf16 / 2, bf16 from %s (of measured)" % bf16_src
        launches = max(2 * (pmx["nt"] - 1), 1)
    mma_flops = pmx["offband_flops"] * mult
    ach_mx = mma_flops / t_off / 1e12 if t_off > 0 else 0.0
    ops_per_launch = pmx["offband_flops"] * mult / max(pmx["evals"], 1) / launches
    bpo, tsrc = ncu_traffic("xg_sliced_left_kernel" if sliced else "xg_offband_gemm_kernel")
    roofline = {"bound": "tensor", "kernel": kname,
                "achieved": ach_mx, "peak": peak, "unit": unit, "frac": ach_mx / peak,
                "peak_source": psrc,
                "traffic": bpo * ops_per_launch if bpo else None,
                "traffic_source": ("dram__bytes_read.sum + dram__bytes_write.sum per algorithmic op from the ncu "
                                   "capture in profiles/ncu_traffic.json (%s), times this launch's ops" %
                                   tsrc.get("case", "")) if bpo else None,
                "algorithmic_ops_per_launch": ops_per_launch,
                "useful_fp64_equivalent_tflops": pmx["offband_flops"] / t_off / 1e12 if t_off > 0 else 0.0,
                "share_of_step": t_off / pmx["t_total"],
                "phases_s_per_eval": {k: pmx[k] / pmx["evals"] for k in
                                      ("t_gen", "t_potrf", "t_trsm", "t_gemm", "t_offband", "t_band")}}
    # the reference's banded mixed-precision scheme (FP32 off-band tiles on TF32 tensor cores), reported
    other = None
    if sliced and not args.no_mixed_leg:
        sess.set_mixed(band=args.band, passes=args.passes)
        for _ in range(2):
            sess.loglik(THETA)
        sess.set_profiling(True)
        llm = [sess.loglik(THETA) for _ in range(args.steps)]
        pm = sess.profile()
        sess.set_profiling(False)
        tm = max_over_ranks(pm["t_total"])
        ach = pm["offband_flops"] * args.passes / pm["t_offband"] / 1e12 if pm["t_offband"] > 0 else 0.0
        other = {"scheme": "FP64 band of %d tiles + FP32 off-band tiles, TF32 x%d tensor cores (psdportf.c)" % (
                     args.band, args.passes),
                 "value": world * args.steps / tm, "unit": UNIT, "ms_per_step": 1e3 * tm / args.steps,
                 "rel_err_vs_fp64": abs(llm[-1] - lls64[-1]) / abs(lls64[-1]),
                 "offband_tf32_tflops": ach, "offband_frac_of_tf32_peak": ach / tf32_peak}
        sess.set_sliced()
    tpf, tsrc64 = ncu_traffic("xg_syrk_gemm_kernel")
    fp64 = {"value": fp64_value, "unit": UNIT, "ms_per_step": 1e3 * t64 / args.steps, "loglik": lls64[-1],
            "roofline": {"bound": "tensor", "kernel": "xg_syrk_gemm_kernel (FP64 DMMA trailing update)",
                         "achieved": ach64, "peak": fp64_peak, "unit": "TFLOP/s", "frac": ach64 / fp64_peak,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this process (of measured)",
                         "traffic": (tpf * p64["gemm_flops"] / p64["evals"] / max(2 * (p64["nt"] - 1) - 1, 1))
                         if tpf else None,
                         "traffic_source": ("ncu capture in profiles/ncu_traffic.json (%s), scaled by flops" %
                                            tsrc64.get("case", "")) if tpf else None,
                         "share_of_step": p64["t_gemm"] / p64["t_total"]}}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tmx / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": ("f64 tiles, trailing updates as int8 digit products (4 slices, s32 accumulate)" if sliced
                      else "f64 band + f32 off-band (tf32x%d tensor cores)" % passes), "data": "synthetic",
            "config": {"workload": workload(N), "tile": int(pmx["ts"]), "tiles_per_side": int(pmx["nt"]),
                       "band_tiles": args.band, "scheme": args.scheme,
                       "tf32_passes": None if sliced else passes,
                       "sm_share": os.environ.get("EXAGEOSTAT_B200_SL_SHARE", "static"),
                       "panel_k": int(os.environ.get("EXAGEOSTAT_B200_PANEL_K", "4")),
                       "parallelism": "replicas" if world > 1 else "single-gpu",
                       "l2": "inputs larger than L2 (20-40 GB of covariance tiles per step)",
                       "loglik_reduced": llsmx[-1], "loglik_fp64": lls64[-1], "rel_err_vs_fp64": rel_err,
                       "loglik_e2e": ll_e2e, "wall_s_timed": wall},
            "fp64": fp64, "speedup_vs_fp64": value / fp64_value, "banded_mixed_tf32": other,
            "roofline": roofline, "e2e": e2e, "clocks": clocks,
            "gpu_launches": int(round(pmx["launches"] / max(pmx["evals"], 1) * args.steps))}
    sess.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        pair = c2_pair(xg, args.seed, args.ts)
        line["c2_measured"] = pair
        line["cpu_baseline"] = cpu_baseline_from(N, pair["n"], pair["cpu_seconds_per_eval"], pair["cpu_phases"],
                                                 "C2 pair")
        # the same baseline's speed-up over the extrapolated CPU time at this N, for reading beside the C2 pair
        line["cpu_baseline"]["gpu_speedup_extrapolated"] = value / line["cpu_baseline"]["value"]
    if rank == 0 and world == 1 and not args.no_mle:
        line["time_to_mle"] = mle_block(xg, args.seed, args.ts)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
