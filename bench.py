"""Benchmark of the B200 GRN evaluator (one JSON line on stdout, rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
                  [--impl ours|reference] [--models M] [--no-cpu-baseline]

A bench step is one pass of the hot path over one batch: every model of the
workload simulated for all its Euler steps and scored (default workload
uneven_64x64: 4096 models, 2-8 genes, 1-24 links, 64x64 grid, 2000 steps).

  value   fitness evaluations/s with the packed batch resident on the device:
          K launches timed with CUDA events on the launching stream, each
          launch bracketed by its own events; between launches a 256 MiB
          buffer is written to flush L2 (outside the events).
  e2e     the same metric through grn_evaluate_batch with host buffers:
          host compile of the batch, pinned H2D copy, kernel, D2H of the raw
          errors and host rounding inside the timed region (wall clock,
          synchronised on both sides).
  roofline  MUFU (SFU pipe) bound.  achieved = algorithmic MUFU ops of a
          launch -- 3 per used link per cell-update (lg2, ex2, rcp of each
          Hill term in the reference formulation) -- over the mean launch
          time, against 16 MUFU/clk/SM x SMs x max SM clock.  The kernel
          issues fewer MUFU ops than that (one lg2 per regulator product and
          one ex2 + rcp per regulated product, in exponent form); those are
          reported as issued_mufu.  fp32_frac: algorithmic FP32 ops
          (6 L + 7 G + 8 G_dif per cell-update) against 128/clk/SM.
  cpu_baseline  the FP64 oracle (a port of the reference's CPU evaluator) on
          the host cores, on a bounded sample of the same workload.

--impl reference times the reference's CPU path (the oracle port; the
reference itself cannot be built here) on the host cores instead.
Multi-GPU: one process per GPU under torchrun; every rank evaluates its own
full batch (seeded by rank), so the work per GPU is fixed (weak scaling) and
no collective touches the data path; timing is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "grn-gpu-performance_b200"))

import synth  # noqa: E402

SFU_PER_CLK_PER_SM = 16  # MUFU results per clock per SM (lg2/ex2/rcp, FP32)
FP32_PER_CLK_PER_SM = 128  # FP32 lanes per SM


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def read_profile(workload):
    """DRAM traffic per launch of the simulation kernel from the committed ncu
    summary (profiles/), or None."""
    path = os.path.join(ROOT, "profiles", "sim_kernel_%s.json" % workload)
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
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
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _ref_module():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_binding  # the reference's own CPU path (oracle/_ref): baseline only
    return ref_binding


def cpu_baseline(workload, seed, budget_s=15.0, threads=None, euler_steps=None):
    """Times the reference's CPU fitness path on the host cores, on a bounded
    sample of the workload: one model per host thread per round, full Euler
    steps (or `euler_steps`), rounds until ~budget_s.

    It is the reference's own code -- EvaluatorMorphogens on Simulator /
    ModelSimulator, compiled from its unchanged sources into
    oracle/_ref/libgrn_ref_o3.so (-O3 -march=x86-64-v3) -- run by a pool of
    threads with one evaluator each, as its CPU calculator threads run.  It
    takes the experiments as RGB images (its input format) and has only its
    thresholded-log fitness.  Where oracle/_ref was not shipped, the FP64
    restatement (oracle port) stands in for it."""
    threads = threads or os.cpu_count() or 1
    over = {"steps": euler_steps} if euler_steps else {}
    ref = _ref_module()
    if ref.available(timed=True) or ref.available():
        timed = ref.available(timed=True)

        def run(n, n_threads):
            params, batch, init, tgt = synth.workload(workload, seed=seed + 1000, n_models=n,
                                                      **over)
            params = dict(params, fitness_kind=0)
            ipx = np.stack([ref.encode_rgb(e) for e in init])
            tpx = np.stack([ref.encode_rgb(e) for e in tgt])
            texts = ref.batch_texts(batch)
            t0 = time.perf_counter()
            ref.evaluate_texts(params, ipx, tpx, texts, n_threads=n_threads, timed=timed)
            return time.perf_counter() - t0, params
        kind = "reference"
        build = ("oracle/_ref/libgrn_ref_o3.so (-O3 -march=x86-64-v3)" if timed else
                 "oracle/_ref/libgrn_ref.so (-O2)")
    else:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import binding as oracle  # the FP64 port: baseline only

        def run(n, n_threads):
            params, batch, init, tgt = synth.workload(workload, seed=seed + 1000, n_models=n,
                                                      **over)
            t0 = time.perf_counter()
            oracle.evaluate_batch(params, init, tgt, batch, n_threads=n_threads)
            return time.perf_counter() - t0, params
        kind = "port"
        build = "oracle/_build/libgrn_oracle.so (FP64 restatement, -O2)"
    t1, _ = run(1, 1)
    rounds = max(1, min(8, int(budget_s / max(t1, 1e-3))))
    n = threads * rounds
    dt, params = run(n, threads)
    cells = params["dim_x"] * params["dim_y"] * params["num_sim_steps"] * n
    return {"value": n / dt, "unit": "evals/s", "cores": threads, "kind": kind,
            "sample": "%d models of %s (%d Euler steps), %d threads, %.1f s; %s"
                      % (n, workload, params["num_sim_steps"], threads, dt, build),
            "cell_updates_per_s": cells / dt, "seconds": dt}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU evaluator (oracle port) on the
    host cores, rank 0 only."""
    if rank != 0:
        return
    if args.workload not in synth.WORKLOADS:
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no %s workload "
                          "(its surrogate-free CPU evaluator only)" % args.workload}), flush=True)
        return
    threads = os.cpu_count() or 1
    wl = synth.WORKLOADS[args.workload]
    vals = []
    # Each step is a bounded sample; the whole run stays near 150 s of CPU
    # time whatever --steps / --warmup ask for (2 s per sample at least).
    budget = max(2.0, min(args.ref_budget, 150.0 / max(1, args.warmup + args.steps)))
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(args.workload, seed=i, budget_s=budget, threads=threads)
        if i >= args.warmup:
            vals.append(cb)
    value = statistics.mean(v["value"] for v in vals)
    line = {
        "impl": "reference", "metric": "GRN fitness evals/sec", "value": value,
        "unit": "evals/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * statistics.mean(v["seconds"] for v in vals),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "models": wl["n_models"],
                   "grid": "%dx%d" % (wl["W"], wl["H"]), "euler_steps": wl["steps"]},
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": threads,
                         "kind": vals[-1]["kind"], "sample": vals[-1]["sample"]},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "cell_updates_per_s": statistics.mean(v["cell_updates_per_s"] for v in vals),
    }
    print(json.dumps(line), flush=True)


def _search_arm(grn, ev, evo_p, n_morph, gens, surrogate=None, audit=False, sur_kw=None,
                score=None):
    """One seeded island search: per generation (elapsed wall s, best error,
    stats)."""
    evo = grn.Evolution(evo_p, n_morph, evaluator=ev)
    evo.set_skip_clones(True)
    if surrogate is not None:
        evo.set_surrogate(surrogate, **(sur_kw or {}))
        if score is not None:
            evo.set_surrogate_score(score)
        if audit:
            evo.set_surrogate_audit(True)
    out, t0 = [], time.perf_counter()
    for _ in range(gens):
        st = evo.step()
        out.append((time.perf_counter() - t0, st["best_error"], st))
    evo.close()
    return out


def run_surrogate_ablation(args, rank, world):
    """Surrogate-assisted against plain island evolution on the same seed
    (islands_100x100: 16 demes x 512, 100x100, 1500 Euler steps; both arms
    skip exact clones).  The surrogate MLP (128 -> 256 x 3 -> 1, BF16
    tcgen05 GEMMs, FP32 accumulate) trains online on every simulated
    (model, error) pair of its run (a 200k-pair ring), and from the
    generation its set holds `min_train` pairs it ranks every generation's
    children and only the best 25% are simulated.
    value = wall-clock seconds of the plain run to reach its final best error
    within 1%, divided by the surrogate run's seconds to reach that same
    error (null if it never does): > 1 means the surrogate run got there
    faster.  A second, audited surrogate run (every child simulated, the
    search unchanged) reports the screen's recall; it is not timed."""
    if rank != 0:
        return
    import torch
    import grn_b200 as grn
    torch.cuda.set_device(0)
    wl = synth.WORKLOADS[args.workload]
    params = synth.sim_params(wl)
    init, tgt = synth.experiments(wl, args.seed)
    n_demes, deme = 16, (args.models or wl["n_models"]) // 16
    evo_p = dict(n_demes=n_demes, deme_size=deme, migration_period=10, n_max_products=8,
                 n_max_links=24, n_host_threads=0, seed=args.seed)
    n_morph = wl["n_in"] + wl["n_target"]
    gens = args.warmup + args.steps
    sur_kw = dict(simulate_fraction=0.25, min_train_pairs=args.min_train,
                  batches_per_generation=32, batch_size=512, lr=1e-3)
    ev = grn.Evaluator(params)
    ev.set_experiments(init, tgt)
    plain = _search_arm(grn, ev, evo_p, n_morph, gens)
    sur = grn.Surrogate(seed=args.seed, capacity=200000)
    score = {"paired": grn.SCORE_PAIRED, "parent": grn.SCORE_PARENT_ERROR}[args.score]
    screened = _search_arm(grn, ev, evo_p, n_morph, gens, sur, sur_kw=sur_kw, score=score)
    sur.close()
    audit = None
    if args.audit:
        sur2 = grn.Surrogate(seed=args.seed, capacity=200000)
        audit = _search_arm(grn, ev, evo_p, n_morph, gens, sur2, audit=True, sur_kw=sur_kw,
                            score=score)
        sur2.close()
    ev.close()
    target = plain[-1][1] * 1.01

    def reach(run):
        for t, b, _ in run:
            if b <= target:
                return t
        return None

    t_plain, t_sur = reach(plain), reach(screened)

    def summary(run):
        sims = sum(st["n_evaluated"] for _, _, st in run)
        rows = [st for _, _, st in run if st["n_screened"] > 0]
        mean = (lambda k: float(np.nanmean([r[k] for r in rows])) if rows and
                np.isfinite([r[k] for r in rows]).any() else None)
        return {"seconds": run[-1][0], "ms_per_generation": 1000 * run[-1][0] / len(run),
                "final_best_error": run[-1][1], "simulations": sims,
                "time_to_target_s": reach(run),
                "best_by_generation": [round(b, 6) for _, b, _ in run],
                "screened_generations": len(rows),
                "surrogate_rho_mean": mean("surrogate_rho"),
                "surrogate_recall_mean": mean("surrogate_recall"),
                "surrogate_improver_recall_mean": mean("surrogate_improver_recall"),
                "surrogate_ms_per_generation": float(np.mean([st["surrogate_ms"]
                                                              for _, _, st in run]))}
    line = {
        "metric": "surrogate vs plain evolution: wall-clock to equal best fitness",
        "value": (t_plain / t_sur) if (t_plain and t_sur) else None, "unit": "x",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "none", "vs_baseline": None, "dtype": "f32/bf16",
        "data": "synthetic",
        "config": {"workload": args.workload, "demes": n_demes, "deme_size": deme,
                   "grid": "%dx%d" % (wl["W"], wl["H"]), "euler_steps": wl["steps"],
                   "generations": gens, "skip_clones": True,
                   "surrogate": "128-256-256-256-1 ReLU MLP, BF16 tcgen05, online, 200k ring, "
                                "top 25%% simulated from %d pairs" % args.min_train,
                   "score": args.score,
                   "target": "plain run's final best error x 1.01"},
        "target_error": target,
        "plain": summary(plain), "surrogate": summary(screened),
        "audit": summary(audit) if audit else None,
    }
    print(json.dumps(line), flush=True)


def run_surrogate_mlp(args, rank, world):
    """The surrogate MLP alone (128 -> 256 -> 256 -> 256 -> 1, ReLU; GEMMs on
    the tcgen05 tensor cores fed by a 4-stage TMA ring, BF16 operands, FP32
    accumulate), at the C4 workload's sizes: screening 8192 offspring per
    call (forward) and Adam training steps at batch 8192 drawn from a
    200k-pair set.
    FLOPs per row: forward 2 (128*256 + 2*256*256 + 256); a training step
    3x forward.  A step of this bench is one screening call plus 16 training
    batches.  Roofline: tensor, against the measured BF16 GEMM peak (burst:
    each call is timed alone).  Whole calls are timed (host encodings in,
    predictions out, launches included), so at these sizes the figure shows
    how far the MLP is from tensor-bound; the ncu summary in profiles/ gives
    the GEMM kernel itself."""
    if rank != 0:
        return
    import torch
    import grn_b200 as grn
    torch.cuda.set_device(0)
    rng = np.random.default_rng(args.seed)
    n_pairs, screen, batch, n_batches = 200000, 8192, 8192, 16
    X = (rng.standard_normal((n_pairs, grn.N_FEATURES)) * 0.5).astype(np.float32)
    y = (0.1 * X[:, :16].sum(1) + 0.05 * rng.standard_normal(n_pairs)).astype(np.float32)
    Xs = X[:screen].copy()
    sur = grn.Surrogate(seed=args.seed, capacity=n_pairs)
    sur.add_data(X, y)
    fwd = 2 * (128 * 256 + 2 * 256 * 256 + 256)
    for _ in range(args.warmup):
        sur.predict(Xs)
        sur.train_batches(n_batches, batch_size=batch)
    torch.cuda.synchronize()
    tp, tt = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        sur.predict(Xs)
        tp.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        sur.train_batches(n_batches, batch_size=batch)
        tt.append(time.perf_counter() - t0)
    sur.close()
    peaks, peak_kind = read_peaks()
    peak = peaks.get("bf16_tflops", 1590.0)
    p_s, t_s = statistics.mean(tp), statistics.mean(tt) / n_batches
    pred_tf = fwd * screen / p_s / 1e12
    train_tf = 3 * fwd * batch / t_s / 1e12
    line = {
        "metric": "surrogate MLP TFLOP/s", "value": train_tf, "unit": "TFLOP/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * (p_s + t_s * n_batches), "higher_is_better": True,
        "scaling": "none", "vs_baseline": None, "dtype": "bf16 operands, fp32 accumulate",
        "data": "synthetic",
        "config": {"workload": "surrogate_mlp", "layers": "128-256-256-256-1 ReLU",
                   "screen_rows": screen, "train_batch": batch, "pairs": n_pairs,
                   "step": "one screening call + %d training batches" % n_batches},
        "screen_ms": 1000 * p_s, "screen_tflops": pred_tf,
        "train_step_ms": 1000 * t_s, "train_tflops": train_tf,
        "roofline": {"bound": "tensor", "achieved": train_tf, "peak": peak, "unit": "TFLOP/s",
                     "frac": train_tf / peak, "traffic": None,
                     "algorithmic": "3 x 2 x B x (128*256 + 2*256*256 + 256) per training step",
                     "peak_source": "%s bf16_tflops (burst)" % peak_kind},
        # per step: a screening call (row conversion, 3 GEMMs, output layer)
        # and per training batch 17 (gather, 3 + 2 GEMMs, 3 weight-gradient
        # GEMMs with their split-K sums, output layer, loss, last-layer
        # backward, bias row sums, Adam)
        "gpu_launches": args.steps * (5 + 17 * n_batches),
    }
    print(json.dumps(line), flush=True)


def run_evolution(args, rank, world):
    """Island evolution workload (islands_100x100: 16 demes x 512 models,
    100x100 grid, <= 8 products and <= 24 links in use, 1500 Euler steps):
    a step is one generation -- host crossover/mutation of every deme, one
    batched GPU evaluation of all 8192 children, deterministic-crowding
    selection.  value = models evaluated per second of generation time.
    time_to_best_within_1pct_s: wall clock from the first generation until
    the best error first came within 1% of the run's final best (the
    search-level metric for island runs)."""
    import torch
    import grn_b200 as grn
    torch.cuda.set_device(rank if world > 1 else 0)
    wl = synth.WORKLOADS[args.workload]
    params = synth.sim_params(wl)
    init, tgt = synth.experiments(wl, args.seed + rank)
    n_demes, deme = 16, (args.models or wl["n_models"]) // 16
    evo_p = dict(n_demes=n_demes, deme_size=deme, migration_period=10, n_max_products=8,
                 n_max_links=24, n_host_threads=0, seed=args.seed + rank)
    ev = grn.Evaluator(params, device=torch.cuda.current_device())
    ev.set_experiments(init, tgt)
    if args.schedule != "auto":
        ev.set_schedule({v: k for k, v in grn.SCHEDULE_NAMES.items()}[args.schedule])
    evo = grn.Evolution(evo_p, wl["n_in"] + wl["n_target"], evaluator=ev)
    if args.skip_clones:
        evo.set_skip_clones(True)
    if args.pipeline:
        evo.set_pipeline(True)
    isl = None
    if world > 1:
        import sharded
        isl = sharded.IslandShards(evo, n_demes, deme, period=10, seed=args.seed)
    gens = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        st = isl.step() if isl else evo.step()
        st["wall_ms"] = 1000 * (time.perf_counter() - t0)
        gens.append(st)
    timed = gens[args.warmup:]
    wall = sum(g["wall_ms"] for g in timed) / 1000.0
    # Search progress over all generations (warm-up included: the search
    # starts at generation 0).
    best_key = "global_best_error" if isl else "best_error"
    final_best = gens[-1][best_key]
    elapsed, t_target, g_target = 0.0, None, None
    for g in gens:
        elapsed += g["wall_ms"] / 1000.0
        if t_target is None and g[best_key] <= final_best * 1.01:
            t_target, g_target = elapsed, g["generation"]
    # Children whose fitness was settled: simulated, or accepted as clones of
    # their parent (--skip-clones; exact, see grn_evolution_set_skip_clones).
    n_sim = sum(g["n_evaluated"] for g in timed)
    n_eval = n_sim + sum(g["n_clones"] for g in timed)
    if rank == 0:
        line = {
            "metric": "GRN fitness evals/sec", "value": n_eval * world / wall, "unit": "evals/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * wall / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "demes": n_demes, "deme_size": deme,
                       "grid": "%dx%d" % (wl["W"], wl["H"]), "euler_steps": wl["steps"],
                       "step": "one generation (reproduce, evaluate, select)",
                       "skip_clones": bool(args.skip_clones),
                       "pipeline": bool(args.pipeline),
                       "migration": "demes every 10 generations; across ranks every 10"
                                    if world > 1 else "demes every 10 generations",
                       "l2": "state and inputs exceed no cache; timed by wall clock per generation"},
            "generations": [{k: round(v, 6) if isinstance(v, float) else v
                             for k, v in g.items()} for g in gens],
            "eval_fraction": sum(g["eval_ms"] for g in timed) / (1000 * wall),
            "simulated_per_s": n_sim * world / wall,
            "final_best_error": final_best,
            "time_to_best_within_1pct_s": t_target,
            "generation_reaching_it": g_target,
            # the autotuner's candidates and times ('*' = kept), per batch shape
            "autotune": [l.strip() for l in ev.autotune_report().splitlines() if l.strip()],
        }
        print(json.dumps(line), flush=True)
    evo.close()
    ev.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="uneven_64x64",
                    choices=sorted(synth.WORKLOADS) + ["surrogate_mlp"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--models", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-budget", type=float, default=12.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--euler-steps", type=int, default=None,
                    help="override the workload's Euler step count (small profiling cases)")
    ap.add_argument("--schedule", default="auto",
                    choices=["auto", "fixed_items", "walk_items", "global", "cluster", "stream",
                             "stream2"],
                    help="force a kernel schedule instead of the autotuner's choice")
    ap.add_argument("--pipeline", action="store_true",
                    help="island workloads: two deme halves alternate on the GPU while the "
                         "host breeds the other (same populations)")
    ap.add_argument("--shard", action="store_true",
                    help="split one batch over the ranks through sharded.deal and all-gather "
                         "the errors (the default when WORLD_SIZE > 1; with one rank it runs "
                         "the same path on a one-rank process group)")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the large_256x256 sub-record of the default workload")
    ap.add_argument("--large-steps", type=int, default=500,
                    help="Euler steps of the large_256x256 sub-record (the configuration: 5000)")
    ap.add_argument("--surrogate", action="store_true",
                    help="islands_100x100: surrogate-screened against plain evolution, same seed")
    ap.add_argument("--audit", action="store_true",
                    help="with --surrogate: a third, audited run that measures the screen's recall")
    ap.add_argument("--score", default="paired", choices=["paired", "parent"],
                    help="with --surrogate: rank children by predicted change against the "
                         "predicted (paired) or the simulated (parent) parent error")
    ap.add_argument("--min-train", type=int, default=8192,
                    help="with --surrogate: pairs the surrogate holds before it screens")
    ap.add_argument("--skip-clones", action="store_true",
                    help="island workloads: accept children whose simulated program equals "
                         "their parent's without simulating them")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "surrogate_mlp":
        run_surrogate_mlp(args, rank, world)
        return
    if args.workload == "islands_100x100" and args.surrogate:
        run_surrogate_ablation(args, rank, world)
        return
    if args.workload == "islands_100x100":
        run_evolution(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    import grn_b200 as grn

    torch.cuda.set_device(local)
    sharded_run = world > 1 or args.shard
    if sharded_run:
        from datetime import timedelta
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29531")
        dist.init_process_group("nccl", rank=rank, world_size=world,
                                timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return t.item()

    over = {"steps": args.euler_steps} if args.euler_steps else {}
    if sharded_run:
        # One global batch (the same seed on every rank), dealt to the ranks
        # by compiled cost (sharded.deal); every rank evaluates its shard and
        # the errors are all-gathered.  Per-GPU work stays at the workload's
        # model count: weak scaling.
        import sharded
        n_per_gpu = args.models or synth.WORKLOADS[args.workload]["n_models"]
        params, gbatch, init, tgt = synth.workload(args.workload, seed=args.seed,
                                                   n_models=n_per_gpu * world, **over)
        n_morph = params["n_input_morphogens"] + params["n_target_morphogens"]
        ranks = sharded.deal(grn.model_costs(gbatch, n_morph), world)
        mine = np.nonzero(ranks == rank)[0]
        batch = gbatch.subset(mine)
        shard_max = int(np.bincount(ranks, minlength=world).max())
    else:
        params, batch, init, tgt = synth.workload(args.workload, seed=args.seed,
                                                  n_models=args.models, **over)
        gbatch = batch
    n = batch.n_models
    ev = grn.Evaluator(params, device=local)
    ev.set_experiments(init, tgt)
    if world > 1:  # the ranks of this node share its cores for compiling batches
        local_world = int(os.environ.get("LOCAL_WORLD_SIZE", str(world)))
        ev.set_host_threads(max(1, (os.cpu_count() or 1) // local_world))
    if args.schedule != "auto":  # a fixed schedule: no autotuning launches (profiling)
        ev.set_schedule({v: k for k, v in grn.SCHEDULE_NAMES.items()}[args.schedule])
    pk = ev.pack(batch)
    info = pk.info
    me = torch.full((n,), 1000.0, dtype=torch.float64, device="cuda")
    raw = torch.zeros(n, dtype=torch.float64, device="cuda")
    steps_out = torch.zeros(n, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # A dedicated stream: the kernel, the flush and the events all run on it
    # (the legacy default stream's handle is 0, which the C ABI reads as
    # "the context's own stream").
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    if sharded_run:
        gather_buf = torch.zeros(shard_max, dtype=torch.float64, device="cuda")
        gather_parts = [torch.empty_like(gather_buf) for _ in range(world)]

    def launch():
        pk.run(me.data_ptr(), raw.data_ptr(), steps_out.data_ptr(), stream.cuda_stream)
        if sharded_run:
            # The step's only exchange: every rank's raw errors to every rank.
            gather_buf[:n].copy_(raw)
            dist.all_gather(gather_parts, gather_buf)

    for _ in range(args.warmup):
        flush.fill_(1)
        launch()
    torch.cuda.synchronize()
    pk.status(stream.cuda_stream)  # a kernel error flag raises here

    # ---- device-resident timing (value) ----
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    barrier()
    torch.cuda.synchronize()
    evs = []
    for i in range(args.steps):
        flush.fill_(i & 0xff)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        launch()
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    barrier()
    pk.status(stream.cuda_stream)
    launch_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(sum(launch_ms))
    clocks = sampler.stop() if sampler else None
    steps_run = int(steps_out.sum().item())
    cells = params["dim_x"] * params["dim_y"]

    # ---- end-to-end through the C ABI with host buffers (e2e) ----
    e2e_times = []
    stats = None
    api = sharded.ShardedEvaluator(ev, n_morph) if sharded_run else ev
    for i in range(max(1, args.warmup // 2) + args.steps):
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        err, rawh, stats = api.evaluate_batch(gbatch)
        t1 = time.perf_counter()
        if i >= max(1, args.warmup // 2):
            e2e_times.append(t1 - t0)
    e2e_s = max_over_ranks(sum(e2e_times))
    assert np.isfinite(rawh).all()
    if sharded_run:
        np.testing.assert_array_equal(rawh[mine], raw.cpu().numpy())
        full = torch.cat(gather_parts).cpu().numpy()
        order = np.concatenate([np.nonzero(ranks == r)[0] for r in range(world)])
        starts = np.arange(world) * shard_max
        counts = np.bincount(ranks, minlength=world)
        got = np.concatenate([full[starts[r]:starts[r] + counts[r]] for r in range(world)])
        np.testing.assert_array_equal(got, rawh[order])
    else:
        np.testing.assert_array_equal(rawh, raw.cpu().numpy())
    g_models = gbatch.n_models

    if rank != 0:
        pk.free()
        ev.close()
        dist.destroy_process_group()
        return

    peaks, peak_kind = read_peaks()
    sm_max = peaks.get("sm_max_mhz", 1965.0)
    props = torch.cuda.get_device_properties(local)
    n_sm = props.multi_processor_count
    mean_ms = statistics.mean(launch_ms)
    # sfu_ops_per_step sums every model's MUFU ops of one Euler step over the
    # grid; steps_run / n is the Euler steps each model ran (all equal here:
    # min_conc_change 0 never stops a simulation early).
    model_steps = steps_run / max(n, 1)
    achieved = info["alg_sfu_ops_per_step"] * model_steps / (mean_ms / 1000.0) / 1e9
    issued = info["sfu_ops_per_step"] * model_steps / (mean_ms / 1000.0) / 1e9
    fp32 = info["alg_fp32_ops_per_step"] * model_steps / (mean_ms / 1000.0) / 1e9
    peak = SFU_PER_CLK_PER_SM * n_sm * sm_max * 1e6 / 1e9
    fp32_peak = FP32_PER_CLK_PER_SM * n_sm * sm_max * 1e6 / 1e9
    prof = read_profile(args.workload)
    value = g_models * args.steps / (total_ms / 1000.0)
    line = {
        "metric": "GRN fitness evals/sec",
        "value": value,
        "unit": "evals/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": args.workload, "models_per_gpu": n, "models_total": g_models,
            "grid": "%dx%d" % (params["dim_x"], params["dim_y"]),
            "genes": "%d-%d" % synth.WORKLOADS[args.workload]["genes"],
            "links": "%d-%d" % synth.WORKLOADS[args.workload]["links"],
            "mean_genes": round(info["mean_genes"], 3), "mean_links": round(info["mean_links"], 3),
            "euler_steps": params["num_sim_steps"], "experiments": int(init.shape[0]),
            "fitness": ["ref_logthresh", "mse"][params["fitness_kind"]],
            "state": "fp32, fitness sums fp64",
            "l2": "256 MiB buffer written between timed launches (outside the launch events)",
            "schedule": grn.SCHEDULE_NAMES.get(stats.get("schedule"), stats.get("schedule")),
            "threads_per_block": stats.get("threads_per_block"), "blocks": stats.get("blocks"),
            "parallelism": ("one batch dealt over %d GPUs by compiled cost, errors all-gathered "
                            "(NCCL) every step" % world) if sharded_run else "1 GPU",
        },
        "cell_updates_per_s": steps_run * cells * world * args.steps / (total_ms / 1000.0),
        "e2e": {
            "value": g_models * args.steps / e2e_s,
            "unit": "evals/s",
            "h2d_bytes_per_step": int(stats.get("h2d_bytes", 0)),
            "d2h_bytes_per_step": int(stats.get("d2h_bytes", 0)),
            "host_pack_ms": round(stats.get("pack_ms", 0.0), 3),
            "api": "sharded.ShardedEvaluator.evaluate_batch" if sharded_run else
                   "grn_evaluate_batch",
        },
        "roofline": {
            "bound": "sfu",
            "achieved": achieved,
            "peak": peak,
            "unit": "Gop/s (MUFU lg2/ex2/rcp)",
            "frac": achieved / peak,
            "algorithmic": "3 MUFU ops per used link per cell-update (mean %.3f links)" % (
                info["mean_links"]),
            "issued_mufu": {"achieved": issued, "frac": issued / peak},
            "fp32_frac": fp32 / fp32_peak,
            "peak_source": "16 MUFU/clk/SM x %d SMs x %.0f MHz (%s sm_max_mhz)" % (
                n_sm, sm_max, peak_kind),
            "traffic": prof.get("dram_bytes_per_launch") if prof else None,
            "kernel": "sim_kernel",
            "launch_ms": round(mean_ms, 3),
        },
        "clocks": clocks,
        "gpu_launches": args.steps,
    }
    if clocks and clocks.get("sm_mhz"):
        line["roofline"]["frac_at_sampled_clock"] = achieved / (
            SFU_PER_CLK_PER_SM * n_sm * clocks["sm_mhz"] * 1e6 / 1e9)
    pk.free()
    ev.close()
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(args.workload, args.seed)
    if not args.no_secondary and world == 1 and args.workload == "uneven_64x64":
        line["secondary"] = [secondary_large(args, grn, torch, local, peaks, peak_kind, n_sm)]
        line["gpu_launches"] += line["secondary"][0]["gpu_launches"]
    print(json.dumps(line), flush=True)
    if sharded_run:
        dist.destroy_process_group()


def secondary_large(args, grn, torch, local, peaks, peak_kind, n_sm):
    """The large-grid stress configuration as a sub-record: large_256x256
    (1024 models, 8 genes, 24 links, 256x256, dt 0.05) at args.large_steps
    Euler steps instead of 5000, so that the default run stays short.  Its
    state (2 x 8 planes of 256 x 256 per model) does not fit on chip; the
    bound is HBM: algorithmic bytes per cell-update = 2 x 8 genes x 4 B / T,
    T = Euler steps fused per pass over the state (the plan's temporal
    blocking depth)."""
    wl = "large_256x256"
    params, batch, init, tgt = synth.workload(wl, seed=args.seed, steps=args.large_steps)
    n = batch.n_models
    ev = grn.Evaluator(params, device=local)
    ev.set_experiments(init, tgt)
    pk = ev.pack(batch)
    me = torch.full((n,), 1000.0, dtype=torch.float64, device="cuda")
    raw = torch.zeros(n, dtype=torch.float64, device="cuda")
    steps_out = torch.zeros(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    for _ in range(2):  # the first launch autotunes the plan
        pk.run(me.data_ptr(), raw.data_ptr(), steps_out.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    launches = 3
    evs = []
    for _ in range(launches):  # 1024 x 2 x 8 x 256 x 256 x 4 B of state > L2
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pk.run(me.data_ptr(), raw.data_ptr(), steps_out.data_ptr(), stream.cuda_stream)
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    pk.status(stream.cuda_stream)
    ms = statistics.mean(a.elapsed_time(b) for a, b in evs)
    # The plan the autotuner kept for this batch (marked '*' in its report).
    kept = [l for l in ev.autotune_report().splitlines() if l.lstrip().startswith("*")]
    plan = kept[-1].lstrip("* ").strip() if kept else None
    pk.free()
    ev.close()
    cells = params["dim_x"] * params["dim_y"]
    cu = int(steps_out.sum().item()) * cells / (ms / 1000.0)
    genes, t_fused = 8, 1
    alg_bytes = 2 * genes * 4 / t_fused
    achieved = cu * alg_bytes / 1e9
    prof = read_profile(wl)
    traffic = None
    if prof and prof.get("dram_bytes_per_cell_update"):
        traffic = prof["dram_bytes_per_cell_update"] * n * args.large_steps * cells
    rec = {
        "config": {"workload": wl, "models": n, "grid": "256x256", "genes": 8, "links": 24,
                   "euler_steps": args.large_steps, "euler_steps_full": 5000, "dt": 0.05,
                   "l2": "state of the batch (4.3 GB) exceeds L2"},
        "metric": "GRN fitness evals/sec", "unit": "evals/s",
        "value": n / (ms / 1000.0),
        "value_at_full_steps": cu / (cells * 5000),
        "cell_updates_per_s": cu, "ms_per_launch": ms, "gpu_launches": launches + 2,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks.get("hbm_gbs"),
                     "unit": "GB/s", "frac": achieved / peaks.get("hbm_gbs", 6545.0),
                     "algorithmic": "%d B per cell-update (2 x %d genes x 4 B, T=%d)" % (
                         alg_bytes, genes, t_fused),
                     "traffic": traffic, "peak_source": "%s hbm_gbs" % peak_kind},
        "plan": plan,
    }
    if not args.no_cpu_baseline:
        rec["cpu_baseline"] = cpu_baseline(wl, args.seed, budget_s=8.0,
                                           euler_steps=args.large_steps)
    return rec


if __name__ == "__main__":
    main()
