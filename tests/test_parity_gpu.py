"""GPU parity tests: the CUDA path, called through the C ABI, against the
FP64 oracle on the same seeded inputs.

Tolerance: the kernels keep FP32 state and use the MUFU lg2/ex2/rcp
approximations; the oracle is FP64.  Raw (unrounded) errors must agree to
RTOL = 1e-4 relative (ATOL = 1e-7 absolute for errors near zero), rounded
errors to the same tolerance or one unit of the last rounded digit, and the
selection ranking of ties-free populations must be identical.  Different
kernel schedules run the same arithmetic and must agree bit for bit.
"""
import json
import math
import os

import numpy as np
import pytest

import binding as oracle
import grn_b200 as grn
import synth
from grn_b200 import LINK_DTYPE, PRODUCT_DTYPE, ModelBatch

pytestmark = pytest.mark.gpu

RTOL = 1e-4
ATOL = 1e-7
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def assert_raw_close(gpu, ref, rtol=RTOL, atol=ATOL, what=""):
    gpu, ref = np.asarray(gpu), np.asarray(ref)
    both_nan = np.isnan(gpu) & np.isnan(ref)
    ok = both_nan | (np.abs(gpu - ref) <= atol + rtol * np.abs(ref))
    if not ok.all():
        bad = np.where(~ok)[0]
        rel = np.abs(gpu - ref) / np.maximum(np.abs(ref), 1e-300)
        raise AssertionError("%s: %d/%d outside tolerance, worst rel %.3g at %d (gpu %r ref %r)"
                             % (what, len(bad), len(ok), rel[bad].max(), bad[rel[bad].argmax()],
                                gpu[bad[rel[bad].argmax()]], ref[bad[rel[bad].argmax()]]))


def assert_rounded_close(gpu, ref, precision):
    for g, r in zip(gpu, ref):
        if r == 100.0 or g == 100.0:
            assert g == r
            continue
        unit = 10.0 ** (math.ceil(math.log10(abs(r))) - precision) if r else 0.0
        assert abs(g - r) <= max(unit * 1.001, ATOL + RTOL * abs(r)), (g, r)


def assert_same_ranking(gpu, ref, rtol=2 * RTOL):
    """Pairs the oracle separates by more than the tolerance keep their order."""
    gpu, ref = np.asarray(gpu), np.asarray(ref)
    o = np.argsort(ref, kind="stable")
    r, g = ref[o], gpu[o]
    for i in range(len(r) - 1):
        for j in range(i + 1, len(r)):
            if r[j] - r[i] > rtol * max(abs(r[i]), abs(r[j])) + ATOL:
                assert g[i] < g[j], (o[i], o[j], r[i], r[j], g[i], g[j])


def run_both(params, batch, init, tgt, max_error=None, schedule=None, threads=None):
    with grn.Evaluator(params) as ev:
        if schedule is not None:
            ev.set_schedule(schedule)
        ev.set_experiments(init, tgt)
        err, raw, stats = ev.evaluate_batch(batch, max_error)
    oe, oraw, osteps = oracle.evaluate_batch(params, init, tgt, batch, max_error, n_threads=threads)
    return err, raw, stats, oe, oraw, osteps


def load_golden():
    with open(os.path.join(GOLDEN, "oracle_small.json")) as f:
        cases = json.load(f)["cases"]
    out = []
    for c in cases:
        batch = ModelBatch(c["product_offsets"],
                           np.array([tuple(r) for r in c["products"]], PRODUCT_DTYPE),
                           c["link_offsets"], np.array([tuple(r) for r in c["links"]], LINK_DTYPE))
        out.append((c, batch))
    return out


@pytest.mark.parametrize("W,H,steps", [(8, 8, 1), (8, 8, 30), (13, 5, 40), (64, 64, 50)])
def test_final_states_match_oracle(W, H, steps):
    """Final simulated state planes against the oracle's, cell by cell."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=W * H + steps, n_models=12,
                                              steps=steps, W=W, H=H)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        raw, states = ev.evaluate_states(batch, max_planes=16)
    for m in range(batch.n_models):
        pr, li = batch.model(m)
        ref, _, _ = oracle.simulate(params, init[0], pr, li, steps)
        got = states[m, 0, :len(ref)].astype(np.float64)
        err = np.abs(got - ref)
        tol = 1e-6 + 1e-4 * np.abs(ref)
        if not (err <= tol).all():
            k, y, x = np.unravel_index(np.argmax(err - tol), err.shape)
            raise AssertionError("model %d: gene %d cell (%d,%d): gpu %r oracle %r (%d genes)"
                                 % (m, k, x, y, got[k, y, x], ref[k, y, x], len(ref)))


def test_golden_fixtures():
    for c, batch in load_golden():
        p = c["params"]
        with grn.Evaluator(p) as ev:
            ev.set_experiments(np.array(c["initial"]), np.array(c["target"]))
            err, raw, stats = ev.evaluate_batch(batch, c["max_error"])
        assert_raw_close(raw, c["raw_error"], what="golden %dx%d" % (p["dim_x"], p["dim_y"]))
        assert_rounded_close(err, c["error"], p["error_precision"])


def test_small_32x32_full_config():
    """64 models, 3 genes, 32x32, 500 steps, MSE fitness: the CPU-runnable
    configuration at full size."""
    params, batch, init, tgt = synth.workload("small_32x32", seed=1)
    err, raw, stats, oe, oraw, _ = run_both(params, batch, init, tgt)
    assert_raw_close(raw, oraw, what="small_32x32")
    assert_rounded_close(err, oe, params["error_precision"])
    assert_same_ranking(raw, oraw)
    assert stats["cell_updates"] == 64 * 500 * 32 * 32


def test_small_32x32_ref_fitness():
    params, batch, init, tgt = synth.workload("small_32x32", seed=2, fitness=0)
    err, raw, _, oe, oraw, _ = run_both(params, batch, init, tgt)
    assert_raw_close(raw, oraw, what="small_32x32 logthresh")
    assert_same_ranking(raw, oraw)


def test_uneven_64x64_sample():
    """Uneven 2-8 genes / 1-24 links at 64x64 (the headline grid)."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=3, n_models=40, steps=300)
    err, raw, stats, oe, oraw, osteps = run_both(params, batch, init, tgt)
    assert_raw_close(raw, oraw, what="uneven_64x64")
    assert_same_ranking(raw, oraw)


def test_uneven_64x64_full_steps_sample():
    """A few models of the headline workload at the full 2000 steps."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=4, n_models=6)
    err, raw, stats, oe, oraw, osteps = run_both(params, batch, init, tgt)
    assert_raw_close(raw, oraw, what="uneven_64x64 2000 steps")


@pytest.mark.parametrize("W,H", [(10, 7), (13, 1), (1, 13), (1, 1), (33, 17), (5, 64), (64, 3)])
def test_ragged_grids(W, H):
    """Widths that are not multiples of 4, single rows/columns, 1x1."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=W * 100 + H, n_models=24,
                                              steps=120, W=W, H=H)
    err, raw, _, oe, oraw, _ = run_both(params, batch, init, tgt)
    assert_raw_close(raw, oraw, what="%dx%d" % (W, H))


@pytest.mark.parametrize("W,H,steps", [(100, 100, 40), (256, 256, 12), (140, 90, 30)])
def test_large_grids(W, H, steps):
    """Grids that do not fit shared memory at 8 genes (hybrid / global)."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=W + H, n_models=10,
                                              steps=steps, W=W, H=H, genes=(6, 8))
    err, raw, _, oe, oraw, _ = run_both(params, batch, init, tgt)
    assert_raw_close(raw, oraw, what="%dx%d" % (W, H))


def test_large_256x256_long_run_fp32_vs_fp64():
    """The large workload's configuration (256 x 256, 8 products, 24 links,
    dt 0.05) over 1000 Euler steps, two models: FP32 state against the FP64
    oracle within the suite's tolerance (rel 1e-4).  At the full 5000 steps
    the 8-model sample stays within 3.9e-6."""
    params, batch, init, tgt = synth.workload("large_256x256", seed=7, n_models=8, steps=1000)
    batch = batch.subset([4, 7])  # the two with the largest deviation at 5000 steps
    err, raw, _, oe, oraw, _ = run_both(params, batch, init, tgt, threads=2)
    assert_raw_close(raw, oraw, what="256x256 1000 steps")


def test_large_config_fp32_vs_fp64_full_steps():
    """The large-grid stress configuration at its full length: 32 seeded
    models (256 x 256, 8 products, 24 links, dt 0.05, 5000 Euler steps), the
    FP32 CUDA path against the FP64 oracle on all host cores.  Every model's
    raw fitness stays within the suite's tolerance (rel 1e-4); the
    per-model error distribution is printed."""
    import os
    params, batch, init, tgt = synth.workload("large_256x256", seed=11, n_models=32)
    assert params["num_sim_steps"] == 5000 and params["dt"] == 0.05
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        _, raw, _ = ev.evaluate_batch(batch)
    _, oraw, _ = oracle.evaluate_batch(params, init, tgt, batch, n_threads=os.cpu_count() or 1)
    rel = np.abs(raw - oraw) / np.maximum(np.abs(oraw), 1e-300)
    print("FP32 vs FP64, 32 models x 5000 steps: median %.3g, p90 %.3g, max %.3g"
          % (np.median(rel), np.percentile(rel, 90), rel.max()))
    assert_raw_close(raw, oraw, what="256x256 5000 steps")


def test_schedules_agree_bitwise():
    """Fixed-item, walking-item and all-global-memory schedules run the same
    arithmetic: identical simulated states; the FP64 fitness sums may differ
    in the last bits (summation order follows the block size)."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=5, n_models=30, steps=80,
                                              W=36, H=20)
    outs = {}
    for sched in (grn.SCHEDULE_AUTO, grn.SCHEDULE_FIXED_ITEMS, grn.SCHEDULE_WALK_ITEMS,
                  grn.SCHEDULE_GLOBAL):
        with grn.Evaluator(params) as ev:
            ev.set_schedule(sched)
            ev.set_experiments(init, tgt)
            raw, states = ev.evaluate_states(batch, max_planes=8)
            _, raw_b, st = ev.evaluate_batch(batch)
        outs[sched] = (raw, states, st["schedule"])
        assert np.array_equal(raw, raw_b)
    base_raw, base_states, _ = outs[grn.SCHEDULE_AUTO]
    for sched, (raw, states, used) in outs.items():
        assert np.array_equal(states, base_states), (sched, used)
        assert_raw_close(raw, base_raw, rtol=1e-12, atol=0, what="schedule %d" % used)
    oe, oraw, _ = oracle.evaluate_batch(params, init, tgt, batch)
    assert_raw_close(base_raw, oraw, what="schedules")


@pytest.mark.parametrize("W,H,clusters", [(36, 20, (2, 4)), (30, 37, (2, 4, 8)),
                                           (64, 64, (2, 4, 16)), (100, 100, (4, 8))])
def test_cluster_schedule_matches_one_cta_bitwise(W, H, clusters):
    """A cluster of CTAs per model, each with a band of rows and halo rows
    pushed through distributed shared memory, runs the same per-cell
    arithmetic as one CTA per model: identical states."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=15, n_models=24, steps=60,
                                              W=W, H=H, n_exp=2)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        ev.set_schedule(grn.SCHEDULE_WALK_ITEMS)
        base_raw, base_states = ev.evaluate_states(batch, max_planes=8)
        for c in clusters:
            ev.set_schedule(grn.SCHEDULE_CLUSTER, cluster_size=c)
            raw, states = ev.evaluate_states(batch, max_planes=8)
            _, raw_b, st = ev.evaluate_batch(batch)
            assert st["schedule"] == grn.SCHEDULE_CLUSTER and st["cluster_size"] == c
            assert np.array_equal(raw, raw_b)
            assert np.array_equal(states, base_states), c
            assert_raw_close(raw, base_raw, rtol=1e-12, atol=0, what="cluster %d" % c)
    oe, oraw, _ = oracle.evaluate_batch(params, init, tgt, batch)
    assert_raw_close(base_raw, oraw, what="cluster base")


def test_cluster_schedule_with_global_genes():
    """256 x 256 with 8 genes: a 16-CTA cluster keeps 6 genes' bands in
    shared memory and 2 in global slots; halo rows of both kinds."""
    params, batch, init, tgt = synth.workload("large_256x256", seed=16, n_models=6, steps=40)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        ev.set_schedule(grn.SCHEDULE_GLOBAL)
        base_raw, base_states = ev.evaluate_states(batch, max_planes=8)
        for c in (8, 16):
            ev.set_schedule(grn.SCHEDULE_CLUSTER, cluster_size=c)
            raw, states = ev.evaluate_states(batch, max_planes=8)
            assert np.array_equal(states, base_states), c
            assert_raw_close(raw, base_raw, rtol=1e-12, atol=0, what="cluster %d" % c)


def test_autotuned_plan_is_cached_and_exact():
    """The measured autotuner picks one plan per batch shape and keeps it;
    whatever it picks computes the same states as the heuristic's plan."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=18, n_models=300, steps=50)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        ev.set_autotune(False)
        h_raw, h_states = ev.evaluate_states(batch, max_planes=8)
        ev.set_autotune(True)
        _, raw1, st1 = ev.evaluate_batch(batch)
        _, raw2, st2 = ev.evaluate_batch(batch)
        a_raw, a_states = ev.evaluate_states(batch, max_planes=8)
    keys = ("schedule", "threads_per_block", "cluster_size", "blocks")
    assert [st1[k] for k in keys] == [st2[k] for k in keys]
    assert np.array_equal(raw1, raw2) and np.array_equal(raw1, a_raw)
    assert np.array_equal(a_states, h_states)
    assert_raw_close(a_raw, h_raw, rtol=1e-12, atol=0, what="autotune")


def test_autotune_key_ignores_exact_link_count():
    """Batches that differ only in their largest link count, as a search's
    generations do, share one tuning run (the report's first line counts
    the runs)."""
    params, b20, init, tgt = synth.workload("uneven_64x64", seed=19, n_models=400, steps=50,
                                            genes=(8, 8), links=(1, 20))
    _, b24, _, _ = synth.workload("uneven_64x64", seed=20, n_models=400, steps=50,
                                  genes=(8, 8), links=(1, 24))
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        infos = [ev.pack(b).info for b in (b20, b24)]
        assert infos[0]["max_genes"] == infos[1]["max_genes"]
        assert infos[0]["max_links"] != infos[1]["max_links"]
        ev.evaluate_batch(b20)
        ev.evaluate_batch(b24)
        head = ev.autotune_report().splitlines()[0]
    assert head.startswith("# autotuning runs 1,"), head


@pytest.mark.parametrize("W,H,steps,genes", [(256, 256, 12, (8, 8)), (100, 100, 30, (6, 8)),
                                             (30, 37, 25, (2, 8)), (250, 90, 15, (8, 16))])
def test_stream_schedule_matches_global_bitwise(W, H, steps, genes):
    """Bands staged through shared memory by bulk copies (streaming
    schedule): the same per-cell arithmetic as the all-global schedule,
    identical states, including ragged widths, a last band shorter than the
    others, 16-gene models and the exact path (links with K = 0)."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=23, n_models=12, steps=steps,
                                              W=W, H=H, genes=genes, links=(1, 24), n_exp=2)
    batch.links["dis_const"][0] = 0.0  # model 0 takes the exact path
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        ev.set_schedule(grn.SCHEDULE_GLOBAL)
        base_raw, base_states = ev.evaluate_states(batch, max_planes=16)
        ev.set_schedule(grn.SCHEDULE_STREAM)
        raw, states = ev.evaluate_states(batch, max_planes=16)
        _, raw_b, st = ev.evaluate_batch(batch)
    assert st["schedule"] == grn.SCHEDULE_STREAM
    assert np.array_equal(states, base_states)
    assert np.array_equal(raw, raw_b)
    assert_raw_close(raw, base_raw, rtol=1e-12, atol=0, what="stream")


def test_stream_schedule_early_exit_bitwise():
    """Early exit under the streaming schedule: final states and step counts
    match the all-global schedule."""
    params, batch, init, tgt = synth.workload("small_32x32", seed=25, n_models=24, steps=3000,
                                              W=40, H=36, min_conc_change=1e-2, fitness=0,
                                              n_exp=2)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        ev.set_schedule(grn.SCHEDULE_GLOBAL)
        base_raw, base_states = ev.evaluate_states(batch, max_planes=8)
        _, _, base_st = ev.evaluate_batch(batch)
        ev.set_schedule(grn.SCHEDULE_STREAM)
        raw, states = ev.evaluate_states(batch, max_planes=8)
        _, _, st = ev.evaluate_batch(batch)
    assert st["schedule"] == grn.SCHEDULE_STREAM
    assert st["total_steps"] == base_st["total_steps"] < 24 * 2 * 3000
    assert np.array_equal(states, base_states)
    assert_raw_close(raw, base_raw, rtol=1e-12, atol=0, what="stream early exit")


@pytest.mark.parametrize("W,H,steps,genes", [(256, 256, 12, (8, 8)), (100, 100, 31, (6, 8)),
                                             (30, 37, 25, (2, 8)), (250, 90, 15, (8, 16)),
                                             (64, 5, 9, (2, 6))])
def test_stream2_schedule_matches_global_bitwise(W, H, steps, genes):
    """Temporal blocking (two Euler steps per pass, GRN_SCHEDULE_STREAM2):
    the same per-cell arithmetic as the all-global schedule, identical
    states, including an odd step count (the last step alone), ragged
    widths, a last band shorter than the others, a grid of one band,
    16-gene models and the exact path."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=23, n_models=12, steps=steps,
                                              W=W, H=H, genes=genes, links=(1, 24), n_exp=2)
    batch.links["dis_const"][0] = 0.0  # model 0 takes the exact path
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        ev.set_schedule(grn.SCHEDULE_GLOBAL)
        base_raw, base_states = ev.evaluate_states(batch, max_planes=16)
        ev.set_schedule(grn.SCHEDULE_STREAM2)
        raw, states = ev.evaluate_states(batch, max_planes=16)
        _, raw_b, st = ev.evaluate_batch(batch)
    assert st["schedule"] == grn.SCHEDULE_STREAM2
    assert np.array_equal(states, base_states)
    assert np.array_equal(raw, raw_b)
    assert_raw_close(raw, base_raw, rtol=1e-12, atol=0, what="stream2")


def test_stream2_early_exit_bitwise():
    """Early exit under temporal blocking: where the change after the first
    step of a pass ends the simulation, that step is redone alone, so final
    states and step counts match the all-global schedule."""
    params, batch, init, tgt = synth.workload("small_32x32", seed=25, n_models=24, steps=3000,
                                              W=40, H=36, min_conc_change=1e-2, fitness=0,
                                              n_exp=2)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        ev.set_schedule(grn.SCHEDULE_GLOBAL)
        base_raw, base_states = ev.evaluate_states(batch, max_planes=8)
        _, _, base_st = ev.evaluate_batch(batch)
        ev.set_schedule(grn.SCHEDULE_STREAM2)
        raw, states = ev.evaluate_states(batch, max_planes=8)
        _, _, st = ev.evaluate_batch(batch)
    assert st["schedule"] == grn.SCHEDULE_STREAM2
    assert st["total_steps"] == base_st["total_steps"] < 24 * 2 * 3000
    assert np.array_equal(states, base_states)
    assert_raw_close(raw, base_raw, rtol=1e-12, atol=0, what="stream2 early exit")


def test_stream_copy_wait_times_out_cleanly():
    """A bulk copy that never arrives (test hook): the kernel's bounded wait
    runs out after about a second, the call reports it, and the context
    keeps working."""
    import time
    params, batch, init, tgt = synth.workload("large_256x256", seed=24, n_models=2, steps=5)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        ev.set_schedule(grn.SCHEDULE_STREAM)
        ev.set_test_hooks(grn.TEST_WITHHOLD_BAND_COPY)
        t0 = time.perf_counter()
        with pytest.raises(grn.GrnError) as e:
            ev.evaluate_batch(batch)
        assert "timed out" in str(e.value)
        assert time.perf_counter() - t0 < 30
        ev.set_test_hooks(0)
        _, raw, _ = ev.evaluate_batch(batch)
        ev.set_schedule(grn.SCHEDULE_GLOBAL)
        _, want, _ = ev.evaluate_batch(batch)
    assert np.isfinite(raw).all()
    np.testing.assert_array_equal(raw, want)


def test_device_allocation_failure_is_reported_and_recoverable():
    """Injected on the host: every device allocation of the context fails
    (test hook).  The call returns GRN_ERR_OUT_OF_MEMORY instead of
    aborting, and once allocation works again the same context gives the
    same results as a fresh one."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=26, n_models=20, steps=30,
                                              W=40, H=30)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        _, want, _ = ev.evaluate_batch(batch)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        ev.set_test_hooks(grn.TEST_FAIL_DEVICE_ALLOC)
        with pytest.raises(grn.GrnError) as e:
            ev.evaluate_batch(batch)
        assert e.value.status == 4  # GRN_ERR_OUT_OF_MEMORY
        ev.set_test_hooks(0)
        _, raw, _ = ev.evaluate_batch(batch)
    np.testing.assert_array_equal(raw, want)


def test_corrupt_record_is_rejected_by_the_kernel():
    """Injected on the host: the first compiled record reaches the kernel
    with a gene count of 0 (test hook).  The kernel's record check rejects
    it without touching memory past the record, the call returns
    GRN_ERR_KERNEL, and the context keeps working."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=27, n_models=20, steps=30,
                                              W=40, H=30)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        _, want, _ = ev.evaluate_batch(batch)
        ev.set_test_hooks(grn.TEST_CORRUPT_RECORD)
        with pytest.raises(grn.GrnError) as e:
            ev.evaluate_batch(batch)
        assert e.value.status == 10 and "rejected a model record" in str(e.value)
        ev.set_test_hooks(0)
        _, raw, _ = ev.evaluate_batch(batch)
    np.testing.assert_array_equal(raw, want)


def test_cluster_schedule_rejects_empty_bands():
    params, batch, init, tgt = synth.workload("small_32x32", seed=17, n_models=4, steps=10,
                                              W=32, H=20)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        ev.set_schedule(grn.SCHEDULE_CLUSTER, cluster_size=16)  # 15 * 2 rows >= 20
        with pytest.raises(grn.GrnError) as e:
            ev.evaluate_batch(batch)
        assert "CAPACITY" in str(e.value)


def test_trace_frames_match_shorter_runs():
    """Frame f of a trace is the state after f * every steps: bitwise the
    final state of the same model simulated for that many steps."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=19, n_models=3, steps=30,
                                              W=20, H=14, n_exp=2)
    every, n_frames = 7, 5
    prods, links = batch.model(1)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        frames, labels = ev.trace(prods, links, experiment=1, every=every,
                                  max_frames=n_frames, max_planes=8)
    assert frames.shape == (n_frames, 8, 14, 20)
    assert labels[0] == 0 and (np.diff(labels[labels >= 0]) > 0).all()
    np.testing.assert_array_equal(frames[0, 0], init[1, 0].astype(np.float32))
    assert not frames[0, 1:].any()  # products other than the input start at 0
    one = grn.ModelBatch.from_models([(prods, links)])
    for f in range(1, n_frames):
        p = dict(params, num_sim_steps=f * every)
        with grn.Evaluator(p) as ev:
            ev.set_experiments(init, tgt)
            _, states = ev.evaluate_states(one, max_planes=8)
        np.testing.assert_array_equal(frames[f], states[0, 1], err_msg="frame %d" % f)


def test_trace_stops_with_the_simulation():
    params, batch, init, tgt = synth.workload("small_32x32", seed=20, n_models=1, steps=4000,
                                              min_conc_change=1e-2, fitness=0)
    prods, links = batch.model(0)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        _, _, st = ev.evaluate_batch(batch)
        frames, _ = ev.trace(prods, links, every=10, max_frames=1000, max_planes=4)
    assert len(frames) == st["total_steps"] // 10 + 1 < 1000


def test_graph_mode_with_growing_gene_counts():
    """A search's population grows: batches whose largest gene count changes
    inside one gene-capacity class (at 64 x 64, 5 genes keep 10 planes in
    shared memory, 6 and 8 genes 12).  A kept plan that is not among a
    batch's candidates is tuned again, outside any capture, on that batch's
    own records; graph mode gives the plain launches' errors bit for bit."""
    params, b5, init, tgt = synth.workload("uneven_64x64", seed=31, n_models=320, steps=40,
                                           genes=(5, 5))
    _, b6, _, _ = synth.workload("uneven_64x64", seed=32, n_models=320, steps=40, genes=(6, 6))
    _, b8, _, _ = synth.workload("uneven_64x64", seed=33, n_models=320, steps=40, genes=(8, 8))
    batches = [b5, b6, b8, b5]
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        genes = [ev.pack(b).info["max_genes"] for b in batches[:3]]
        assert len(set(genes)) == 3, genes
        want = [ev.evaluate_batch(b)[1] for b in batches]
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        ev.set_graphs(True)
        got = [ev.evaluate_batch(b)[1] for b in batches]
    for w, g in zip(want, got):
        np.testing.assert_array_equal(g, w)


def test_graph_mode_matches_stream_launches():
    """Graph mode (one captured graph per job, updated in place) gives the
    same errors as plain stream launches, across batch sizes that change
    the graph's copy sizes and kernel arguments, and through submit/wait."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=22, n_models=200, steps=60,
                                              W=24, H=20)
    subsets = [np.arange(200), np.arange(37), np.arange(5, 180), np.arange(200)]
    me = np.linspace(0.01, 5.0, 200)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        want = [ev.evaluate_batch(batch.subset(ix), me[ix])[:2] for ix in subsets]
        ev.set_graphs(True)
        for ix, (we, wr) in zip(subsets, want):
            err, raw, st = ev.evaluate_batch(batch.subset(ix), me[ix])
            np.testing.assert_array_equal(raw, wr)
            np.testing.assert_array_equal(err, we)
            assert st["kernel_ms"] > 0
        for t, ix in enumerate(subsets[:3]):
            ev.submit(t, batch.subset(ix), me[ix])
        got = {}
        for _ in range(3):
            t, err, raw = ev.wait_any()
            got[t] = (err, raw)
        for t in range(3):
            np.testing.assert_array_equal(got[t][1], want[t][1])
            np.testing.assert_array_equal(got[t][0], want[t][0])


def test_early_exit_and_steps():
    """minConcChange stops simulations early; the non-convergence penalty
    uses the running change sum."""
    params, batch, init, tgt = synth.workload("small_32x32", seed=6, n_models=32, steps=3000,
                                              min_conc_change=1e-3, fitness=0, n_exp=2)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        err, raw, stats = ev.evaluate_batch(batch)
    oe, oraw, osteps = oracle.evaluate_batch(params, init, tgt, batch)
    assert_raw_close(raw, oraw, rtol=1e-3, what="early exit")
    assert stats["total_steps"] < 32 * 2 * 3000  # something converged


def test_max_error_abandon():
    params, batch, init, tgt = synth.workload("small_32x32", seed=7, n_models=32, steps=100,
                                              n_exp=3, fitness=0)
    _, _, _, _, oraw, _ = run_both(params, batch, init, tgt)
    # parents' errors: half the models get a bound below their own error
    me = np.where(np.arange(32) % 2 == 0, oraw * 0.5, 1000.0)
    err, raw, _, oe, oraw2, _ = run_both(params, batch, init, tgt, max_error=me)
    assert np.array_equal(err == 100.0, oe == 100.0)
    assert (err[::2] == 100.0).all()
    assert_rounded_close(err, oe, params["error_precision"])


def test_edge_models():
    """Zero regulation (no activator), Hill coefficient 0, K = 0 (NaN Hill
    values at x = 0, which the reference propagates), duplicate links."""
    rng = np.random.default_rng(8)
    models = []
    for t in range(24):
        pr, li = synth.random_model(rng, 4, 8, 2)
        if t % 4 == 0:
            li["hill_coef"] = -np.abs(li["hill_coef"])  # no activator anywhere
        if t % 4 == 1:
            li["hill_coef"][:3] = 0.0
        if t % 4 == 2:
            li["dis_const"][:2] = 0.0
        if t % 4 == 3:
            li = np.concatenate([li, li[:2]])
        models.append((pr, li))
    batch = ModelBatch.from_models(models)
    params, _, init, tgt = synth.workload("small_32x32", seed=9, n_models=1, steps=150, fitness=0,
                                          n_target=1, W=12, H=9)
    err, raw, _, oe, oraw, _ = run_both(params, batch, init, tgt)
    assert_raw_close(raw, oraw, what="edge models")


def test_reference_test_model():
    """The reference's built-in test model (13 products, 19 links) on
    synthetic patterns with 2 morphogens."""
    with open(os.path.join(GOLDEN, "reference_test_model.json")) as f:
        pr, li = oracle.parse_model(json.load(f)["model"])
    batch = ModelBatch.from_models([(pr, li)] * 4)
    params, _, init, tgt = synth.workload("small_32x32", seed=10, n_models=1, steps=400,
                                          n_target=1, fitness=0, n_exp=2)
    err, raw, _, oe, oraw, _ = run_both(params, batch, init, tgt)
    assert_raw_close(raw, oraw, what="reference test model")
    assert len(set(raw.tolist())) == 1


def test_single_evaluate_matches_batch():
    params, batch, init, tgt = synth.workload("small_32x32", seed=11, n_models=8, steps=60)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        err, raw, _ = ev.evaluate_batch(batch, 1000.0)
        singles = [ev.evaluate(*batch.model(i), 1000.0) for i in range(batch.n_models)]
    assert np.array_equal(np.array(singles), err)


def test_submit_wait_any():
    """ErrorCalculator::process / waitForAnyDeme semantics."""
    params, batch, init, tgt = synth.workload("small_32x32", seed=12, n_models=40, steps=80)
    demes = [batch.subset(range(i * 10, (i + 1) * 10)) for i in range(4)]
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        ref = [ev.evaluate_batch(d)[0] for d in demes]
        for i, d in enumerate(demes):
            ev.submit(i, d)
        seen = set()
        for _ in range(4):
            tag, err, raw = ev.wait_any(timeout_ms=60000)
            assert tag not in seen
            seen.add(tag)
            assert np.array_equal(err, ref[tag])
        with pytest.raises(grn.GrnError) as e:
            ev.wait_any(timeout_ms=10)
        assert e.value.status == 9


def test_rgb_experiments_match_planar():
    rng = np.random.default_rng(13)
    params, batch, _, _ = synth.workload("small_32x32", seed=13, n_models=6, steps=50, n_target=1)
    W, H = params["dim_x"], params["dim_y"]
    pin = rng.integers(0, 2 ** 32, size=(2, H, W), dtype=np.uint64).astype(np.uint32)
    pout = rng.integers(0, 2 ** 32, size=(2, H, W), dtype=np.uint64).astype(np.uint32)
    init = np.stack([grn.decode_rgb(p, 1) for p in pin])
    tgt = np.stack([grn.decode_rgb(p, 1) for p in pout])
    with grn.Evaluator(params) as ev:
        ev.set_experiments_rgb(pin, pout)
        a = ev.evaluate_batch(batch)[1]
        ev.set_experiments(init, tgt)
        b = ev.evaluate_batch(batch)[1]
    assert np.array_equal(a, b)


def test_run_packed_device_buffers():
    """Device-level entry point on a caller stream equals the host path."""
    torch = pytest.importorskip("torch")
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=14, n_models=64, steps=50)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        _, raw_ref, _ = ev.evaluate_batch(batch)
        pk = ev.pack(batch)
        me = torch.full((64,), 1000.0, dtype=torch.float64, device="cuda")
        raw = torch.zeros(64, dtype=torch.float64, device="cuda")
        steps = torch.zeros(64, dtype=torch.int32, device="cuda")
        # A stream of its own: the legacy default stream's handle is 0, which
        # the C ABI reads as "the evaluator's stream".
        s = torch.cuda.Stream()
        torch.cuda.synchronize()
        pk.run(me.data_ptr(), raw.data_ptr(), steps.data_ptr(), s.cuda_stream)
        s.synchronize()
        assert np.array_equal(raw.cpu().numpy(), raw_ref)
        assert (steps.cpu().numpy() == 50).all()
        assert pk.info["n_models"] == 64
        pk.free()


def test_full_headline_workload_properties():
    """All 4096 models x 2000 steps of the headline workload: deterministic
    across runs, finite, every step run (min_conc_change 0), and a sample
    agrees with the oracle."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=0)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        err1, raw1, st1 = ev.evaluate_batch(batch)
        err2, raw2, st2 = ev.evaluate_batch(batch)
    assert np.array_equal(raw1, raw2)
    assert np.isfinite(raw1).all()
    assert st1["cell_updates"] == 4096 * 2000 * 64 * 64
    idx = np.arange(0, 4096, 512)
    sub = batch.subset(idx)
    oe, oraw, _ = oracle.evaluate_batch(params, init, tgt, sub)
    assert_raw_close(raw1[idx], oraw, what="headline sample")


def test_host_thread_count_does_not_change_results():
    """Batches compiled by one host thread or by many give the same errors
    bit for bit (the record order is the cost order either way)."""
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=43, n_models=600, steps=30)
    out = []
    for n in (1, 0, 5):
        with grn.Evaluator(params) as ev:
            ev.set_experiments(init, tgt)
            ev.set_host_threads(n)
            out.append(ev.evaluate_batch(batch)[1])
    np.testing.assert_array_equal(out[0], out[1])
    np.testing.assert_array_equal(out[0], out[2])
