"""Parity pinned to the reference itself (CPU).

oracle/_ref is the reference's own CPU fitness path -- EvaluatorMorphogens,
Simulator, ModelSimulator, the SimOp classes, SimState and Model -- compiled
from its unchanged sources (oracle/build_ref.py).  These tests check:

  - the FP64 restatement (oracle/grn_oracle.cpp) against the committed
    reference-produced fixtures (tests/golden/ref_pinned.json): rounded
    errors, final states, changes and step counts bit for bit, NaN and inf
    cells included;
  - the restatement against the live reference library on random batches,
    including the full 64-model 32x32 500-step configuration and a sample of
    the 64x64 uneven configuration at its full 2000 steps;
  - the text format, image decoding, ceilS rounding and labels-in-use of
    the product's C ABI and of the restatement against the reference's.

The live-library tests skip where oracle/_ref is neither built nor buildable
(no reference checkout); the fixture tests run everywhere.
"""
import numpy as np
import pytest

import binding as oracle
import grn_b200 as grn
import ref_binding as ref
import ref_golden
import synth
from grn_b200 import ModelBatch

needs_ref = pytest.mark.skipif(not (ref.available() or ref.build()),
                               reason="oracle/_ref is not built and the reference is absent")


def _oracle_inputs(case):
    p = case["params"]
    init = np.stack([oracle.decode_rgb(px, p["n_input_morphogens"]) for px in case["input_px"]])
    tgt = np.stack([oracle.decode_rgb(px, p["n_target_morphogens"]) for px in case["target_px"]])
    return init, tgt


def _batch(texts, parse=oracle.parse_model):
    return ModelBatch.from_models([parse(t) for t in texts])


@pytest.mark.parametrize("case", ref_golden.load_cases(), ids=lambda c: c["name"])
def test_restatement_matches_reference_fixtures(case, built_libs):
    p = case["params"]
    init, tgt = _oracle_inputs(case)
    batch = _batch(case["models"])
    err, _, _ = oracle.evaluate_batch(p, init, tgt, batch, case["max_error"])
    assert np.array_equal(err, case["errors"], equal_nan=True), (err, case["errors"])
    for run in case["runs"]:
        pr, li = batch.model(run["model"])
        state, change, steps = oracle.simulate(p, init[0], pr, li, p["num_sim_steps"])
        assert np.array_equal(state, run["state"], equal_nan=True), run["model"]
        assert change == run["change"] or (np.isnan(change) and np.isnan(run["change"]))
        assert steps == run["steps"]


def test_reference_fixtures_cover_the_special_cases():
    cases = {c["name"]: c for c in ref_golden.load_cases()}
    assert (cases["uneven_ragged_2exp"]["errors"] == 100.0).any()        # abandoned models
    assert len({r["steps"] for r in cases["early_exit"]["runs"]}) > 1     # early exit
    assert any(np.isnan(r["state"]).any() for r in cases["unstable_dt"]["runs"])
    assert any(np.isnan(r["state"]).any() for r in cases["edge_models"]["runs"])  # K = 0


@needs_ref
@pytest.mark.parametrize("config", [
    # The full 64-model 32x32 500-step configuration (thresholded-log fitness:
    # the reference has no other).
    dict(name="small_32x32", n_models=64, kw=dict(fitness=0)),
    # A sample of the 64x64 uneven configuration at its full 2000 steps.
    dict(name="uneven_64x64", n_models=24, kw=dict()),
    # Ragged grid, two experiments, two target channels, max-error abandon.
    dict(name="uneven_64x64", n_models=32, kw=dict(steps=250, W=27, H=19, n_exp=2, n_target=2)),
])
def test_restatement_matches_reference_library(config, built_libs):
    params, batch, init, tgt = synth.workload(config["name"], seed=77, n_models=config["n_models"],
                                              **config["kw"])
    assert params["fitness_kind"] == 0
    ipx = np.stack([ref.encode_rgb(e) for e in init])
    tpx = np.stack([ref.encode_rgb(e) for e in tgt])
    dinit = np.stack([ref.decode_rgb(px, params["n_input_morphogens"]) for px in ipx])
    dtgt = np.stack([ref.decode_rgb(px, params["n_target_morphogens"]) for px in tpx])
    me = np.full(batch.n_models, 1000.0)
    me[1::7] = 0.2
    want = ref.evaluate_batch(params, ipx, tpx, batch, me, n_threads=8)
    got, _, _ = oracle.evaluate_batch(params, dinit, dtgt, batch, me)
    assert np.array_equal(got, want, equal_nan=True)
    for m in range(0, batch.n_models, max(1, batch.n_models // 4)):
        pr, li = batch.model(m)
        s_ref, ch_ref, st_ref, _ = ref.simulate(params, ipx[0], pr, li, params["num_sim_steps"])
        s_or, ch_or, st_or = oracle.simulate(params, dinit[0], pr, li, params["num_sim_steps"])
        assert np.array_equal(s_or, s_ref, equal_nan=True)
        assert (ch_or, st_or) == (ch_ref, st_ref)


@needs_ref
def test_decode_and_rounding_match_reference(built_libs):
    rng = np.random.default_rng(5)
    px = rng.integers(0, 2 ** 32, size=(11, 17), dtype=np.uint64).astype(np.uint32)
    for n in (1, 2, 3):
        want = ref.decode_rgb(px, n)
        assert np.array_equal(oracle.decode_rgb(px, n), want)
        assert np.array_equal(grn.decode_rgb(px, n), want)
    for x in np.concatenate([rng.uniform(0, 2, 200), 10.0 ** rng.uniform(-9, 3, 200),
                             [0.0, 1.0, 0.1, 0.048701011019999997]]):
        for d in (1, 4, 8, 12):
            want = ref.ceil_s(x, d)
            assert oracle.ceil_s(x, d) == want
            assert grn.round_error(x, 1e300, d) == want


@needs_ref
def test_model_text_and_labels_match_reference(built_libs):
    texts = [ref_golden.load_cases()[-4]["models"][0]]  # the reference's test model
    b = synth.random_batch(40, (2, 9), (0, 30), 3, seed=8)
    texts += [ref.model_text(*b.model(i)) for i in range(b.n_models)]
    for text in texts:
        pr, li = grn.parse_model(text)
        # The reference's own writer (6 significant digits) and ours agree.
        assert grn.format_model(pr, li) == ref.format_model(text)
        opr, oli = oracle.parse_model(text)
        assert np.array_equal(opr, pr) and np.array_equal(oli, li)
        for n_morph in (1, 2, 3):
            want = ref.labels_in_use(pr, li, n_morph).tolist()
            assert oracle.labels_in_use(pr, li, n_morph) == want
