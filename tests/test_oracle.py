"""CPU tests of the FP64 oracle: pinned against the reference's fixtures
where they exist, cross-checked against the independent pure-Python
restatement, and frozen against the committed golden outputs."""
import json
import math
import os

import numpy as np
import pytest

import binding as oracle
import pyoracle
import synth
from grn_b200 import LINK_DTYPE, PRODUCT_DTYPE, ModelBatch

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _dicts(a):
    return [dict(zip(a.dtype.names, [x.item() for x in r])) for r in a]


def _ref_model():
    with open(os.path.join(GOLDEN, "reference_test_model.json")) as f:
        return json.load(f)


def test_parse_reference_test_model(built_libs):
    """The reference's test-model string (errorcalculatormultithread.cpp:61)
    parses to 13 products and 19 links with the fields it spells out."""
    pr, li = oracle.parse_model(_ref_model()["model"])
    assert len(pr) == 13 and len(li) == 19
    assert pr["label"][0] == 87889 and pr["lim"][0] == 0.614236 and pr["dif"][0] == 0.912483
    # label 1 is the green morphogen (init -2), label 0 the red one (init -1)
    one = pr[pr["label"] == 1][0]
    assert one["init"] == -2 and one["lim"] == 0.828329 and one["dif"] == 0
    zero = pr[pr["label"] == 0][0]
    assert zero["init"] == -1 and zero["deg"] == 0.00487246
    assert (li["regulator"][1], li["regulated"][1]) == (132569, 132569)
    assert li["hill_coef"][1] == -4.91105 and li["is_and"][1] == 1
    assert li["dis_const"][3] == 0.0162271 and li["is_and"][3] == 0


def test_reference_model_round_trip(built_libs):
    text = _ref_model()["model"]
    pr, li = oracle.parse_model(text)
    assert oracle.format_model(pr, li) == text


def test_reference_model_labels_in_use(built_libs):
    """Model::calcProductLabelsInUse on the test model with 2 morphogens."""
    pr, li = oracle.parse_model(_ref_model()["model"])
    labels = oracle.labels_in_use(pr, li, 2)
    assert labels == pyoracle.labels_in_use(pr, _dicts(li), 2)
    # 0 and 1 are regulated by 64653, 107652, 1 (chains through 64653 <- 0)
    assert labels == sorted(labels) and labels[:2] == [0, 1]
    assert 64653 in labels and 107652 in labels
    assert 87889 not in labels  # regulates only 136389, which is not in use


def test_reference_model_program(built_libs):
    """Op program of the test model: OR links before AND links, repression
    for negative Hill coefficients, zero for products without activators."""
    pr, li = oracle.parse_model(_ref_model()["model"])
    prog = oracle.dump_program(pr, li, 2).splitlines()
    labels = oracle.labels_in_use(pr, li, 2)
    idx = {lab: i for i, lab in enumerate(labels)}
    # label 1 has links 0->1 (act, OR), 1->1 (act, OR), 107652->1 (rep, AND)
    p1 = [l for l in prog if l.split()[1] in (str(idx[1]), "-1")]
    assert prog[0].startswith("hillact") or prog[0].startswith("zero")
    want_first = "hillact %d %d " % (idx[1], idx[0])
    assert any(l.startswith(want_first) for l in prog)
    assert any(l == "or %d" % idx[1] for l in prog)
    assert any(l == "and %d" % idx[1] for l in prog)
    assert any(l.startswith("hillrep -1 %d " % idx[107652]) for l in prog)
    assert p1


def test_oracle_matches_python_restatement(built_libs):
    """The C++ oracle and the pure-Python oracle agree bit for bit on random
    tiny cases, including K = 0 (NaN Hill values), Hill coefficient 0,
    clamping, early exit and both fitness kinds."""
    rng = np.random.default_rng(7)
    for t in range(30):
        W, H = int(rng.integers(1, 6)), int(rng.integers(1, 6))
        nin, nt = 1, int(rng.integers(1, 3))
        G = int(rng.integers(nin + nt, 6))
        pr, li = synth.random_model(rng, G, int(rng.integers(0, 10)), nin + nt)
        if t % 5 == 0 and len(li):
            li["dis_const"][0] = 0.0
        if t % 7 == 0 and len(li):
            li["hill_coef"][0] = 0.0
        params = dict(dim_x=W, dim_y=H, n_input_morphogens=nin, n_target_morphogens=nt,
                      num_sim_steps=int(rng.integers(0, 25)), error_precision=6,
                      fitness_kind=t % 2, dt=0.1, min_conc=0.0 if t % 3 else 0.05,
                      min_conc_change=1e-3 if t % 4 == 0 else 0.0, dist_error_threshold=0.05)
        nexp = int(rng.integers(1, 3))
        init, tgt = rng.random((nexp, nin, H, W)), rng.random((nexp, nt, H, W))
        e, r, s = oracle.evaluate_batch(params, init, tgt, ModelBatch.from_models([(pr, li)]),
                                        [5.0], n_threads=1)
        pe, praw, ps = pyoracle.evaluate(params, init.tolist(), tgt.tolist(), _dicts(pr),
                                         _dicts(li), 5.0)
        assert (math.isnan(r[0]) and math.isnan(praw)) or r[0] == praw, t
        assert (math.isnan(e[0]) and math.isnan(pe)) or e[0] == pe, t
        assert s[0] == ps, t


def test_oracle_golden_fixtures(built_libs):
    """The oracle still reproduces the committed golden outputs exactly."""
    with open(os.path.join(GOLDEN, "oracle_small.json")) as f:
        cases = json.load(f)["cases"]
    assert len(cases) >= 5
    for c in cases:
        batch = ModelBatch(c["product_offsets"],
                           np.array([tuple(r) for r in c["products"]], PRODUCT_DTYPE),
                           c["link_offsets"], np.array([tuple(r) for r in c["links"]], LINK_DTYPE))
        e, r, s = oracle.evaluate_batch(c["params"], np.array(c["initial"]), np.array(c["target"]),
                                        batch, c["max_error"], n_threads=2)
        assert r.tolist() == c["raw_error"]
        assert e.tolist() == c["error"]
        assert s.tolist() == c["steps"]


def test_oracle_thread_pool_is_deterministic(built_libs):
    params, batch, init, tgt = synth.workload("small_32x32", seed=3, n_models=12, steps=20)
    a = oracle.evaluate_batch(params, init, tgt, batch, n_threads=1)
    b = oracle.evaluate_batch(params, init, tgt, batch, n_threads=4)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("x,d,want", [(0.048701011019999997, 10, 0.04870101102),
                                      (0.0, 5, 0.0), (1.23451, 3, 1.24), (99.0001, 2, 100.0),
                                      (0.000123456, 2, 0.00013)])
def test_ceil_s(built_libs, x, d, want):
    """MathAlgo::ceilS rounds UP to d significant digits (mathalgo.h:55-62)."""
    assert oracle.ceil_s(x, d) == pytest.approx(want, rel=1e-12, abs=0)
    assert oracle.ceil_s(x, d) == pyoracle.ceil_s(x, d)


def test_decode_rgb_flips_y(built_libs):
    """SimState::loadMorphologyImage: scanline j -> row H-1-j, channel k =
    byte (16 - 8k) / 255 of 0xAARRGGBB."""
    px = np.array([[0xFF102030, 0xFF405060], [0xFF708090, 0xFFA0B0C0]], np.uint32)
    out = oracle.decode_rgb(px, 3)
    assert out[0, 1, 0] == 0x10 / 255.0 and out[1, 1, 0] == 0x20 / 255.0
    assert out[2, 1, 1] == 0x60 / 255.0 and out[0, 0, 0] == 0x70 / 255.0
