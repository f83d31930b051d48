"""The reference's model text format (grn_model_format / grn_model_parse),
pinned on the reference's own test-model string."""
import json
import os

import numpy as np
import pytest

import binding as oracle
import grn_b200 as grn
import synth

HERE = os.path.dirname(os.path.abspath(__file__))


def _ref_model():
    with open(os.path.join(HERE, "golden", "reference_test_model.json")) as f:
        return json.load(f)["model"]


def test_reference_string_roundtrips_byte_for_byte(built_libs):
    text = _ref_model()
    pr, li = grn.parse_model(text)
    assert len(pr) == 13 and len(li) == 19
    assert grn.format_model(pr, li) == text  # 6 significant digits, as the reference writes
    opr, oli = oracle.parse_model(text)
    for f in ("label", "init", "lim", "deg", "dif"):
        np.testing.assert_array_equal(pr[f], opr[f])
    for f in ("regulator", "regulated", "dis_const", "hill_coef", "is_and"):
        np.testing.assert_array_equal(li[f], oli[f])


def test_exact_roundtrip_of_random_models(built_libs):
    b = synth.random_batch(200, (1, 8), (0, 24), 3, 9)
    for i in range(b.n_models):
        pr, li = b.model(i)
        pr2, li2 = grn.parse_model(grn.format_model(pr, li, precision=17))
        np.testing.assert_array_equal(pr2, pr)
        np.testing.assert_array_equal(li2, li)


def test_parse_edge_cases(built_libs):
    pr, li = grn.parse_model("(0 -1 0.5 0.25 0*)")
    assert len(pr) == 1 and len(li) == 0 and pr[0]["init"] == -1
    pr, li = grn.parse_model(" ( 0 -1 1e-05 inf 0 | 3 0 1 2 3 * 3 0 0.5 -2 7 ) ")
    assert pr[0]["lim"] == 1e-05 and np.isinf(pr[0]["deg"]) and li[0]["is_and"] == 1
    assert grn.format_model(pr, li) == "(0 -1 1e-05 inf 0|3 0 1 2 3*3 0 0.5 -2 1)"
    for bad in ("", "(", "()", "(0 1 2 3*)", "(0 1 2 3 4|*)", "(0 1 2 3 4*1 2 3 4)",
                "(0 1 2 3 4*1 2 3 4 0", "(0 1 2 3 4*) trailing", "(x 1 2 3 4*)",
                "(0 1 2 3 4*1 2 3 4 0|)"):
        with pytest.raises(grn.GrnError) as e:
            grn.parse_model(bad)
        assert "MODEL" in str(e.value), bad
