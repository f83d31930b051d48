"""The C++ host layer (include/grn_gpu.hpp): the reference's evaluator
classes -- CEvaluatorMorphogens, ErrorCalculator, Individual, Model -- over
the C ABI.  A small driver (tests/cpp/evaluator_layer.cpp) is compiled with
g++ against the header and the built library.

CPU: model text round trip, batch view, no device -> grn::Error
(GRN_ERR_NO_DEVICE).  GPU: one-by-one, batched and deme-by-deme
(ErrorCalculatorB200) evaluations agree bit for bit and match the oracle
within the parity tolerance (raw errors to 1e-4 relative, so rounded errors
to one unit of their last digit)."""
import json
import math
import os
import subprocess

import numpy as np
import pytest

import binding as oracle
import grn_b200 as grn
import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "evaluator_layer.cpp")
GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_test_model.json")


@pytest.fixture(scope="module")
def driver(built_libs, tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "evaluator_layer")
    libdir = os.path.dirname(grn.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L", libdir, "-l:" + os.path.basename(grn.LIB_PATH),
                    "-Wl,-rpath," + libdir], check=True)
    return exe


@pytest.mark.skipif(__import__("conftest").HAS_GPU, reason="checks the no-device path")
def test_cpp_layer_host_side(driver, tmp_path):
    model = json.load(open(GOLDEN))["model"]
    f = tmp_path / "model.txt"
    f.write_text(model + "\n")
    out = subprocess.run([driver, "cpu", str(f)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "ok"


def _write_input(path, params, init, tgt, batch, deme, max_error):
    lines = [" ".join(str(params[k]) for k in (
        "dim_x", "dim_y", "n_input_morphogens", "n_target_morphogens", "num_sim_steps",
        "error_precision", "fitness_kind")) + " " + " ".join(repr(float(params[k])) for k in (
        "dt", "min_conc", "min_conc_change", "dist_error_threshold")),
        str(init.shape[0]),
        " ".join(repr(float(v)) for v in init.ravel()),
        " ".join(repr(float(v)) for v in tgt.ravel()),
        "%d %d" % (batch.n_models, int(max(deme)) + 1)]
    for m in range(batch.n_models):
        prods, links = batch.model(m)
        lines.append("%d %r %s" % (deme[m], float(max_error[m]),
                                   grn.format_model(prods, links, precision=17)))
    path.write_text("\n".join(lines) + "\n")


@pytest.mark.gpu
def test_cpp_layer_matches_oracle(driver, tmp_path):
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=41, n_models=36, steps=120,
                                              W=24, H=18, n_exp=2)
    rng = np.random.default_rng(41)
    deme = rng.integers(0, 5, batch.n_models)
    deme[:5] = np.arange(5)  # every deme non-empty
    max_error = np.where(rng.random(batch.n_models) < 0.25, 0.05, 1000.0)
    inp, outp = tmp_path / "in.txt", tmp_path / "out.txt"
    _write_input(inp, params, init, tgt, batch, deme, max_error)
    out = subprocess.run([driver, "gpu", str(inp), str(outp)], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    res = np.loadtxt(outp, ndmin=2)
    one, batched, calc, sim_time = res[:, 1], res[:, 2], res[:, 3], res[:, 4]
    assert np.array_equal(one, batched) and np.array_equal(one, calc)
    assert (sim_time > 0).all()
    oe, oraw, _ = oracle.evaluate_batch(params, init, tgt, batch, max_error)
    assert (one == 100.0).sum() > 0  # the maxError abandon path is exercised
    for g, r in zip(one, oe):
        if r == 100.0 or g == 100.0:
            assert g == r
            continue
        unit = 10.0 ** (math.ceil(math.log10(abs(r))) - params["error_precision"]) if r else 0.0
        assert abs(g - r) <= max(unit * 1.001, 1e-7 + 1e-4 * abs(r)), (g, r)
