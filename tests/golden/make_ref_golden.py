"""Writes tests/golden/ref_pinned.json: evaluation cases with the outputs of
the reference's OWN CPU fitness path, compiled from its unchanged sources
into oracle/_ref (oracle/build_ref.py).

  python tests/golden/make_ref_golden.py [--reference DIR]

DIR is the reference checkout (default $GRN_REFERENCE_ROOT, else
/root/reference); it is needed only if oracle/_ref is not built yet.

Every case gives the simulation parameters, the experiments as the 32-bit RGB
images the reference loads (SimState::loadMorphologyImage,
Src/Simulator/simstate.cpp:71-90), the models as reference model strings
(Model::loadFromString, Src/Model/model.cpp:639-706) and the max errors, and
records what the reference computed for them:

  errors    EvaluatorMorphogens::evaluate (Src/Search/evaluatormorphogens.cpp:48-76),
            the rounded error or 100, for every model;
  runs      for the first models, one Simulator run over experiment 0
            (Src/Simulator/simulator.cpp:35-63): the final state of every
            product in use, the last step's change, the steps taken and the
            thresholded log distance to the target (simstate.cpp:135-158).

Doubles are stored exactly: scalars as float.hex strings, arrays as base64
of little-endian float64 bytes.  The cases cover uneven random models on a
ragged grid with two experiments, abandoned models (max error), early exit
(min_conc_change > 0), a minConc clamp, hand-made edge models (K = 0,
n = 0, a repeated link, no activator, no links, negative K), an unstable
step (dt * dif > 1/4: cells overflow to inf and NaN), the reference's own
test model, and one-cell, one-row and one-column grids.
"""
import argparse
import base64
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "grn-gpu-performance_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import ref_binding as ref  # noqa: E402
import synth  # noqa: E402
from grn_b200 import LINK_DTYPE, PRODUCT_DTYPE, ModelBatch  # noqa: E402

OUT = os.path.join(HERE, "ref_pinned.json")
RUNS_PER_CASE = 3


def f64(a):
    return base64.b64encode(np.ascontiguousarray(a, "<f8").tobytes()).decode()


def u32(a):
    return base64.b64encode(np.ascontiguousarray(a, "<u4").tobytes()).decode()


def _params(W, H, n_in, n_target, steps, dt=0.1, min_conc=0.0, min_conc_change=0.0,
            precision=8, threshold=0.05):
    return dict(dim_x=W, dim_y=H, n_input_morphogens=n_in, n_target_morphogens=n_target,
                num_sim_steps=steps, error_precision=precision, fitness_kind=0, dt=dt,
                min_conc=min_conc, min_conc_change=min_conc_change,
                dist_error_threshold=threshold)


def _images(params, n_exp, seed):
    """Seeded input (radial or gradient) and target (stripe) images."""
    rng = np.random.default_rng(seed)
    W, H = params["dim_x"], params["dim_y"]
    ins, outs = [], []
    for e in range(n_exp):
        planes = [synth.radial_pattern(rng, W, H) if k % 2 == 0 else
                  synth.gradient_pattern(rng, W, H)
                  for k in range(params["n_input_morphogens"])]
        ins.append(ref.encode_rgb(np.array(planes)))
        tg = [synth.stripe_pattern(rng, W, H) * rng.uniform(0.6, 1.0)
              for _ in range(params["n_target_morphogens"])]
        outs.append(ref.encode_rgb(np.array(tg)))
    return np.array(ins), np.array(outs)


def _model(prods, links):
    p = np.zeros(len(prods), PRODUCT_DTYPE)
    for i, (lab, lim, deg, dif) in enumerate(prods):
        p[i] = (lab, 0, -(lab + 1) if lab < 3 else 0, lim, deg, dif)
    l = np.zeros(len(links), LINK_DTYPE)
    for i, (a, b, k, n, is_and) in enumerate(links):
        l[i] = (a, b, k, n, is_and, 0)
    return p, l


def edge_models():
    """Hand-made models that reach the reference's special cases
    (Src/Simulator/modelsimulator.cpp:71-280, simophillact.cpp:9-20)."""
    base = [(0, 0.5, 0.2, 0.3), (1, 0.7, 0.4, 0.0), (2, 0.6, 0.3, 0.2), (3, 0.9, 0.5, 0.4)]
    return [
        _model(base, [(3, 1, 0.0, 2.0, 0), (1, 2, 0.4, 2.0, 1), (1, 3, 0.6, 1.0, 0)]),  # K = 0
        # K = 0 as the first and as the second OR term: a NaN Hill value is
        # dropped as the running value and kept as the new term
        # (simopor.cpp:20-22 with MathAlgo::max).
        _model(base, [(3, 1, 0.0, 2.0, 0), (2, 1, 0.5, 1.5, 0), (1, 2, 0.4, 2.0, 1),
                      (1, 3, 0.6, 1.0, 0)]),
        _model(base, [(2, 1, 0.5, 1.5, 0), (3, 1, 0.0, 2.0, 0), (1, 2, 0.4, 2.0, 1),
                      (1, 3, 0.6, 1.0, 0)]),
        _model(base, [(0, 1, 0.5, 0.0, 0), (2, 1, 0.4, 3.0, 1), (1, 3, 0.3, 2.0, 0)]),  # n = 0
        _model(base, [(0, 1, 0.5, 2.0, 0), (0, 1, 0.3, -1.5, 1), (1, 2, 0.6, 2.5, 0)]),  # repeat
        _model(base, [(0, 1, 0.5, -2.0, 1), (2, 1, 0.3, -1.0, 1), (1, 2, 0.6, 2.5, 0)]),  # no act
        _model(base, []),                                                                # no links
        _model(base, [(0, 1, -0.4, 2.0, 0), (1, 2, 0.6, 1.5, 1)]),                      # K < 0
        _model(base, [(1, 1, 0.3, 4.0, 0), (2, 2, 0.2, -3.5, 1), (0, 3, 0.9, 1.0, 1),
                      (3, 0, 0.1, 2.0, 0), (2, 0, 0.7, -2.0, 1)]),                      # loops
    ]


def reference_test_model_case():
    with open(os.path.join(HERE, "reference_test_model.json")) as f:
        text = json.load(f)["model"]
    return text


def random_texts(n, genes, links, n_morph, seed):
    b = synth.random_batch(n, genes, links, n_morph, seed)
    return [ref.model_text(*b.model(i)) for i in range(b.n_models)], b


def make_cases():
    cases = []

    def add(name, params, n_exp, texts, max_error, seed):
        ins, outs = _images(params, n_exp, seed)
        errors = ref.evaluate_texts(params, ins, outs, texts, max_error, n_threads=8)
        runs = []
        for i in range(min(RUNS_PER_CASE, len(texts))):
            prods, links = _parse(texts[i])
            state, change, steps, dist = ref.simulate(params, ins[0], prods, links,
                                                      params["num_sim_steps"], target_px=outs[0])
            runs.append({"model": i, "planes": int(state.shape[0]), "state": f64(state),
                         "change": change.hex(), "steps": steps, "distance": dist.hex()})
        cases.append({"name": name, "params": params, "n_exp": n_exp,
                      "input_px": u32(ins), "target_px": u32(outs), "models": texts,
                      "max_error": [float(x).hex() for x in max_error],
                      "errors": [float(x).hex() for x in errors], "runs": runs})

    p = _params(18, 13, 1, 2, 300)
    texts, _ = random_texts(24, (2, 8), (1, 24), 3, seed=101)
    me = np.full(len(texts), 1000.0)
    me[::4] = 0.3
    add("uneven_ragged_2exp", p, 2, texts, me, seed=201)

    p = _params(20, 20, 1, 1, 2000, min_conc_change=0.02)
    texts, _ = random_texts(12, (2, 6), (1, 12), 2, seed=102)
    add("early_exit", p, 1, texts, np.full(len(texts), 1000.0), seed=202)

    p = _params(16, 12, 1, 1, 200, min_conc=0.002)
    texts, _ = random_texts(12, (2, 6), (1, 12), 2, seed=103)
    add("min_conc_clamp", p, 1, texts, np.full(len(texts), 1000.0), seed=203)

    p = _params(15, 11, 1, 1, 150)
    texts = [ref.model_text(*m) for m in edge_models()]
    add("edge_models", p, 1, texts, np.full(len(texts), 1000.0), seed=204)

    p = _params(12, 10, 1, 1, 1500, dt=1.0)
    texts, b = random_texts(8, (2, 5), (1, 10), 2, seed=105)
    for i in range(b.n_models):
        pr, li = b.model(i)
        pr["dif"] = np.linspace(0.5, 1.0, len(pr))
    texts = [ref.model_text(*b.model(i)) for i in range(b.n_models)]
    add("unstable_dt", p, 1, texts, np.full(len(texts), 1000.0), seed=205)

    p = _params(32, 32, 1, 1, 500, precision=10)
    add("reference_test_model", p, 1, [reference_test_model_case()], [1000.0], seed=206)

    for W, H in ((1, 1), (1, 7), (9, 1)):
        p = _params(W, H, 1, 1, 120)
        texts, _ = random_texts(5, (2, 5), (1, 10), 2, seed=106 + W * 10 + H)
        add("grid_%dx%d" % (W, H), p, 1, texts, np.full(len(texts), 1000.0), seed=207 + W + H)
    return cases


def _parse(text):
    """Model string -> (products, links) with the reference's parser's
    meaning (label init lim deg dif | regulator regulated K n isAnd)."""
    body = text.strip()[1:-1]
    ptxt, ltxt = body.split("*")
    prods = [s.split() for s in ptxt.split("|") if s.strip()]
    links = [s.split() for s in ltxt.split("|") if s.strip()]
    p = np.zeros(len(prods), PRODUCT_DTYPE)
    for i, f in enumerate(prods):
        p[i] = (int(f[0]), 0, float(f[1]), float(f[2]), float(f[3]), float(f[4]))
    l = np.zeros(len(links), LINK_DTYPE)
    for i, f in enumerate(links):
        l[i] = (int(f[0]), int(f[1]), float(f[2]), float(f[3]), int(f[4]), 0)
    return p, l


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None,
                    help="reference checkout (default $GRN_REFERENCE_ROOT or /root/reference)")
    args = ap.parse_args()
    if args.reference:
        os.environ["GRN_REFERENCE_ROOT"] = args.reference
    if not ref.available():
        ref.build()
    cases = make_cases()
    with open(OUT, "w") as f:
        json.dump({"source": "oracle/_ref: the reference's CPU fitness path compiled from its "
                             "unchanged sources (oracle/build_ref.py)",
                   "generator": "tests/golden/make_ref_golden.py", "cases": cases}, f)
        f.write("\n")
    print("wrote %s: %d cases, %d models" % (OUT, len(cases),
                                             sum(len(c["models"]) for c in cases)))


if __name__ == "__main__":
    main()
