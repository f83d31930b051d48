"""Regenerates the golden fixtures in tests/golden/.

  python tests/golden/make_golden.py [--reference DIR]

reference_test_model.json
    The reference's only known-answer fixture: the test-model string of
    ErrorCalculatorMultiThread::testPerformance
    (Src/UI/Evolution/errorcalculatormultithread.cpp:61) and its expected
    error (:62).  Read from the reference source tree when it is mounted;
    the expected error cannot be re-run (its experiment images live in an
    unshipped database) and is recorded for documentation only.

oracle_small.json
    Seeded small evaluation cases (models, initial/target patterns,
    parameters) with the FP64 oracle's outputs.  Every case is computed by
    both oracle restatements (C++ oracle/grn_oracle.cpp and pure-Python
    oracle/pyoracle.py) and written only if they agree bit for bit.
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "grn-gpu-performance_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import binding as oracle  # noqa: E402
import pyoracle  # noqa: E402
import synth  # noqa: E402
from grn_b200 import ModelBatch  # noqa: E402

REF_FILE = os.path.join("Src", "UI", "Evolution", "errorcalculatormultithread.cpp")


def reference_source(root):
    """The reference file holding its test model, under the checkout `root`
    (the --reference argument, else $GRN_REFERENCE_ROOT, else
    /root/reference)."""
    root = root or os.environ.get("GRN_REFERENCE_ROOT", "/root/reference")
    return os.path.join(root, REF_FILE)


def reference_test_model(path):
    with open(path) as f:
        lines = f.read().splitlines()
    model = re.search(r'QString modelStr\("(.*)"\);', lines[60]).group(1)
    expected = re.search(r"double expectedError = ([0-9.eE+-]+);", lines[61]).group(1)
    return {"source": "Src/UI/Evolution/errorcalculatormultithread.cpp:61-62",
            "model": model, "expected_error_text": expected}


def _records(a):
    return [[x.item() for x in r] for r in a]


def small_cases():
    cases = []
    rng = np.random.default_rng(20261203)
    specs = [
        # (W, H, n_in, n_target, steps, n_exp, fitness, min_conc, min_conc_change, genes, links)
        (8, 8, 1, 1, 60, 1, 0, 0.0, 0.0, (2, 5), (1, 10)),
        (8, 6, 1, 2, 40, 2, 0, 0.0, 0.0, (3, 6), (2, 12)),
        (5, 7, 1, 1, 80, 1, 1, 0.0, 0.0, (2, 4), (1, 8)),
        (6, 6, 2, 1, 50, 2, 0, 0.02, 0.0, (3, 6), (1, 12)),
        (4, 4, 1, 1, 400, 1, 0, 0.0, 1e-3, (2, 4), (1, 6)),  # early exit
        (1, 1, 1, 1, 30, 1, 0, 0.0, 0.0, (2, 3), (1, 4)),
        (9, 3, 1, 2, 45, 1, 1, 0.0, 0.0, (3, 7), (3, 14)),
    ]
    for ci, (W, H, nin, nt, steps, nexp, fk, mc, mcc, genes, links) in enumerate(specs):
        params = dict(dim_x=W, dim_y=H, n_input_morphogens=nin, n_target_morphogens=nt,
                      num_sim_steps=steps, error_precision=6, fitness_kind=fk, dt=0.1,
                      min_conc=mc, min_conc_change=mcc, dist_error_threshold=0.05)
        models = []
        for _ in range(6):
            g = int(rng.integers(genes[0], genes[1] + 1))
            l = int(rng.integers(links[0], links[1] + 1))
            models.append(synth.random_model(rng, max(g, nin + nt), l, nin + nt))
        batch = ModelBatch.from_models(models)
        init = rng.random((nexp, nin, H, W))
        tgt = (rng.random((nexp, nt, H, W)) > 0.5).astype(np.float64)
        max_error = np.full(batch.n_models, 1000.0)
        max_error[-1] = 0.05  # exercise the abandon-on-maxError path
        err, raw, st = oracle.evaluate_batch(params, init, tgt, batch, max_error, n_threads=1)
        for m in range(batch.n_models):
            pr, li = batch.model(m)
            todict = lambda a: [dict(zip(a.dtype.names, [x.item() for x in r])) for r in a]
            pe, praw, ps = pyoracle.evaluate(params, init.tolist(), tgt.tolist(), todict(pr),
                                             todict(li), float(max_error[m]))
            assert praw == raw[m] and pe == err[m] and ps == st[m], (ci, m, praw, raw[m])
        cases.append({
            "params": params,
            "product_offsets": batch.product_offsets.tolist(),
            "products": _records(batch.products),
            "link_offsets": batch.link_offsets.tolist(),
            "links": _records(batch.links),
            "initial": init.tolist(), "target": tgt.tolist(),
            "max_error": max_error.tolist(),
            "error": err.tolist(), "raw_error": raw.tolist(), "steps": st.tolist(),
        })
    return cases


def main():
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="reference checkout")
    src = reference_source(ap.parse_args().reference)
    if os.path.exists(src):
        with open(os.path.join(HERE, "reference_test_model.json"), "w") as f:
            json.dump(reference_test_model(src), f, indent=1)
    with open(os.path.join(HERE, "oracle_small.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": small_cases()}, f)
    print("fixtures written")


if __name__ == "__main__":
    main()
