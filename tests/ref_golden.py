"""Loader of tests/golden/ref_pinned.json, the fixtures produced by the
reference's own CPU fitness path (oracle/_ref; generator
tests/golden/make_ref_golden.py)."""
import base64
import json
import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_pinned.json")


def _f64(s):
    return np.frombuffer(base64.b64decode(s), "<f8").copy()


def _u32(s):
    return np.frombuffer(base64.b64decode(s), "<u4").copy()


def load_cases():
    """Cases with decoded arrays: params, n_exp, input_px / target_px
    [n_exp][H][W] uint32, models (texts), max_error, errors (the reference's
    rounded errors) and runs (model, state [planes][H][W], change, steps,
    distance)."""
    with open(PATH) as f:
        data = json.load(f)
    cases = []
    for c in data["cases"]:
        p = c["params"]
        H, W = p["dim_y"], p["dim_x"]
        runs = []
        for r in c["runs"]:
            runs.append({"model": r["model"],
                         "state": _f64(r["state"]).reshape(r["planes"], H, W),
                         "change": float.fromhex(r["change"]), "steps": r["steps"],
                         "distance": float.fromhex(r["distance"])})
        cases.append({"name": c["name"], "params": p, "n_exp": c["n_exp"],
                      "input_px": _u32(c["input_px"]).reshape(c["n_exp"], H, W),
                      "target_px": _u32(c["target_px"]).reshape(c["n_exp"], H, W),
                      "models": c["models"],
                      "max_error": np.array([float.fromhex(x) for x in c["max_error"]]),
                      "errors": np.array([float.fromhex(x) for x in c["errors"]]),
                      "runs": runs})
    return cases
