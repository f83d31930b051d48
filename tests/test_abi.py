"""CPU tests of the C-ABI library: it loads, exports every function that
include/grn_gpu.h declares, refuses to run without a device, and its host
logic (model compilation, rounding, image decode) matches the oracle."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

import binding as oracle
import grn_b200 as grn
import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "grn_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("typedef"))
    return sorted(set(re.findall(r"^[A-Za-z_][\w \*]*?\b(grn_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    for want in ("grn_create", "grn_destroy", "grn_set_experiments", "grn_evaluate",
                 "grn_evaluate_batch", "grn_submit", "grn_wait_any", "grn_pack",
                 "grn_run_packed"):
        assert want in names


def test_library_exports_every_declared_symbol(built_libs):
    out = subprocess.run(["nm", "-D", "--defined-only", grn.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    lib = grn.load_library()
    for n in declared_functions():
        assert getattr(lib, n) is not None


def test_abi_version(built_libs):
    assert grn.load_library().grn_abi_version() == 2


@pytest.mark.skipif(__import__("conftest").HAS_GPU, reason="checks the no-device path")
def test_create_without_device_fails_loudly(built_libs):
    params, _, _, _ = synth.workload("small_32x32", n_models=1)
    with pytest.raises(grn.GrnError) as e:
        grn.Evaluator(params)
    assert e.value.status == 2  # GRN_ERR_NO_DEVICE: no CPU fallback


def test_create_rejects_bad_params(built_libs):
    params, _, _, _ = synth.workload("small_32x32", n_models=1)
    params["dim_x"] = 0
    with pytest.raises(grn.GrnError) as e:
        grn.Evaluator(params)
    assert e.value.status == 1


def test_round_error_matches_reference_rounding(built_libs):
    rng = np.random.default_rng(1)
    for x in np.concatenate([rng.random(200) * 10.0 ** rng.integers(-6, 2, 200), [0.0]]):
        for d in (3, 6, 8):
            assert grn.round_error(x, 1000.0, d) == oracle.ceil_s(x, d)
    assert grn.round_error(0.5, 0.4, 6) == 100.0   # > maxError -> 100
    assert grn.round_error(0.4, 0.4, 6) == oracle.ceil_s(0.4, 6)


def test_decode_rgb_matches_oracle(built_libs):
    rng = np.random.default_rng(2)
    px = rng.integers(0, 2 ** 32, size=(7, 5), dtype=np.uint64).astype(np.uint32)
    for n in (1, 2, 3):
        assert np.array_equal(grn.decode_rgb(px, n), oracle.decode_rgb(px, n))


def _oracle_gene_ops(dump, n_genes):
    """Per gene: list of (kind, regulator index, K, n) Hill links in program
    order, and counts of OR / AND combine ops; zero genes get None."""
    genes = {p: {"hill": [], "or": 0, "and": 0, "zero": False} for p in range(n_genes)}
    pending = None
    for line in dump.splitlines():
        f = line.split()
        if f[0] in ("hillact", "hillrep"):
            to, frm, K, n = int(f[1]), int(f[2]), float(f[3]), float(f[4])
            if to >= 0:
                genes[to]["hill"].append((f[0], frm, K, n))
            else:
                pending = (f[0], frm, K, n)
        elif f[0] in ("or", "and"):
            p = int(f[1])
            genes[p]["hill"].append(pending)
            genes[p][f[0]] += 1
        elif f[0] == "zero":
            genes[int(f[1])]["zero"] = True
    return genes


def _check_compile(pr, li, n_morph):
    desc = grn.describe_model(pr, li, n_morph).splitlines()
    labels = oracle.labels_in_use(pr, li, n_morph)
    ops = _oracle_gene_ops(oracle.dump_program(pr, li, n_morph), len(labels))
    head = desc[0].split()
    assert int(head[2]) == len(labels)
    gene_lines = [l.split() for l in desc if l.startswith("gene ")]
    link_lines = [l.split() for l in desc if l.startswith("link ")]
    assert len(gene_lines) == len(labels)
    for g in gene_lines:
        i, lab = int(g[1]), int(g[3])
        n_or, n_and = int(g[11]), int(g[13])
        assert lab == labels[i]
        want = ops[i]
        if want["zero"]:
            assert n_or + n_and == 0
            continue
        hills = want["hill"]
        assert n_or + n_and == len(hills)
        if n_or >= 1:
            assert want["or"] == n_or - 1 and want["and"] == n_and
        else:
            assert want["or"] == 0 and want["and"] == n_and - 1
        mine = [l for l in link_lines if int(l[1]) == i]
        for (kind, frm, K, n), l in zip(hills, mine):
            slot, a, b = int(l[3]), float(l[5]), float(l[7])
            if n == 0:
                assert slot == 255 and a == 0 and b == 0
                continue
            assert slot == frm
            lk = np.log2(K) if K > 0 else (-np.inf if K == 0 else np.nan)
            wa, wb = (-n, n * lk) if kind == "hillact" else (n, -n * lk)
            assert np.float32(a) == np.float32(wa)
            if np.isfinite(wb):
                assert np.float32(b) == np.float32(wb)
            else:
                assert (np.isnan(b) and np.isnan(wb)) or b == wb


def test_host_compiler_matches_oracle_program_reference_model(built_libs):
    with open(os.path.join(ROOT, "tests", "golden", "reference_test_model.json")) as f:
        pr, li = oracle.parse_model(json.load(f)["model"])
    for n_morph in (1, 2):  # labels 0 and 1 are its morphogens
        _check_compile(pr, li, n_morph)


def test_host_compiler_matches_oracle_program_random(built_libs):
    rng = np.random.default_rng(11)
    for t in range(60):
        G = int(rng.integers(2, 9))
        pr, li = synth.random_model(rng, G, int(rng.integers(0, 24)), 2)
        if t % 6 == 0 and len(li):
            li["hill_coef"][int(rng.integers(len(li)))] = 0.0
        if t % 9 == 0 and len(li):
            li["dis_const"][0] = 0.0
        _check_compile(pr, li, 2)


def test_host_compiler_rejects_missing_product(built_libs):
    pr = np.zeros(1, grn.PRODUCT_DTYPE)
    pr["label"] = 0
    li = np.zeros(1, grn.LINK_DTYPE)
    li[0] = (7, 0, 0.5, 2.0, 0, 0)  # regulator 7 is in use but has no product
    with pytest.raises(grn.GrnError) as e:
        grn.describe_model(pr, li, 1)
    assert e.value.status == 5


def test_host_compiler_capacity(built_libs):
    G = 20
    pr = np.zeros(G, grn.PRODUCT_DTYPE)
    pr["label"] = np.arange(G)
    li = np.zeros(G - 1, grn.LINK_DTYPE)
    li["regulator"] = np.arange(1, G)
    li["regulated"] = 0
    li["dis_const"] = 0.5
    li["hill_coef"] = 2.0
    with pytest.raises(grn.GrnError) as e:
        grn.describe_model(pr, li, 1)
    assert e.value.status == 6
