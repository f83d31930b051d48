"""TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.

ctypes binding of the FP64 CPU oracle (oracle/_build/libgrn_oracle.so),
used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg.  Builds the library on first use when the sources are present.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "grn-gpu-performance_b200"))
from grn_b200 import LINK_DTYPE, PRODUCT_DTYPE, ModelBatchC, SimParams  # noqa: E402

LIB_PATH = os.path.join(HERE, "_build", "libgrn_oracle.so")
_lib = None
_P = ctypes.c_void_p
_I = ctypes.c_int


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        sys.path.insert(0, HERE)
        import build as oracle_build  # noqa: E402
        oracle_build.build()
    lib = ctypes.CDLL(LIB_PATH)
    lib.grno_evaluate_batch.argtypes = [ctypes.POINTER(SimParams), _I, _P, _P,
                                        ctypes.POINTER(ModelBatchC), _P, _P, _P, _P, _I]
    lib.grno_evaluate_batch.restype = _I
    lib.grno_simulate.argtypes = [ctypes.POINTER(SimParams), _P, _P, _I, _P, _I, _I, _P, _I,
                                  ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(_I)]
    lib.grno_simulate.restype = _I
    lib.grno_labels_in_use.argtypes = [_P, _I, _P, _I, _I, _P, _I, ctypes.POINTER(_I)]
    lib.grno_labels_in_use.restype = _I
    lib.grno_dump_program.argtypes = [_P, _I, _P, _I, _I, ctypes.c_char_p, _I]
    lib.grno_dump_program.restype = _I
    lib.grno_ceil_s.argtypes = [ctypes.c_double, _I]
    lib.grno_ceil_s.restype = ctypes.c_double
    lib.grno_decode_rgb.argtypes = [_I, _I, _I, _P, _P]
    lib.grno_decode_rgb.restype = _I
    lib.grno_parse_model.argtypes = [ctypes.c_char_p, _P, _I, ctypes.POINTER(_I), _P, _I,
                                     ctypes.POINTER(_I)]
    lib.grno_parse_model.restype = _I
    lib.grno_format_model.argtypes = [_P, _I, _P, _I, ctypes.c_char_p, _I]
    lib.grno_format_model.restype = _I
    _lib = lib
    return lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None and a.size else None


def _ok(st, what):
    if st != 0:
        raise RuntimeError("oracle %s failed with status %d" % (what, st))


def evaluate_batch(params, initial, target, batch, max_error=None, n_threads=None):
    """Returns (rounded errors, raw errors, steps) for a grn_b200.ModelBatch."""
    lib = load()
    p = SimParams.from_dict(params)
    ini = np.ascontiguousarray(initial, np.float64)
    tgt = np.ascontiguousarray(target, np.float64)
    n = batch.n_models
    me = np.full(n, 1000.0) if max_error is None else \
        np.ascontiguousarray(np.broadcast_to(np.asarray(max_error, np.float64), (n,)))
    err = np.zeros(n)
    raw = np.zeros(n)
    steps = np.zeros(n, np.int32)
    cb = batch.as_c()
    nt = n_threads or os.cpu_count() or 1
    _ok(lib.grno_evaluate_batch(ctypes.byref(p), ini.shape[0], _ptr(ini), _ptr(tgt),
                                ctypes.byref(cb), _ptr(me), _ptr(err), _ptr(raw), _ptr(steps),
                                int(nt)), "evaluate_batch")
    return err, raw, steps


def simulate(params, initial_one, products, links, n_steps, max_planes=64):
    """Final state [n_products][H][W], change, steps of one experiment."""
    lib = load()
    p = SimParams.from_dict(params)
    ini = np.ascontiguousarray(initial_one, np.float64)
    pr = np.ascontiguousarray(products, PRODUCT_DTYPE)
    li = np.ascontiguousarray(links, LINK_DTYPE)
    out = np.zeros((max_planes, params["dim_y"], params["dim_x"]))
    npl, steps = _I(), _I()
    ch = ctypes.c_double()
    _ok(lib.grno_simulate(ctypes.byref(p), _ptr(ini), _ptr(pr), len(pr), _ptr(li), len(li),
                          int(n_steps), _ptr(out), max_planes, ctypes.byref(npl),
                          ctypes.byref(ch), ctypes.byref(steps)), "simulate")
    return out[:npl.value].copy(), ch.value, steps.value


def labels_in_use(products, links, n_morph):
    lib = load()
    pr = np.ascontiguousarray(products, PRODUCT_DTYPE)
    li = np.ascontiguousarray(links, LINK_DTYPE)
    out = np.zeros(1024, np.int32)
    n = _I()
    _ok(lib.grno_labels_in_use(_ptr(pr), len(pr), _ptr(li), len(li), n_morph, _ptr(out), 1024,
                               ctypes.byref(n)), "labels_in_use")
    return out[:n.value].tolist()


def dump_program(products, links, n_morph):
    lib = load()
    pr = np.ascontiguousarray(products, PRODUCT_DTYPE)
    li = np.ascontiguousarray(links, LINK_DTYPE)
    buf = ctypes.create_string_buffer(1 << 16)
    _ok(lib.grno_dump_program(_ptr(pr), len(pr), _ptr(li), len(li), n_morph, buf, len(buf)),
        "dump_program")
    return buf.value.decode()


def ceil_s(x, d):
    return load().grno_ceil_s(float(x), int(d))


def decode_rgb(pixels, n_channels):
    lib = load()
    px = np.ascontiguousarray(pixels, np.uint32)
    h, w = px.shape
    out = np.zeros((n_channels, h, w))
    _ok(lib.grno_decode_rgb(w, h, n_channels, _ptr(px), _ptr(out)), "decode_rgb")
    return out


def parse_model(text):
    lib = load()
    pr = np.zeros(4096, PRODUCT_DTYPE)
    li = np.zeros(16384, LINK_DTYPE)
    npr, nli = _I(), _I()
    _ok(lib.grno_parse_model(text.encode(), _ptr(pr), len(pr), ctypes.byref(npr), _ptr(li),
                             len(li), ctypes.byref(nli)), "parse_model")
    return pr[:npr.value].copy(), li[:nli.value].copy()


def format_model(products, links):
    lib = load()
    pr = np.ascontiguousarray(products, PRODUCT_DTYPE)
    li = np.ascontiguousarray(links, LINK_DTYPE)
    buf = ctypes.create_string_buffer(1 << 20)
    _ok(lib.grno_format_model(_ptr(pr), len(pr), _ptr(li), len(li), buf, len(buf)),
        "format_model")
    return buf.value.decode()
