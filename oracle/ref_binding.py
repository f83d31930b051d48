"""TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.

ctypes binding of oracle/_ref/libgrn_ref.so: the reference's own CPU fitness
path (EvaluatorMorphogens, Simulator, ModelSimulator, SimState, Model),
compiled from its unchanged sources by oracle/build_ref.py.  Used by tests/
to pin the FP64 restatement and the CUDA path to the reference, by
tests/golden/make_ref_golden.py to write reference-produced fixtures, and by
bench.py's CPU baseline and reference arm (the -O3 build).

Experiments go in as the reference stores them, 32-bit RGB images
(0xAARRGGBB, scan lines top to bottom; encode_rgb turns planar channels into
one), and models as the reference's text (model_text, 17 significant digits,
so every double arrives exactly).
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "grn-gpu-performance_b200"))
from grn_b200 import SimParams  # noqa: E402  (the grn_sim_params layout)

LIB_PATH = os.path.join(HERE, "_ref", "libgrn_ref.so")
LIB_O3_PATH = os.path.join(HERE, "_ref", "libgrn_ref_o3.so")
_libs = {}
_P = ctypes.c_void_p
_I = ctypes.c_int


def _cpu_runs_x86_64_v3():
    """The timed build targets x86-64-v3 (AVX2, FMA, BMI2)."""
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
        return all(" %s" % x in flags for x in ("avx2", "fma", "bmi2", "movbe"))
    except OSError:
        return False


def available(timed=False):
    if timed:
        return os.path.exists(LIB_O3_PATH) and _cpu_runs_x86_64_v3()
    return os.path.exists(LIB_PATH)


def build():
    sys.path.insert(0, HERE)
    import build_ref  # noqa: E402
    return build_ref.build()


def load(timed=False):
    """The parity build, or with timed=True the -O3 build (falls back to the
    parity build where the host CPU cannot run it)."""
    path = LIB_O3_PATH if timed and available(timed=True) else LIB_PATH
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        build()
    if not os.path.exists(path):
        raise RuntimeError("oracle/_ref is not built and the reference checkout is absent")
    lib = ctypes.CDLL(path)
    lib.grnr_assert_failures.restype = _I
    lib.grnr_ceil_s.argtypes = [ctypes.c_double, _I]
    lib.grnr_ceil_s.restype = ctypes.c_double
    lib.grnr_decode_rgb.argtypes = [_I, _I, _I, _P, _P]
    lib.grnr_decode_rgb.restype = _I
    lib.grnr_labels_in_use.argtypes = [ctypes.c_char_p, _I, _P, _I, ctypes.POINTER(_I)]
    lib.grnr_labels_in_use.restype = _I
    lib.grnr_format_model.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _I]
    lib.grnr_format_model.restype = _I
    lib.grnr_simulate.argtypes = [ctypes.POINTER(SimParams), _P, _P, ctypes.c_char_p, _I, _P, _I,
                                  ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_double)]
    lib.grnr_simulate.restype = _I
    lib.grnr_evaluate_batch.argtypes = [ctypes.POINTER(SimParams), _I, _P, _P, _I,
                                        ctypes.POINTER(ctypes.c_char_p), _P, _P, _I]
    lib.grnr_evaluate_batch.restype = _I
    _libs[path] = lib
    return lib


def _ok(st, what):
    if st != 0:
        raise RuntimeError("reference %s failed with status %d" % (what, st))


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def model_text(products, links):
    """The reference's model string (Src/Model/model.cpp:639-706) with 17
    significant digits."""
    p = ["%d %.17g %.17g %.17g %.17g" % (int(r["label"]), r["init"], r["lim"], r["deg"], r["dif"])
         for r in products]
    l = ["%d %d %.17g %.17g %d" % (int(r["regulator"]), int(r["regulated"]), r["dis_const"],
                                  r["hill_coef"], int(r["is_and"] != 0)) for r in links]
    return "(" + "|".join(p) + "*" + "|".join(l) + ")"


def batch_texts(batch):
    return [model_text(*batch.model(i)) for i in range(batch.n_models)]


def encode_rgb(planes):
    """Planar channels [n<=3][H][W] in [0, 1] -> RGB image [H][W] (0xFFRRGGBB):
    channel k in byte 2-k, rounded to the nearest 1/255, with the reference's
    y flip (image row j holds y = H-1-j, Src/Simulator/simstate.cpp:80-88)."""
    planes = np.asarray(planes, np.float64)
    n, h, w = planes.shape
    if n > 3:
        raise ValueError("an RGB image holds at most 3 channels")
    px = np.full((h, w), 0xFF000000, np.uint64)
    for k in range(n):
        b = np.rint(np.clip(planes[k], 0.0, 1.0) * 255.0).astype(np.uint64)
        px |= b[::-1] << np.uint64(16 - 8 * k)
    return px.astype(np.uint32)


def decode_rgb(pixels, n_channels):
    lib = load()
    px = np.ascontiguousarray(pixels, np.uint32)
    h, w = px.shape
    out = np.zeros((n_channels, h, w))
    _ok(lib.grnr_decode_rgb(w, h, n_channels, _ptr(px), _ptr(out)), "decode")
    return out


def ceil_s(n, digits):
    return load().grnr_ceil_s(float(n), int(digits))


def labels_in_use(products, links, n_morphogens):
    lib = load()
    out = np.zeros(256, np.int32)
    n = _I(0)
    _ok(lib.grnr_labels_in_use(model_text(products, links).encode(), n_morphogens, _ptr(out),
                               len(out), ctypes.byref(n)), "labels_in_use")
    return out[:n.value].copy()


def format_model(text):
    """Model::loadFromString then Model::toString (6 significant digits)."""
    lib = load()
    buf = ctypes.create_string_buffer(1 << 16)
    _ok(lib.grnr_format_model(text.encode(), buf, len(buf)), "format_model")
    return buf.value.decode()


def simulate(params, input_px, products, links, n_steps, target_px=None, max_planes=64):
    """Simulator run of one model on one experiment image.  Returns
    (state [n_products][H][W], change, steps, distance or None)."""
    lib = load()
    p = SimParams.from_dict(params)
    ipx = np.ascontiguousarray(input_px, np.uint32)
    tpx = None if target_px is None else np.ascontiguousarray(target_px, np.uint32)
    H, W = params["dim_y"], params["dim_x"]
    state = np.zeros((max_planes, H, W))
    n = _I(0)
    change = ctypes.c_double(0)
    steps = _I(0)
    dist = ctypes.c_double(0)
    _ok(lib.grnr_simulate(ctypes.byref(p), _ptr(ipx), None if tpx is None else _ptr(tpx),
                          model_text(products, links).encode(), n_steps, _ptr(state),
                          max_planes, ctypes.byref(n), ctypes.byref(change), ctypes.byref(steps),
                          None if tpx is None else ctypes.byref(dist)), "simulate")
    return state[:n.value].copy(), change.value, steps.value, (None if tpx is None else dist.value)


def evaluate_texts(params, input_px, target_px, texts, max_error=None, n_threads=1, timed=False):
    """EvaluatorMorphogens::evaluate of every model text: the reference's
    rounded errors (100 past max_error)."""
    lib = load(timed=timed)
    p = SimParams.from_dict(params)
    ipx = np.ascontiguousarray(input_px, np.uint32)
    tpx = np.ascontiguousarray(target_px, np.uint32)
    if ipx.ndim == 2:
        ipx, tpx = ipx[None], tpx[None]
    n = len(texts)
    me = np.full(n, 1000.0) if max_error is None else \
        np.ascontiguousarray(np.broadcast_to(np.asarray(max_error, np.float64), (n,)))
    arr = (ctypes.c_char_p * max(n, 1))(*[t.encode() for t in texts])
    out = np.zeros(n)
    _ok(lib.grnr_evaluate_batch(ctypes.byref(p), ipx.shape[0], _ptr(ipx), _ptr(tpx), n, arr,
                                _ptr(me), _ptr(out), int(n_threads)), "evaluate_batch")
    return out


def evaluate_batch(params, input_px, target_px, batch, max_error=None, n_threads=1, timed=False):
    return evaluate_texts(params, input_px, target_px, batch_texts(batch), max_error, n_threads,
                          timed)
