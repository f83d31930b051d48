"""Python binding of the B200 GRN evaluator (ctypes over libgrn_b200.so).

The product is the C ABI in include/grn_gpu.h; this module is thin glue for
tests, benchmarks and Python callers.  It loads the in-tree library and
fails loudly if it is missing: there is no Python or CPU fallback.

Models travel as numpy structured arrays whose layout is the C structs
grn_product / grn_link.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgrn_b200.so")

PRODUCT_DTYPE = np.dtype([("label", "<i4"), ("reserved0", "<i4"), ("init", "<f8"),
                          ("lim", "<f8"), ("deg", "<f8"), ("dif", "<f8")])
LINK_DTYPE = np.dtype([("regulator", "<i4"), ("regulated", "<i4"), ("dis_const", "<f8"),
                       ("hill_coef", "<f8"), ("is_and", "<i4"), ("reserved0", "<i4")])
assert PRODUCT_DTYPE.itemsize == 40 and LINK_DTYPE.itemsize == 32

GRN_OK = 0
STATUS_NAMES = {0: "GRN_OK", 1: "GRN_ERR_INVALID_ARGUMENT", 2: "GRN_ERR_NO_DEVICE",
                3: "GRN_ERR_CUDA", 4: "GRN_ERR_OUT_OF_MEMORY", 5: "GRN_ERR_MODEL",
                6: "GRN_ERR_CAPACITY", 7: "GRN_ERR_NO_EXPERIMENTS", 8: "GRN_ERR_TIMEOUT",
                9: "GRN_ERR_NOT_FOUND", 10: "GRN_ERR_KERNEL"}
FITNESS_REF_LOGTHRESH = 0
FITNESS_MSE = 1
SCHEDULE_AUTO, SCHEDULE_FIXED_ITEMS, SCHEDULE_WALK_ITEMS, SCHEDULE_GLOBAL = 0, 1, 2, 3
SCHEDULE_CLUSTER = 4
SCHEDULE_STREAM = 5
SCHEDULE_STREAM2 = 6
TEST_WITHHOLD_BAND_COPY = 1
TEST_FAIL_DEVICE_ALLOC = 2
TEST_CORRUPT_RECORD = 4
SCORE_PARENT_ERROR, SCORE_PAIRED = 0, 1
SCHEDULE_NAMES = {0: "auto", 1: "fixed_items", 2: "walk_items", 3: "global", 4: "cluster",
                  5: "stream", 6: "stream2"}


class SimParams(ctypes.Structure):
    _fields_ = [("dim_x", ctypes.c_int32), ("dim_y", ctypes.c_int32),
                ("n_input_morphogens", ctypes.c_int32), ("n_target_morphogens", ctypes.c_int32),
                ("num_sim_steps", ctypes.c_int32), ("error_precision", ctypes.c_int32),
                ("fitness_kind", ctypes.c_int32), ("reserved0", ctypes.c_int32),
                ("dt", ctypes.c_double), ("min_conc", ctypes.c_double),
                ("min_conc_change", ctypes.c_double), ("dist_error_threshold", ctypes.c_double)]

    @classmethod
    def from_dict(cls, d):
        p = cls()
        for name, _ in cls._fields_:
            if name in d:
                setattr(p, name, d[name])
        return p


class EvolutionParams(ctypes.Structure):
    _fields_ = [("n_demes", ctypes.c_int32), ("deme_size", ctypes.c_int32),
                ("migration_period", ctypes.c_int32), ("n_max_products", ctypes.c_int32),
                ("n_max_links", ctypes.c_int32), ("n_host_threads", ctypes.c_int32),
                ("seed", ctypes.c_uint64)]


class GenerationStats(ctypes.Structure):
    _fields_ = [("generation", ctypes.c_int32), ("n_evaluated", ctypes.c_int32),
                ("best_error", ctypes.c_double), ("best_complexity", ctypes.c_int32),
                ("pareto_size", ctypes.c_int32), ("mean_error", ctypes.c_double),
                ("host_ms", ctypes.c_double), ("eval_ms", ctypes.c_double),
                ("migrated", ctypes.c_int32), ("n_screened", ctypes.c_int32),
                ("surrogate_ms", ctypes.c_double), ("surrogate_loss", ctypes.c_double),
                ("n_clones", ctypes.c_int32), ("n_audited", ctypes.c_int32),
                ("surrogate_rho", ctypes.c_double), ("surrogate_recall", ctypes.c_double),
                ("surrogate_improver_recall", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved0"}


class ModelBatchC(ctypes.Structure):
    _fields_ = [("n_models", ctypes.c_int32), ("reserved0", ctypes.c_int32),
                ("product_offsets", ctypes.c_void_p), ("products", ctypes.c_void_p),
                ("link_offsets", ctypes.c_void_p), ("links", ctypes.c_void_p)]


class EvalStats(ctypes.Structure):
    _fields_ = [("n_models", ctypes.c_int64), ("cell_updates", ctypes.c_int64),
                ("total_steps", ctypes.c_int64), ("kernel_ms", ctypes.c_double),
                ("pack_ms", ctypes.c_double), ("h2d_bytes", ctypes.c_int64),
                ("d2h_bytes", ctypes.c_int64), ("schedule", ctypes.c_int32),
                ("threads_per_block", ctypes.c_int32), ("blocks", ctypes.c_int32),
                ("cluster_size", ctypes.c_int32)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved0"}


class PackedInfo(ctypes.Structure):
    _fields_ = [("n_models", ctypes.c_int64), ("device_bytes", ctypes.c_int64),
                ("cell_update_bound", ctypes.c_int64), ("sfu_ops_per_step", ctypes.c_int64),
                ("max_genes", ctypes.c_int32), ("max_links", ctypes.c_int32),
                ("mean_genes", ctypes.c_double), ("mean_links", ctypes.c_double),
                ("mean_dif_genes", ctypes.c_double),
                ("alg_sfu_ops_per_step", ctypes.c_int64),
                ("alg_fp32_ops_per_step", ctypes.c_int64)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
# grn_error_calculator_fn
CALCULATOR_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ModelBatchC),
                                 ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double))
_SIGNATURES = {
    "grn_abi_version": ([], _I),
    "grn_status_str": ([_I], ctypes.c_char_p),
    "grn_last_error": ([_P], ctypes.c_char_p),
    "grn_round_error": ([_D, _D, _I], _D),
    "grn_create": ([ctypes.POINTER(_P), _I, ctypes.POINTER(SimParams)], _I),
    "grn_destroy": ([_P], _I),
    "grn_set_schedule": ([_P, _I, _I], _I),
    "grn_set_cluster_size": ([_P, _I], _I),
    "grn_set_autotune": ([_P, _I], _I),
    "grn_autotune_report": ([_P, _P, _I], _I),
    "grn_set_graphs": ([_P, _I], _I),
    "grn_set_host_threads": ([_P, _I], _I),
    "grn_set_test_hooks": ([_P, _I], _I),
    "grn_set_experiments": ([_P, _I, _P, _P], _I),
    "grn_set_experiments_rgb": ([_P, _I, _P, _P], _I),
    "grn_decode_rgb": ([_I, _I, _I, _P, _P], _I),
    "grn_evaluate": ([_P, _P, _I, _P, _I, _D, ctypes.POINTER(_D)], _I),
    "grn_evaluate_batch": ([_P, ctypes.POINTER(ModelBatchC), _P, _P, _P,
                            ctypes.POINTER(EvalStats)], _I),
    "grn_evaluate_states": ([_P, ctypes.POINTER(ModelBatchC), _P, _P, _P, _I], _I),
    "grn_submit": ([_P, _I, ctypes.POINTER(ModelBatchC), _P, _P, _P], _I),
    "grn_wait_any": ([_P, _I, ctypes.POINTER(_I)], _I),
    "grn_pack": ([_P, ctypes.POINTER(ModelBatchC), ctypes.POINTER(_P)], _I),
    "grn_packed_free": ([_P], _I),
    "grn_packed_get_info": ([_P, ctypes.POINTER(PackedInfo)], _I),
    "grn_run_packed": ([_P, _P, _P, _P, _P, _P], _I),
    "grn_run_packed_status": ([_P, _P], _I),
    "grn_describe_model": ([_P, _I, _P, _I, _I, ctypes.c_char_p, _I], _I),
    "grn_evolution_create": ([ctypes.POINTER(EvolutionParams), _I, _P, ctypes.POINTER(_P)], _I),
    "grn_evolution_create_cb": ([ctypes.POINTER(EvolutionParams), _I, CALCULATOR_FN, _P,
                                 ctypes.POINTER(_P)], _I),
    "grn_evolution_step": ([_P, ctypes.POINTER(GenerationStats)], _I),
    "grn_evolution_individual": ([_P, _I, _I, _P, _I, ctypes.POINTER(_I), _P, _I,
                                  ctypes.POINTER(_I), ctypes.POINTER(_D), ctypes.POINTER(_I)], _I),
    "grn_evolution_best": ([_P, ctypes.POINTER(_I), ctypes.POINTER(_I)], _I),
    "grn_evolution_destroy": ([_P], _I),
    "grn_encode_models": ([ctypes.POINTER(ModelBatchC), _I, _P], _I),
    "grn_model_costs": ([ctypes.POINTER(ModelBatchC), _I, _P], _I),
    "grn_trace_model": ([_P, _P, _I, _P, _I, _I, _I, _I, _I, _P, ctypes.POINTER(_I), _P], _I),
    "grn_render_cells": ([_P, _I, _I, _I, _I, _P], _I),
    "grn_render_concentrations": ([_P, _I, _I, _I, _D, _P], _I),
    "grn_write_ppm": ([ctypes.c_char_p, _P, _I, _I], _I),
    "grn_model_format": ([_P, _I, _P, _I, _I, _P, _I, ctypes.POINTER(_I)], _I),
    "grn_model_parse": ([ctypes.c_char_p, _P, _I, ctypes.POINTER(_I), _P, _I,
                         ctypes.POINTER(_I)], _I),
    "grn_evolution_set_individual": ([_P, _I, _I, _P, _I, _P, _I, _D], _I),
    "grn_evolution_set_generation": ([_P, _I], _I),
    "grn_evolution_checkpoint": ([_P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)], _I),
    "grn_evolution_restore": ([_P, _P, ctypes.c_size_t], _I),
    "grn_evolution_set_pipeline": ([_P, _I], _I),
    "grn_surrogate_create": ([_I, ctypes.c_uint64, _I, ctypes.POINTER(_P)], _I),
    "grn_surrogate_destroy": ([_P], _I),
    "grn_surrogate_add_data": ([_P, _P, _P, _I], _I),
    "grn_surrogate_data_count": ([_P], _I),
    "grn_surrogate_train": ([_P, _I, _I, ctypes.c_float, ctypes.POINTER(_D)], _I),
    "grn_surrogate_train_batches": ([_P, _I, _I, ctypes.c_float, ctypes.POINTER(_D)], _I),
    "grn_surrogate_predict": ([_P, _P, _I, _P], _I),
    "grn_surrogate_use_tcgen05": ([_P, _I], _I),
    "grn_surrogate_checkpoint": ([_P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)], _I),
    "grn_surrogate_restore": ([_P, _P, ctypes.c_size_t], _I),
    "grn_surrogate_params": ([_P, _P, _I], _I),
    "grn_surrogate_set_params": ([_P, _P, _I], _I),
    "grn_surrogate_gradients": ([_P, _P, _P, _I, _P, ctypes.POINTER(_D)], _I),
    "grn_evolution_set_skip_clones": ([_P, _I], _I),
    "grn_evolution_set_surrogate": ([_P, _P, _D, _I, _I, _I, ctypes.c_float], _I),
    "grn_evolution_set_surrogate_audit": ([_P, _I], _I),
    "grn_evolution_set_surrogate_score": ([_P, _I], _I),
    "grn_evaluate_batch_noalloc": ([ctypes.POINTER(SimParams), _I, _P, _P,
                                    ctypes.POINTER(ModelBatchC), _P, _P, _P, _P,
                                    ctypes.c_char_p, _I], _I),
    "grn_evaluate_batch_noalloc_status": ([_P, ctypes.c_char_p, _I], _I),
}

_lib = None


class GrnError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__("%s%s" % (STATUS_NAMES.get(status, str(status)), (": " + msg) if msg else ""))


def load_library(path=LIB_PATH):
    """Loads libgrn_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("libgrn_b200.so not built: run `python grn-gpu-performance_b200/build.py`"
                           " (there is no fallback path)")
    lib = ctypes.CDLL(path)
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class ModelBatch:
    """Models in genome form (the C struct grn_model_batch)."""

    def __init__(self, product_offsets, products, link_offsets, links):
        self.product_offsets = np.ascontiguousarray(product_offsets, dtype=np.int32)
        self.products = np.ascontiguousarray(products, dtype=PRODUCT_DTYPE)
        self.link_offsets = np.ascontiguousarray(link_offsets, dtype=np.int32)
        self.links = np.ascontiguousarray(links, dtype=LINK_DTYPE)
        assert len(self.product_offsets) == len(self.link_offsets)

    @property
    def n_models(self):
        return len(self.product_offsets) - 1

    @classmethod
    def from_models(cls, models):
        """models: list of (products array, links array)."""
        po, lo = [0], [0]
        for p, l in models:
            po.append(po[-1] + len(p))
            lo.append(lo[-1] + len(l))
        prods = np.concatenate([np.asarray(p, PRODUCT_DTYPE) for p, _ in models]) if models else \
            np.zeros(0, PRODUCT_DTYPE)
        links = np.concatenate([np.asarray(l, LINK_DTYPE) for _, l in models]) if models else \
            np.zeros(0, LINK_DTYPE)
        return cls(po, prods, lo, links)

    def model(self, i):
        return (self.products[self.product_offsets[i]:self.product_offsets[i + 1]],
                self.links[self.link_offsets[i]:self.link_offsets[i + 1]])

    def subset(self, idx):
        """The models at `idx`, in that order (vectorised gather)."""
        idx = np.asarray(idx, np.int64).reshape(-1)

        def gather(offsets, rows):
            start, end = offsets[idx].astype(np.int64), offsets[idx + 1].astype(np.int64)
            lens = end - start
            out_off = np.zeros(len(idx) + 1, np.int64)
            np.cumsum(lens, out=out_off[1:])
            # row r of the result comes from start[m] + (r - out_off[m]) of model m
            pos = np.arange(out_off[-1]) - np.repeat(out_off[:-1], lens) + np.repeat(start, lens)
            return out_off, rows[pos]
        po, prods = gather(self.product_offsets, self.products)
        lo, links = gather(self.link_offsets, self.links)
        return ModelBatch(po, prods, lo, links)

    def as_c(self):
        c = ModelBatchC()
        c.n_models = self.n_models
        c.product_offsets = _ptr(self.product_offsets)
        c.products = _ptr(self.products) if len(self.products) else None
        c.link_offsets = _ptr(self.link_offsets)
        c.links = _ptr(self.links) if len(self.links) else None
        return c


def round_error(raw, max_error, precision):
    return load_library().grn_round_error(float(raw), float(max_error), int(precision))


def decode_rgb(pixels, n_channels):
    """0xAARRGGBB pixels [H][W] -> planar channels [n][H][W] (reference y flip)."""
    lib = load_library()
    px = np.ascontiguousarray(pixels, dtype=np.uint32)
    h, w = px.shape
    out = np.zeros((n_channels, h, w), np.float64)
    _check(lib.grn_decode_rgb(w, h, n_channels, _ptr(px), _ptr(out)))
    return out


def describe_model(products, links, n_morphogens):
    """Text listing of the compiled program of one model (see grn_gpu.h)."""
    lib = load_library()
    p = np.ascontiguousarray(products, PRODUCT_DTYPE)
    l = np.ascontiguousarray(links, LINK_DTYPE)
    buf = ctypes.create_string_buffer(1 << 16)
    _check(lib.grn_describe_model(_ptr(p), len(p), _ptr(l) if len(l) else None, len(l),
                                  n_morphogens, buf, len(buf)))
    return buf.value.decode()


def _check(status, ctx=None):
    if status != GRN_OK:
        msg = ""
        if ctx:
            msg = load_library().grn_last_error(ctx).decode()
        raise GrnError(status, msg)


def evaluate_batch_noalloc(params, n_experiments, d_initial, d_target, batch, d_max_error,
                           d_raw_error, d_steps=None, stream=None):
    """grn_evaluate_batch_noalloc: device pointers (ints) for the experiments,
    max errors in and raw errors / steps out; `batch` is a host ModelBatch.
    Allocates no device memory; asynchronous on `stream` (cudaStream_t as int,
    None = legacy default stream)."""
    lib = load_library()
    p = SimParams.from_dict(params)
    cb = batch.as_c()
    buf = ctypes.create_string_buffer(512)
    st = lib.grn_evaluate_batch_noalloc(ctypes.byref(p), int(n_experiments),
                                        ctypes.c_void_p(d_initial), ctypes.c_void_p(d_target),
                                        ctypes.byref(cb), ctypes.c_void_p(d_max_error),
                                        ctypes.c_void_p(d_raw_error),
                                        ctypes.c_void_p(d_steps) if d_steps else None,
                                        ctypes.c_void_p(stream) if stream else None, buf, len(buf))
    if st != GRN_OK:
        raise GrnError(st, buf.value.decode())


def evaluate_batch_noalloc_status(stream=None):
    """grn_evaluate_batch_noalloc_status: waits for `stream` and raises
    GrnError (GRN_ERR_KERNEL) if the last no-allocation call's kernel flagged
    an error."""
    lib = load_library()
    buf = ctypes.create_string_buffer(512)
    st = lib.grn_evaluate_batch_noalloc_status(ctypes.c_void_p(stream) if stream else None, buf,
                                               len(buf))
    if st != GRN_OK:
        raise GrnError(st, buf.value.decode())


class Evaluator:
    """One grn_ctx: a device, a stream, the uploaded experiments."""

    def __init__(self, params, device=0):
        self.lib = load_library()
        self.params = dict(params)
        self._p = SimParams.from_dict(self.params)
        ctx = ctypes.c_void_p()
        _check(self.lib.grn_create(ctypes.byref(ctx), device, ctypes.byref(self._p)))
        self.ctx = ctx
        self._keep = {}

    def close(self):
        if self.ctx:
            self.lib.grn_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_schedule(self, schedule, threads=0, cluster_size=0):
        _check(self.lib.grn_set_schedule(self.ctx, schedule, threads), self.ctx)
        _check(self.lib.grn_set_cluster_size(self.ctx, cluster_size), self.ctx)

    def set_test_hooks(self, hooks):
        _check(self.lib.grn_set_test_hooks(self.ctx, int(hooks)), self.ctx)

    def set_graphs(self, enable=True):
        _check(self.lib.grn_set_graphs(self.ctx, int(bool(enable))), self.ctx)

    def autotune_report(self):
        buf = ctypes.create_string_buffer(8192)
        self.lib.grn_autotune_report(self.ctx, buf, len(buf))
        return buf.value.decode()

    def set_host_threads(self, n_threads):
        """Threads that compile a batch (0: the CPUs this process may use)."""
        _check(self.lib.grn_set_host_threads(self.ctx, int(n_threads)), self.ctx)

    def set_autotune(self, enable=True):
        _check(self.lib.grn_set_autotune(self.ctx, int(bool(enable))), self.ctx)

    def set_experiments(self, initial, target):
        """initial [n_exp][n_in][H][W], target [n_exp][n_target][H][W] (float64)."""
        ini = np.ascontiguousarray(initial, np.float64)
        tgt = np.ascontiguousarray(target, np.float64)
        _check(self.lib.grn_set_experiments(self.ctx, ini.shape[0], _ptr(ini), _ptr(tgt)), self.ctx)
        self._n_exp = ini.shape[0]

    def set_experiments_rgb(self, input_pixels, target_pixels):
        a = np.ascontiguousarray(input_pixels, np.uint32)
        b = np.ascontiguousarray(target_pixels, np.uint32)
        _check(self.lib.grn_set_experiments_rgb(self.ctx, a.shape[0], _ptr(a), _ptr(b)), self.ctx)
        self._n_exp = a.shape[0]

    def evaluate(self, products, links, max_error=1000.0):
        p = np.ascontiguousarray(products, PRODUCT_DTYPE)
        l = np.ascontiguousarray(links, LINK_DTYPE)
        out = ctypes.c_double()
        _check(self.lib.grn_evaluate(self.ctx, _ptr(p), len(p), _ptr(l) if len(l) else None,
                                     len(l), float(max_error), ctypes.byref(out)), self.ctx)
        return out.value

    def evaluate_batch(self, batch, max_error=None):
        """Returns (rounded errors, raw errors, stats dict)."""
        n = batch.n_models
        me = np.full(n, 1000.0) if max_error is None else \
            np.ascontiguousarray(np.broadcast_to(np.asarray(max_error, np.float64), (n,)))
        err = np.zeros(n, np.float64)
        raw = np.zeros(n, np.float64)
        st = EvalStats()
        cb = batch.as_c()
        _check(self.lib.grn_evaluate_batch(self.ctx, ctypes.byref(cb), _ptr(me), _ptr(err),
                                           _ptr(raw), ctypes.byref(st)), self.ctx)
        return err, raw, st.as_dict()

    def evaluate_states(self, batch, max_error=None, max_planes=16):
        """Returns (raw errors, final states [n][n_exp][max_planes][H][W] float32)."""
        n = batch.n_models
        me = np.full(n, 1000.0) if max_error is None else \
            np.ascontiguousarray(np.broadcast_to(np.asarray(max_error, np.float64), (n,)))
        raw = np.zeros(n, np.float64)
        n_exp = self._n_exp
        st = np.zeros((n, n_exp, max_planes, self.params["dim_y"], self.params["dim_x"]),
                      np.float32)
        cb = batch.as_c()
        _check(self.lib.grn_evaluate_states(self.ctx, ctypes.byref(cb), _ptr(me), _ptr(raw),
                                            _ptr(st), max_planes), self.ctx)
        return raw, st

    def submit(self, tag, batch, max_error=None):
        n = batch.n_models
        me = np.full(n, 1000.0) if max_error is None else \
            np.ascontiguousarray(np.broadcast_to(np.asarray(max_error, np.float64), (n,)))
        err = np.zeros(n, np.float64)
        raw = np.zeros(n, np.float64)
        cb = batch.as_c()
        _check(self.lib.grn_submit(self.ctx, int(tag), ctypes.byref(cb), _ptr(me), _ptr(err),
                                   _ptr(raw)), self.ctx)
        self._keep[int(tag)] = (err, raw, me, batch)
        return err, raw

    def wait_any(self, timeout_ms=-1):
        tag = ctypes.c_int()
        _check(self.lib.grn_wait_any(self.ctx, int(timeout_ms), ctypes.byref(tag)), self.ctx)
        err, raw, _, _ = self._keep.pop(tag.value)
        return tag.value, err, raw

    def trace(self, products, links, experiment=0, every=1, max_frames=64, max_planes=16):
        """grn_trace_model: (frames [n][planes][H][W], labels [planes])."""
        p = np.ascontiguousarray(products, PRODUCT_DTYPE)
        l = np.ascontiguousarray(links, LINK_DTYPE)
        H, W = self.params["dim_y"], self.params["dim_x"]
        frames = np.zeros((max_frames, max_planes, H, W), np.float32)
        labels = np.zeros(max_planes, np.int32)
        n = ctypes.c_int(0)
        _check(self.lib.grn_trace_model(self.ctx, _ptr(p) if len(p) else None, len(p),
                                        _ptr(l) if len(l) else None, len(l), experiment, every,
                                        max_frames, max_planes, _ptr(frames), ctypes.byref(n),
                                        _ptr(labels)), self.ctx)
        return frames[:n.value], labels

    def pack(self, batch):
        return Packed(self, batch)


class Packed:
    """A batch compiled and resident on the device (grn_pack)."""

    def __init__(self, ev, batch):
        self.ev = ev
        h = ctypes.c_void_p()
        cb = batch.as_c()
        _check(ev.lib.grn_pack(ev.ctx, ctypes.byref(cb), ctypes.byref(h)), ev.ctx)
        self.handle = h
        info = PackedInfo()
        _check(ev.lib.grn_packed_get_info(h, ctypes.byref(info)))
        self.info = {name: getattr(info, name) for name, _ in PackedInfo._fields_}

    def run(self, d_max_error, d_raw_error, d_steps=None, stream=None):
        """Device pointers (ints); stream is a cudaStream_t as int, or None for
        the evaluator's own stream (a handle of 0 also maps to it)."""
        _check(self.ev.lib.grn_run_packed(self.ev.ctx, self.handle, ctypes.c_void_p(d_max_error),
                                          ctypes.c_void_p(d_raw_error),
                                          ctypes.c_void_p(d_steps) if d_steps else None,
                                          ctypes.c_void_p(stream) if stream is not None else None),
               self.ev.ctx)

    def status(self, stream=None):
        """grn_run_packed_status: waits for `stream` and raises GrnError
        (GRN_ERR_KERNEL) if a launch flagged an error since the last call."""
        _check(self.ev.lib.grn_run_packed_status(
            self.ev.ctx, ctypes.c_void_p(stream) if stream is not None else None), self.ev.ctx)

    def free(self):
        if self.handle:
            self.ev.lib.grn_packed_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def batch_from_c(cb):
    """ModelBatch copy of a grn_model_batch passed to a calculator callback."""
    n = cb.contents.n_models
    po = np.ctypeslib.as_array(ctypes.cast(cb.contents.product_offsets,
                                           ctypes.POINTER(ctypes.c_int32)), (n + 1,)).copy()
    lo = np.ctypeslib.as_array(ctypes.cast(cb.contents.link_offsets,
                                           ctypes.POINTER(ctypes.c_int32)), (n + 1,)).copy()
    npr, nli = int(po[-1]), int(lo[-1])
    prods = np.frombuffer(ctypes.string_at(cb.contents.products, npr * PRODUCT_DTYPE.itemsize),
                          PRODUCT_DTYPE).copy() if npr else np.zeros(0, PRODUCT_DTYPE)
    links = np.frombuffer(ctypes.string_at(cb.contents.links, nli * LINK_DTYPE.itemsize),
                          LINK_DTYPE).copy() if nli else np.zeros(0, LINK_DTYPE)
    return ModelBatch(po, prods, lo, links)


class Evolution:
    """Island search (grn_evolution_*).  Pass an Evaluator to evaluate on the
    GPU, or a Python callable calculator(batch, max_error) -> errors."""

    def __init__(self, params, n_morphogens, evaluator=None, calculator=None):
        self.lib = load_library()
        self._p = EvolutionParams(**params)
        h = ctypes.c_void_p()
        if evaluator is not None:
            self._keep = evaluator
            _check(self.lib.grn_evolution_create(ctypes.byref(self._p), n_morphogens,
                                                 evaluator.ctx, ctypes.byref(h)))
        else:
            def trampoline(user, cb, max_error, error_out):
                try:
                    batch = batch_from_c(cb)
                    n = batch.n_models
                    me = np.ctypeslib.as_array(max_error, (n,)).copy()
                    out = np.asarray(calculator(batch, me), np.float64)
                    np.ctypeslib.as_array(error_out, (n,))[:] = out
                    return GRN_OK
                except Exception:  # surfaced as a status, not an unwind through C
                    import traceback
                    traceback.print_exc()
                    return 3
            self._cb = CALCULATOR_FN(trampoline)
            _check(self.lib.grn_evolution_create_cb(ctypes.byref(self._p), n_morphogens,
                                                    self._cb, None, ctypes.byref(h)))
        self.handle = h

    def step(self):
        st = GenerationStats()
        _check(self.lib.grn_evolution_step(self.handle, ctypes.byref(st)))
        return st.as_dict()

    def individual(self, deme, index):
        npr, nli, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        err = ctypes.c_double()
        _check(self.lib.grn_evolution_individual(self.handle, deme, index, None, 0,
                                                 ctypes.byref(npr), None, 0, ctypes.byref(nli),
                                                 ctypes.byref(err), ctypes.byref(c)))
        prods = np.zeros(npr.value, PRODUCT_DTYPE)
        links = np.zeros(nli.value, LINK_DTYPE)
        _check(self.lib.grn_evolution_individual(self.handle, deme, index, _ptr(prods),
                                                 npr.value, None, _ptr(links), nli.value, None,
                                                 None, None))
        return prods, links, err.value, c.value

    def set_individual(self, deme, index, products, links, error):
        p = np.ascontiguousarray(products, PRODUCT_DTYPE)
        l = np.ascontiguousarray(links, LINK_DTYPE)
        _check(self.lib.grn_evolution_set_individual(
            self.handle, deme, index, _ptr(p) if len(p) else None, len(p),
            _ptr(l) if len(l) else None, len(l), float(error)))

    def set_pipeline(self, enable=True):
        _check(self.lib.grn_evolution_set_pipeline(self.handle, int(bool(enable))))

    def set_generation(self, generation):
        _check(self.lib.grn_evolution_set_generation(self.handle, generation))

    def checkpoint(self):
        """The search's exact state as bytes (grn_evolution_checkpoint)."""
        n = ctypes.c_size_t()
        _check(self.lib.grn_evolution_checkpoint(self.handle, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        _check(self.lib.grn_evolution_checkpoint(self.handle, buf, n.value, ctypes.byref(n)))
        return buf.raw[:n.value]

    def restore(self, state):
        """Continues from a checkpoint of a search with the same parameters."""
        _check(self.lib.grn_evolution_restore(self.handle, state, len(state)))

    def set_skip_clones(self, enable=True):
        _check(self.lib.grn_evolution_set_skip_clones(self.handle, int(bool(enable))))

    def set_surrogate(self, surrogate, simulate_fraction=0.25, min_train_pairs=2048,
                      batches_per_generation=32, batch_size=512, lr=1e-3):
        self._sur = surrogate
        _check(self.lib.grn_evolution_set_surrogate(
            self.handle, surrogate.handle if surrogate else None, simulate_fraction,
            min_train_pairs, batches_per_generation, batch_size, lr))

    def set_surrogate_score(self, score):
        """grn_evolution_set_surrogate_score: SCORE_PARENT_ERROR or SCORE_PAIRED."""
        _check(self.lib.grn_evolution_set_surrogate_score(self.handle, int(score)))

    def set_surrogate_audit(self, enable=True):
        """grn_evolution_set_surrogate_audit: also simulate rejected children
        to measure the screen's recall (the search is unchanged)."""
        _check(self.lib.grn_evolution_set_surrogate_audit(self.handle, 1 if enable else 0))

    def best(self):
        d, i = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.grn_evolution_best(self.handle, ctypes.byref(d), ctypes.byref(i)))
        return d.value, i.value

    def close(self):
        if self.handle:
            self.lib.grn_evolution_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


N_FEATURES = 128
N_PARAMS = 164865


def render_cells(planes, n_morphogens):
    """grn_render_cells: [H][W][3] uint8 of planes [n][H][W]."""
    p = np.ascontiguousarray(planes, np.float32)
    out = np.zeros(p.shape[1:] + (3,), np.uint8)
    _check(load_library().grn_render_cells(_ptr(p), p.shape[0], n_morphogens, p.shape[2],
                                           p.shape[1], _ptr(out)))
    return out


def render_concentrations(planes, factor=1.0):
    """grn_render_concentrations: [H][W][3] uint8 of planes [n][H][W]."""
    p = np.ascontiguousarray(planes, np.float32)
    out = np.zeros(p.shape[1:] + (3,), np.uint8)
    _check(load_library().grn_render_concentrations(_ptr(p), p.shape[0], p.shape[2], p.shape[1],
                                                    factor, _ptr(out)))
    return out


def write_ppm(path, rgb):
    rgb = np.ascontiguousarray(rgb, np.uint8)
    _check(load_library().grn_write_ppm(str(path).encode(), _ptr(rgb), rgb.shape[1],
                                        rgb.shape[0]))


def format_model(products, links, precision=6):
    """grn_model_format: the reference's model string."""
    lib = load_library()
    p = np.ascontiguousarray(products, PRODUCT_DTYPE)
    l = np.ascontiguousarray(links, LINK_DTYPE)
    need = ctypes.c_int(0)
    args = (_ptr(p) if len(p) else None, len(p), _ptr(l) if len(l) else None, len(l), precision)
    st = lib.grn_model_format(*args, None, 0, ctypes.byref(need))
    if st not in (0, 6):  # GRN_ERR_CAPACITY just reports the size
        _check(st)
    buf = ctypes.create_string_buffer(need.value)
    _check(lib.grn_model_format(*args, buf, need.value, ctypes.byref(need)))
    return buf.value.decode()


def parse_model(text):
    """grn_model_parse: (products, links) arrays of a model string."""
    lib = load_library()
    raw = text.encode()
    npr, nli = ctypes.c_int(0), ctypes.c_int(0)
    st = lib.grn_model_parse(raw, None, 0, ctypes.byref(npr), None, 0, ctypes.byref(nli))
    if st not in (0, 6):
        _check(st)
    pr = np.zeros(npr.value, PRODUCT_DTYPE)
    li = np.zeros(nli.value, LINK_DTYPE)
    _check(lib.grn_model_parse(raw, _ptr(pr) if len(pr) else None, len(pr), ctypes.byref(npr),
                               _ptr(li) if len(li) else None, len(li), ctypes.byref(nli)))
    return pr, li


def model_costs(batch, n_morphogens):
    """grn_model_costs: relative work of one cell-step of each model."""
    out = np.zeros(batch.n_models, np.float64)
    cb = batch.as_c()
    _check(load_library().grn_model_costs(ctypes.byref(cb), n_morphogens, _ptr(out)))
    return out


def encode_models(batch, n_morphogens):
    """grn_encode_models: [n][128] float32 encodings (host only)."""
    out = np.zeros((batch.n_models, N_FEATURES), np.float32)
    cb = batch.as_c()
    _check(load_library().grn_encode_models(ctypes.byref(cb), n_morphogens, _ptr(out)))
    return out


class Surrogate:
    """The surrogate MLP (grn_surrogate_*)."""

    def __init__(self, device=0, seed=0, capacity=200000):
        self.lib = load_library()
        h = ctypes.c_void_p()
        _check(self.lib.grn_surrogate_create(device, seed, capacity, ctypes.byref(h)))
        self.handle = h

    def add_data(self, features, log_error):
        f = np.ascontiguousarray(features, np.float32)
        t = np.ascontiguousarray(log_error, np.float32)
        _check(self.lib.grn_surrogate_add_data(self.handle, _ptr(f), _ptr(t), len(t)))

    @property
    def data_count(self):
        return self.lib.grn_surrogate_data_count(self.handle)

    def train(self, epochs=1, batch_size=512, lr=1e-3):
        loss = ctypes.c_double()
        _check(self.lib.grn_surrogate_train(self.handle, epochs, batch_size, lr,
                                            ctypes.byref(loss)))
        return loss.value

    def use_tcgen05(self, enable=True):
        _check(self.lib.grn_surrogate_use_tcgen05(self.handle, int(bool(enable))))

    def checkpoint(self):
        """Weights, optimiser state and training set as bytes."""
        n = ctypes.c_size_t()
        _check(self.lib.grn_surrogate_checkpoint(self.handle, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        _check(self.lib.grn_surrogate_checkpoint(self.handle, buf, n.value, ctypes.byref(n)))
        return buf.raw[:n.value]

    def restore(self, state):
        _check(self.lib.grn_surrogate_restore(self.handle, state, len(state)))

    def train_batches(self, n_batches, batch_size=512, lr=1e-3):
        loss = ctypes.c_double()
        _check(self.lib.grn_surrogate_train_batches(self.handle, n_batches, batch_size, lr,
                                                    ctypes.byref(loss)))
        return loss.value

    def predict(self, features):
        f = np.ascontiguousarray(features, np.float32)
        out = np.zeros(len(f), np.float32)
        _check(self.lib.grn_surrogate_predict(self.handle, _ptr(f), len(f), _ptr(out)))
        return out

    def params(self):
        out = np.zeros(N_PARAMS, np.float32)
        _check(self.lib.grn_surrogate_params(self.handle, _ptr(out), N_PARAMS))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        _check(self.lib.grn_surrogate_set_params(self.handle, _ptr(p), N_PARAMS))

    def gradients(self, features, log_error):
        f = np.ascontiguousarray(features, np.float32)
        t = np.ascontiguousarray(log_error, np.float32)
        g = np.zeros(N_PARAMS, np.float32)
        loss = ctypes.c_double()
        _check(self.lib.grn_surrogate_gradients(self.handle, _ptr(f), _ptr(t), len(t), _ptr(g),
                                                ctypes.byref(loss)))
        return loss.value, g

    def close(self):
        if self.handle:
            self.lib.grn_surrogate_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
