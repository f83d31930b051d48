"""grn_evaluate_batch_noalloc, the entry point for callers that cannot
allocate device memory (their host owns the whole device memory budget, or
they must not touch the allocator mid-run).  On two calls in a row (the
scratch array it uses keeps the previous call's contents) it must give the
raw errors and step counts of grn_evaluate_batch / grn_run_packed on the same
inputs, agree with the FP64 oracle within the parity tolerance, leave the
device's free memory unchanged, and reject work that does not fit its fixed
scratch.

This file is collected last on purpose: a failure here leaves every other
test already run.  The buffers below are the test's own (the test may
allocate; the entry point does not)."""
import numpy as np
import pytest

import binding as oracle
import grn_b200 as grn
import synth

pytestmark = pytest.mark.gpu

RTOL = 1e-4
ATOL = 1e-7


def _device_inputs(torch, batch, init, tgt, max_error):
    return (torch.tensor(init, dtype=torch.float32, device="cuda").contiguous(),
            torch.tensor(tgt, dtype=torch.float32, device="cuda").contiguous(),
            torch.tensor(max_error, dtype=torch.float64, device="cuda"),
            torch.full((batch.n_models,), -1.0, dtype=torch.float64, device="cuda"),
            torch.zeros(batch.n_models, dtype=torch.int32, device="cuda"))


def _noalloc_call(params, batch, n_exp, bufs, stream):
    d_init, d_tgt, d_me, d_raw, d_steps = bufs
    grn.evaluate_batch_noalloc(params, n_exp, d_init.data_ptr(), d_tgt.data_ptr(), batch,
                               d_me.data_ptr(), d_raw.data_ptr(), d_steps.data_ptr(),
                               stream.cuda_stream)
    grn.evaluate_batch_noalloc_status(stream.cuda_stream)  # kernel error flag
    return d_raw.cpu().numpy(), d_steps.cpu().numpy()


def _close(a, b):
    return np.abs(a - b) <= ATOL + RTOL * np.abs(b)


@pytest.mark.parametrize("name,over", [
    ("small_32x32", dict(n_models=64, steps=200)),
    ("uneven_64x64", dict(n_models=96, steps=150)),      # genes 7-8 spill to scratch slots
    ("uneven_64x64", dict(n_models=12, steps=20, W=150, H=70)),
])
def test_noalloc_matches_evaluate_batch_twice(name, over):
    torch = pytest.importorskip("torch")
    params, batch, init, tgt = synth.workload(name, seed=31, **over)
    me = np.full(batch.n_models, 1000.0)
    me[::5] = 0.01  # some models abandoned after the first experiment
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        _, ref, _ = ev.evaluate_batch(batch, me)
        # Step counts through the device-buffer entry point.
        pk = ev.pack(batch)
        d_me = torch.tensor(me, dtype=torch.float64, device="cuda")
        d_raw = torch.zeros(batch.n_models, dtype=torch.float64, device="cuda")
        d_steps = torch.zeros(batch.n_models, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        pk.run(d_me.data_ptr(), d_raw.data_ptr(), d_steps.data_ptr())
        pk.status()
        ref_steps = d_steps.cpu().numpy()
        pk.free()
    _, o_raw, o_steps = oracle.evaluate_batch(params, init, tgt, batch, me)
    stream = torch.cuda.Stream()
    bufs = _device_inputs(torch, batch, init, tgt, me)
    torch.cuda.synchronize()
    free = []
    for _ in range(2):
        raw, steps = _noalloc_call(params, batch, init.shape[0], bufs, stream)
        free.append(torch.cuda.mem_get_info()[0])
        assert _close(raw, ref).all(), (np.where(~_close(raw, ref))[0], raw, ref)
        assert np.array_equal(steps, ref_steps)
        assert _close(raw, o_raw).all(), (np.where(~_close(raw, o_raw))[0], raw, o_raw)
        assert np.array_equal(steps, o_steps)
    # The second call reserved nothing the first had not.
    assert free[1] == free[0]


def test_noalloc_empty_batch_sets_up_and_allocates_nothing_more():
    torch = pytest.importorskip("torch")
    params, batch, init, tgt = synth.workload("small_32x32", seed=33, n_models=1, steps=5)
    empty = batch.subset([])
    d = torch.zeros(init.size + tgt.size + 16, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    # A call with no models loads the module (reserving the scratch array).
    grn.evaluate_batch_noalloc(params, 1, d.data_ptr(), d.data_ptr(), empty, 0, 0)
    bufs = _device_inputs(torch, batch, init, tgt, np.full(1, 1000.0))
    torch.cuda.synchronize()
    before = torch.cuda.mem_get_info()[0]
    stream = torch.cuda.Stream()
    _noalloc_call(params, batch, 1, bufs, stream)
    assert torch.cuda.mem_get_info()[0] == before


def test_noalloc_rejects_work_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    # One block's state slot for a 1024 x 1024 grid with 8 genes is larger
    # than the whole scratch array.
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=32, n_models=1, steps=1,
                                              W=1024, H=1024, genes=(8, 8))
    d_init = torch.zeros(init.shape, dtype=torch.float32, device="cuda")
    d_tgt = torch.zeros(tgt.shape, dtype=torch.float32, device="cuda")
    d_me = torch.full((1,), 1000.0, dtype=torch.float64, device="cuda")
    d_raw = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(grn.GrnError) as e:
        grn.evaluate_batch_noalloc(params, 1, d_init.data_ptr(), d_tgt.data_ptr(), batch,
                                   d_me.data_ptr(), d_raw.data_ptr())
    assert e.value.status == 6
    assert "GRN_NOALLOC_SCRATCH_BYTES" in str(e.value)
