"""grn_evaluate_batch_noalloc, the entry point for callers that cannot
allocate device memory (their host owns the whole device memory budget, or
they must not touch the allocator mid-run).  It must give the same errors as
grn_evaluate_batch on the same inputs, on two calls in a row (the scratch
array it uses keeps the previous call's contents), and reject work that does
not fit its fixed scratch.

This file is collected last on purpose: a failure here leaves every other
test already run.  The buffers below are the test's own (the test may
allocate; the entry point does not)."""
import numpy as np
import pytest

import grn_b200 as grn
import synth

pytestmark = pytest.mark.gpu

RTOL = 1e-4
ATOL = 1e-7


def _noalloc_raw(torch, params, batch, init, tgt, max_error, stream):
    d_init = torch.tensor(init, dtype=torch.float32, device="cuda").contiguous()
    d_tgt = torch.tensor(tgt, dtype=torch.float32, device="cuda").contiguous()
    d_me = torch.tensor(max_error, dtype=torch.float64, device="cuda")
    d_raw = torch.full((batch.n_models,), -1.0, dtype=torch.float64, device="cuda")
    d_steps = torch.zeros(batch.n_models, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    grn.evaluate_batch_noalloc(params, init.shape[0], d_init.data_ptr(), d_tgt.data_ptr(), batch,
                               d_me.data_ptr(), d_raw.data_ptr(), d_steps.data_ptr(),
                               stream.cuda_stream)
    stream.synchronize()
    return d_raw.cpu().numpy(), d_steps.cpu().numpy()


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
    stream = torch.cuda.Stream()
    for _ in range(2):
        raw, steps = _noalloc_raw(torch, params, batch, init, tgt, me, stream)
        ok = np.abs(raw - ref) <= ATOL + RTOL * np.abs(ref)
        assert ok.all(), (np.where(~ok)[0], raw[~ok], ref[~ok])
        assert (steps > 0).all()


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
