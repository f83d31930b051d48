"""Cases run through both the normal and the bounds-checked library
(lib/libgrn_b200_checked.so) by tests/test_bounds_checked.py: every kernel
schedule on small grids -- fixed and walking items, all-global, streaming,
cluster-split with shared-memory and global-slot genes, trace frames, the
no-allocation entry's scratch layout -- including ragged widths, short last
bands, 16-gene models and the exact path.

Run as a script it loads the library named on the command line and writes
the results to an .npz: python tests/bounds_cases.py LIB OUT.npz
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "grn-gpu-performance_b200"))

import grn_b200 as grn  # noqa: E402
import synth  # noqa: E402


def _states(out, name, params, batch, init, tgt, schedule, cluster=0, planes=16):
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        ev.set_schedule(schedule, cluster_size=cluster)
        raw, states = ev.evaluate_states(batch, max_planes=planes)
        _, raw_b, st = ev.evaluate_batch(batch)
    out[name + "/raw"] = raw
    out[name + "/raw_batch"] = raw_b
    out[name + "/states"] = states
    out[name + "/schedule"] = np.array([st["schedule"], st["cluster_size"]])


def run_cases():
    out = {}
    # One CTA per model, state on chip / spilled to global slots.
    for W, H in ((36, 20), (13, 5), (64, 64)):
        params, batch, init, tgt = synth.workload("uneven_64x64", seed=3, n_models=20, steps=40,
                                                  W=W, H=H, n_exp=2)
        batch.links["dis_const"][0] = 0.0  # model 0 takes the exact path
        for sched in (grn.SCHEDULE_FIXED_ITEMS, grn.SCHEDULE_WALK_ITEMS, grn.SCHEDULE_GLOBAL):
            _states(out, "grid%dx%d_s%d" % (W, H, sched), params, batch, init, tgt, sched,
                    planes=8)
    # Degenerate grids: one cell, one column, one row, one float4 group per
    # row (the zero group that ends it), every schedule including streaming.
    for W, H in ((1, 1), (1, 37), (53, 1), (4, 9)):
        params, batch, init, tgt = synth.workload("uneven_64x64", seed=9, n_models=6, steps=12,
                                                  W=W, H=H)
        for sched in (grn.SCHEDULE_FIXED_ITEMS, grn.SCHEDULE_WALK_ITEMS, grn.SCHEDULE_GLOBAL,
                      grn.SCHEDULE_STREAM):
            _states(out, "edge%dx%d_s%d" % (W, H, sched), params, batch, init, tgt, sched,
                    planes=8)
    # Clusters whose bands are one row high (halo rows only) and a short last band.
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=10, n_models=4, steps=12,
                                              W=17, H=2)
    _states(out, "cluster17x2_c2", params, batch, init, tgt, grn.SCHEDULE_CLUSTER, cluster=2,
            planes=8)
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=11, n_models=4, steps=12,
                                              W=9, H=7)
    _states(out, "cluster9x7_c4", params, batch, init, tgt, grn.SCHEDULE_CLUSTER, cluster=4,
            planes=8)
    # 100x100 walking: 2 genes on chip, the rest in global slots.
    params, batch, init, tgt = synth.workload("islands_100x100", seed=4, n_models=10, steps=20)
    _states(out, "islands_walk", params, batch, init, tgt, grn.SCHEDULE_WALK_ITEMS, planes=8)
    # Streaming: ragged width with a short last band, 256 x 256, 16-gene models.
    for W, H, steps, genes in ((30, 37, 15, (2, 8)), (256, 256, 6, (8, 8)),
                               (250, 90, 6, (8, 16))):
        params, batch, init, tgt = synth.workload("uneven_64x64", seed=5, n_models=6,
                                                  steps=steps, W=W, H=H, genes=genes,
                                                  links=(1, 24), n_exp=2)
        batch.links["dis_const"][0] = 0.0
        _states(out, "stream%dx%d" % (W, H), params, batch, init, tgt, grn.SCHEDULE_STREAM)
        _states(out, "stream2_%dx%d" % (W, H), params, batch, init, tgt, grn.SCHEDULE_STREAM2)
    # Cluster-split: halo rows through distributed shared memory and, at
    # 256 x 256, through neighbouring blocks' global slots.
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=6, n_models=8, steps=20,
                                              W=30, H=37, n_exp=2)
    for c in (2, 4, 8):
        _states(out, "cluster30x37_c%d" % c, params, batch, init, tgt, grn.SCHEDULE_CLUSTER,
                cluster=c, planes=8)
    params, batch, init, tgt = synth.workload("large_256x256", seed=7, n_models=3, steps=8)
    for c in (8, 16):
        _states(out, "cluster256_c%d" % c, params, batch, init, tgt, grn.SCHEDULE_CLUSTER,
                cluster=c, planes=8)
    # Trace frames (their own kernel variant).
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=8, n_models=2, steps=30,
                                              W=41, H=23)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        prods, links = batch.model(1)
        frames, labels = ev.trace(prods, links, every=7, max_frames=8, max_planes=8)
    out["trace/frames"] = frames
    out["trace/labels"] = labels
    # The no-allocation entry: records, offsets and the state slots of the
    # genes that spill (7-8 gene models at 64 x 64) in its fixed scratch
    # array, with its own slot layout and a capped block count.
    import torch
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=12, n_models=24, steps=15,
                                              genes=(7, 8))
    d_init = torch.tensor(init, dtype=torch.float32, device="cuda")
    d_tgt = torch.tensor(tgt, dtype=torch.float32, device="cuda")
    d_me = torch.full((batch.n_models,), 1000.0, dtype=torch.float64, device="cuda")
    d_raw = torch.zeros(batch.n_models, dtype=torch.float64, device="cuda")
    d_steps = torch.zeros(batch.n_models, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    grn.evaluate_batch_noalloc(params, init.shape[0], d_init.data_ptr(), d_tgt.data_ptr(), batch,
                               d_me.data_ptr(), d_raw.data_ptr(), d_steps.data_ptr())
    grn.evaluate_batch_noalloc_status()  # raises on a bounds-check flag
    out["noalloc/raw"] = d_raw.cpu().numpy()
    out["noalloc/steps"] = d_steps.cpu().numpy()
    return out


if __name__ == "__main__":
    grn.load_library(sys.argv[1])
    np.savez(sys.argv[2], **run_cases())
    print("ok")
