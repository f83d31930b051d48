"""Rank bodies of the multi-process (gloo, CPU) tests of sharded.py.  Each
runs in a spawned process: it sets up its import path, joins the process
group on 127.0.0.1 and writes its result to a .npz file."""
import os
import sys


def _setup(root, rank, world, port):
    for p in (os.path.join(root, "grn-gpu-performance_b200"), os.path.join(root, "oracle"),
              os.path.join(root, "tests"), root):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    return dist


class OracleEvaluator:
    """evaluate_batch through the FP64 oracle (test stand-in for a GPU)."""

    def __init__(self, sim, init, tgt):
        self.sim, self.init, self.tgt = sim, init, tgt
        self.seen = 0

    def evaluate_batch(self, batch, max_error=None):
        import binding as oracle
        self.seen += batch.n_models
        err, raw, steps = oracle.evaluate_batch(self.sim, self.init, self.tgt, batch, max_error,
                                                n_threads=1)
        return err, raw, {"n_models": batch.n_models}


def sharded_eval(rank, world, port, root, out):
    dist = _setup(root, rank, world, port)
    import numpy as np
    import synth
    import sharded
    params, batch, init, tgt = synth.workload("small_32x32", seed=21, n_models=23, steps=40,
                                              W=12, H=10)
    ev = OracleEvaluator(params, init, tgt)
    me = np.linspace(0.05, 1000.0, batch.n_models)
    sh = sharded.ShardedEvaluator(ev, params["n_input_morphogens"] +
                                  params["n_target_morphogens"])
    err, raw, _ = sh.evaluate_batch(batch, me)
    np.savez(os.path.join(out, "rank%d.npz" % rank), err=err, raw=raw, seen=ev.seen)
    dist.barrier()
    dist.destroy_process_group()


def island_shards(rank, world, port, root, out):
    dist = _setup(root, rank, world, port)
    import numpy as np
    import grn_b200 as grn
    import synth
    import sharded
    sim = dict(dim_x=8, dim_y=8, n_input_morphogens=1, n_target_morphogens=1, num_sim_steps=20,
               error_precision=6, fitness_kind=0, dt=0.1, min_conc=0.0, min_conc_change=1e-3,
               dist_error_threshold=0.05)
    wl = dict(synth.WORKLOADS["uneven_64x64"], W=8, H=8, n_exp=1)
    init, tgt = synth.experiments(wl, 3)
    ev = OracleEvaluator(sim, init, tgt)
    evo = grn.Evolution(dict(n_demes=2, deme_size=8, migration_period=0, n_max_products=5,
                             n_max_links=8, n_host_threads=1, seed=100 + rank), 2,
                        calculator=lambda b, me: ev.evaluate_batch(b, me)[0])
    isl = sharded.IslandShards(evo, 2, 8, period=2, seed=9)
    stats = [isl.step() for _ in range(4)]
    ex = isl.last_exchange
    after = [evo.individual(ex["deme"], i) for i in ex["slots"]]
    import pickle
    with open(os.path.join(out, "rank%d.pkl" % rank), "wb") as f:
        pickle.dump({"stats": stats, "after": after, "exchange": ex}, f)
    evo.close()
    dist.barrier()
    dist.destroy_process_group()


def cuda_one_rank(rank, world, port, root, out):
    """ShardedEvaluator and IslandShards over the CUDA evaluator on a
    one-rank NCCL process group (the same code paths a multi-GPU run takes:
    deal, shard evaluation, all_gather; deme steps and the global-best
    all_reduce)."""
    for p in (os.path.join(root, "grn-gpu-performance_b200"), os.path.join(root, "oracle"),
              os.path.join(root, "tests"), root):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    import grn_b200 as grn
    import sharded
    import synth
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", 0))
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=41, n_models=37, steps=120)
    me = np.full(batch.n_models, 1000.0)
    me[::6] = 0.05
    n_morph = params["n_input_morphogens"] + params["n_target_morphogens"]
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        err_s, raw_s, _ = sharded.ShardedEvaluator(ev, n_morph).evaluate_batch(batch, me)
        err_p, raw_p, _ = ev.evaluate_batch(batch, me)
        evo_p = dict(n_demes=4, deme_size=16, migration_period=2, n_max_products=6,
                     n_max_links=10, n_host_threads=2, seed=5)
        evo = grn.Evolution(evo_p, n_morph, evaluator=ev)
        isl = sharded.IslandShards(evo, 4, 16, period=2, seed=3)
        best_sharded = [isl.step()["global_best_error"] for _ in range(4)]
        evo.close()
        evo = grn.Evolution(evo_p, n_morph, evaluator=ev)
        best_plain = [evo.step()["best_error"] for _ in range(4)]
        evo.close()
    np.savez(os.path.join(out, "rank%d.npz" % rank), err_s=err_s, raw_s=raw_s, err_p=err_p,
             raw_p=raw_p, best_sharded=best_sharded, best_plain=best_plain)
    dist.barrier()
    dist.destroy_process_group()


def sharded_rank_dies(rank, world, port, root, out):
    """Rank 1 dies between steps (after a completed gather, before the
    next); rank 0's next gather must end in an error, not wait for good."""
    import datetime
    import time
    dist = _setup(root, rank, world, port)
    import numpy as np
    import synth
    import sharded
    params, batch, init, tgt = synth.workload("small_32x32", seed=22, n_models=9, steps=20,
                                              W=8, H=8)
    ev = OracleEvaluator(params, init, tgt)
    sh = sharded.ShardedEvaluator(ev, params["n_input_morphogens"] +
                                  params["n_target_morphogens"])
    err, raw, _ = sh.evaluate_batch(batch)  # one step that both ranks finish
    if rank == 1:
        os._exit(3)  # no clean-up: the process is gone
    t0 = time.monotonic()
    try:
        sh.evaluate_batch(batch)
        outcome = "returned"
    except Exception as e:  # the backend's error for a lost peer
        outcome = "raised " + type(e).__name__
    np.savez(os.path.join(out, "rank0.npz"), outcome=outcome, seconds=time.monotonic() - t0,
             first=raw)
