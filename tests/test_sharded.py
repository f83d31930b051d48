"""Multi-GPU sharding logic (sharded.py) run as 2 gloo ranks on the CPU,
with the FP64 oracle standing in for each rank's GPU evaluator."""
import os
import pickle
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import binding as oracle
import dist_workers
import sharded
import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_deal_balances_count_and_cost():
    rng = np.random.default_rng(0)
    costs = rng.lognormal(size=1001)
    for world in (1, 2, 3, 8):
        ranks = sharded.deal(costs, world)
        counts = np.bincount(ranks, minlength=world)
        assert counts.max() - counts.min() <= 1
        per = np.array([costs[ranks == r].sum() for r in range(world)])
        assert per.max() - per.min() <= costs.max()
    assert (sharded.deal([3.0, 1.0, 2.0, 5.0], 2) == [1, 0, 1, 0]).all()


def test_sharded_evaluator_matches_one_process(built_libs, tmp_path):
    mp.spawn(dist_workers.sharded_eval, args=(2, _port(), ROOT, str(tmp_path)), nprocs=2,
             join=True)
    r0 = np.load(tmp_path / "rank0.npz")
    r1 = np.load(tmp_path / "rank1.npz")
    params, batch, init, tgt = synth.workload("small_32x32", seed=21, n_models=23, steps=40,
                                              W=12, H=10)
    me = np.linspace(0.05, 1000.0, batch.n_models)
    err, raw, _ = oracle.evaluate_batch(params, init, tgt, batch, me, n_threads=2)
    for r in (r0, r1):
        np.testing.assert_array_equal(r["err"], err)
        np.testing.assert_array_equal(r["raw"], raw)
    assert int(r0["seen"]) + int(r1["seen"]) == 23 and abs(int(r0["seen"]) - int(r1["seen"])) <= 1


def test_island_shards_migrate_across_ranks(built_libs, tmp_path):
    mp.spawn(dist_workers.island_shards, args=(2, _port(), ROOT, str(tmp_path)), nprocs=2,
             join=True)
    res = [pickle.load(open(tmp_path / ("rank%d.pkl" % r), "rb")) for r in (0, 1)]
    for r in (0, 1):
        st = res[r]["stats"]
        assert [s.get("migrated_ranks", 0) for s in st] == [0, 1, 0, 1]
        for s in st:
            assert s["global_best_error"] <= s["best_error"]
    # the global best is the min over both ranks, identical on both
    for g in range(4):
        gb = [res[r]["stats"][g]["global_best_error"] for r in (0, 1)]
        assert gb[0] == gb[1] == min(res[r]["stats"][g]["best_error"] for r in (0, 1))

    # the last migration swapped half a deme: what each rank received is what
    # its partner sent, and it now sits in the receiving rank's deme
    e0, e1 = res[0]["exchange"], res[1]["exchange"]
    assert e0["partner"] == 1 and e1["partner"] == 0
    assert len(e0["slots"]) == 4
    for mine, other, got in ((e0, e1, res[0]["after"]), (e1, e0, res[1]["after"])):
        for (p1, l1, err1, _), (p2, l2, err2, _), (p3, l3, err3, _) in zip(
                mine["received"], other["sent"], got):
            assert np.array_equal(p1, p2) and np.array_equal(l1, l2) and err1 == err2
            assert np.array_equal(p3, p2) and np.array_equal(l3, l2) and err3 == err2


def test_lost_rank_ends_the_next_gather_with_an_error(built_libs, tmp_path):
    """Failure detection on the host: a rank that dies between steps (with
    nothing of its own in flight) makes the survivor's next collective
    raise within the process group's timeout instead of hanging."""
    ctx = mp.start_processes(dist_workers.sharded_rank_dies,
                             args=(2, _port(), ROOT, str(tmp_path)), nprocs=2, join=False,
                             start_method="spawn")
    deadline = 90.0
    for p in ctx.processes:
        p.join(deadline)
    alive = [p for p in ctx.processes if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank did not finish"
    assert [p.exitcode for p in ctx.processes] == [0, 3]
    r = np.load(tmp_path / "rank0.npz")
    print("survivor:", str(r["outcome"]), "after %.1f s" % float(r["seconds"]))
    assert str(r["outcome"]).startswith("raised"), str(r["outcome"])
    assert float(r["seconds"]) < 70.0


@pytest.mark.gpu
def test_sharding_runs_over_the_cuda_evaluator(built_libs, tmp_path):
    """The sharding code over the real CUDA evaluator on a one-rank NCCL
    group: the dealt-and-gathered errors equal a plain evaluate_batch bit for
    bit and the FP64 oracle within the parity tolerance, and an island search
    through IslandShards follows the plain search's trajectory."""
    mp.spawn(dist_workers.cuda_one_rank, args=(1, _port(), ROOT, str(tmp_path)), nprocs=1,
             join=True)
    r = np.load(tmp_path / "rank0.npz")
    np.testing.assert_array_equal(r["err_s"], r["err_p"])
    np.testing.assert_array_equal(r["raw_s"], r["raw_p"])
    params, batch, init, tgt = synth.workload("uneven_64x64", seed=41, n_models=37, steps=120)
    me = np.full(batch.n_models, 1000.0)
    me[::6] = 0.05
    _, o_raw, _ = oracle.evaluate_batch(params, init, tgt, batch, me)
    assert (np.abs(r["raw_s"] - o_raw) <= 1e-7 + 1e-4 * np.abs(o_raw)).all()
    np.testing.assert_array_equal(r["best_sharded"], r["best_plain"])
