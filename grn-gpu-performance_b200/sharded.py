"""Multi-GPU sharding of the batched evaluator and of the island search.

One process per GPU under torch.distributed (NCCL between GPUs; gloo runs the
same code on CPU).  A fitness evaluation has no exchange step: every rank
simulates its own shard of the batch and the only collective is the gather of
two doubles (rounded and raw error) per model.  The reference spreads models
over one evaluator thread per GPU (Src/GPUSimulator/cevaluatormorphogens.cpp:
64-90, CalculatorThreadGPU in Src/UI/Evolution/errorcalculatormultithread.cpp:
233-254); here the split is decided once per batch from the models' compiled
cost.

Island search across GPUs: every rank runs whole demes (its own
grn_evolution); every `period` generations ranks are paired at random (the
same pairing on every rank, from a shared seed) and each pair swaps a random
half of one deme's individuals -- the reference's deme migration
(Src/Search/search.cpp:263-311) with one deme of the pair on each GPU.
"""
import numpy as np
import torch
import torch.distributed as dist

import grn_b200 as grn


def deal(costs, world):
    """Rank of every model: models in decreasing cost are dealt to the ranks
    in boustrophedon order (0, 1, .., W-1, W-1, .., 0, 0, ..), so that every
    rank gets the same number of models (+-1) and about the same total cost.
    (Contiguous ranges of the cost order would hand one GPU a few long models,
    fewer than its SMs can run at once.)"""
    costs = np.asarray(costs, np.float64)
    order = np.argsort(-costs, kind="stable")
    ranks = np.empty(len(costs), np.int64)
    i = np.arange(len(costs))
    lap, pos = np.divmod(i, world)
    ranks[order] = np.where(lap % 2 == 0, pos, world - 1 - pos)
    return ranks


def _gather_device(group):
    backend = dist.get_backend(group)
    if backend == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


class ShardedEvaluator:
    """evaluate_batch over all ranks of `group`: every rank passes the same
    batch and gets every model's errors.  `evaluator` is this rank's
    evaluator (grn_b200.Evaluator, or anything with the same
    evaluate_batch(batch, max_error) -> (err, raw, stats))."""

    def __init__(self, evaluator, n_morphogens, group=None):
        self.ev = evaluator
        self.n_morph = n_morphogens
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def evaluate_batch(self, batch, max_error=None):
        n = batch.n_models
        me = np.full(n, 1000.0) if max_error is None else \
            np.ascontiguousarray(np.broadcast_to(np.asarray(max_error, np.float64), (n,)))
        ranks = deal(grn.model_costs(batch, self.n_morph), self.world)
        mine = np.nonzero(ranks == self.rank)[0]
        stats = {}
        if len(mine):
            err, raw, stats = self.ev.evaluate_batch(batch.subset(mine), me[mine])
        else:
            err = raw = np.zeros(0)
        counts = np.bincount(ranks, minlength=self.world)
        dev = _gather_device(self.group)
        buf = torch.zeros((int(counts.max()) if n else 0, 2), dtype=torch.float64, device=dev)
        buf[:len(mine), 0] = torch.as_tensor(err, dtype=torch.float64)
        buf[:len(mine), 1] = torch.as_tensor(raw, dtype=torch.float64)
        parts = [torch.empty_like(buf) for _ in range(self.world)]
        dist.all_gather(parts, buf, group=self.group)
        full = np.zeros((n, 2))
        for r in range(self.world):
            idx = np.nonzero(ranks == r)[0]
            full[idx] = parts[r][:len(idx)].cpu().numpy()
        return full[:, 0], full[:, 1], stats


class IslandShards:
    """An island search with whole demes on every rank and migration across
    ranks.  `evo` is this rank's grn_b200.Evolution (its own demes and seed);
    every rank must construct it with the same deme count and size."""

    def __init__(self, evo, n_demes, deme_size, period=10, seed=0, group=None):
        self.evo = evo
        self.n_demes = n_demes
        self.deme_size = deme_size
        self.period = period
        self.seed = seed
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.generation = 0

    def step(self):
        """One generation on every rank, migration across ranks every
        `period` generations, and the best error over all ranks."""
        st = self.evo.step()
        self.generation += 1
        if self.world > 1 and self.period > 0 and self.generation % self.period == 0:
            self.migrate()
            st["migrated_ranks"] = 1
        best = torch.tensor([st["best_error"]], dtype=torch.float64,
                            device=_gather_device(self.group))
        dist.all_reduce(best, op=dist.ReduceOp.MIN, group=self.group)
        st["global_best_error"] = float(best.item())
        return st

    def migrate(self):
        """Pairs ranks at random (shared seed: the same pairs everywhere);
        each pair swaps a random half of one deme each."""
        rng = np.random.default_rng([self.seed, self.generation])
        perm = rng.permutation(self.world)
        partner = -1
        for i in range(0, self.world - 1, 2):
            a, b = int(perm[i]), int(perm[i + 1])
            if self.rank == a:
                partner = b
            elif self.rank == b:
                partner = a
        local = np.random.default_rng([self.seed, self.generation, self.rank])
        deme = int(local.integers(self.n_demes))
        slots = local.permutation(self.deme_size)[:self.deme_size // 2]
        payload = None
        if partner >= 0:
            payload = [self.evo.individual(deme, int(i)) for i in slots]
        everyone = [None] * self.world
        dist.all_gather_object(everyone, (partner, payload), group=self.group)
        self.last_exchange = None
        if partner >= 0:
            their_partner, theirs = everyone[partner]
            assert their_partner == self.rank
            for i, (prods, links, err, _) in zip(slots, theirs):
                self.evo.set_individual(deme, int(i), prods, links, err)
            self.last_exchange = {"partner": partner, "deme": deme,
                                  "slots": [int(i) for i in slots], "sent": payload,
                                  "received": theirs}
