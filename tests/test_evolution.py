"""Island evolution host (grn_evolution_*): model-operator invariants,
determinism and deterministic-crowding selection, driven on the CPU by the
FP64 oracle as the batch evaluator, and on the GPU by the library's own
evaluator."""
import numpy as np
import pytest

import binding as oracle
import grn_b200 as grn
import synth

SIM = dict(dim_x=8, dim_y=8, n_input_morphogens=1, n_target_morphogens=1, num_sim_steps=25,
           error_precision=6, fitness_kind=0, dt=0.1, min_conc=0.0, min_conc_change=1e-3,
           dist_error_threshold=0.05)
EVO = dict(n_demes=4, deme_size=10, migration_period=2, n_max_products=6, n_max_links=10,
           n_host_threads=2, seed=7)


def _experiments(sim, seed=3):
    wl = dict(synth.WORKLOADS["uneven_64x64"], W=sim["dim_x"], H=sim["dim_y"], n_exp=2)
    return synth.experiments(wl, seed)


class OracleCalculator:
    def __init__(self, sim):
        self.sim = sim
        self.init, self.tgt = _experiments(sim)
        self.calls = []

    def __call__(self, batch, max_error):
        self.calls.append((batch.n_models, max_error.copy()))
        err, _, _ = oracle.evaluate_batch(self.sim, self.init, self.tgt, batch, max_error,
                                          n_threads=2)
        return err


def _check_model(prods, links, n_morph, max_prods, max_links):
    labels = set(prods["label"].tolist())
    assert set(range(n_morph)) <= labels  # morphogens are never removed
    for l in links:
        assert l["regulator"] in labels and l["regulated"] in labels
    in_use = oracle.labels_in_use(prods, links, n_morph)
    assert len(in_use) <= max_prods
    used = [l for l in links if l["regulator"] in in_use and l["regulated"] in in_use]
    assert len(used) <= max_links
    assert all((l["hill_coef"] >= 0) or l["is_and"] for l in links)  # repressors are AND


def test_evolution_invariants_with_oracle(built_libs):
    calc = OracleCalculator(SIM)
    evo = grn.Evolution(EVO, 2, calculator=calc)
    stats = [evo.step() for _ in range(6)]
    assert stats[0]["generation"] == 0 and stats[0]["n_evaluated"] == 40
    assert all(s["n_evaluated"] == 40 for s in stats)
    # the global best never gets worse (children replace parents only if not worse)
    best = [s["best_error"] for s in stats]
    assert all(b2 <= b1 for b1, b2 in zip(best, best[1:]))
    assert [s["migrated"] for s in stats] == [0, 0, 1, 0, 1, 0]
    # initial individuals are evaluated with maxError 1000, children with their parent's error
    assert (calc.calls[0][1] == 1000.0).all()
    assert (calc.calls[1][1] <= 1000.0).all() and (calc.calls[1][1] < 1000.0).any()
    for d in range(4):
        for i in range(10):
            prods, links, err, comp = evo.individual(d, i)
            _check_model(prods, links, 2, EVO["n_max_products"], EVO["n_max_links"])
            # stored errors are the evaluator's (re-evaluate with maxError 1000)
            e, _, _ = oracle.evaluate_batch(SIM, calc.init, calc.tgt,
                                            grn.ModelBatch.from_models([(prods, links)]),
                                            [1000.0], n_threads=1)
            assert e[0] == err or err == 100.0
    d, i = evo.best()
    assert evo.individual(d, i)[2] == best[-1]
    evo.close()


def test_evolution_is_deterministic(built_libs):
    runs = []
    for _ in range(2):
        calc = OracleCalculator(SIM)
        evo = grn.Evolution(dict(EVO, seed=11), 2, calculator=calc)
        st = [evo.step() for _ in range(4)]
        models = [evo.individual(d, i) for d in range(4) for i in range(10)]
        runs.append((st, models))
        evo.close()
    (s1, m1), (s2, m2) = runs
    assert [x["best_error"] for x in s1] == [x["best_error"] for x in s2]
    for a, b in zip(m1, m2):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]


def test_skip_clones_keeps_the_search_identical(built_libs):
    """Accepting children whose simulated program equals their parent's
    without simulating them changes nothing but the number of simulations."""
    runs = []
    for skip in (False, True):
        calc = OracleCalculator(SIM)
        evo = grn.Evolution(dict(EVO, seed=13), 2, calculator=calc)
        evo.set_skip_clones(skip)
        st = [evo.step() for _ in range(6)]
        models = [evo.individual(d, i) for d in range(4) for i in range(10)]
        runs.append((st, models, sum(c[0] for c in calc.calls)))
        evo.close()
    (s1, m1, n1), (s2, m2, n2) = runs
    assert all(x["n_clones"] == 0 for x in s1)
    clones = sum(x["n_clones"] for x in s2)
    assert clones > 0 and n2 == n1 - clones
    assert all(a["n_evaluated"] + a["n_clones"] == 40 for a in s2)
    assert [x["best_error"] for x in s1] == [x["best_error"] for x in s2]
    for a, b in zip(m1, m2):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]


def test_evolution_models_grow_within_limits(built_libs):
    """Duplication mutations add products; excess removal keeps the
    products and links in use within the limits."""
    rng_err = np.random.default_rng(0)
    evo = grn.Evolution(dict(EVO, deme_size=16, n_max_products=4, n_max_links=5, seed=3), 2,
                        calculator=lambda b, me: rng_err.random(b.n_models))
    for _ in range(30):
        evo.step()
    sizes = []
    for d in range(4):
        for i in range(16):
            prods, links, _, _ = evo.individual(d, i)
            _check_model(prods, links, 2, 4, 5)
            sizes.append(len(prods))
    assert max(sizes) > 2
    evo.close()


@pytest.mark.gpu
def test_evolution_on_gpu_matches_oracle_errors():
    sim = dict(SIM, dim_x=16, dim_y=16, num_sim_steps=60)
    init, tgt = _experiments(sim)
    with grn.Evaluator(sim) as ev:
        ev.set_experiments(init, tgt)
        evo = grn.Evolution(dict(EVO, deme_size=32, n_max_products=8, n_max_links=24), 2,
                            evaluator=ev)
        stats = [evo.step() for _ in range(5)]
        best = [s["best_error"] for s in stats]
        assert all(b2 <= b1 for b1, b2 in zip(best, best[1:]))
        models, errs = [], []
        for d in range(4):
            for i in range(0, 32, 4):
                prods, links, err, _ = evo.individual(d, i)
                models.append((prods, links))
                errs.append(err)
        evo.close()
    batch = grn.ModelBatch.from_models(models)
    oe, oraw, _ = oracle.evaluate_batch(sim, init, tgt, batch)
    errs = np.array(errs)
    ok = (np.abs(errs - oe) <= 1e-7 + 1e-4 * np.abs(oe)) | (errs == 100.0)
    assert ok.all(), (errs[~ok], oe[~ok])


def test_pipeline_needs_gpu_evaluator(built_libs):
    evo = grn.Evolution(EVO, 2, calculator=OracleCalculator(SIM))
    with pytest.raises(grn.GrnError):
        evo.set_pipeline(True)
    evo.close()


@pytest.mark.gpu
def test_pipelined_generations_match_synchronous():
    """Two halves of the demes alternating on the GPU while the host breeds
    the other half: the same populations as the synchronous search."""
    sim = dict(SIM, dim_x=16, dim_y=16, num_sim_steps=60)
    init, tgt = _experiments(sim)
    runs = []
    for pipe in (False, True):
        with grn.Evaluator(sim) as ev:
            ev.set_experiments(init, tgt)
            evo = grn.Evolution(dict(EVO, deme_size=32, n_max_products=8, n_max_links=24,
                                     migration_period=3, seed=31), 2, evaluator=ev)
            evo.set_skip_clones(True)
            if pipe:
                evo.set_pipeline(True)
            st = [evo.step() for _ in range(8)]
            models = [evo.individual(d, i) for d in range(4) for i in range(32)]
            if pipe:  # replacing an individual drops the children in flight
                p, l, e, _ = models[5]
                evo.set_individual(0, 0, p, l, e)
                evo.step()
            evo.close()
        runs.append((st, models))
    (s1, m1), (s2, m2) = runs
    for k in ("generation", "best_error", "mean_error", "n_evaluated", "n_clones", "migrated"):
        assert [x[k] for x in s1] == [x[k] for x in s2], k
    for a, b in zip(m1, m2):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]


def _populations(evo):
    return [evo.individual(d, i) for d in range(EVO["n_demes"]) for i in range(EVO["deme_size"])]


def _same_populations(a, b):
    return len(a) == len(b) and all(
        np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1]) and x[2] == y[2] and
        x[3] == y[3] for x, y in zip(a, b))


def test_checkpoint_restore_continues_the_run_exactly(built_libs):
    """A search restored from a checkpoint of generation 2 of another run
    (created with a different seed) goes through generations 3-6 exactly as
    the original did: populations, errors and statistics, migrations
    included."""
    evo = grn.Evolution(dict(EVO, seed=17), 2, calculator=OracleCalculator(SIM))
    for _ in range(3):
        evo.step()
    state = evo.checkpoint()
    tail = [evo.step() for _ in range(4)]
    want = _populations(evo)
    evo2 = grn.Evolution(dict(EVO, seed=99), 2, calculator=OracleCalculator(SIM))
    evo2.restore(state)
    tail2 = [evo2.step() for _ in range(4)]
    keys = ("generation", "n_evaluated", "best_error", "best_complexity", "mean_error",
            "migrated")
    assert [[s[k] for k in keys] for s in tail2] == [[s[k] for k in keys] for s in tail]
    assert _same_populations(_populations(evo2), want)
    # the checkpoint of the restored search at the same point equals the original's
    assert evo2.checkpoint() == evo.checkpoint()
    evo.close()
    evo2.close()


def test_restore_rejects_foreign_or_damaged_checkpoints(built_libs):
    evo = grn.Evolution(dict(EVO, seed=17), 2, calculator=OracleCalculator(SIM))
    evo.step()
    state = evo.checkpoint()
    before = _populations(evo)
    for bad in (state[:-1], state + b"x", b"GRNEVOCK" + state[8:20], b"x" * 64,
                state[:8] + b"\x02" + state[9:]):
        with pytest.raises(grn.GrnError):
            evo.restore(bad)
    other = grn.Evolution(dict(EVO, seed=17, deme_size=12), 2, calculator=OracleCalculator(SIM))
    with pytest.raises(grn.GrnError):
        other.restore(state)
    assert _same_populations(_populations(evo), before)  # a failed restore changes nothing
    evo.close()
    other.close()


@pytest.mark.gpu
def test_checkpoint_of_a_pipelined_search():
    """A pipelined search holds children in flight and cannot be
    checkpointed; switched back to synchronous mode (which drops them) it
    can, and a restored copy continues exactly like it on the GPU
    evaluator."""
    sim = dict(SIM, dim_x=16, dim_y=16, num_sim_steps=60)
    init, tgt = _experiments(sim)
    with grn.Evaluator(sim) as ev:
        ev.set_experiments(init, tgt)
        p = dict(EVO, deme_size=32, n_max_products=8, n_max_links=24, seed=37)
        evo = grn.Evolution(p, 2, evaluator=ev)
        evo.set_pipeline(True)
        for _ in range(3):
            evo.step()
        with pytest.raises(grn.GrnError):
            evo.checkpoint()
        evo.set_pipeline(False)
        state = evo.checkpoint()
        evo2 = grn.Evolution(dict(p, seed=1), 2, evaluator=ev)
        evo2.restore(state)
        a = [evo.step()["best_error"] for _ in range(3)]
        b = [evo2.step()["best_error"] for _ in range(3)]
        assert a == b and evo.checkpoint() == evo2.checkpoint()
        evo.close()
        evo2.close()
