"""Surrogate fitness MLP (grn_surrogate_*, grn_encode_models): the model
encoding on the CPU, the FP64 numpy MLP's own backward pass against finite
differences, and on the GPU the tensor-core forward/backward/Adam kernels
against that FP64 MLP with BF16 rounding emulated at the points where the
kernels store BF16."""
import math

import numpy as np
import pytest

import grn_b200 as grn
import mlp_ref
import synth

N_MORPH = 2


def _one_model_batch():
    prods = np.zeros(2, grn.PRODUCT_DTYPE)
    prods["label"] = [0, 1]
    prods["lim"] = [0.5, 0.25]
    prods["deg"] = [0.125, 0.75]
    prods["dif"] = [0.0, 0.375]
    links = np.zeros(3, grn.LINK_DTYPE)
    # 1 -> 0 OR (n 1, K 1), 0 -> 1 OR (n 2, K 0.5), 1 -> 1 AND repression (n 3, K 0.25)
    links["regulator"] = [1, 0, 1]
    links["regulated"] = [0, 1, 1]
    links["hill_coef"] = [1.0, 2.0, -3.0]
    links["dis_const"] = [1.0, 0.5, 0.25]
    links["is_and"] = [0, 0, 1]
    return grn.ModelBatch.from_models([(prods, links)])


def test_encoding_layout(built_libs):
    f = grn.encode_models(_one_model_batch(), 1)[0]
    assert f.shape == (128,)
    np.testing.assert_allclose(f[:8], [0.5, 0.125, 0.0, 1.0, 0.25, 0.75, 0.375, 1.0], rtol=1e-7)
    assert not f[8:32].any()  # genes 2..7 absent
    links = f[32:44].reshape(3, 4)
    # program order: gene 0's OR link, gene 1's OR link, gene 1's AND link
    np.testing.assert_allclose(links[0], [1 / 8, 1.0, 1 / 5, 1 / 8], rtol=1e-6)
    np.testing.assert_allclose(links[1], [0 / 8, 0.5, 2 / 5, 2 / 8], rtol=1e-6)
    np.testing.assert_allclose(links[2], [1 / 8, 0.25, -3 / 5, -2 / 8], rtol=1e-6)
    assert not f[44:].any()


def test_encoding_batch_bounds(built_libs):
    b = synth.random_batch(500, (2, 8), (1, 24), N_MORPH, 5)
    f = grn.encode_models(b, N_MORPH)
    assert f.shape == (500, 128) and np.isfinite(f).all()
    assert np.abs(f).max() <= 4.0
    # genes in use are flagged, and the flags are a prefix
    flags = f[:, 3:32:4]
    assert ((flags == 0) | (flags == 1)).all()
    assert (np.diff(flags, axis=1) <= 0).all()


def test_encoding_rejects_bad_model(built_libs):
    prods = np.zeros(1, grn.PRODUCT_DTYPE)
    links = np.zeros(1, grn.LINK_DTYPE)
    links["regulator"], links["regulated"] = 5, 0  # regulator 5 has no product
    links["hill_coef"], links["dis_const"] = 1.0, 0.5
    with pytest.raises(grn.GrnError):
        grn.encode_models(grn.ModelBatch.from_models([(prods, links)]), 1)


def test_fp64_mlp_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    P = {name: rng.normal(size=shape) * (0.1 if name[0] == "W" else 0.05)
         for name, shape in mlp_ref.SHAPES}
    p = mlp_ref.pack(P)
    x = rng.normal(size=(6, 128))
    t = rng.normal(size=6)
    loss, g = mlp_ref.loss_and_grads(p, x, t, emulate_bf16=False)
    offsets = np.cumsum([0] + [int(np.prod(s)) for _, s in mlp_ref.SHAPES])
    for k, (name, _) in enumerate(mlp_ref.SHAPES):
        n = offsets[k + 1] - offsets[k]
        for i in rng.choice(n, min(3, n), replace=False):
            j = offsets[k] + i
            e = np.zeros_like(p)
            e[j] = 1e-6
            fd = (mlp_ref.loss_and_grads(p + e, x, t, False)[0] -
                  mlp_ref.loss_and_grads(p - e, x, t, False)[0]) / 2e-6
            assert abs(fd - g[j]) <= 1e-6 + 1e-5 * abs(g[j]), (name, i, fd, g[j])


def test_surrogate_needs_device(built_libs):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(grn.GrnError) as e:
        grn.Surrogate()
    assert "NO_DEVICE" in str(e.value)


def _blocks(v):
    o, out = 0, {}
    for name, shape in mlp_ref.SHAPES:
        n = int(np.prod(shape))
        out[name] = v[o:o + n]
        o += n
    return out


@pytest.mark.gpu
def test_surrogate_gradients_match_fp64(built_libs):
    rng = np.random.default_rng(1)
    s = grn.Surrogate(seed=11)
    p = s.params().astype(np.float64)
    x = rng.normal(size=(300, 128)).astype(np.float32)  # 300: ragged 64-row tiles
    t = (rng.normal(size=300) - 1).astype(np.float32)
    loss, g = s.gradients(x, t)
    ref_loss, ref_g = mlp_ref.loss_and_grads(p, x, t, emulate_bf16=True)
    _, g64 = mlp_ref.loss_and_grads(p, x, t, emulate_bf16=False)
    assert abs(loss - ref_loss) <= 1e-4 * ref_loss
    y = s.predict(x)
    y_ref, _ = mlp_ref.forward(p, x, emulate_bf16=True)
    assert np.linalg.norm(y - y_ref) <= 2e-3 * np.linalg.norm(y_ref)
    gb, rb, fb = _blocks(g), _blocks(ref_g), _blocks(g64)
    for name, _ in mlp_ref.SHAPES:
        # BF16-emulating FP64 reference: the same roundings, FP64 sums (tolerance 5e-3)
        assert np.linalg.norm(gb[name] - rb[name]) <= 5e-3 * np.linalg.norm(rb[name]), name
        # plain FP64 gradient: BF16 operands keep the direction (cosine >= 0.99)
        cos = gb[name] @ fb[name] / (np.linalg.norm(gb[name]) * np.linalg.norm(fb[name]))
        assert cos >= 0.99, (name, cos)


@pytest.mark.gpu
def test_tcgen05_and_mma_sync_paths_agree(built_libs):
    """The GEMMs on tcgen05 (accumulator in tensor memory) and on warp-level
    mma.sync give the same predictions and gradients up to FP32 summation
    order (and the BF16 roundings it can flip)."""
    rng = np.random.default_rng(5)
    s = grn.Surrogate(seed=15)
    x = rng.normal(size=(333, 128)).astype(np.float32)  # ragged 128-row tiles
    t = rng.normal(size=333).astype(np.float32)
    out = {}
    for tc in (True, False):
        s.use_tcgen05(tc)
        out[tc] = (s.predict(x), s.gradients(x, t))
    (y1, (l1, g1)), (y0, (l0, g0)) = out[True], out[False]
    assert np.linalg.norm(y1 - y0) <= 2e-3 * np.linalg.norm(y0)
    assert abs(l1 - l0) <= 1e-3 * abs(l0)
    b1, b0 = _blocks(g1), _blocks(g0)
    for name, _ in mlp_ref.SHAPES:
        assert np.linalg.norm(b1[name] - b0[name]) <= 5e-3 * np.linalg.norm(b0[name]), name


@pytest.mark.gpu
def test_surrogate_adam_step(built_libs):
    rng = np.random.default_rng(2)
    s = grn.Surrogate(seed=12, capacity=256)
    p0 = s.params().astype(np.float64)
    x = rng.normal(size=(256, 128)).astype(np.float32)
    t = rng.normal(size=256).astype(np.float32)
    s.add_data(x, t)
    assert s.data_count == 256
    lr = 1e-3
    s.train(epochs=1, batch_size=256, lr=lr)  # one minibatch: the whole set
    p1 = s.params().astype(np.float64)
    _, g = mlp_ref.loss_and_grads(p0, x, t, emulate_bf16=True)
    p_ref, _, _ = mlp_ref.adam(p0, g, np.zeros_like(p0), np.zeros_like(p0), 1, lr)
    d, d_ref = p1 - p0, p_ref - p0
    # Adam's first step is lr * g / (|g| + eps): at most lr per parameter
    assert np.abs(d).max() <= lr * 1.0001
    assert np.linalg.norm(d - d_ref) <= 0.05 * np.linalg.norm(d_ref)


@pytest.mark.gpu
def test_surrogate_params_roundtrip_and_ring(built_libs):
    s = grn.Surrogate(seed=13, capacity=100)
    p = np.random.default_rng(3).normal(size=grn.N_PARAMS).astype(np.float32)
    s.set_params(p)
    np.testing.assert_array_equal(s.params(), p)
    x = np.zeros((150, 128), np.float32)
    s.add_data(x, np.zeros(150, np.float32))
    assert s.data_count == 100  # ring buffer keeps the newest 100


@pytest.mark.gpu
def test_surrogate_learns_smooth_function(built_libs):
    rng = np.random.default_rng(4)
    n = 12000
    X = rng.uniform(-1, 1, size=(n, 128)).astype(np.float32)
    u = rng.normal(size=128) / math.sqrt(128)
    v = rng.normal(size=128) / math.sqrt(128)
    T = (np.sin(2 * X @ u) + 0.5 * (X @ v) ** 2).astype(np.float32)
    s = grn.Surrogate(seed=14, capacity=10000)
    s.add_data(X[:10000], T[:10000])
    first = s.train(epochs=1, batch_size=256, lr=1e-3)
    for _ in range(14):
        last = s.train(epochs=1, batch_size=256, lr=1e-3)
    assert last < 0.2 * first
    P = s.predict(X[10000:])
    assert np.mean((P - T[10000:]) ** 2) <= 0.15 * np.var(T[10000:])


@pytest.mark.gpu
def test_evolution_with_surrogate_screening(built_libs):
    params = dict(dim_x=16, dim_y=16, n_input_morphogens=1, n_target_morphogens=1,
                  num_sim_steps=100, error_precision=6, fitness_kind=0, dt=0.1, min_conc=0.0,
                  min_conc_change=1e-3, dist_error_threshold=0.05)
    wl = dict(synth.WORKLOADS["uneven_64x64"], W=16, H=16, n_exp=2)
    init, tgt = synth.experiments(wl, 3)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        evo = grn.Evolution(dict(n_demes=4, deme_size=64, migration_period=5, n_max_products=6,
                                 n_max_links=12, n_host_threads=2, seed=5), 2, evaluator=ev)
        sur = grn.Surrogate(seed=6, capacity=4096)
        evo.set_surrogate(sur, simulate_fraction=0.25, min_train_pairs=512,
                          batches_per_generation=8, batch_size=128)
        stats = [evo.step() for _ in range(8)]
        # generation 0 simulates the initial 256; clones of their parent are
        # never simulated; screening starts once 512 pairs exist
        assert stats[0]["n_evaluated"] == 256 and stats[0]["n_screened"] == 0
        assert all(s["n_evaluated"] + s["n_clones"] == 256 for s in stats[1:] if
                   not s["n_screened"])
        screened = [s for s in stats if s["n_screened"]]
        assert screened and all(s["n_screened"] + s["n_clones"] == 256 and
                                s["n_evaluated"] == math.ceil(0.25 * s["n_screened"])
                                for s in screened)
        assert sur.data_count == sum(s["n_evaluated"] for s in stats)
        best = [s["best_error"] for s in stats]
        assert all(b2 <= b1 for b1, b2 in zip(best, best[1:]))
        assert all(math.isfinite(s["surrogate_loss"]) for s in stats)
        evo.close()
        sur.close()


def _search(ev, gens, seed, sur_seed=None, audit=False, score=None, fraction=0.25):
    evo = grn.Evolution(dict(n_demes=8, deme_size=64, migration_period=5, n_max_products=6,
                             n_max_links=12, n_host_threads=2, seed=seed), 2, evaluator=ev)
    evo.set_skip_clones(True)
    sur = None
    if sur_seed is not None:
        sur = grn.Surrogate(seed=sur_seed, capacity=20000)
        evo.set_surrogate(sur, simulate_fraction=fraction, min_train_pairs=1024,
                          batches_per_generation=16, batch_size=256)
        if score is not None:
            evo.set_surrogate_score(score)
        if audit:
            evo.set_surrogate_audit(True)
    stats = [evo.step() for _ in range(gens)]
    evo.close()
    if sur:
        sur.close()
    return stats


@pytest.mark.gpu
def test_surrogate_screen_quality_against_no_network(built_libs):
    """What the trained network gains over screening without it.  An audited
    run (every child also simulated, the search unchanged) measures, per
    screened generation, the share of the children that beat their parents
    which the screen kept.  Without a network a screen keeping 25% of the
    children keeps 25% of the improvers on average.  Measured on B200: the
    trained network's screen keeps 26.5% (Spearman rho 0.19 between
    predicted and simulated change) -- hardly better than chance -- and the
    screened search still reaches the plain search's best error, with 41% of
    its simulations, on this small problem.  The test holds that relation:
    no worse than chance, the same best error, far fewer simulations.  The
    audit must not change the search: its trajectory equals the unaudited
    run's."""
    params = dict(dim_x=16, dim_y=16, n_input_morphogens=1, n_target_morphogens=1,
                  num_sim_steps=150, error_precision=8, fitness_kind=0, dt=0.1, min_conc=0.0,
                  min_conc_change=0.0, dist_error_threshold=0.05)
    wl = dict(synth.WORKLOADS["uneven_64x64"], W=16, H=16, n_exp=1)
    init, tgt = synth.experiments(wl, 11)
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        plain = _search(ev, 24, seed=7)
        screened = _search(ev, 24, seed=7, sur_seed=3)
        audited = _search(ev, 24, seed=7, sur_seed=3, audit=True)
    assert [s["best_error"] for s in audited] == [s["best_error"] for s in screened]
    assert [s["n_evaluated"] for s in audited] == [s["n_evaluated"] for s in screened]
    rows = [s for s in audited if s["n_screened"]]
    assert len(rows) >= 10
    assert all(s["n_audited"] == s["n_screened"] for s in rows)
    rec = np.array([s["surrogate_improver_recall"] for s in rows], np.float64)
    rho = np.array([s["surrogate_rho"] for s in rows], np.float64)
    rec, rho = rec[np.isfinite(rec)], rho[np.isfinite(rho)]
    print("improver recall %.3f (no network: 0.25), rho %.3f, best plain %.5f screened %.5f, "
          "simulations plain %d screened %d" % (
              rec.mean(), rho.mean(), plain[-1]["best_error"], screened[-1]["best_error"],
              sum(s["n_evaluated"] for s in plain), sum(s["n_evaluated"] for s in screened)))
    assert len(rec) >= 5 and 0.22 <= rec.mean() <= 1.0
    assert rho.mean() > 0.05
    assert screened[-1]["best_error"] <= 1.01 * plain[-1]["best_error"]
    # The screened search simulates far fewer children than the plain one.
    assert sum(s["n_evaluated"] for s in screened) < 0.6 * sum(s["n_evaluated"] for s in plain)


def _spearman(a, b):
    ra = np.argsort(np.argsort(a)).astype(np.float64)
    rb = np.argsort(np.argsort(b)).astype(np.float64)
    ra -= ra.mean()
    rb -= rb.mean()
    return float((ra * rb).sum() / np.sqrt((ra * ra).sum() * (rb * rb).sum()))


@pytest.mark.gpu
def test_short_run_screen_fades_as_population_converges(built_libs):
    """Why no screen pays on the island workload: a cheap low-fidelity
    simulation (the same child, 10% of the Euler steps) ranks the children
    like the full simulation in the first generations and at chance once the
    population has converged -- the children then share their parents'
    plateau error, and the rare improvers are not the ones a short run
    favours.  The search runs at the island workload's grid and steps
    (100 x 100, 1500 steps) with 8 demes of 512; every generation's children
    are also simulated without the abandon bound (the full fitness) and for
    150 steps.  An improver beats its parent's rounded error.  Measured on
    B200: Spearman rho between the short and the full errors falls from 0.61
    (generation 2) to -0.17 (generation 26), and keeping the best 25% by the
    short run keeps 18% of the improvers on average -- below chance from the
    start, because an improving mutation shows late.  The test holds those
    relations (the search is seeded and the evaluator deterministic)."""
    wl = synth.WORKLOADS["islands_100x100"]
    params = synth.sim_params(wl)
    init, tgt = synth.experiments(wl, 0)
    short_params = dict(params, num_sim_steps=params["num_sim_steps"] // 10)
    rows = []
    with grn.Evaluator(params) as ev, grn.Evaluator(short_params) as evs:
        ev.set_experiments(init, tgt)
        evs.set_experiments(init, tgt)

        def calc(batch, max_error):
            err, _, _ = ev.evaluate_batch(batch, max_error)
            if np.all(max_error >= 100.0):  # the random first population
                return err
            full_err, full, _ = ev.evaluate_batch(batch)
            _, short, _ = evs.evaluate_batch(batch)
            k = len(short) // 4
            keep = np.zeros(len(short), bool)
            keep[np.argsort(short, kind="stable")[:k]] = True
            imp = full_err < max_error
            rows.append((_spearman(short, full),
                         float((keep & imp).sum() / imp.sum()) if imp.sum() >= 10 else np.nan))
            return err

        evo = grn.Evolution(dict(n_demes=8, deme_size=512, migration_period=10, n_max_products=8,
                                 n_max_links=24, n_host_threads=0, seed=0),
                            wl["n_in"] + wl["n_target"], calculator=calc)
        for _ in range(26):
            evo.step()
        evo.close()
    rho = np.array([r[0] for r in rows])
    rec = np.array([r[1] for r in rows])
    print("rho by generation", np.round(rho, 3).tolist())
    print("improver recall by generation", np.round(rec, 3).tolist())
    assert len(rows) == 25
    assert rho[:3].mean() > 0.4          # ranks like the full run at first
    assert rho[-5:].mean() < 0.1         # and at chance once the population converged
    assert np.nanmean(rec) < 0.25        # no better than keeping children at random


@pytest.mark.gpu
def test_surrogate_tiny_and_ragged_batches(built_libs):
    """Batches smaller than one 128-row tile and weight-gradient GEMMs whose
    reduction (the batch) is shorter than one 64-wide slice: the tensor maps
    zero-fill past the edges.  Predictions and gradients on the tcgen05 path
    against the BF16-emulating FP64 MLP (tolerances as in the gradient
    check)."""
    rng = np.random.default_rng(9)
    s = grn.Surrogate(seed=19)
    p = s.params().astype(np.float64)
    for n in (1, 5, 7, 64, 129):
        x = rng.normal(size=(n, 128)).astype(np.float32)
        t = (rng.normal(size=n) - 1).astype(np.float32)
        y = s.predict(x)
        y_ref, _ = mlp_ref.forward(p, x, emulate_bf16=True)
        assert np.linalg.norm(y - y_ref) <= 2e-3 * np.linalg.norm(y_ref), n
        loss, g = s.gradients(x, t)
        ref_loss, ref_g = mlp_ref.loss_and_grads(p, x, t, emulate_bf16=True)
        assert abs(loss - ref_loss) <= 1e-4 * ref_loss, n
        gb, rb = _blocks(g), _blocks(ref_g)
        for name, _ in mlp_ref.SHAPES:
            assert np.linalg.norm(gb[name] - rb[name]) <= 5e-3 * np.linalg.norm(rb[name]) + 1e-7, \
                (n, name)


@pytest.mark.gpu
def test_screened_search_resumes_exactly(built_libs):
    """A surrogate-screened search checkpointed after generation 7 (search
    and surrogate) and restored into new objects with other seeds goes on
    exactly like the original: the same screening, simulations, losses and
    best errors."""
    params = dict(dim_x=16, dim_y=16, n_input_morphogens=1, n_target_morphogens=1,
                  num_sim_steps=100, error_precision=8, fitness_kind=0, dt=0.1, min_conc=0.0,
                  min_conc_change=0.0, dist_error_threshold=0.05)
    wl = dict(synth.WORKLOADS["uneven_64x64"], W=16, H=16, n_exp=1)
    init, tgt = synth.experiments(wl, 12)
    evo_p = dict(n_demes=4, deme_size=64, migration_period=5, n_max_products=6, n_max_links=12,
                 n_host_threads=2, seed=9)
    sur_kw = dict(simulate_fraction=0.25, min_train_pairs=512, batches_per_generation=8,
                  batch_size=128)
    keys = ("generation", "n_evaluated", "n_screened", "best_error", "mean_error",
            "surrogate_loss", "n_clones")
    with grn.Evaluator(params) as ev:
        ev.set_experiments(init, tgt)
        evo = grn.Evolution(evo_p, 2, evaluator=ev)
        sur = grn.Surrogate(seed=4, capacity=5000)
        evo.set_surrogate(sur, **sur_kw)
        for _ in range(8):
            evo.step()
        state, sstate = evo.checkpoint(), sur.checkpoint()
        tail = [evo.step() for _ in range(6)]
        evo2 = grn.Evolution(dict(evo_p, seed=1), 2, evaluator=ev)
        sur2 = grn.Surrogate(seed=8, capacity=5000)
        evo2.set_surrogate(sur2, **sur_kw)
        evo2.restore(state)
        sur2.restore(sstate)
        tail2 = [evo2.step() for _ in range(6)]
        assert sum(s["n_screened"] for s in tail) > 0
        assert [[s[k] for k in keys] for s in tail2] == [[s[k] for k in keys] for s in tail]
        assert evo2.checkpoint() == evo.checkpoint()
        with pytest.raises(grn.GrnError):
            grn.Surrogate(seed=8, capacity=4000).restore(sstate)  # another capacity
        for e in (evo, evo2):
            e.close()
        for s in (sur, sur2):
            s.close()
