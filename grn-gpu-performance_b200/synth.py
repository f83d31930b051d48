"""Seeded synthetic workloads: GRN models, initial patterns and targets.

The reference's experiments are morphology images stored in a database that
does not ship; these generators stand in for them with the shapes, sizes and
parameter ranges of the benchmark configurations:

  small_32x32      64 models, 3 genes, 2-6 links, 32x32, 500 steps, dt 0.1,
                   linear-gradient inputs, stripe targets, MSE fitness
  uneven_64x64     4096 models, 2-8 genes, 1-24 links, 64x64, 2000 steps,
                   radial/gradient inputs, multi-stripe targets
  islands_100x100  16 x 512 models, <=8 genes, <=24 links, 100x100, 1500 steps
  large_256x256    1024 models, 8 genes, 24 links, 256x256, 5000 steps, dt 0.05

Model parameters: Hill coefficient magnitude U[1,4] with activation or
repression equally likely (repression links are AND links, activation links
AND or OR with equal probability, as the reference's ModelLink constructor,
Src/Model/modellink.cpp:10-22), K ~ U[0.1,1], production, degradation and
diffusion ~ U[0.01,1].  Labels 0..G-1; morphogens are labels
0..n_input+n_target-1.  Links are distinct (regulator, regulated) pairs, as
the reference's addOrReplaceRandomLink keeps them (Src/Model/model.cpp:449-453).
"""
import numpy as np

from grn_b200 import LINK_DTYPE, PRODUCT_DTYPE, FITNESS_MSE, FITNESS_REF_LOGTHRESH, ModelBatch

WORKLOADS = {
    "small_32x32": dict(n_models=64, genes=(3, 3), links=(2, 6), W=32, H=32, steps=500,
                        dt=0.1, n_in=1, n_target=2, fitness=FITNESS_MSE, inputs="gradient",
                        n_exp=1),
    "uneven_64x64": dict(n_models=4096, genes=(2, 8), links=(1, 24), W=64, H=64, steps=2000,
                         dt=0.1, n_in=1, n_target=1, fitness=FITNESS_REF_LOGTHRESH,
                         inputs="radial", n_exp=1),
    "islands_100x100": dict(n_models=8192, genes=(2, 8), links=(1, 24), W=100, H=100,
                            steps=1500, dt=0.1, n_in=1, n_target=1,
                            fitness=FITNESS_REF_LOGTHRESH, inputs="radial", n_exp=1),
    "large_256x256": dict(n_models=1024, genes=(8, 8), links=(24, 24), W=256, H=256,
                          steps=5000, dt=0.05, n_in=1, n_target=1,
                          fitness=FITNESS_REF_LOGTHRESH, inputs="radial", n_exp=1),
}


def sim_params(wl, **over):
    """grn_sim_params dict of a workload.  min_conc_change 0 never stops a
    simulation early unless every rate is exactly zero."""
    p = dict(dim_x=wl["W"], dim_y=wl["H"], n_input_morphogens=wl["n_in"],
             n_target_morphogens=wl["n_target"], num_sim_steps=wl["steps"],
             error_precision=8, fitness_kind=wl["fitness"], dt=wl["dt"], min_conc=0.0,
             min_conc_change=0.0, dist_error_threshold=0.05)
    p.update(over)
    return p


def random_model(rng, n_genes, n_links, n_morph, hill=(1.0, 4.0), k=(0.1, 1.0),
                 rates=(0.01, 1.0)):
    prods = np.zeros(n_genes, PRODUCT_DTYPE)
    prods["label"] = np.arange(n_genes)
    prods["init"] = [-(i + 1) if i < min(n_morph, 3) else 0 for i in range(n_genes)]
    prods["lim"] = rng.uniform(*rates, n_genes)
    prods["deg"] = rng.uniform(*rates, n_genes)
    prods["dif"] = rng.uniform(*rates, n_genes)
    n_links = min(n_links, n_genes * n_genes)
    pairs = rng.choice(n_genes * n_genes, size=n_links, replace=False)
    links = np.zeros(n_links, LINK_DTYPE)
    links["regulator"] = pairs // n_genes
    links["regulated"] = pairs % n_genes
    links["dis_const"] = rng.uniform(*k, n_links)
    mag = rng.uniform(*hill, n_links)
    rep = rng.random(n_links) < 0.5
    links["hill_coef"] = np.where(rep, -mag, mag)
    links["is_and"] = np.where(rep, 1, (rng.random(n_links) < 0.5).astype(np.int32))
    return prods, links


def random_batch(n_models, genes, links, n_morph, seed):
    rng = np.random.default_rng(seed)
    models = []
    for _ in range(n_models):
        g = int(rng.integers(genes[0], genes[1] + 1))
        l = int(rng.integers(links[0], links[1] + 1))
        models.append(random_model(rng, max(g, n_morph), l, n_morph))
    return ModelBatch.from_models(models)


def gradient_pattern(rng, W, H):
    th = rng.uniform(0, 2 * np.pi)
    y, x = np.mgrid[0:H, 0:W]
    u = (x * np.cos(th) + y * np.sin(th))
    u = (u - u.min()) / max(u.max() - u.min(), 1e-12)
    lo, hi = rng.uniform(0.0, 0.3), rng.uniform(0.7, 1.0)
    return lo + (hi - lo) * u


def radial_pattern(rng, W, H):
    cx, cy = rng.uniform(0.2, 0.8) * W, rng.uniform(0.2, 0.8) * H
    s = rng.uniform(0.15, 0.4) * max(W, H)
    y, x = np.mgrid[0:H, 0:W]
    return np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * s * s))


def stripe_pattern(rng, W, H, n_stripes=None):
    n = n_stripes or int(rng.integers(1, 4))
    th = rng.uniform(0, np.pi)
    ph = rng.uniform(0, 2 * np.pi)
    y, x = np.mgrid[0:H, 0:W]
    u = (x * np.cos(th) + y * np.sin(th)) / max(W, H)
    return (np.sin(2 * np.pi * n * u + ph) > 0).astype(np.float64)


def experiments(wl, seed):
    """(initial [n_exp][n_in][H][W], target [n_exp][n_target][H][W])."""
    rng = np.random.default_rng(seed + 7919)
    W, H = wl["W"], wl["H"]
    init = np.zeros((wl["n_exp"], wl["n_in"], H, W))
    tgt = np.zeros((wl["n_exp"], wl["n_target"], H, W))
    for e in range(wl["n_exp"]):
        for k in range(wl["n_in"]):
            if wl["inputs"] == "gradient" or (wl["inputs"] == "radial" and k % 2 == 1):
                init[e, k] = gradient_pattern(rng, W, H)
            else:
                init[e, k] = radial_pattern(rng, W, H)
        for k in range(wl["n_target"]):
            tgt[e, k] = stripe_pattern(rng, W, H)
    return init, tgt


def workload(name, seed=0, n_models=None, **over):
    """(sim params dict, ModelBatch, initial, target) of a named workload."""
    wl = dict(WORKLOADS[name])
    for k in list(over):
        if k in wl:
            wl[k] = over.pop(k)
    if n_models is not None:
        wl["n_models"] = n_models
    params = sim_params(wl, **over)
    batch = random_batch(wl["n_models"], wl["genes"], wl["links"], wl["n_in"] + wl["n_target"],
                         seed)
    init, tgt = experiments(wl, seed)
    return params, batch, init, tgt
