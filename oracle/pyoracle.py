"""TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.

Second, independent restatement of the reference's CPU fitness path in pure
Python (FP64), for tiny grids only.  It exists to cross-check the C++ oracle
(oracle/grn_oracle.cpp): the two are written differently (this one evaluates
each product's regulation directly instead of compiling an op list) and must
agree to the last bit on the same inputs.

Parity status: numerics unpinned (the reference itself cannot be built or run
here; see grn_oracle.h).

Reference lines followed (lobolab/grn-gpu-performance):
  labels in use       Src/Model/model.cpp:243-283
  regulation program  Src/Simulator/modelsimulator.cpp:99-203
  Hill terms          Src/Simulator/simophillact.cpp:17-20, simophillrep.cpp:17-20
  OR / AND            simopor.cpp:20-22, simopand.cpp:20-22, Src/Common/mathalgo.h:208-216
  Euler step          Src/Simulator/modelsimulator.cpp:205-280
  step loop           Src/Simulator/simulator.cpp:54-63
  distance            Src/Simulator/simstate.cpp:135-158
  evaluation          Src/Search/evaluatormorphogens.cpp:48-76
  ceilS               Src/Common/mathalgo.h:55-62
"""
import math


def ref_max(a, b):
    return b if a < b else a


def ref_min(a, b):
    return a if not (b < a) else b


def labels_in_use(products, links, n_morph):
    regs = {}
    for ln in links:
        regs.setdefault(ln["regulated"], []).append(ln["regulator"])
    in_use = set(range(n_morph))
    queue = list(range(n_morph))
    while queue:
        lab = queue.pop(0)
        for r in regs.get(lab, []):
            if r not in in_use:
                in_use.add(r)
                queue.append(r)
    return sorted(in_use)


def _hill(x, link):
    n = link["hill_coef"]
    if n >= 0:
        kn = math.pow(link["dis_const"], n)
        rcn = math.pow(x, n)
        return _div(rcn, rcn + kn)
    n = -1.0 * n
    kn = math.pow(link["dis_const"], n)
    rcn = math.pow(x, n)
    return _div(kn, rcn + kn)


def _div(a, b):
    if b == 0:
        if a == 0 or math.isnan(a):
            return math.nan
        return math.copysign(math.inf, a)
    return a / b


def regulation(label, labels, links, conc):
    """Regulation value of one product at one cell: the result of the ops the
    reference compiles for it (OR links first, then AND links)."""
    in_use = set(labels)
    index = {lab: i for i, lab in enumerate(labels)}
    mine = [ln for ln in links if ln["regulated"] == label]
    if not any(ln["hill_coef"] >= 0 for ln in mine):
        return 0.0
    ors = [ln for ln in mine if ln["regulator"] in in_use and not ln["is_and"]]
    ands = [ln for ln in mine if ln["regulator"] in in_use and ln["is_and"]]
    val = None
    for ln in ors:
        h = _hill(conc[index[ln["regulator"]]], ln)
        val = h if val is None else ref_max(h, val)
    for ln in ands:
        h = _hill(conc[index[ln["regulator"]]], ln)
        val = h if val is None else ref_min(h, val)
    return 0.0 if val is None else val


def simulate(params, initial, products, links, n_steps):
    """Returns (state [np][H][W] nested lists, change, steps)."""
    W, H = params["dim_x"], params["dim_y"]
    n_morph = params["n_input_morphogens"] + params["n_target_morphogens"]
    labels = labels_in_use(products, links, n_morph)
    prods = {}
    for p in products:
        prods.setdefault(p["label"], p)
    np_ = len(labels)
    state = [[[0.0] * W for _ in range(H)] for _ in range(np_)]
    for k in range(min(params["n_input_morphogens"], np_)):
        for y in range(H):
            for x in range(W):
                state[k][y][x] = float(initial[k][y][x])
    change, step = 1.0, 0
    dt, min_conc = params["dt"], params["min_conc"]
    while step < n_steps and change > params["min_conc_change"]:
        old = [[row[:] for row in plane] for plane in state]
        max_change = 0.0
        for y in range(H):
            for x in range(W):
                conc = [old[k][y][x] for k in range(np_)]
                for k, lab in enumerate(labels):
                    p = prods[lab]
                    reg = regulation(lab, labels, links, conc)
                    rate = p["lim"] * reg - p["deg"] * conc[k]
                    if p["dif"] > 0:
                        s, tot = 0.0, 0.0
                        if x > 0:
                            s += old[k][y][x - 1]; tot += 1
                        if x < W - 1:
                            s += old[k][y][x + 1]; tot += 1
                        if y > 0:
                            s += old[k][y - 1][x]; tot += 1
                        if y < H - 1:
                            s += old[k][y + 1][x]; tot += 1
                        if s > 0 or (tot > 0 and conc[k] > 0):
                            rate += p["dif"] * (s - tot * conc[k])
                    if rate != 0:  # NaN counts as non-zero, like `if (ratio)`
                        c = conc[k] + dt * rate
                        state[k][y][x] = 0.0 if c < min_conc else c
                        max_change = ref_max(max_change, abs(rate))
        change = max_change
        step += 1
    return state, change, step


def distance(params, state, target):
    W, H = params["dim_x"], params["dim_y"]
    n_in, n_t = params["n_input_morphogens"], params["n_target_morphogens"]
    d = 0.0
    if params.get("fitness_kind", 0) == 1:
        for x in range(W):
            for y in range(H):
                for k in range(n_t):
                    e = state[n_in + k][y][x] - target[k][y][x]
                    d += e * e
        return d / (W * H * n_t)
    for x in range(W):
        for y in range(H):
            for k in range(n_t):
                sub = abs(state[n_in + k][y][x] - target[k][y][x]) - params["dist_error_threshold"]
                if sub > 0:
                    d += math.log(1 + sub)
    return d / (W * H)


def ceil_s(n, d):
    if n == 0.0:
        return 0.0
    factor = math.pow(10.0, d - math.ceil(math.log10(abs(n))))
    return math.ceil(n * factor) / factor


def evaluate(params, initial, target, products, links, max_error):
    """Returns (rounded error, raw error, steps run)."""
    n_exp = len(initial)
    error, change, steps, i = 0.0, 0.0, 0, 0
    while i < n_exp and error <= max_error:
        state, ch, s = simulate(params, initial[i], products, links, params["num_sim_steps"])
        change += ch
        steps += s
        e = distance(params, state, target[i])
        if change > params["min_conc_change"]:
            e += change - params["min_conc_change"]
        error += e / n_exp
        i += 1
    rounded = 100.0 if error > max_error else ceil_s(error, params["error_precision"])
    return rounded, error, steps
