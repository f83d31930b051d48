"""FP64 numpy restatement of the surrogate MLP (128-256-256-256-1, ReLU,
mean squared loss) for the tests: forward, backward and Adam, optionally
rounding operands to BF16 at the points where the CUDA kernels store BF16
(inputs, hidden activations, weight copies, hidden-layer deltas)."""
import numpy as np

F, H = 128, 256
SHAPES = [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)),
          ("b3", (H,)), ("w4", (H,)), ("b4", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16(a):
    """Round float32 values to the nearest BF16 (ties to even), as float64."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(p):
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], np.float64).reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SHAPES])


def forward(p, x, emulate_bf16=True):
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float64))
    P = unpack(p)
    X = r(x)
    h1 = r(np.maximum(X @ r(P["W1"]).T + P["b1"], 0))
    h2 = r(np.maximum(h1 @ r(P["W2"]).T + P["b2"], 0))
    h3 = r(np.maximum(h2 @ r(P["W3"]).T + P["b3"], 0))
    y = h3 @ P["w4"] + P["b4"][0]
    return y, (X, h1, h2, h3)


def loss_and_grads(p, x, t, emulate_bf16=True):
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float64))
    P = unpack(p)
    y, (X, h1, h2, h3) = forward(p, x, emulate_bf16)
    B = len(t)
    d = y - np.asarray(t, np.float64)
    loss = float(np.mean(d * d))
    dy = 2 * d / B
    g = {"w4": h3.T @ dy, "b4": np.array([dy.sum()])}
    dz3 = r(np.where(h3 > 0, dy[:, None] * P["w4"][None, :], 0))
    g["W3"], g["b3"] = dz3.T @ h2, dz3.sum(0)
    dz2 = r(np.where(h2 > 0, dz3 @ r(P["W3"]), 0))
    g["W2"], g["b2"] = dz2.T @ h1, dz2.sum(0)
    dz1 = r(np.where(h1 > 0, dz2 @ r(P["W2"]), 0))
    g["W1"], g["b1"] = dz1.T @ X, dz1.sum(0)
    return loss, pack(g)


def adam(p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return p, m, v


def spearman(a, b):
    ra = np.argsort(np.argsort(a)).astype(np.float64)
    rb = np.argsort(np.argsort(b)).astype(np.float64)
    ra -= ra.mean()
    rb -= rb.mean()
    return float((ra * rb).sum() / np.sqrt((ra * ra).sum() * (rb * rb).sum()))
