"""CPU restatement of the learned selector's network -- TEST INFRASTRUCTURE ONLY.

Mirrors xmp_b200/csrc/selector.cu (features, 4 -> 64 -> 64 -> 48 MLP with ReLU,
mean squared error of log2(ms) over valid entries) in float64 numpy, with an
analytic backward pass.  tests/ check it against finite differences and then
check the CUDA gradients against it.
"""
import numpy as np

NIN, NH, NOUT = 4, 64, 48
OFF = {}
_o = 0
for name, size in (("W1", NIN * NH), ("b1", NH), ("W2", NH * NH), ("b2", NH), ("W3", NH * NOUT), ("b3", NOUT)):
    OFF[name] = (_o, _o + size)
    _o += size
NPARAMS = _o


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    g = lambda k: p[OFF[k][0]:OFF[k][1]]
    return g("W1").reshape(NIN, NH), g("b1"), g("W2").reshape(NH, NH), g("b2"), g("W3").reshape(NH, NOUT), g("b3")


def features(shapes):
    s = np.asarray(shapes, dtype=np.float64)
    op, bits, exp_bits, count = s[:, 0], s[:, 1], s[:, 2], s[:, 3]
    return np.stack([op - 1.0, (np.log2(np.maximum(bits, 1)) - 10.0) / 4.0,
                     (np.log2(np.maximum(count, 1)) - 13.0) / 7.0, (np.log2(exp_bits + 1.0) - 7.0) / 7.0], axis=1)


def targets(ms):
    ms = np.asarray(ms, dtype=np.float64)
    mask = np.isfinite(ms) & (ms > 0)
    t = np.where(mask, np.log2(np.where(mask, ms, 1.0)), 0.0)
    return t, mask.astype(np.float64)


def forward(p, x):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    h1 = np.maximum(x @ W1 + b1, 0.0)
    h2 = np.maximum(h1 @ W2 + b2, 0.0)
    return h1, h2, h2 @ W3 + b3


def loss_and_grad(p, shapes, ms):
    x = features(shapes)
    t, mask = targets(ms)
    W1, b1, W2, b2, W3, b3 = unpack(p)
    h1, h2, y = forward(p, x)
    cnt = mask.sum()
    d = (y - t) * mask
    loss = (d * d).sum() / cnt
    dy = 2.0 * d / cnt
    gW3, gb3 = h2.T @ dy, dy.sum(0)
    dh2 = (dy @ W3.T) * (h2 > 0)
    gW2, gb2 = h1.T @ dh2, dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (h1 > 0)
    gW1, gb1 = x.T @ dh1, dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def init(seed=0):
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAMS)
    for name, fan in (("W1", NIN), ("W2", NH), ("W3", NH)):
        a, b = OFF[name]
        p[a:b] = rng.uniform(-1, 1, b - a) * np.sqrt(6.0 / fan)
    return p
