"""The selector's CPU restatement (oracle/selector_ref.py) against finite
differences, and the tuning-grid / regret bookkeeping, without a GPU."""
import numpy as np

from oracle import selector_ref as ref


def _data(seed, n=12):
    rng = np.random.default_rng(seed)
    shapes = [(int(rng.integers(0, 3)), int(32 * rng.integers(4, 128)), int(rng.integers(0, 4096)),
               int(2 ** rng.integers(6, 20))) for _ in range(n)]
    ms = rng.uniform(0.01, 50.0, size=(n, 48))
    ms[rng.uniform(size=ms.shape) < 0.3] = -1.0  # invalid slots
    return shapes, ms


def test_gradient_matches_finite_differences():
    shapes, ms = _data(1)
    p = ref.init(3)
    loss, g = ref.loss_and_grad(p, shapes, ms)
    rng = np.random.default_rng(4)
    for k in rng.choice(ref.NPARAMS, 60, replace=False):
        e = np.zeros(ref.NPARAMS)
        e[k] = 1e-6
        num = (ref.loss_and_grad(p + e, shapes, ms)[0] - ref.loss_and_grad(p - e, shapes, ms)[0]) / 2e-6
        assert abs(num - g[k]) <= 1e-5 * max(1.0, abs(num)), (k, num, g[k])


def test_grid_and_regret_bookkeeping():
    from xmp_b200 import tuning
    g = tuning.grid(25.0)
    assert len(g) > 100
    assert {s[0] for s in g} == {0, 1, 2}
    tr, te, held = tuning.split_cells(g)
    cells = {(s[0], s[1]) for s in g}
    assert 0.15 <= len(held) / len(cells) <= 0.25
    assert not ({(g[i][0], g[i][1]) for i in tr} & set(held))
    # held-out shapes within the measured precisions: disjoint, complete, ~20%, deterministic
    tr2, te2 = tuning.split_shapes(g)
    assert not (set(tr2) & set(te2)) and sorted(tr2 + te2) == list(range(len(g)))
    assert 0.18 <= len(te2) / len(g) <= 0.22
    assert (tr2, te2) == tuning.split_shapes(g)
    assert set(tuning.splits(g)) == {"cells", "shapes"}
    row = np.full(48, -1.0, dtype=np.float32)
    row[[0, 1, 6]] = [2.0, 1.0, 4.0]
    row[7] = np.nan
    assert tuning.regret_of(row, 1) == 0.0
    assert abs(tuning.regret_of(row, 0) - 1.0) < 1e-9
    assert tuning.regret_of(row, 7) >= 3.0  # untimed window of a slow distribution


def test_window_rules_agree_on_dataset_exponents():
    """The evaluation maps a selector slot to the window the library would run with the
    sliding-window rule; the fixed-window kernels' rule must give the same window at every
    exponent length the dataset holds, or that mapping would be inexact for them."""
    from xmp_b200 import tuning
    lengths = {s[2] for s in tuning.grid(150.0) if s[0] == tuning.OPS["powm"]}
    assert lengths
    for k in sorted(lengths):
        assert tuning.analytic_window(k, sliding=True) == tuning.analytic_window(k, sliding=False), k

