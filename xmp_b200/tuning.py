"""Autotuning and the learned configuration selector (host orchestration).

The tuner and the selector themselves are C/CUDA in libxmp.so
(include/xmp_b200.h: xmpTuneMeasure, xmpSelectorTrain/Gradients/Predict/Load[Ensemble]);
this module drives them:

  collect  -- time every candidate configuration of every shape of the grid
              (op in {mul, divmod, powm} x bits x batch x powm exponent length)
              on the GPU with the exhaustive tuner; writes a dataset file;
  train    -- fit an ensemble of independently seeded selector MLPs with the
              library's CUDA training kernels on 80% of the shapes (--split
              shapes, the shipped selector) or on the shapes of 80% of the
              (op, bits) cells (--split cells); the members' mean prediction
              picks the configuration;
  evaluate -- regret t(chosen)/t(best) - 1 of the selector and of the built-in
              heuristic against the exhaustive tuner, on both held-out sets:
              shapes within the measured precisions, and whole precisions.

  python -m xmp_b200.tuning collect --out xmp_b200/tuning/b200_dataset.json
  python -m xmp_b200.tuning train --data xmp_b200/tuning/b200_dataset.json --out xmp_b200/tuning/b200_selector.f32

The selector only chooses a schedule, so every result stays bit-exact.
"""
import argparse
import ctypes
import json
import math
import os
import random
import time

import numpy as np

import xmp_b200 as xmp

OPS = {"mul": 0, "divmod": 1, "powm": 2}
OP_NAMES = {v: k for k, v in OPS.items()}
NCAND = 48
NPARAMS = 4 * 64 + 64 + 64 * 64 + 64 + 64 * 48 + 48
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_DATA = os.path.join(HERE, "tuning", "b200_dataset.json")
DEFAULT_WEIGHTS = os.path.join(HERE, "tuning", "b200_selector.f32")

BITS = [128, 192, 256, 384, 512, 768, 1024, 1536, 2048, 3072, 4096, 6144, 8192]
BATCH_LOG2 = list(range(6, 21, 2))  # 2^6 .. 2^20
EXP = [17, 256, 1024, None]          # None = full length


class Shape(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int32), ("bits", ctypes.c_uint32), ("exp_bits", ctypes.c_uint32),
                ("count", ctypes.c_uint32)]


def shapes_array(shapes):
    arr = (Shape * len(shapes))()
    for i, s in enumerate(shapes):
        arr[i] = Shape(*s)
    return arr


def estimated_ms(op, bits, exp_bits, count):
    """Rough cost of the best kernel, used only to keep the collection bounded."""
    n = max(count, 4096) / 65536.0
    if op == OPS["powm"]:
        return 260.0 * n * (bits / 2048.0) ** 2 * (exp_bits / 2048.0)
    per = (bits / 1024.0) ** 2 * (2.0 if op == OPS["divmod"] else 1.0)
    return 0.05 + 0.02 * per * max(count, 4096) / 4096.0


def grid(max_ms=25.0, max_count_log2=20):
    out = []
    for op in (OPS["mul"], OPS["divmod"], OPS["powm"]):
        for bits in BITS:
            for lb in BATCH_LOG2:
                if lb > max_count_log2:
                    continue
                count = 1 << lb
                exps = [None] if op != OPS["powm"] else EXP
                for e in exps:
                    eb = 0 if op != OPS["powm"] else (bits if e is None else e)
                    if estimated_ms(op, bits, eb, count) > max_ms:
                        continue
                    out.append((op, bits, eb, count))
    return out


def candidate_valid(op, bits):
    lib = xmp.lib()
    v = ctypes.c_int32(0)
    res = []
    for s in range(NCAND):
        xmp.check(lib.xmpTuneCandidate(op, bits, s, ctypes.byref(v), None), "xmpTuneCandidate")
        res.append(bool(v.value))
    return res


def measure(h, shape, reps=1):
    ms = np.zeros(NCAND, dtype=np.float32)
    sh = Shape(*shape)
    xmp.check(xmp.lib().xmpTuneMeasure(h.h, ctypes.byref(sh), reps, ms.ctypes.data), "xmpTuneMeasure")
    return ms


def collect(h, shapes, reps=1, log=None):
    rows = []
    t0 = time.time()
    for i, s in enumerate(shapes):
        ms = measure(h, s, reps)
        rows.append(ms)
        if log:
            v = ms[np.isfinite(ms) & (ms > 0)]
            log("%4d/%d %-6s bits=%5d exp=%5d count=%7d best=%.3f ms  (%.0f s)" % (
                i + 1, len(shapes), OP_NAMES[s[0]], s[1], s[2], s[3], v.min() if len(v) else -1, time.time() - t0))
    return np.stack(rows) if rows else np.zeros((0, NCAND), dtype=np.float32)


def save_dataset(path, shapes, ms, meta=None):
    doc = {"shapes": [list(map(int, s)) for s in shapes],
           "ms": [[None if not np.isfinite(v) else float(v) for v in row] for row in ms],
           "meta": meta or {}}
    with open(path, "w") as f:
        json.dump(doc, f)


def load_dataset(path):
    with open(path) as f:
        doc = json.load(f)
    shapes = [tuple(s) for s in doc["shapes"]]
    ms = np.array([[np.nan if v is None else v for v in row] for row in doc["ms"]], dtype=np.float32)
    return shapes, ms, doc.get("meta", {})


def split_cells(shapes, holdout=0.2, seed=7):
    """80/20 split by (op, bits) cell."""
    cells = sorted({(s[0], s[1]) for s in shapes})
    rnd = random.Random(seed)
    rnd.shuffle(cells)
    k = max(1, int(round(len(cells) * holdout)))
    held = set(cells[:k])
    train = [i for i, s in enumerate(shapes) if (s[0], s[1]) not in held]
    test = [i for i, s in enumerate(shapes) if (s[0], s[1]) in held]
    return train, test, sorted(held)


def split_shapes(shapes, holdout=0.2, seed=7):
    """80/20 split by shape within the measured precisions: every (op, bits) cell keeps most of its
    shapes for training and holds out the others (other batch sizes and exponent lengths at the
    same precision).  The held-out list is the selector's use within the precisions it was
    measured on; `split_cells` holds out whole precisions instead (extrapolation)."""
    rnd = random.Random(seed)
    idx = list(range(len(shapes)))
    rnd.shuffle(idx)
    k = max(1, int(round(len(shapes) * holdout)))
    held = set(idx[:k])
    return [i for i in range(len(shapes)) if i not in held], sorted(held)


def splits(shapes):
    """(train, heldout) indices of both evaluations: 'cells' (whole held-out precisions) and
    'shapes' (held-out shapes within the measured precisions)."""
    tr_c, te_c, _ = split_cells(shapes)
    tr_s, te_s = split_shapes(shapes)
    return {"cells": (tr_c, te_c), "shapes": (tr_s, te_s)}


def train(h, shapes, ms, epochs=3000, lr=3e-3, seed=1, params=None):
    p = np.zeros(NPARAMS, dtype=np.float32) if params is None else np.array(params, dtype=np.float32)
    loss = ctypes.c_float(0)
    sa = shapes_array(shapes)
    m = np.ascontiguousarray(np.where(np.isfinite(ms), ms, -1.0), dtype=np.float32)
    xmp.check(xmp.lib().xmpSelectorTrain(h.h, sa, m.ctypes.data, len(shapes), epochs, lr, seed,
                                         0 if params is None else 1, p.ctypes.data, ctypes.byref(loss)),
              "xmpSelectorTrain")
    return p, loss.value


def train_ensemble(h, shapes, ms, members=5, epochs=3000, lr=3e-3, seed=1):
    """`members` networks trained from seeds seed, seed+1, ...; parameters back to back."""
    ps, losses = [], []
    for k in range(members):
        p, loss = train(h, shapes, ms, epochs, lr, seed + k)
        ps.append(p)
        losses.append(loss)
    return np.concatenate(ps), losses


def members_of(params):
    p = np.ascontiguousarray(params, dtype=np.float32)
    assert p.size % NPARAMS == 0 and p.size > 0, "selector weights must be a multiple of %d floats" % NPARAMS
    return p.reshape(-1, NPARAMS)


def predict(h, params, shapes):
    """Predicted log2(ms) per slot; for an ensemble the members' mean (what the grid table uses)."""
    out = np.zeros((len(shapes), NCAND), dtype=np.float64)
    mem = members_of(params)
    for p in mem:
        pred = np.zeros((len(shapes), NCAND), dtype=np.float32)
        p = np.ascontiguousarray(p)
        xmp.check(xmp.lib().xmpSelectorPredict(h.h, p.ctypes.data, shapes_array(shapes), len(shapes),
                                               pred.ctypes.data), "xmpSelectorPredict")
        out += pred
    return (out / len(mem)).astype(np.float32)


def gradients(h, params, shapes, ms):
    g = np.zeros(NPARAMS, dtype=np.float32)
    loss = ctypes.c_float(0)
    p = np.ascontiguousarray(params, dtype=np.float32)
    m = np.ascontiguousarray(np.where(np.isfinite(ms), ms, -1.0), dtype=np.float32)
    xmp.check(xmp.lib().xmpSelectorGradients(h.h, p.ctypes.data, shapes_array(shapes), m.ctypes.data, len(shapes),
                                             ctypes.byref(loss), g.ctypes.data), "xmpSelectorGradients")
    return loss.value, g


def choose(pred_row, valid):
    best, bv = -1, float("inf")
    for s in range(NCAND):
        if valid[s] and pred_row[s] < bv:
            best, bv = s, pred_row[s]
    return best


_HEURISTIC = {}


def heuristic_slot(h, shape):
    """The built-in heuristic's choice (no tuned entries, no selector).  Asked of a
    handle of its own with the tuner cleared: every new handle starts with the
    compiled-in selector, whose choice xmpTuneGetChoice would report instead."""
    hh = _HEURISTIC.get("h")
    if hh is None:
        hh = _HEURISTIC["h"] = xmp.Handle()
        xmp.check(xmp.lib().xmpTuneClear(hh.h), "xmpTuneClear")
    s = ctypes.c_int32(0)
    src = ctypes.c_int32(0)
    xmp.check(xmp.lib().xmpTuneGetChoice(hh.h, ctypes.byref(Shape(*shape)), ctypes.byref(s), ctypes.byref(src)))
    assert src.value == 0
    return s.value


def analytic_window(exp_bits, wmax=7, sliding=True):
    """window_for_bits in the library: the window minimising the table build plus one multiply per
    window -- 1.25 * 2^(W-1) + ceil(k / (W+1)) for the register kernels' sliding window, (2^W - 2) +
    ceil(k / W) for the digit-serial kernel's fixed window."""
    if exp_bits <= 1:
        return 1
    best, cost = 1, None
    for w in range(1, wmax + 1):
        c = 1.25 * (1 << (w - 1)) + -(-exp_bits // (w + 1)) if sliding else (1 << w) - 2 + -(-exp_bits // w)
        if cost is None or c < cost:
            best, cost = w, c
    return best


def runtime_slot(shape, slot):
    """The configuration the library runs for a selector choice (tuner_lookup_powm): for powm the
    chosen kernel with the chosen window kept within one of the analytic window's (the analytic
    window alone where it is beyond the six windows the tuner times).  Register kernels take the
    sliding-window rule here; the fixed-window kernels' rule gives the same window at every
    exponent length of the dataset (17, 256, 1024 and the full precisions)."""
    if shape[0] != OPS["powm"]:
        return slot
    d, w = slot // 6, slot % 6 + 1
    wa = analytic_window(shape[2], sliding=d < 6)
    if wa > 6:
        return d * 6 + 5
    return d * 6 + max(wa - 1, min(wa + 1, w)) - 1


def regret_of(ms_row, slot):
    """t(slot)/t(best) - 1; a slot left untimed (NaN) counts as its distribution's first timing (a lower bound)."""
    finite = ms_row[np.isfinite(ms_row) & (ms_row > 0)]
    best = finite.min()
    t = ms_row[slot]
    if not np.isfinite(t) or t <= 0:
        if t < 0:
            return float("inf")
        # untimed window of a hopeless distribution: charge the distribution's slowest timed window
        d = slot // 6
        same = ms_row[d * 6:(d + 1) * 6]
        same = same[np.isfinite(same) & (same > 0)]
        t = same.max() if len(same) else best * 20
    return float(t / best - 1.0)


def evaluate(h, params, shapes, ms, idx):
    pred = predict(h, params, [shapes[i] for i in idx]) if len(idx) else np.zeros((0, NCAND))
    sel, heu = [], []
    for k, i in enumerate(idx):
        valid = candidate_valid(shapes[i][0], shapes[i][1])
        sel.append(regret_of(ms[i], runtime_slot(shapes[i], choose(pred[k], valid))))
        heu.append(regret_of(ms[i], heuristic_slot(h, shapes[i])))
    sel, heu = np.array(sel), np.array(heu)
    return {"n": len(idx), "selector_mean_regret": float(sel.mean()) if len(sel) else None,
            "selector_median_regret": float(np.median(sel)) if len(sel) else None,
            "selector_max_regret": float(sel.max()) if len(sel) else None,
            "heuristic_mean_regret": float(heu.mean()) if len(heu) else None,
            "heuristic_median_regret": float(np.median(heu)) if len(heu) else None,
            "heuristic_max_regret": float(heu.max()) if len(heu) else None}


def save_weights(path, params):
    np.asarray(params, dtype="<f4").tofile(path)


def load_weights(path=DEFAULT_WEIGHTS):
    p = np.fromfile(path, dtype="<f4")
    members_of(p)
    return p


def install(h, params):
    """Loads a trained selector (one network or an ensemble) into the handle (CUDA grid inference ->
    lookup table)."""
    mem = members_of(params)
    p = np.ascontiguousarray(mem.reshape(-1))
    xmp.check(xmp.lib().xmpSelectorLoadEnsemble(h.h, p.ctypes.data, len(mem)), "xmpSelectorLoadEnsemble")


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--out", default=DEFAULT_DATA)
    c.add_argument("--max-ms", type=float, default=25.0)
    c.add_argument("--reps", type=int, default=1)
    c.add_argument("--append", default=None,
                   help="existing dataset: only shapes it lacks are timed, the result is the union")
    t = sub.add_parser("train")
    t.add_argument("--data", default=DEFAULT_DATA)
    t.add_argument("--out", default=DEFAULT_WEIGHTS)
    t.add_argument("--epochs", type=int, default=4000)
    t.add_argument("--lr", type=float, default=3e-3)
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--members", type=int, default=5, help="ensemble size (seeds seed .. seed+members-1)")
    t.add_argument("--report", default=None)
    t.add_argument("--split", default="shapes", choices=["shapes", "cells"],
                   help="training shapes: all but the held-out shapes (default) or all but the held-out cells")
    ev = sub.add_parser("evaluate", help="regret of given weights on a dataset's held-out and training cells")
    ev.add_argument("--data", default=DEFAULT_DATA)
    ev.add_argument("--weights", default=DEFAULT_WEIGHTS)
    ev.add_argument("--report", default=None)
    a = ap.parse_args()
    import torch
    torch.cuda.set_device(0)
    h = xmp.Handle()
    if a.cmd == "collect":
        shapes = grid(a.max_ms)
        meta = {"device": torch.cuda.get_device_name(0), "reps": a.reps, "max_ms": a.max_ms}
        old_shapes, old_ms = [], np.zeros((0, NCAND), dtype=np.float32)
        if a.append:
            old_shapes, old_ms, old_meta = load_dataset(a.append)
            meta["appended_to"] = old_meta
            have = set(old_shapes)
            shapes = [s for s in shapes if s not in have]
        ms = collect(h, shapes, a.reps, log=lambda s: print(s, flush=True))
        save_dataset(a.out, list(old_shapes) + list(shapes), np.concatenate([old_ms, ms]), meta)
    elif a.cmd == "evaluate":
        shapes, ms, meta = load_dataset(a.data)
        params = load_weights(a.weights)
        _, _, held = split_cells(shapes)
        rep = {"weights": os.path.basename(a.weights), "heldout_cells": [[OP_NAMES[o], b] for o, b in held]}
        for name, (tr, te) in splits(shapes).items():
            rep[name] = {"heldout": evaluate(h, params, shapes, ms, te), "train": evaluate(h, params, shapes, ms, tr)}
        print(json.dumps(rep, indent=1))
        if a.report:
            with open(a.report, "w") as f:
                json.dump(rep, f, indent=1)
    else:
        shapes, ms, meta = load_dataset(a.data)
        tr, te = splits(shapes)[a.split]
        _, _, held = split_cells(shapes)
        t0 = time.time()
        params, loss = train_ensemble(h, [shapes[i] for i in tr], ms[tr], a.members, a.epochs, a.lr, a.seed)
        rep = {"members": a.members, "split": a.split, "train_loss": loss, "train_seconds": time.time() - t0,
               "train_shapes": len(tr), "heldout": evaluate(h, params, shapes, ms, te),
               "train": evaluate(h, params, shapes, ms, tr)}
        if a.split == "cells":
            rep["heldout_cells"] = [[OP_NAMES[o], b] for o, b in held]
        save_weights(a.out, params)
        print(json.dumps(rep, indent=1))
        if a.report:
            with open(a.report, "w") as f:
                json.dump(rep, f, indent=1)
    h.destroy()


if __name__ == "__main__":
    main()
