"""Shared helpers for the tests: big-int <-> limb-row conversion, golden-case decoding."""
import numpy as np


def rows_from_ints(vals, nlimbs):
    out = np.zeros((len(vals), nlimbs), dtype=np.uint32)
    for i, v in enumerate(vals):
        v %= 1 << (32 * nlimbs)
        out[i] = np.frombuffer(v.to_bytes(4 * nlimbs, "little"), dtype="<u4")
    return out


def ints_from_rows(rows):
    rows = np.ascontiguousarray(rows, dtype="<u4")
    return [int.from_bytes(r.tobytes(), "little") for r in rows]


def hexs(col):
    return [int(v, 16) for v in col]


def cases(golden, op):
    return [c for c in golden["cases"] if c["op"] == op]
