"""CPU oracle for the batched multi-precision path -- TEST INFRASTRUCTURE ONLY.

Python bindings of oracle/_build/libxmporacle.so (built from oracle/xmp_oracle.c
by oracle/Makefile).  Only tests/, the smoke test and bench.py's CPU-baseline
leg use it, as the checker; the product path never does.

Also holds the seeded workload generators shared by tests and bench
(splitmix64 limbs; full-length odd moduli; bases uniform in [0, m)).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libxmporacle.so")

OP = {"add": 0, "sub": 1, "and": 2, "ior": 3, "xor": 4, "mul": 5, "div": 6, "mod": 7}


class _In(ctypes.Structure):
    _fields_ = [("limbs", ctypes.c_void_p), ("n", ctypes.c_uint32), ("count", ctypes.c_uint32),
                ("index", ctypes.c_void_p), ("index_count", ctypes.c_uint32)]


class _Out(ctypes.Structure):
    _fields_ = [("limbs", ctypes.c_void_p), ("n", ctypes.c_uint32), ("count", ctypes.c_uint32),
                ("index", ctypes.c_void_p)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_binary.argtypes = [ctypes.c_int, _Out, _In, _In, ctypes.c_uint32, ctypes.c_int]
        L.oracle_divmod.argtypes = [_Out, _Out, _In, _In, ctypes.c_uint32, ctypes.c_int]
        L.oracle_not.argtypes = [_Out, _In, ctypes.c_uint32]
        L.oracle_shf.argtypes = [_Out, _In, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]
        L.oracle_cmp.argtypes = [ctypes.c_void_p, _In, _In, ctypes.c_uint32]
        L.oracle_popc.argtypes = [ctypes.c_void_p, _In, ctypes.c_uint32]
        L.oracle_powm.argtypes = [_Out, _In, _In, _In, ctypes.c_uint32, ctypes.c_int, ctypes.c_int]
        L.oracle_powm_mont.argtypes = [_Out, _In, _In, _In, ctypes.c_uint32]
        L.oracle_crt_key.argtypes = [ctypes.c_void_p] * 8 + []
        L.oracle_crt_key.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32] + [ctypes.c_void_p] * 6
        L.oracle_max_threads.argtypes = []
        _lib = L
    return _lib


def _keep(*arrs):
    return [np.ascontiguousarray(a, dtype=np.uint32) if a is not None else None for a in arrs]


def _in(rows, index=None):
    rows = np.ascontiguousarray(rows, dtype=np.uint32)
    idx = None if index is None else np.ascontiguousarray(index, dtype=np.uint32)
    s = _In(rows.ctypes.data, rows.shape[1], rows.shape[0], None if idx is None else idx.ctypes.data,
            0 if idx is None else len(idx))
    return s, (rows, idx)


def _out(nlimbs, count, index=None, init=None):
    out = np.zeros((count, nlimbs), dtype=np.uint32) if init is None else np.array(init, dtype=np.uint32, copy=True)
    idx = None if index is None else np.ascontiguousarray(index, dtype=np.uint32)
    s = _Out(out.ctypes.data, out.shape[1], out.shape[0], None if idx is None else idx.ctypes.data)
    return s, out, idx


def binary(op, a, b, out_limbs, count, out_count=None, out_index=None, a_index=None, b_index=None, init=None,
           threads=0):
    """out[o(i)] = op(a[ea(i)], b[eb(i)]) mod 2^(32 out_limbs) for i < count."""
    so, out, _i0 = _out(out_limbs, out_count or count, out_index, init)
    sa, _ka = _in(a, a_index)
    sb, _kb = _in(b, b_index)
    r = lib().oracle_binary(OP[op], so, sa, sb, count, threads)
    assert r == 0
    return out


def divmod_(a, b, q_limbs, r_limbs, count, q_count=None, r_count=None, q_index=None, r_index=None, a_index=None,
            b_index=None, q_init=None, r_init=None, threads=0):
    sq, q, _1 = _out(q_limbs, q_count or count, q_index, q_init)
    sr, r, _2 = _out(r_limbs, r_count or count, r_index, r_init)
    sa, _ka = _in(a, a_index)
    sb, _kb = _in(b, b_index)
    lib().oracle_divmod(sq, sr, sa, sb, count, threads)
    return q, r


def not_(a, out_limbs, count, out_count=None, out_index=None, a_index=None, init=None):
    so, out, _1 = _out(out_limbs, out_count or count, out_index, init)
    sa, _ka = _in(a, a_index)
    lib().oracle_not(so, sa, count)
    return out


def shf(a, shifts, out_limbs, count, out_count=None, out_index=None, a_index=None, init=None):
    so, out, _1 = _out(out_limbs, out_count or count, out_index, init)
    sa, _ka = _in(a, a_index)
    s = np.ascontiguousarray(shifts, dtype=np.int32)
    lib().oracle_shf(so, sa, s.ctypes.data, len(s), count)
    return out


def cmp(a, b, count, a_index=None, b_index=None):
    out = np.zeros(count, dtype=np.int32)
    sa, _ka = _in(a, a_index)
    sb, _kb = _in(b, b_index)
    lib().oracle_cmp(out.ctypes.data, sa, sb, count)
    return out


def popc(a, count, a_index=None):
    out = np.zeros(count, dtype=np.uint32)
    sa, _ka = _in(a, a_index)
    lib().oracle_popc(out.ctypes.data, sa, count)
    return out


def powm(base, exp, mod, count, out_count=None, out_index=None, base_index=None, exp_index=None, mod_index=None,
         init=None, threads=0, sec=False):
    """GMP mpz_powm (or mpz_powm_sec) per instance with XMP index rules."""
    so, out, _1 = _out(mod.shape[1], out_count or count, out_index, init)
    sb, _kb = _in(base, base_index)
    se, _ke = _in(exp, exp_index)
    sm, _km = _in(mod, mod_index)
    used = lib().oracle_powm(so, sb, se, sm, count, threads, 1 if sec else 0)
    return out, used


def powm_mont(base, exp, mod, count):
    """Plain-C fixed-window Montgomery restatement of the reference algorithm."""
    so, out, _1 = _out(mod.shape[1], count)
    sb, _kb = _in(base)
    se, _ke = _in(exp)
    sm, _km = _in(mod)
    lib().oracle_powm_mont(so, sb, se, sm, count)
    return out


def crt_key(p0, q0):
    hn = len(p0)
    p0, q0 = _keep(p0, q0)
    outs = [np.zeros(hn, dtype=np.uint32) for _ in range(5)]
    n = np.zeros(2 * hn, dtype=np.uint32)
    r = lib().oracle_crt_key(p0.ctypes.data, q0.ctypes.data, hn, *[o.ctypes.data for o in outs], n.ctypes.data)
    if r != 0:
        return None
    p, q, dp, dq, qinv = outs
    return dict(p=p, q=q, dp=dp, dq=dq, qinv=qinv, n=n)


def max_threads():
    return lib().oracle_max_threads()


# ---- seeded generators -------------------------------------------------------

_M64 = (1 << 64) - 1


def splitmix64(seed, n):
    """n outputs of the splitmix64 stream started at `seed` (numpy uint64)."""
    out = np.empty(n, dtype=np.uint64)
    s = seed & _M64
    # vectorised: state_k = seed + k * gamma
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(s) + k * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    out[:] = z
    return out


def random_limbs(seed, count, nlimbs):
    w = splitmix64(seed, (count * nlimbs + 1) // 2)
    return w.view(np.uint32)[: count * nlimbs].reshape(count, nlimbs).copy()


def full_length_odd(seed, count, nlimbs):
    """Uniform moduli with the top and bottom bits forced (odd, full length)."""
    m = random_limbs(seed, count, nlimbs)
    m[:, 0] |= np.uint32(1)
    m[:, -1] |= np.uint32(0x80000000)
    return m


def below(seed, mod):
    """Per row x uniform in [0, m) by rejection on the top limb, then exact check."""
    count, n = mod.shape
    x = random_limbs(seed, count, n)
    # x mod m on the top limb keeps it below m's top limb; fix up exact order with Python ints where needed
    top_m = mod[:, -1].astype(np.uint64)
    x[:, -1] = (x[:, -1].astype(np.uint64) % np.maximum(top_m, 1)).astype(np.uint32)
    return x


def to_int(row):
    return int.from_bytes(np.ascontiguousarray(row, dtype="<u4").tobytes(), "little")


def from_int(v, nlimbs):
    return np.frombuffer((v % (1 << (32 * nlimbs))).to_bytes(4 * nlimbs, "little"), dtype="<u4").copy()
