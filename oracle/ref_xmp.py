"""The reference XMP library as a second parity oracle -- TEST INFRASTRUCTURE ONLY.

ctypes bindings of oracle/_ref/libxmp_ref_<variant>.so, the reference's own
sources compiled for sm_100a by oracle/build_ref.sh (variant "imad": -DIMAD,
the 32-bit multiply-add path; "xmad": the reference's default 16-bit
emulation).  The tests run the same seeded inputs through this library and
through libxmp.so and require identical results; bench.py times it as the
same-box reference GPU figure.  The product never loads it.

Only inputs the reference handles with every lane of every warp active are
given to it (its warp-distributed kernels use full-mask shuffles, and its
digit-serial division and multiplication call __syncthreads inside their
per-instance loops):
  * instance counts that are multiples of 128 (whole blocks of its kernels),
    and for the digit-serial mul/divmod paths at most one wave, so that every
    thread runs exactly one instance;
  * powm above 512 bits with full-length moduli (top bit set): its a*R mod N
    set-up divides by the modulus with a loop whose trip count follows the
    modulus' leading zeros;
  * divmod with the divisor's top bit set, for the same reason.
`check_safe_*` enforce these before any call.

Host buffers: the reference tells host from device pointers with
cudaPointerGetAttributes and takes anything but cudaMemoryTypeHost for device
memory; since CUDA 11 pageable host memory reports cudaMemoryTypeUnregistered,
so a pageable buffer would be handed to its kernels as a device pointer.  Only
its native-order import/export (one cudaMemcpyDefault copy) takes pageable
memory here; the cmp/popc outputs and the shf shift array are device buffers,
and other import/export formats are refused.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")

ALG_DEFAULT, ALG_REGMP, ALG_DIGITMP, ALG_DISTRIBUTEDMP = 0, 1, 2, 3

_VP = ctypes.c_void_p
_U32 = ctypes.c_uint32
_I32 = ctypes.c_int32
_SZ = ctypes.c_size_t

_SIGS = {
    "xmpHandleCreate": [ctypes.POINTER(_VP)],
    "xmpHandleDestroy": [_VP],
    "xmpHandleSetExecutionPolicy": [_VP, _VP],
    "xmpExecutionPolicyCreate": [_VP, ctypes.POINTER(_VP)],
    "xmpExecutionPolicyDestroy": [_VP, _VP],
    "xmpExecutionPolicySetParameter": [_VP, _VP, ctypes.c_int, ctypes.c_uint64],
    "xmpIntegersCreate": [_VP, ctypes.POINTER(_VP), _U32, _U32],
    "xmpIntegersDestroy": [_VP, _VP],
    "xmpIntegersImport": [_VP, _VP, _U32, _I32, _SZ, _I32, _U32, _VP, _U32],
    "xmpIntegersExport": [_VP, _VP, ctypes.POINTER(_U32), _I32, _SZ, _I32, _U32, _VP, _U32],
    "xmpIntegersShf": [_VP, _VP, _VP, _VP, _U32, _U32],
    "xmpIntegersNot": [_VP, _VP, _VP, _U32],
    "xmpIntegersPopc": [_VP, _VP, _VP, _U32],
    "xmpIntegersCmp": [_VP, _VP, _VP, _VP, _U32],
    "xmpIntegersDivMod": [_VP, _VP, _VP, _VP, _VP, _U32],
    "xmpIntegersPowm": [_VP, _VP, _VP, _VP, _VP, _U32],
    "xmpIntegersPowmAsync": [_VP, _VP, _VP, _VP, _VP, _U32],
}
for _n in ("Add", "Sub", "Mul", "Ior", "And", "Xor"):
    _SIGS["xmpIntegers" + _n] = [_VP, _VP, _VP, _VP, _U32]


def path(variant="imad"):
    return os.path.join(REF_DIR, "libxmp_ref_%s.so" % variant)


def available(variant="imad"):
    return os.path.exists(path(variant))


class RefError(RuntimeError):
    pass


def _check(code, what):
    if code != 0:
        raise RefError("reference %s returned xmpError %d" % (what, code))


def check_safe_count(count, one_wave=False):
    if count % 128:
        raise ValueError("reference runs take whole blocks: count %d is not a multiple of 128" % count)
    if one_wave and count > 148 * 128:
        raise ValueError("reference digit-serial paths run one instance per thread: count %d exceeds one wave" % count)


def check_full_length(rows, what):
    if not np.all(rows[:, -1] & np.uint32(0x80000000)):
        raise ValueError("reference %s needs the top bit of every %s set" % (what, what))


class Ref:
    """One reference handle on the current CUDA device."""

    def __init__(self, variant="imad"):
        if not available(variant):
            raise FileNotFoundError(path(variant))
        L = ctypes.CDLL(path(variant))
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        self.lib = L
        h = _VP()
        _check(L.xmpHandleCreate(ctypes.byref(h)), "xmpHandleCreate")
        self.h = h
        self.policy = None
        self._arrays = []

    def set_algorithm(self, alg):
        if self.policy is None:
            p = _VP()
            _check(self.lib.xmpExecutionPolicyCreate(self.h, ctypes.byref(p)), "xmpExecutionPolicyCreate")
            self.policy = p
        _check(self.lib.xmpExecutionPolicySetParameter(self.h, self.policy, 0, alg), "SetParameter")
        _check(self.lib.xmpHandleSetExecutionPolicy(self.h, self.policy), "SetExecutionPolicy")

    def default_algorithm(self):
        if self.policy is not None:
            self.set_algorithm(ALG_DEFAULT)

    def integers(self, precision, count, rows=None):
        x = _VP()
        _check(self.lib.xmpIntegersCreate(self.h, ctypes.byref(x), precision, count), "xmpIntegersCreate")
        self._arrays.append(x)
        if rows is not None:
            self.import_(x, rows)
        return x

    def import_(self, x, rows, order=-1, size=4, endian=-1, nails=0):
        if (order, endian, nails) != (-1, -1, 0):
            raise ValueError("reference import of host rows only in its native format")
        rows = np.ascontiguousarray(rows)
        words = rows.shape[1] if rows.ndim == 2 else rows.size // rows.shape[0]
        _check(self.lib.xmpIntegersImport(self.h, x, words, order, size, endian, nails, rows.ctypes.data,
                                          rows.shape[0]), "xmpIntegersImport")

    def export(self, x, precision, count, order=-1, size=4, endian=-1, nails=0):
        if (order, endian, nails) != (-1, -1, 0):
            raise ValueError("reference export to host rows only in its native format")
        dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[size]
        out = np.zeros((count, precision // (8 * size)), dtype=dt)
        w = _U32(0)
        _check(self.lib.xmpIntegersExport(self.h, out.ctypes.data, ctypes.byref(w), order, size, endian, nails, x,
                                          count), "xmpIntegersExport")
        return out

    def binary(self, op, a, b, out_bits, count):
        """op in add, sub, mul, ior, and, xor on compact uint32 rows."""
        self.default_algorithm()
        check_safe_count(count, one_wave=(op == "mul"))
        A = self.integers(a.shape[1] * 32, a.shape[0], a)
        B = self.integers(b.shape[1] * 32, b.shape[0], b)
        C = self.integers(out_bits, count)
        name = {"add": "Add", "sub": "Sub", "mul": "Mul", "ior": "Ior", "and": "And", "xor": "Xor"}[op]
        _check(getattr(self.lib, "xmpIntegers" + name)(self.h, C, A, B, count), "xmpIntegers" + name)
        return self.export(C, out_bits, count)

    def not_(self, a, out_bits, count):
        self.default_algorithm()
        check_safe_count(count)
        A = self.integers(a.shape[1] * 32, a.shape[0], a)
        C = self.integers(out_bits, count)
        _check(self.lib.xmpIntegersNot(self.h, C, A, count), "xmpIntegersNot")
        return self.export(C, out_bits, count)

    def shf(self, a, shifts, out_bits, count):
        import torch
        self.default_algorithm()
        check_safe_count(count)
        A = self.integers(a.shape[1] * 32, a.shape[0], a)
        C = self.integers(out_bits, count)
        s = torch.from_numpy(np.ascontiguousarray(shifts, dtype=np.int32)).cuda()
        _check(self.lib.xmpIntegersShf(self.h, C, A, s.data_ptr(), s.numel(), count), "xmpIntegersShf")
        return self.export(C, out_bits, count)

    def cmp(self, a, b, count):
        import torch
        self.default_algorithm()
        check_safe_count(count)
        A = self.integers(a.shape[1] * 32, a.shape[0], a)
        B = self.integers(b.shape[1] * 32, b.shape[0], b)
        out = torch.zeros(count, dtype=torch.int32, device="cuda")
        _check(self.lib.xmpIntegersCmp(self.h, out.data_ptr(), A, B, count), "xmpIntegersCmp")
        torch.cuda.synchronize()
        return out.cpu().numpy()

    def popc(self, a, count):
        import torch
        self.default_algorithm()
        check_safe_count(count)
        A = self.integers(a.shape[1] * 32, a.shape[0], a)
        out = torch.zeros(count, dtype=torch.int32, device="cuda")
        _check(self.lib.xmpIntegersPopc(self.h, out.data_ptr(), A, count), "xmpIntegersPopc")
        torch.cuda.synchronize()
        return out.cpu().numpy().view(np.uint32)

    def divmod_(self, a, b, count):
        self.default_algorithm()
        check_safe_count(count, one_wave=True)
        check_full_length(b, "divisor")
        A = self.integers(a.shape[1] * 32, a.shape[0], a)
        B = self.integers(b.shape[1] * 32, b.shape[0], b)
        Q = self.integers(a.shape[1] * 32, count)
        R = self.integers(b.shape[1] * 32, count)
        _check(self.lib.xmpIntegersDivMod(self.h, Q, R, A, B, count), "xmpIntegersDivMod")
        return self.export(Q, a.shape[1] * 32, count), self.export(R, b.shape[1] * 32, count)

    def powm_arrays(self, base, exp, mod):
        """Device arrays (out, base, exp, mod) for repeated powm calls.

        Up to 512 bits the per-thread algorithm is requested, above it the
        warp-distributed one.  Above 512 bits the reference splits a call into
        launches of whole waves of its chosen kernel (instances per SM from
        its tuning table times the SM count) plus a tail; at most 4,096
        instances fit one wave of every distributed kernel at 1024 and 2048
        bits, and 65,536 x 2048 bits splits into 56,832 + 8,704 instances on
        148 SMs, both whole blocks.  Other shapes above 512 bits are refused."""
        count, n = mod.shape
        check_safe_count(count)
        bits = 32 * n
        if bits > 512:
            check_full_length(mod, "modulus")
            if not (count <= 4096 and bits in (1024, 1536, 2048)) and (bits, count) != (2048, 65536):
                raise ValueError("reference powm at %d bits x %d instances is not a checked launch shape"
                                 % (bits, count))
            self.set_algorithm(ALG_DISTRIBUTEDMP)
        else:
            self.set_algorithm(ALG_REGMP)
        return (self.integers(bits, count), self.integers(bits, count, base),
                self.integers(32 * exp.shape[1], count, exp), self.integers(bits, count, mod))

    def powm(self, base, exp, mod):
        count, n = mod.shape
        O, X, E, M = self.powm_arrays(base, exp, mod)
        _check(self.lib.xmpIntegersPowm(self.h, O, X, E, M, count), "xmpIntegersPowm")
        return self.export(O, 32 * n, count)

    def powm_async(self, O, X, E, M, count):
        _check(self.lib.xmpIntegersPowmAsync(self.h, O, X, E, M, count), "xmpIntegersPowmAsync")

    def close(self):
        for x in self._arrays:
            self.lib.xmpIntegersDestroy(self.h, x)
        self._arrays = []
        if self.policy is not None:
            self.lib.xmpExecutionPolicyDestroy(self.h, self.policy)
            self.policy = None
        if self.h:
            self.lib.xmpHandleDestroy(self.h)
            self.h = None
