"""Python bindings of the B200-native XMP-compatible C API (libxmp.so).

The library itself is C/C++/CUDA behind the C ABI declared in include/xmp.h;
this module only binds it with ctypes for tests, benchmarks and scripting.
Names mirror the reference C API (src/include/xmp.h): Handle wraps
xmpHandle_t, Integers wraps xmpIntegers_t, Policy wraps xmpExecutionPolicy_t,
and the op functions (add, sub, mul, div, mod, divmod, powm, shf, ior, and_,
xor, not_, popc, cmp) call the synchronous xmpIntegers* entry points.
Any non-success xmpError_t raises XmpError carrying the code.
There is no CPU fallback: importing without a built libxmp.so raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libxmp.so")

ERROR_NAMES = [
    "xmpErrorSuccess", "xmpErrorInvalidDispatchTable", "xmpErrorInvalidParameter", "xmpErrorInvalidMalloc",
    "xmpErrorInvalidCudaMalloc", "xmpErrorInvalidCount", "xmpErrorInvalidDevice", "xmpErrorInvalidFormat",
    "xmpErrorInvalidPrecision", "xmpErrorIncreaseScratchLimit", "xmpErrorUnsupported", "xmpErrorUnspecified",
    "xmpErrorCuda",
]
ERR = {n: i for i, n in enumerate(ERROR_NAMES)}

ALG_DEFAULT, ALG_REGMP, ALG_DIGITMP, ALG_DISTRIBUTEDMP = 0, 1, 2, 3
PARAM_ALGORITHM, PARAM_SCRATCH_LIMIT = 0, 1


class XmpError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        name = ERROR_NAMES[code] if 0 <= code < len(ERROR_NAMES) else "xmpErrorUnknown(%d)" % code
        super().__init__("%s%s" % (name, (" in " + what) if what else ""))
        self.name = name


_lib = None

_VP = ctypes.c_void_p
_U32 = ctypes.c_uint32
_I32 = ctypes.c_int32
_SZ = ctypes.c_size_t

# name -> argtypes (restype is xmpError_t = int for all)
_SIGS = {
    "xmpHandleCreate": [ctypes.POINTER(_VP)],
    "xmpHandleCreateWithMemoryFunctions": [ctypes.POINTER(_VP), _VP, _VP, _VP, _VP],
    "xmpHandleDestroy": [_VP],
    "xmpHandleSetStream": [_VP, _VP],
    "xmpHandleGetStream": [_VP, ctypes.POINTER(_VP)],
    "xmpHandleSetExecutionPolicy": [_VP, _VP],
    "xmpHandleGetMemoryFunctions": [_VP, _VP, _VP, _VP, _VP],
    "xmpHandleSetCudaStream": [_VP, _VP],
    "xmpHandleGetCudaStream": [_VP, ctypes.POINTER(_VP)],
    "xmpHandleGetDevice": [_VP, ctypes.POINTER(_I32)],
    "xmpExecutionPolicyCreate": [_VP, ctypes.POINTER(_VP)],
    "xmpExecutionPolicyDestroy": [_VP, _VP],
    "xmpExecutionPolicySetIndices": [_VP, _VP, _U32, _VP, _U32],
    "xmpExecutionPolicySetIndicesAsync": [_VP, _VP, _U32, _VP, _U32],
    "xmpExecutionPolicySetParameter": [_VP, _VP, ctypes.c_int, ctypes.c_uint64],
    "xmpExecutionPolicyGetParameter": [_VP, _VP, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)],
    "xmpIntegersCreate": [_VP, ctypes.POINTER(_VP), _U32, _U32],
    "xmpIntegersDestroy": [_VP, _VP],
    "xmpIntegersGetPrecision": [_VP, _VP, ctypes.POINTER(_U32)],
    "xmpIntegersGetCount": [_VP, _VP, ctypes.POINTER(_U32)],
    "xmpIntegersImport": [_VP, _VP, _U32, _I32, _SZ, _I32, _U32, _VP, _U32],
    "xmpIntegersImportAsync": [_VP, _VP, _U32, _I32, _SZ, _I32, _U32, _VP, _U32],
    "xmpIntegersExport": [_VP, _VP, ctypes.POINTER(_U32), _I32, _SZ, _I32, _U32, _VP, _U32],
    "xmpIntegersExportAsync": [_VP, _VP, ctypes.POINTER(_U32), _I32, _SZ, _I32, _U32, _VP, _U32],
    "xmpIntegersSet": [_VP, _VP, _VP, _U32],
    "xmpIntegersSetAsync": [_VP, _VP, _VP, _U32],
    "xmpIntegersShf": [_VP, _VP, _VP, _VP, _U32, _U32],
    "xmpIntegersShfAsync": [_VP, _VP, _VP, _VP, _U32, _U32],
    "xmpIntegersNot": [_VP, _VP, _VP, _U32],
    "xmpIntegersNotAsync": [_VP, _VP, _VP, _U32],
    "xmpIntegersPopc": [_VP, _VP, _VP, _U32],
    "xmpIntegersPopcAsync": [_VP, _VP, _VP, _U32],
    "xmpIntegersCmp": [_VP, _VP, _VP, _VP, _U32],
    "xmpIntegersCmpAsync": [_VP, _VP, _VP, _VP, _U32],
    "xmpIntegersDivMod": [_VP, _VP, _VP, _VP, _VP, _U32],
    "xmpIntegersDivModAsync": [_VP, _VP, _VP, _VP, _VP, _U32],
    "xmpIntegersPowm": [_VP, _VP, _VP, _VP, _VP, _U32],
    "xmpIntegersPowmAsync": [_VP, _VP, _VP, _VP, _VP, _U32],
    "xmpIntegersPowmNoAlloc": [_VP, _VP, _VP, _VP, _VP, _U32, _U32, _U32, _U32],
    "xmpIntegersPowmCRT": [_VP] * 8 + [_U32],
    "xmpIntegersPowmCRTAsync": [_VP] * 8 + [_U32],
    "xmpPowmKernelCount": [ctypes.POINTER(_I32)],
    "xmpPowmKernelGet": [_I32, ctypes.POINTER(_I32), ctypes.POINTER(_I32)],
    "xmpPowmGetConfig": [_VP, _U32, _U32, _U32, _VP],
    "xmpIntegersPowmWithConfigAsync": [_VP, _VP, _VP, _VP, _VP, _U32, _VP],
    "xmpTuneCandidate": [_I32, _U32, _I32, ctypes.POINTER(_I32), _VP],
    "xmpTuneMeasure": [_VP, _VP, _I32, _VP],
    "xmpTuneSetChoice": [_VP, _VP, _I32],
    "xmpTuneGetChoice": [_VP, _VP, ctypes.POINTER(_I32), ctypes.POINTER(_I32)],
    "xmpTuneClear": [_VP],
    "xmpSelectorTrain": [_VP, _VP, _VP, _I32, _I32, ctypes.c_float, ctypes.c_uint64, _I32, _VP, _VP],
    "xmpSelectorGradients": [_VP, _VP, _VP, _VP, _I32, _VP, _VP],
    "xmpSelectorPredict": [_VP, _VP, _VP, _I32, _VP],
    "xmpSelectorLoad": [_VP, _VP],
    "xmpSelectorLoadEnsemble": [_VP, _VP, _I32],
    "xmpPowmBatchPlanCreate": [_VP, _VP, _I32, _VP, _I32, _I32, ctypes.POINTER(_VP)],
    "xmpPowmBatchPlanExecute": [_VP, _VP],
    "xmpPowmBatchPlanDestroy": [_VP, _VP],
    "xmpPowmBatchPlanInfo": [_VP, ctypes.POINTER(_I32), _VP, _VP, _VP, _VP, _I32],
    "xmpServerCreate": [_VP, _VP, _U32, _VP, ctypes.POINTER(_VP)],
    "xmpServerDestroy": [_VP],
    "xmpServerAddKeys": [_VP, _U32, _VP, _U32, ctypes.POINTER(_U32)],
    "xmpServerSubmit": [_VP, _U32, _U32, _VP, _VP, _VP, ctypes.POINTER(ctypes.c_uint64)],
    "xmpServerWait": [_VP, ctypes.c_uint64, _U32, ctypes.POINTER(_I32)],
    "xmpServerStats": [_VP, _VP],
    "xmpServerReplay": [_VP, _U32, _VP, _VP, _VP, _VP, _VP, _VP, _I32, _VP, ctypes.POINTER(ctypes.c_double)],
}
for _n in ("Add", "Sub", "Mul", "Div", "Mod", "Ior", "And", "Xor"):
    _SIGS["xmpIntegers" + _n] = [_VP, _VP, _VP, _VP, _U32]
    _SIGS["xmpIntegers" + _n + "Async"] = [_VP, _VP, _VP, _VP, _U32]

API_NAMES = sorted(_SIGS)


def lib():
    """Loads libxmp.so (built in tree by `python -m xmp_b200.build`)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libxmp.so is not built (%s); run `python -m xmp_b200.build`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def check(code, what=""):
    if code != 0:
        raise XmpError(code, what)


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):  # torch tensor
        return a.data_ptr()
    raise TypeError("unsupported buffer type %r" % type(a))


class Policy:
    def __init__(self, handle):
        self.handle = handle
        p = _VP()
        check(lib().xmpExecutionPolicyCreate(handle.h, ctypes.byref(p)), "xmpExecutionPolicyCreate")
        self.p = p

    def set_indices(self, which, indices):
        if indices is None:
            check(lib().xmpExecutionPolicySetIndices(self.handle.h, self.p, which, None, 0), "SetIndices")
            return
        idx = np.ascontiguousarray(indices, dtype=np.uint32)
        check(lib().xmpExecutionPolicySetIndices(self.handle.h, self.p, which, idx.ctypes.data, len(idx)),
              "xmpExecutionPolicySetIndices")

    def set_algorithm(self, alg):
        check(lib().xmpExecutionPolicySetParameter(self.handle.h, self.p, PARAM_ALGORITHM, alg), "SetParameter")

    def set_scratch_limit(self, nbytes):
        check(lib().xmpExecutionPolicySetParameter(self.handle.h, self.p, PARAM_SCRATCH_LIMIT, nbytes),
              "SetParameter")

    def get(self, param):
        v = ctypes.c_uint64(0)
        check(lib().xmpExecutionPolicyGetParameter(self.handle.h, self.p, param, ctypes.byref(v)), "GetParameter")
        return v.value

    def destroy(self):
        if self.p:
            check(lib().xmpExecutionPolicyDestroy(self.handle.h, self.p), "xmpExecutionPolicyDestroy")
            self.p = None


class Integers:
    """An xmpIntegers_t array of `count` integers of `precision` bits."""

    def __init__(self, handle, precision, count):
        self.handle = handle
        x = _VP()
        check(lib().xmpIntegersCreate(handle.h, ctypes.byref(x), precision, count), "xmpIntegersCreate")
        self.x = x
        self.precision = precision
        self.count = count
        self.nlimbs = precision // 32

    def import_(self, rows, count=None, words=None, order=-1, size=4, endian=-1, nails=0, asynchronous=False):
        """Imports compact rows (numpy array or device pointer)."""
        if isinstance(rows, np.ndarray):
            rows = np.ascontiguousarray(rows)
            if count is None:
                count = rows.shape[0]
            if words is None:
                words = rows.shape[1] if rows.ndim == 2 else self.precision // (8 * size)
        if words is None:
            words = self.precision // (8 * size)
        f = lib().xmpIntegersImportAsync if asynchronous else lib().xmpIntegersImport
        check(f(self.handle.h, self.x, words, order, size, endian, nails, _ptr(rows), count), "xmpIntegersImport")
        return self

    def export(self, count=None, order=-1, size=4, endian=-1, nails=0, out=None, asynchronous=False):
        count = self.count if count is None else count
        dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[size]
        words = self.nlimbs * 4 // size
        if out is None:
            out = np.zeros((count, words), dtype=dt)
        w = _U32(0)
        f = lib().xmpIntegersExportAsync if asynchronous else lib().xmpIntegersExport
        check(f(self.handle.h, _ptr(out), ctypes.byref(w), order, size, endian, nails, self.x, count),
              "xmpIntegersExport")
        return out

    def destroy(self):
        if self.x:
            check(lib().xmpIntegersDestroy(self.handle.h, self.x), "xmpIntegersDestroy")
            self.x = None


class Handle:
    def __init__(self):
        h = _VP()
        check(lib().xmpHandleCreate(ctypes.byref(h)), "xmpHandleCreate")
        self.h = h

    def set_stream(self, stream_ptr):
        check(lib().xmpHandleSetStream(self.h, stream_ptr), "xmpHandleSetStream")

    def get_stream(self):
        s = _VP()
        check(lib().xmpHandleGetStream(self.h, ctypes.byref(s)), "xmpHandleGetStream")
        return s.value or 0

    def set_policy(self, policy):
        check(lib().xmpHandleSetExecutionPolicy(self.h, policy.p if policy else None), "SetExecutionPolicy")

    def integers(self, precision, count, rows=None):
        x = Integers(self, precision, count)
        if rows is not None:
            x.import_(rows)
        return x

    def policy(self):
        return Policy(self)

    def destroy(self):
        if self.h:
            check(lib().xmpHandleDestroy(self.h), "xmpHandleDestroy")
            self.h = None


def _x(v):
    return v.x if isinstance(v, Integers) else v


def _binary(name):
    def f(h, c, a, b, count, asynchronous=False):
        fn = getattr(lib(), "xmpIntegers" + name + ("Async" if asynchronous else ""))
        check(fn(h.h, _x(c), _x(a), _x(b), count), "xmpIntegers" + name)
    f.__name__ = name.lower()
    return f


add = _binary("Add")
sub = _binary("Sub")
mul = _binary("Mul")
div = _binary("Div")
mod = _binary("Mod")
ior = _binary("Ior")
and_ = _binary("And")
xor = _binary("Xor")


def not_(h, c, a, count, asynchronous=False):
    fn = lib().xmpIntegersNotAsync if asynchronous else lib().xmpIntegersNot
    check(fn(h.h, _x(c), _x(a), count), "xmpIntegersNot")


def divmod_(h, q, r, a, b, count, asynchronous=False):
    fn = lib().xmpIntegersDivModAsync if asynchronous else lib().xmpIntegersDivMod
    check(fn(h.h, _x(q), _x(r), _x(a), _x(b), count), "xmpIntegersDivMod")


class PowmConfig(ctypes.Structure):
    """xmpPowmConfig_t (include/xmp_b200.h)."""
    _fields_ = [("distribution", ctypes.c_int32), ("lanes", ctypes.c_int32), ("limbs", ctypes.c_int32),
                ("window", ctypes.c_int32)]

    def __repr__(self):
        return "PowmConfig(dist=%d, lanes=%d, limbs=%d, window=%d)" % (self.distribution, self.lanes, self.limbs,
                                                                        self.window)


def powm_kernels():
    """(lanes, limbs) of every register powm kernel compiled into the library."""
    n = _I32(0)
    check(lib().xmpPowmKernelCount(ctypes.byref(n)))
    out = []
    for i in range(n.value):
        a, b = _I32(0), _I32(0)
        check(lib().xmpPowmKernelGet(i, ctypes.byref(a), ctypes.byref(b)))
        out.append((a.value, b.value))
    return out


def powm_get_config(h, precision, exp_precision, count):
    c = PowmConfig()
    check(lib().xmpPowmGetConfig(h.h, precision, exp_precision, count, ctypes.byref(c)), "xmpPowmGetConfig")
    return c


def powm_with_config(h, out, base, exp, mod_, count, config):
    check(lib().xmpIntegersPowmWithConfigAsync(h.h, _x(out), _x(base), _x(exp), _x(mod_), count,
                                               ctypes.byref(config)), "xmpIntegersPowmWithConfigAsync")


class BatchItem(ctypes.Structure):
    """xmpPowmBatchItem_t: out = base^exp mod mod for `count` instances."""
    _fields_ = [("out", _VP), ("base", _VP), ("exp", _VP), ("mod", _VP), ("count", _U32)]


class CRTItem(ctypes.Structure):
    """xmpPowmCRTItem_t: out = c^d mod pq from (p, q, dp, dq, qinv)."""
    _fields_ = [("out", _VP), ("c", _VP), ("p", _VP), ("q", _VP), ("dp", _VP), ("dq", _VP), ("qinv", _VP),
                ("count", _U32)]


class BatchPlan:
    """A batched mixed-precision powm plan (xmpPowmBatchPlan_t)."""

    def __init__(self, h, items=(), crt=(), use_graph=True):
        self.h = h
        it = (BatchItem * max(1, len(items)))(*[BatchItem(_x(o), _x(b), _x(e), _x(m), c) for o, b, e, m, c in items])
        cr = (CRTItem * max(1, len(crt)))(*[CRTItem(*[_x(v) for v in row[:7]], row[7]) for row in crt])
        p = _VP()
        check(lib().xmpPowmBatchPlanCreate(h.h, it, len(items), cr, len(crt), 1 if use_graph else 0, ctypes.byref(p)),
              "xmpPowmBatchPlanCreate")
        self.p = p

    def execute(self):
        check(lib().xmpPowmBatchPlanExecute(self.h.h, self.p), "xmpPowmBatchPlanExecute")

    def info(self):
        n = _I32(0)
        prec = (_U32 * 64)()
        cnt = (_U32 * 64)()
        cfg = (PowmConfig * 64)()
        blk = (_I32 * 64)()
        check(lib().xmpPowmBatchPlanInfo(self.p, ctypes.byref(n), prec, cnt, cfg, blk, 64))
        return [dict(precision=prec[i], count=cnt[i], config=cfg[i], blocks=blk[i]) for i in range(n.value)]

    def destroy(self):
        if self.p:
            check(lib().xmpPowmBatchPlanDestroy(self.h.h, self.p), "xmpPowmBatchPlanDestroy")
            self.p = None


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_size_t), ("max_wave_ops", _U32), ("streams", _U32), ("max_keys", _U32),
                ("max_slots", _U32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("requests_submitted", ctypes.c_uint64), ("requests_completed", ctypes.c_uint64),
                ("ops_completed", ctypes.c_uint64), ("waves", ctypes.c_uint64),
                ("admission_stalls", ctypes.c_uint64), ("max_inflight_ops", _U32), ("classes", _U32),
                ("device_bytes", ctypes.c_size_t)]


class Server:
    """Continuous-batching modexp server (xmpServer_t).  Operand and result
    buffers are numpy uint32 arrays of shape (nops, precision / 32)."""

    def __init__(self, h, precisions, **config):
        self.h = h
        cfg = ServerConfig(**config)
        prec = (_U32 * len(precisions))(*precisions)
        p = _VP()
        check(lib().xmpServerCreate(h.h, prec, len(precisions), ctypes.byref(cfg), ctypes.byref(p)),
              "xmpServerCreate")
        self.s = p
        self._keep = {}

    def add_keys(self, precision, moduli):
        m = np.ascontiguousarray(moduli, dtype=np.uint32)
        first = _U32(0)
        check(lib().xmpServerAddKeys(self.s, precision, _ptr(m), m.shape[0], ctypes.byref(first)),
              "xmpServerAddKeys")
        return first.value

    def submit(self, key, bases, exps, out):
        """Queues out = bases^exps mod key (row-wise); returns the request id.
        The arrays are kept alive until wait() reports the request done."""
        b = np.ascontiguousarray(bases, dtype=np.uint32)
        e = np.ascontiguousarray(exps, dtype=np.uint32)
        assert out.flags.c_contiguous and out.dtype == np.uint32 and out.shape == b.shape
        rid = ctypes.c_uint64(0)
        check(lib().xmpServerSubmit(self.s, key, b.shape[0], _ptr(b), _ptr(e), _ptr(out), ctypes.byref(rid)),
              "xmpServerSubmit")
        self._keep[rid.value] = (b, e, out)
        return rid.value

    def wait(self, request, timeout_us=10_000_000):
        done = _I32(0)
        check(lib().xmpServerWait(self.s, request, timeout_us, ctypes.byref(done)), "xmpServerWait")
        if done.value:
            self._keep.pop(request, None)
        return bool(done.value)

    def stats(self):
        st = ServerStats()
        check(lib().xmpServerStats(self.s, ctypes.byref(st)), "xmpServerStats")
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def replay(self, keys, arrival_ns, bases, exps, outs, mode=0):
        """Open-loop replay; bases/exps/outs are lists of (nops, n) arrays.
        Returns (latency_ns array, seconds)."""
        n = len(keys)
        k = np.ascontiguousarray(keys, dtype=np.uint32)
        nops = np.array([b.shape[0] for b in bases], dtype=np.uint32)
        arr = np.ascontiguousarray(arrival_ns, dtype=np.uint64)
        bp = (ctypes.c_void_p * n)(*[b.ctypes.data for b in bases])
        ep = (ctypes.c_void_p * n)(*[e.ctypes.data for e in exps])
        op = (ctypes.c_void_p * n)(*[o.ctypes.data for o in outs])
        lat = np.zeros(n, dtype=np.uint64)
        secs = ctypes.c_double(0)
        check(lib().xmpServerReplay(self.s, n, _ptr(k), _ptr(nops), _ptr(arr), bp, ep, op, mode, _ptr(lat),
                                    ctypes.byref(secs)), "xmpServerReplay")
        return lat, secs.value

    def destroy(self):
        if self.s:
            check(lib().xmpServerDestroy(self.s), "xmpServerDestroy")
            self.s = None
            self._keep.clear()


def powm(h, out, base, exp, mod_, count, asynchronous=False):
    fn = lib().xmpIntegersPowmAsync if asynchronous else lib().xmpIntegersPowm
    check(fn(h.h, _x(out), _x(base), _x(exp), _x(mod_), count), "xmpIntegersPowm")


def powm_crt(h, out, c, p, q, dp, dq, qinv, count, asynchronous=False):
    """out = c^d mod pq from the CRT key (p, q, dp, dq, qinv) in one fused kernel (xmpIntegersPowmCRT)."""
    fn = lib().xmpIntegersPowmCRTAsync if asynchronous else lib().xmpIntegersPowmCRT
    check(fn(h.h, _x(out), _x(c), _x(p), _x(q), _x(dp), _x(dq), _x(qinv), count), "xmpIntegersPowmCRT")


def shf(h, c, a, shifts, count, shift_count=None):
    s = np.ascontiguousarray(shifts, dtype=np.int32) if isinstance(shifts, (list, np.ndarray)) else shifts
    n = len(s) if shift_count is None else shift_count
    check(lib().xmpIntegersShf(h.h, _x(c), _x(a), _ptr(s), n, count), "xmpIntegersShf")


def cmp(h, a, b, count, out=None):
    out = np.zeros(count, dtype=np.int32) if out is None else out
    check(lib().xmpIntegersCmp(h.h, _ptr(out), _x(a), _x(b), count), "xmpIntegersCmp")
    return out


def popc(h, a, count, out=None):
    out = np.zeros(count, dtype=np.uint32) if out is None else out
    check(lib().xmpIntegersPopc(h.h, _ptr(out), _x(a), count), "xmpIntegersPopc")
    return out
