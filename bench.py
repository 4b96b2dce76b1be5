"""Benchmark of the batched modular-exponentiation hot path.

Workload (default): 2048-bit batched powm, 65,536 independent instances of
x^e mod m, uint32 limbs; m uniform odd full-length (top and bottom bits set)
from a seeded splitmix64 stream, x in [0, m), e a full-length random 2048-bit
exponent.  Metric: 2048-bit modexp/s (higher is better).

  value  -- whole-job modexp/s with operands resident in HBM: one
            xmpIntegersPowmAsync per step, timed with CUDA events on the
            launching stream, L2 flushed between steps (outside the events).
  e2e    -- the same metric through the public C API with host buffers:
            per step, xmpIntegersImport of base/exp/mod from pinned host memory,
            xmpIntegersPowm, xmpIntegersExport of the result to pinned host
            memory, all inside the timed region.
  roofline -- the powm kernel's algorithmic INT32 multiply-adds per launch
            (k + ceil(k/5)) * (4n^2 + n) per modexp, n = 64 limbs, k = 2048,
            over its event-timed duration, against the IMAD peak measured live
            by libxmpprobe.so on the same device.
  cpu_baseline -- GMP mpz_powm on the host's cores (OpenMP) on a bounded
            sample of the same instances (the oracle, as the reference's own
            perf harness compares against GMP, perf_tests/main.cu:153-229).

Multi-GPU (torchrun, one rank per GPU): replicas -- each rank runs its own
batch (weak scaling), value = all instances / max-over-ranks time.
`--impl reference` times the CPU reference path (GMP under OpenMP, all host
threads) on the same workload and prints the same JSON line.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# One hardware queue per stream for the serving workload's 32 streams (CUDA reads this when the
# context is created; work on a single stream, as in the other workloads, is unaffected).
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

L2_BYTES = 126 * 1024 * 1024


def imad_per_modexp(bits, ebits):
    n = bits // 32
    return (ebits + math.ceil(ebits / 5)) * (4 * n * n + n)


def replica_seed(rank):
    """Each replica (rank) works on its own seeded batch: no data is shared, so
    the ranks need no collective beyond the timing barrier and reduction."""
    return 2048 + 7919 * rank


def aggregate_over_ranks(dist, local_ms, device, instances_per_rank, steps, world):
    """Whole-job throughput from per-rank elapsed times: the max over ranks
    (the job ends when its slowest replica does) and every rank's instances.
    Returns (max_ms, instances per second)."""
    ms = local_ms
    if dist is not None:
        import torch
        t = torch.tensor([local_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, world * instances_per_rank * steps / (ms * 1e-3)


def make_inputs(bits, count, seed=2048):
    import oracle as orc  # seeded generators only
    n = bits // 32
    m = orc.full_length_odd(seed, count, n)
    x = orc.below(seed + 1, m)
    e = orc.random_limbs(seed + 2, count, n)
    e[:, -1] |= np.uint32(0x80000000)
    return x, e, m


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [q.strip() for q in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        loaded = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def profiled_traffic(bits, count):
    """DRAM bytes per powm launch from a committed ncu capture of this exact workload
    (dram__bytes_read.sum + dram__bytes_write.sum), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "powm_kernel_%dbit_traffic.json" % bits)) as f:
            d = json.load(f)
    except (OSError, ValueError):
        return None
    return d.get("dram_bytes_per_launch") if d.get("instances") == count else None


def probe_imad_peak():
    lib = ctypes.CDLL(os.path.join(ROOT, "xmp_b200", "libxmpprobe.so"))
    lib.xmpb_probe_imad.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double)]
    res = {}
    for mode, name in ((0, "imad"), (1, "carry_rows")):
        best = 0.0
        for _ in range(3):
            imads, ms = ctypes.c_double(), ctypes.c_double()
            rc = lib.xmpb_probe_imad(mode, 8, 2048, ctypes.byref(imads), ctypes.byref(ms))
            if rc != 0:
                raise RuntimeError("IMAD probe failed with CUDA error %d" % rc)
            best = max(best, imads.value / (ms.value * 1e-3))
        res[name] = best / 1e12
    return res


def cpu_gmp_rate(x, e, m, target_s=10.0, threads=0, sec=False):
    """GMP mpz_powm (sec: mpz_powm_sec, the side-channel-silent form the reference's perf harness
    times) over a bounded sample on all host threads; returns (ops/s, threads, sample, seconds)."""
    import oracle as orc
    count = len(m)
    n0 = min(count, 256)
    t = time.perf_counter()
    _, used = orc.powm(x[:n0], e[:n0], m[:n0], n0, threads=threads, sec=sec)
    dt = time.perf_counter() - t
    rate0 = n0 / max(dt, 1e-9)
    n1 = int(min(count, max(n0, rate0 * target_s)))
    t = time.perf_counter()
    _, used = orc.powm(x[:n1], e[:n1], m[:n1], n1, threads=threads, sec=sec)
    dt = time.perf_counter() - t
    return n1 / dt, used, n1, dt


def run_reference(args, rank, world):
    """CPU reference arm: GMP mpz_powm under OpenMP on all host threads (rank 0 only)."""
    if rank != 0:
        return
    x, e, m = make_inputs(args.bits, args.count)
    rates = []
    for step in range(args.warmup + args.steps):
        rate, used, sample, dt = cpu_gmp_rate(x, e, m, target_s=args.ref_seconds)
        if step >= args.warmup:
            rates.append(rate)
    value = statistics.median(rates)
    line = {
        "impl": "reference", "metric": "%d-bit modexp/s" % args.bits, "value": value, "unit": "modexp/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * args.count / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": "batched powm %d-bit, %d instances, full-length exponents" % (args.bits, args.count),
                   "bits": args.bits, "instances": args.count, "parallelism": "cpu"},
        "cpu_baseline": {"value": value, "unit": "modexp/s", "cores": used, "kind": "port",
                         "sample": "%d of the %d instances per step (GMP mpz_powm, OpenMP)" % (sample, args.count)},
        "e2e": {"value": value, "unit": "modexp/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _timed_events(fn, stream, flush, steps, warmup):
    """Per-step CUDA-event times (ms) on `stream`, L2 flushed before each step outside the events."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    evs = []
    for _ in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in evs]


def powm_rows(h, x, e, m):
    """x^e mod m row-wise through xmpIntegersPowm (this library)."""
    import xmp_b200 as xmp
    count, n = m.shape
    X, E, M, O = (h.integers(32 * n, count, v) for v in (x, e, m, None))
    try:
        xmp.powm(h, O, X, E, M, count)
        return O.export()
    finally:
        for v in (X, E, M, O):
            v.destroy()


def config1_suite(h, stream, flush, steps, warmup, imad_peak, cpu_seconds):
    """Plain batched powm, 4,096 independent 1024-bit instances with full-length exponents
    (seeded like the headline): device-resident modexp/s, IMAD roofline, end to end through
    the C API with pinned host buffers, GMP on the host, every result checked against GMP."""
    import torch
    import oracle as orc
    import xmp_b200 as xmp
    bits, count = 1024, 4096
    n = bits // 32
    x, e, m = make_inputs(bits, count)
    lib = xmp.lib()
    X, E, M, O = (h.integers(bits, count) for _ in range(4))
    for arr, rows in ((X, x), (E, e), (M, m)):
        arr.import_(rows)
    cfg = xmp.powm_get_config(h, bits, bits, count)

    def step():
        xmp.check(lib.xmpIntegersPowmAsync(h.h, O.x, X.x, E.x, M.x, count), "xmpIntegersPowmAsync")

    ms = statistics.median(_timed_events(step, stream, flush, steps, warmup))
    hx, he, hm = (torch.from_numpy(v).pin_memory() for v in (x, e, m))
    hout = torch.empty((count, n), dtype=torch.int32).pin_memory()
    w = ctypes.c_uint32(0)

    def e2e_step():
        for arr, buf in ((X, hx), (E, he), (M, hm)):
            xmp.check(lib.xmpIntegersImportAsync(h.h, arr.x, n, -1, 4, -1, 0, buf.data_ptr(), count), "Import")
        step()
        xmp.check(lib.xmpIntegersExportAsync(h.h, hout.data_ptr(), ctypes.byref(w), -1, 4, -1, 0, O.x, count),
                  "Export")

    e2e_ms = statistics.median(_timed_events(e2e_step, stream, flush, steps, warmup))
    want, _ = orc.powm(x, e, m, count)
    ok = bool(np.array_equal(hout.numpy().view(np.uint32), want))
    rate, used, sample, dt = cpu_gmp_rate(x, e, m, target_s=cpu_seconds)
    for v in (X, E, M, O):
        v.destroy()
    achieved = imad_per_modexp(bits, bits) * count / (ms * 1e-3) / 1e12
    return {"workload": "batched powm 1024-bit x 4096 instances, full-length exponents",
            "value": count / (ms * 1e-3), "unit": "modexp/s", "ms_per_step": ms,
            "kernel": {"lanes": cfg.lanes, "limbs": cfg.limbs, "window": cfg.window},
            "roofline": {"bound": "imad", "achieved": achieved, "peak": imad_peak, "unit": "TIMAD/s",
                         "frac": achieved / imad_peak},
            "e2e": {"value": count / (e2e_ms * 1e-3), "unit": "modexp/s", "h2d_bytes_per_step": 3 * count * n * 4,
                    "d2h_bytes_per_step": count * n * 4},
            "cpu_baseline": {"value": rate, "unit": "modexp/s", "cores": used, "kind": "port",
                             "sample": "%d instances (%.1f s, GMP mpz_powm via OpenMP)" % (sample, dt)},
            "result_check": ok}


def sweep_suite(h, stream, flush, imad_peak, counts=(4096, 16384, 65536, 262144), steps=3):
    """The 2048-bit workload (full-length exponents) over batch sizes 2^12 .. 2^18: modexp/s and the
    IMAD roofline fraction per size with the library's default choice, 32 results per size checked
    against GMP."""
    import oracle as orc
    import xmp_b200 as xmp
    bits, n = 2048, 64
    out = {}
    for count in counts:
        x, e, m = make_inputs(bits, count)
        X, E, M, O = (h.integers(bits, count) for _ in range(4))
        for arr, rows in ((X, x), (E, e), (M, m)):
            arr.import_(rows)
        cfg = xmp.powm_get_config(h, bits, bits, count)
        step = lambda: xmp.check(xmp.lib().xmpIntegersPowmAsync(h.h, O.x, X.x, E.x, M.x, count), "xmpIntegersPowmAsync")
        ms = statistics.median(_timed_events(step, stream, flush, steps, 1))
        want, _ = orc.powm(x[:32], e[:32], m[:32], 32)
        ok = bool(np.array_equal(O.export()[:32], want))
        achieved = imad_per_modexp(bits, bits) * count / (ms * 1e-3) / 1e12
        out[str(count)] = {"value": count / (ms * 1e-3), "unit": "modexp/s", "ms": ms, "imad_frac": achieved / imad_peak,
                           "kernel": {"distribution": cfg.distribution, "lanes": cfg.lanes, "limbs": cfg.limbs,
                                      "window": cfg.window}, "check": ok}
        for v in (X, E, M, O):
            v.destroy()
    return out


def latency_suite(h, stream, reps=5, sizes=(1024, 2048, 3072, 4096)):
    """One full-exponent modexp alone, per size, through xmpIntegersPowm: the library's default
    choice for a batch of one (one instance per CTA) and the fastest lane kernel for it (the
    warp-distributed heuristic), best of `reps` by CUDA events, both results checked against GMP."""
    import torch
    import oracle as orc
    import xmp_b200 as xmp
    out = {}
    for bits in sizes:
        x, e, m = make_inputs(bits, 1)
        X, E, M, O = (h.integers(bits, 1) for _ in range(4))
        for arr, rows in ((X, x), (E, e), (M, m)):
            arr.import_(rows)
        want, _ = orc.powm(x, e, m, 1)
        res = {}
        for name, alg in (("default", xmp.ALG_DEFAULT), ("lane_kernel", xmp.ALG_DISTRIBUTEDMP)):
            pol = xmp.Policy(h)
            pol.set_algorithm(alg)
            h.set_policy(pol)
            cfg = xmp.powm_get_config(h, bits, bits, 1)
            fn = lambda: xmp.check(xmp.lib().xmpIntegersPowmAsync(h.h, O.x, X.x, E.x, M.x, 1), "xmpIntegersPowmAsync")
            fn()
            torch.cuda.synchronize()
            ts = []
            for _ in range(reps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                fn()
                b.record(stream)
                torch.cuda.synchronize()
                ts.append(a.elapsed_time(b))
            h.set_policy(None)
            pol.destroy()
            res[name] = {"ms": min(ts), "distribution": cfg.distribution, "lanes": cfg.lanes, "limbs": cfg.limbs,
                         "check": bool(np.array_equal(O.export(), want))}
        out[str(bits)] = res
        for v in (X, E, M, O):
            v.destroy()
    return out


def reference_gpu_suite(stream, flush, steps, warmup, ours):
    """The reference XMP's own kernels on this GPU (oracle/_ref, built from its sources for
    sm_100a by oracle/build_ref.sh): modexp/s on the headline workload and the 1024-bit x 4,096
    workload, both variants (-DIMAD and its default XMAD emulation), device-resident operands,
    CUDA events on the default stream it launches on; results compared with this library's
    (`ours`: {(bits, count): rows})."""
    import torch
    from oracle import ref_xmp
    out = {}
    for variant in ("imad", "xmad"):
        if not ref_xmp.available(variant):
            out[variant] = {"unavailable": "oracle/_ref/libxmp_ref_%s.so not built" % variant}
            continue
        r = ref_xmp.Ref(variant)
        res = {}
        try:
            for (bits, count), rows in ours.items():
                x, e, m = make_inputs(bits, count)
                O, X, E, M = r.powm_arrays(x, e, m)
                dflt = torch.cuda.default_stream()
                with torch.cuda.stream(dflt):
                    ms = statistics.median(_timed_events(lambda: r.powm_async(O, X, E, M, count), dflt, flush,
                                                         steps, warmup))
                got = r.export(O, bits, count)
                res["%d_x_%d" % (bits, count)] = {"value": count / (ms * 1e-3), "unit": "modexp/s",
                                                  "ms_per_step": ms,
                                                  "identical_to_ours": bool(np.array_equal(got, rows))}
                r.close()
                r = ref_xmp.Ref(variant)
        finally:
            r.close()
        out[variant] = res
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    import xmp_b200 as xmp

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    stream = torch.cuda.current_stream()
    bits, count = args.bits, args.count
    n = bits // 32
    x, e, m = make_inputs(bits, count, seed=replica_seed(rank))

    h = xmp.Handle()
    h.set_stream(stream.cuda_stream)
    X, E, M, O = (h.integers(bits, count) for _ in range(4))
    for arr, rows in ((X, x), (E, e), (M, m)):
        arr.import_(rows)

    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device="cuda")
    lib = xmp.lib()

    forced = None
    if args.force_config:
        t, l, w = (int(v) for v in args.force_config.split(","))
        forced = xmp.PowmConfig(0, t, l, w)

    def step():
        if forced is not None:  # profiling aid: one kernel configuration regardless of the tuner
            xmp.check(lib.xmpIntegersPowmWithConfigAsync(h.h, O.x, X.x, E.x, M.x, count, ctypes.byref(forced)),
                      "xmpIntegersPowmWithConfigAsync")
        else:
            xmp.check(lib.xmpIntegersPowmAsync(h.h, O.x, X.x, E.x, M.x, count), "xmpIntegersPowmAsync")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- device-resident timing: per-step events, L2 flushed between steps ----
    sampler = ClockSampler(local_rank) if rank == 0 else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    evs = []
    for _ in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step()
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop() if sampler else None
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms, value = aggregate_over_ranks(dist, sum(step_ms), "cuda", count, args.steps, world)

    # ---- end-to-end through the C API with pinned host buffers ----
    hx = torch.from_numpy(x).pin_memory()
    he = torch.from_numpy(e).pin_memory()
    hm = torch.from_numpy(m).pin_memory()
    hout = torch.empty((count, n), dtype=torch.int32).pin_memory()
    out_w = ctypes.c_uint32(0)

    def e2e_step():
        for arr, buf in ((X, hx), (E, he), (M, hm)):
            xmp.check(lib.xmpIntegersImportAsync(h.h, arr.x, n, -1, 4, -1, 0, buf.data_ptr(), count), "Import")
        step()
        xmp.check(lib.xmpIntegersExportAsync(h.h, hout.data_ptr(), ctypes.byref(out_w), -1, 4, -1, 0, O.x, count),
                  "Export")

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        e2e_step()
    b.record(stream)
    torch.cuda.synchronize()
    e2e_ms, e2e_value = aggregate_over_ranks(dist, a.elapsed_time(b), "cuda", count, args.steps, world)

    # result check on a sample against the oracle (outside every timed region)
    res = hout.numpy().view(np.uint32)
    check_ok = None
    if rank == 0 and not args.no_check:
        import oracle as orc
        sample = np.arange(0, count, max(1, count // 64))
        want, _ = orc.powm(x[sample], e[sample], m[sample], len(sample))
        check_ok = bool(np.array_equal(res[sample], want))

    if rank != 0:
        return
    peaks = probe_imad_peak()
    algo = imad_per_modexp(bits, bits) * count  # per launch
    kernel_s = statistics.median(step_ms) * 1e-3
    achieved = algo / kernel_s / 1e12
    roofline = {"bound": "imad", "achieved": achieved, "peak": peaks["imad"], "unit": "TIMAD/s",
                "frac": achieved / peaks["imad"], "traffic": profiled_traffic(bits, count),
                "peak_source": "measured live: libxmpprobe independent mad.lo.u32 chains, all SMs",
                "carry_row_peak": peaks["carry_rows"],
                "algorithmic_imad_per_modexp": imad_per_modexp(bits, bits)}

    cpu = None
    if not args.no_cpu:
        rate, used, sample, dt = cpu_gmp_rate(x, e, m, target_s=args.cpu_seconds)
        rate1, _, sample1, dt1 = cpu_gmp_rate(x, e, m, target_s=max(1.0, args.cpu_seconds / 4), threads=1)
        rates, useds, samples, dts = cpu_gmp_rate(x, e, m, target_s=max(1.0, args.cpu_seconds / 4), sec=True)
        cpu = {"value": rate, "unit": "modexp/s", "cores": used, "kind": "port",
               "sample": "%d instances of the same workload (%.1f s, GMP mpz_powm via OpenMP)" % (sample, dt),
               "single_core": {"value": rate1, "sample": "%d instances (%.1f s, 1 thread)" % (sample1, dt1)},
               "powm_sec": {"value": rates, "cores": useds,
                            "sample": "%d instances (%.1f s, GMP mpz_powm_sec via OpenMP)" % (samples, dts)}}

    extra = None
    if world == 1 and not args.no_extra:
        # the other single-GPU workloads, measured after the headline's timed regions (rank 0, N = 1)
        t0 = time.perf_counter()
        extra = {}
        extra["config1_1024bit_x4096"] = config1_suite(h, stream, flush, args.steps, args.warmup, peaks["imad"],
                                                       min(args.cpu_seconds, 3.0))
        xx, ee, mm = make_inputs(1024, 4096)
        ours1 = {(bits, count): res.copy(), (1024, 4096): powm_rows(h, xx, ee, mm)}
        extra["reference_gpu"] = reference_gpu_suite(stream, flush, 3, 1, ours1)
        ew, ew_cpu, hbm = elementwise_suite(h, stream, 5, 2, peaks["imad"])
        extra["config2_elementwise"] = {"ops": ew, "cpu_baseline_ops_per_s": ew_cpu, "hbm_peak_gbs": hbm,
                                        "imad_peak_timad_s": peaks["imad"]}
        extra["config3_mixed"] = mixed_suite(3, 1, 65536, 16384, 256)
        extra["single_op_latency"] = latency_suite(h, stream)
        extra["powm2048_batch_sweep"] = sweep_suite(h, stream, flush, peaks["imad"])
        extra["config5_serving"] = serving_quick()
        extra["seconds"] = time.perf_counter() - t0

    line = {
        "metric": "%d-bit modexp/s" % bits, "value": value, "unit": "modexp/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded splitmix64 limbs)",
        "config": {"workload": "batched powm %d-bit x %d instances, full-length exponents" % (bits, count),
                   "bits": bits, "instances_per_gpu": count, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "flushed between steps (256 MB write outside the events)"},
        "e2e": {"value": e2e_value, "unit": "modexp/s", "h2d_bytes_per_step": int(3 * count * n * 4),
                "d2h_bytes_per_step": int(count * n * 4)},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": args.steps,
        "result_check": check_ok,
    }
    if extra is not None:
        line["extra_configs"] = extra
    print(json.dumps(line), flush=True)
    for v in (X, E, M, O):
        v.destroy()
    h.destroy()


def _crt_keys(nkeys, half_bits, seed):
    """RSA keys from GMP nextprime on seeded random starts (oracle generators, CPU)."""
    import oracle as orc
    keys, s = [], seed
    while len(keys) < nkeys:
        p0 = orc.random_limbs(s, 1, half_bits // 32)[0]
        q0 = orc.random_limbs(s + 1, 1, half_bits // 32)[0]
        p0[-1] |= np.uint32(0x80000000)
        q0[-1] |= np.uint32(0x80000000)
        s += 2
        k = orc.crt_key(p0, q0)
        if k is not None and orc.to_int(k["p"]) != orc.to_int(k["q"]):
            keys.append(k)
    return keys


def serving_quick():
    """The serving workload (config 5) with floors, peak, one moderate-rate run and the
    70%-of-peak point only.  Returns the p99 at 70% of peak and its parts, or the error."""
    try:
        d = serve_suite(quick=True, seconds=1.0, peak_requests=3000, sync_requests=0)
    except Exception as exc:  # noqa: BLE001 -- reported, not raised: the headline line still prints
        return {"error": "%s: %s" % (type(exc).__name__, exc)}
    at = d["at_70pct"]
    return {"metric": d["metric"], "value": d["value"], "unit": d["unit"], "peak_ops_per_s": d["peak_ops_per_s"],
            "offered_ops_per_s": at["offered_ops_per_s"], "delivered_ops_per_s": at["ops_per_s"],
            "p50_ms": at["p50_ms"], "p99_ms": at["p99_ms"], "p999_ms": at["p999_ms"], "by_bits": at["by_bits"],
            "single_op_latency_ms": d["single_op_latency_ms"], "result_check": d["result_check"],
            "config": d["config"]}


def mixed_suite(steps, warmup, total, ncrt, nkeys):
    """Uneven-size batch: 65,536 instances (40% 1024, 30% 2048, 20% 3072, 10% 4096 bits,
    full-length exponents, bases in [0, m)) plus 16,384 CRT-RSA private operations
    (1024-bit primes from nextprime, e = 65537, Garner with q^-1 mod p, messages
    uniform in [0, pq)).  Plain per-size xmpIntegersPowm calls and the CRT op
    sequence -- with the library's default (compiled-in selector) choices and with
    the static heuristic alone (a handle whose tuner is cleared) -- vs one
    autotuned batch plan replayed as a CUDA graph.  Returns the result dict."""
    import torch
    import oracle as orc
    import xmp_b200 as xmp
    from xmp_b200 import tuning
    torch.cuda.set_device(0)
    mix = [(1024, 0.4), (2048, 0.3), (3072, 0.2), (4096, 0.1)]
    sizes = [(b, int(total * f)) for b, f in mix]
    sizes[0] = (1024, total - sum(c for _, c in sizes[1:]))
    keys = _crt_keys(nkeys, 1024, 777)
    rng = np.random.default_rng(778)
    h = xmp.Handle()
    stream = torch.cuda.current_stream()
    h.set_stream(stream.cuda_stream)
    groups = []
    for k, (bits, cnt) in enumerate(sizes):
        n = bits // 32
        m = orc.full_length_odd(900 + k, cnt, n)
        x = orc.below(910 + k, m)
        e = orc.random_limbs(920 + k, cnt, n)
        e[:, -1] |= np.uint32(0x80000000)
        X, E, M = (h.integers(bits, cnt, v) for v in (x, e, m))
        groups.append(dict(bits=bits, count=cnt, X=X, E=E, M=M, O1=h.integers(bits, cnt), O2=h.integers(bits, cnt),
                           sample=(x[:16], e[:16], m[:16])))
    msgs, cts = [], []
    for i in range(ncrt):
        kk = keys[i % nkeys]
        nn = orc.to_int(kk["n"])
        mm = int.from_bytes(rng.bytes(256), "little") % nn
        msgs.append(mm)
        cts.append(pow(mm, 65537, nn))
    C = h.integers(2048, ncrt, np.stack([orc.from_int(c, 64) for c in cts]))
    ka = {f: h.integers(1024, nkeys, np.stack([kk[f] for kk in keys])) for f in ("p", "q", "dp", "dq", "qinv")}
    outs = [h.integers(2048, ncrt) for _ in range(2)]
    tmp = dict(cp=h.integers(1024, ncrt), cq=h.integers(1024, ncrt), mp=h.integers(1024, ncrt),
               mq=h.integers(1024, ncrt), p2=h.integers(1056, nkeys), t1=h.integers(1056, ncrt),
               d=h.integers(1056, ncrt), e=h.integers(2080, ncrt), hh=h.integers(1024, ncrt), f=h.integers(2048, ncrt))

    heur = xmp.Handle()  # the static register/occupancy heuristic only
    heur.set_stream(stream.cuda_stream)
    xmp.check(xmp.lib().xmpTuneClear(heur.h), "xmpTuneClear")

    def plain(h=h):
        for g in groups:
            xmp.check(xmp.lib().xmpIntegersPowmAsync(h.h, g["O1"].x, g["X"].x, g["E"].x, g["M"].x, g["count"]))
        L = xmp.lib()
        xmp.check(L.xmpIntegersModAsync(h.h, tmp["cp"].x, C.x, ka["p"].x, ncrt))
        xmp.check(L.xmpIntegersModAsync(h.h, tmp["cq"].x, C.x, ka["q"].x, ncrt))
        xmp.check(L.xmpIntegersPowmAsync(h.h, tmp["mp"].x, tmp["cp"].x, ka["dp"].x, ka["p"].x, ncrt))
        xmp.check(L.xmpIntegersPowmAsync(h.h, tmp["mq"].x, tmp["cq"].x, ka["dq"].x, ka["q"].x, ncrt))
        xmp.check(L.xmpIntegersAddAsync(h.h, tmp["p2"].x, ka["p"].x, ka["p"].x, nkeys))
        xmp.check(L.xmpIntegersAddAsync(h.h, tmp["t1"].x, tmp["mp"].x, tmp["p2"].x, ncrt))
        xmp.check(L.xmpIntegersSubAsync(h.h, tmp["d"].x, tmp["t1"].x, tmp["mq"].x, ncrt))
        xmp.check(L.xmpIntegersMulAsync(h.h, tmp["e"].x, tmp["d"].x, ka["qinv"].x, ncrt))
        xmp.check(L.xmpIntegersModAsync(h.h, tmp["hh"].x, tmp["e"].x, ka["p"].x, ncrt))
        xmp.check(L.xmpIntegersMulAsync(h.h, tmp["f"].x, ka["q"].x, tmp["hh"].x, ncrt))
        xmp.check(L.xmpIntegersAddAsync(h.h, outs[0].x, tmp["f"].x, tmp["mq"].x, ncrt))

    # autotuned batch plan, replayed as a graph (every handle starts with the compiled-in selector)
    selector = os.path.exists(tuning.DEFAULT_WEIGHTS)
    plan = xmp.BatchPlan(h, [(g["O2"], g["X"], g["E"], g["M"], g["count"]) for g in groups],
                         [(outs[1], C, ka["p"], ka["q"], ka["dp"], ka["dq"], ka["qinv"], ncrt)], use_graph=True)

    def timed(fn, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return float(np.median(ts))

    # plain launches use the library's default choices (the compiled-in selector), as any caller gets
    t_plain = timed(plain, steps, warmup)
    t_heur = timed(lambda: plain(heur), steps, warmup)
    t_batch = timed(plan.execute, steps, warmup)
    # the CRT part alone: the op sequence above vs one fused xmpIntegersPowmCRT launch
    L = xmp.lib()
    crt_out = h.integers(2048, ncrt)

    def crt_seq():
        xmp.check(L.xmpIntegersModAsync(h.h, tmp["cp"].x, C.x, ka["p"].x, ncrt))
        xmp.check(L.xmpIntegersModAsync(h.h, tmp["cq"].x, C.x, ka["q"].x, ncrt))
        xmp.check(L.xmpIntegersPowmAsync(h.h, tmp["mp"].x, tmp["cp"].x, ka["dp"].x, ka["p"].x, ncrt))
        xmp.check(L.xmpIntegersPowmAsync(h.h, tmp["mq"].x, tmp["cq"].x, ka["dq"].x, ka["q"].x, ncrt))
        xmp.check(L.xmpIntegersAddAsync(h.h, tmp["p2"].x, ka["p"].x, ka["p"].x, nkeys))
        xmp.check(L.xmpIntegersAddAsync(h.h, tmp["t1"].x, tmp["mp"].x, tmp["p2"].x, ncrt))
        xmp.check(L.xmpIntegersSubAsync(h.h, tmp["d"].x, tmp["t1"].x, tmp["mq"].x, ncrt))
        xmp.check(L.xmpIntegersMulAsync(h.h, tmp["e"].x, tmp["d"].x, ka["qinv"].x, ncrt))
        xmp.check(L.xmpIntegersModAsync(h.h, tmp["hh"].x, tmp["e"].x, ka["p"].x, ncrt))
        xmp.check(L.xmpIntegersMulAsync(h.h, tmp["f"].x, ka["q"].x, tmp["hh"].x, ncrt))
        xmp.check(L.xmpIntegersAddAsync(h.h, outs[0].x, tmp["f"].x, tmp["mq"].x, ncrt))

    t_crt_seq = timed(crt_seq, steps, warmup)
    t_crt_fused = timed(lambda: xmp.powm_crt(h, crt_out, C, ka["p"], ka["q"], ka["dp"], ka["dq"], ka["qinv"], ncrt,
                                             asynchronous=True), steps, warmup)
    crt_ok = [orc.to_int(r) for r in crt_out.export()[:256]] == msgs[:256]
    crt_out.destroy()
    # the plain launches one at a time: their sum bounds what any schedule of the same kernels can gain
    parts = {}
    for g in groups:
        parts["powm%d" % g["bits"]] = timed(lambda g=g: xmp.check(xmp.lib().xmpIntegersPowmAsync(
            h.h, g["O1"].x, g["X"].x, g["E"].x, g["M"].x, g["count"])), 2, 1)
    parts["crt"] = t_plain - sum(parts.values())
    ok = all(np.array_equal(g["O1"].export(), g["O2"].export()) for g in groups)
    res = [orc.to_int(r) for r in outs[1].export()[:256]]
    ok = ok and res == msgs[:256] and np.array_equal(outs[0].export(), outs[1].export())
    x, e, m = groups[1]["sample"]
    want, _ = orc.powm(x, e, m, len(m))
    ok = ok and np.array_equal(groups[1]["O2"].export()[:16], want)
    n_ops = total + ncrt
    out = {"speedup_vs_plain_selector": t_plain / t_batch, "speedup_vs_plain_heuristic": t_heur / t_batch,
           "crt_rsa2048_x%d" % ncrt: {"op_sequence_ms": t_crt_seq, "fused_kernel_ms": t_crt_fused,
                                      "speedup": t_crt_seq / t_crt_fused, "fused_result_check": crt_ok},
           "plain_ms": t_plain, "plain_heuristic_ms": t_heur, "batch_ms": t_batch, "plain_parts_ms": parts,
           "plain_ops_per_s": n_ops / (t_plain * 1e-3), "batch_ops_per_s": n_ops / (t_batch * 1e-3),
           "bins": [dict(precision=b["precision"], count=b["count"], blocks=b["blocks"],
                         lanes=b["config"].lanes, limbs=b["config"].limbs, window=b["config"].window)
                    for b in plan.info()],
           "selector": selector, "result_check": ok}
    plan.destroy()
    heur.destroy()
    h.destroy()
    return out


def run_mixed(args):
    """The mixed-size batch (mixed_suite) as its own JSON line."""
    r = mixed_suite(args.steps, args.warmup, args.count, args.crt, args.crt_keys)
    line = {"metric": "mixed-size batch speedup (autotuned batch plan vs plain per-size launches)",
            "value": r["speedup_vs_plain_selector"], "unit": "x", "higher_is_better": True, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["batch_ms"], "dtype": "u32",
            "data": "synthetic (seeded)",
            "config": {"workload": "65,536 mixed powm (40/30/20/10%% of 1024/2048/3072/4096 bits) + %d CRT-RSA-2048"
                       % args.crt, "crt_keys": args.crt_keys, "selector": r["selector"]}}
    line.update({k: v for k, v in r.items() if k != "selector"})
    print(json.dumps(line), flush=True)


def run_serve(args):
    print(json.dumps(serve_suite(args.serve_quick, args.serve_seconds, args.serve_peak_requests,
                                 args.serve_sync_requests)), flush=True)


def serve_suite(quick, seconds, peak_requests, sync_requests):
    """Serving loop: open-loop Poisson arrivals of requests with 1-64 ops under
    one key from a pool of 1,024 odd full-length moduli (512 x 2048, 307 x
    3072, 205 x 4096 bits: a 50/30/20 mix), bases below the key, full-length
    exponents; 8 GiB HBM admission budget.  Peak = saturated throughput (all
    requests at t=0); the sweep reports p50/p99/p999 per offered rate; the
    baseline is plain synchronous per-request calls.  quick: floors, peak, a
    run at 25 k ops/s and the 70%-of-peak point only (no overload points, no
    baseline)."""
    import torch
    import oracle as orc
    import xmp_b200 as xmp
    from xmp_b200 import tuning
    torch.cuda.set_device(0)
    h = xmp.Handle()  # starts with the compiled-in selector
    selector = os.path.exists(tuning.DEFAULT_WEIGHTS)
    classes = [(2048, 512), (3072, 307), (4096, 205)]
    srv = xmp.Server(h, [c for c, _ in classes], hbm_budget=8 << 30, max_keys=512)
    # per class: one block of 64 ops per key (bases below that key); a request
    # takes the first nops ops of a block, results land in that block's rows
    blocks = []
    for ci, (bits, nk) in enumerate(classes):
        n = bits // 32
        keys = orc.full_length_odd(5000 + ci, nk, n)
        first = srv.add_keys(bits, keys)
        mm = np.repeat(keys, 64, axis=0)
        base = orc.below(5100 + ci, mm).reshape(nk, 64, n)
        exp = orc.random_limbs(5200 + ci, nk * 64, n)
        exp[:, -1] |= np.uint32(0x80000000)
        exp = exp.reshape(nk, 64, n)
        out = np.zeros_like(base)
        for k in range(nk):
            blocks.append((first + k, base[k], exp[k], out[k], keys[k], bits))
    rng = np.random.default_rng(4242)

    def stream(n_req, rate):
        """n_req requests; arrival times (ns) of a Poisson process at `rate` ops/s (0: all at once)."""
        ks = rng.integers(0, len(blocks), size=n_req)
        nops = rng.integers(1, 65, size=n_req)
        if rate > 0:
            gaps = rng.exponential(32.5 / rate * 1e9, size=n_req)
            arr = np.cumsum(gaps).astype(np.uint64)
        else:
            arr = np.zeros(n_req, dtype=np.uint64)
        keys = [blocks[k][0] for k in ks]
        bases = [blocks[k][1][:m] for k, m in zip(ks, nops)]
        exps = [blocks[k][2][:m] for k, m in zip(ks, nops)]
        outs = [blocks[k][3][:m] for k, m in zip(ks, nops)]
        return keys, arr, bases, exps, outs, int(nops.sum()), ks, nops

    def run(n_req, rate, mode=0):
        keys, arr, bases, exps, outs, ops, ks, nops = stream(n_req, rate)
        lat, secs = srv.replay(keys, arr, bases, exps, outs, mode=mode)
        ms = lat.astype(np.float64) * 1e-6
        bits = np.array([blocks[k][5] for k in ks])
        by_bits = {int(b): {"p50_ms": float(np.percentile(ms[bits == b], 50)),
                            "p99_ms": float(np.percentile(ms[bits == b], 99))}
                   for b in sorted(set(bits.tolist()))}
        return {"offered_ops_per_s": rate, "requests": n_req, "ops": ops, "ops_per_s": ops / secs,
                "p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)),
                "p999_ms": float(np.percentile(ms, 99.9)), "max_ms": float(ms.max()), "by_bits": by_bits}, ks, nops

    # latency floor: one op alone per size (median of 3)
    floor = {}
    for bits in (2048, 3072, 4096):
        k = next(i for i, b in enumerate(blocks) if b[5] == bits)
        t = []
        for _ in range(3):
            lat, _ = srv.replay([blocks[k][0]], np.zeros(1, np.uint64), [blocks[k][1][:1]], [blocks[k][2][:1]],
                                [blocks[k][3][:1]])
            t.append(float(lat[0]) * 1e-6)
        floor[bits] = statistics.median(t)
    run(200, 0)  # warm-up
    peak, _, _ = run(peak_requests, 0)
    sweep = []
    rates = sorted(set([10000, 25000, 50000, int(0.7 * peak["ops_per_s"]), 100000, 200000, 500000]))
    if quick:
        rates = [25000, int(0.7 * peak["ops_per_s"])]
    at70 = None
    for rate in rates:
        n_req = max(50, int(rate * seconds / 32.5))
        r, _, _ = run(n_req, rate)
        sweep.append(r)
        if rate == int(0.7 * peak["ops_per_s"]):
            at70 = r
    sync = None if quick else run(sync_requests, 10000, mode=1)[0]
    # results check: written rows of a sample of blocks against GMP
    ok = True
    for bi in rng.choice(len(blocks), size=12, replace=False):
        key, base, exp, out, m, bits = blocks[bi]
        rows = [j for j in range(8) if out[j].any()]  # rows some request wrote
        if not rows:
            continue
        mm = np.repeat(m[None, :], len(rows), axis=0)
        want, _ = orc.powm(base[rows], exp[rows], mm, len(rows))
        ok = ok and np.array_equal(out[rows], want)
    st = srv.stats()
    line = {"metric": "serving p99 latency at 70% of peak load", "value": at70["p99_ms"], "unit": "ms",
            "higher_is_better": False, "n_gpus": 1, "dtype": "u32", "data": "synthetic (seeded)",
            "config": {"workload": "open-loop Poisson modexp requests, 1-64 ops each, 1,024 keys "
                                   "(50/30/20% of 2048/3072/4096 bits), full-length exponents",
                       "hbm_budget_gib": 8, "selector": selector},
            "peak_ops_per_s": peak["ops_per_s"], "at_70pct": at70, "sweep": sweep,
            "sync_baseline": sync, "single_op_latency_ms": floor,
            "server": {k: st[k] for k in ("waves", "admission_stalls", "max_inflight_ops", "device_bytes")},
            "result_check": bool(ok)}
    srv.destroy()
    h.destroy()
    return line


def elementwise_suite(h, stream, steps, warmup, imad_peak):
    """Elementwise and contraction suite: add, sub, and, ior, xor, not, shf (shifts
    uniform 0..255), cmp, popc on 2^22 pairs of 256-bit operands (HBM-bound:
    GB/s of algorithmic bytes against the measured HBM copy bandwidth, and against
    a device-to-device copy of the same byte count timed the same way); mul on
    2^18 pairs of 512 x 512 -> 1024 bits; divmod on 2^18 instances of 2048-bit
    dividends by 1024-bit divisors with the top bit set.  Operands resident in
    HBM (every working set exceeds the 126 MB L2); each op checked bit-exact
    against GMP on its first 4,096 instances; GMP multithreaded on the host
    for add, mul and divmod.  Returns (per-op results, GMP rates, HBM peak)."""
    import torch
    import oracle as orc
    import xmp_b200 as xmp
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        pass
    hbm = peaks.get("hbm_gbs") or 6650.0
    E = 1 << 22
    a = orc.random_limbs(31, E, 8)
    b = orc.random_limbs(32, E, 8)
    sh = (orc.splitmix64(33, E) % np.uint64(256)).astype(np.int32)
    A, B, C = h.integers(256, E, a), h.integers(256, E, b), h.integers(256, E)
    SH = torch.from_numpy(sh).cuda()
    I32 = torch.empty(E, dtype=torch.int32, device="cuda")

    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device="cuda")

    def timed(fn):
        """Median device time of one call.  Every step is queued behind an L2
        flush (a 252 MB write), so no step finds its operands in L2, and behind
        a 100 us device spin before its first event, so the GPU is still busy
        while the host makes the library call: the events then bracket the
        call's kernels alone, not the host's time to issue them (a few tens
        of microseconds through ctypes, as long as the shortest kernels here).
        One synchronize at the end."""
        spin = int(100e-6 * torch.cuda.get_device_properties(0).clock_rate * 1e3)
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        evs = []
        for _ in range(steps):
            flush.zero_()
            torch.cuda._sleep(spin)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            evs.append((e0, e1))
        torch.cuda.synchronize()
        return statistics.median([e0.elapsed_time(e1) for e0, e1 in evs])

    S = 4096
    res = {}
    copies = {}

    def copy_gbs(total):
        """GB/s of a device-to-device copy moving `total` bytes (read + write), timed like the ops:
        the bandwidth a launch of this size reaches, launch and ramp included."""
        if total not in copies:
            src = torch.empty(total // 2, dtype=torch.uint8, device="cuda")
            dst = torch.empty_like(src)
            copies[total] = total / (timed(lambda: dst.copy_(src)) * 1e-3) / 1e9
            del src, dst
        return copies[total]

    def row(name, ms, bytes_per_op, count, ok, imad_per_op=0, vs_copy=False):
        r = {"ms": ms, "ops_per_s": count / (ms * 1e-3), "bytes_per_op": bytes_per_op,
             "gbs": bytes_per_op * count / (ms * 1e-3) / 1e9, "check": bool(ok)}
        r["hbm_frac"] = r["gbs"] / hbm
        if vs_copy:
            r["copy_gbs_same_bytes"] = copy_gbs(bytes_per_op * count)
            r["copy_frac"] = r["gbs"] / r["copy_gbs_same_bytes"]
        if imad_per_op:
            r["timad_s"] = imad_per_op * count / (ms * 1e-3) / 1e12
            r["imad_frac"] = r["timad_s"] / imad_peak
        res[name] = r

    for name, fn, op in (("add", xmp.add, "add"), ("sub", xmp.sub, "sub"), ("and", xmp.and_, "and"),
                         ("ior", xmp.ior, "ior"), ("xor", xmp.xor, "xor")):
        ms = timed(lambda fn=fn: fn(h, C, A, B, E, asynchronous=True))
        ok = np.array_equal(C.export(count=E)[:S], orc.binary(op, a[:S], b[:S], 8, S))
        row(name, ms, 96, E, ok, vs_copy=True)
    ms = timed(lambda: xmp.not_(h, C, A, E, asynchronous=True))
    row("not", ms, 64, E, np.array_equal(C.export()[:S], orc.not_(a[:S], 8, S)), vs_copy=True)
    L = xmp.lib()
    ms = timed(lambda: xmp.check(L.xmpIntegersShfAsync(h.h, C.x, A.x, SH.data_ptr(), E, E)))
    row("shf", ms, 68, E, np.array_equal(C.export()[:S], orc.shf(a[:S], sh[:S], 8, S)), vs_copy=True)
    # cmp reads limb groups from the top down and stops at the first that differs: for these random
    # operands the top 16-byte groups decide, so 2 x 16 B read + 4 B written per op
    ms = timed(lambda: xmp.check(L.xmpIntegersCmpAsync(h.h, I32.data_ptr(), A.x, B.x, E)))
    row("cmp", ms, 36, E, np.array_equal(I32[:S].cpu().numpy(), orc.cmp(a[:S], b[:S], S)), vs_copy=True)
    ms = timed(lambda: xmp.check(L.xmpIntegersPopcAsync(h.h, I32.data_ptr(), A.x, E)))
    row("popc", ms, 36, E, np.array_equal(I32[:S].cpu().numpy().view(np.uint32), orc.popc(a[:S], S)),
        vs_copy=True)
    # add through index arrays (random permutations gathering a and b, scattering c): 96 B of
    # operands plus three 4-byte indices per op
    perms = [np.random.default_rng(60 + k).permutation(E).astype(np.uint32) for k in range(3)]
    pol = xmp.Policy(h)
    for k in range(3):
        pol.set_indices(k, perms[k])
    h.set_policy(pol)
    ms = timed(lambda: xmp.add(h, C, A, B, E, asynchronous=True))
    h.set_policy(None)
    got = C.export()
    want = orc.binary("add", a[perms[1][:S]], b[perms[2][:S]], 8, S)
    row("add_indexed", ms, 108, E, np.array_equal(got[perms[0][:S]], want))
    pol.destroy()
    cpu = {}
    t = time.perf_counter()
    orc.binary("add", a, b, 8, E)
    cpu["add"] = E / (time.perf_counter() - t)
    for X in (A, B, C):
        X.destroy()
    # mul: 2^18 x (512 x 512 -> 1024)
    M = 1 << 18
    ma = orc.random_limbs(41, M, 16)
    mb = orc.random_limbs(42, M, 16)
    MA, MB, MC = h.integers(512, M, ma), h.integers(512, M, mb), h.integers(1024, M)
    ms = timed(lambda: xmp.mul(h, MC, MA, MB, M, asynchronous=True))
    row("mul", ms, 256, M, np.array_equal(MC.export()[:S], orc.binary("mul", ma[:S], mb[:S], 32, S)),
        imad_per_op=2 * 16 * 16)
    t = time.perf_counter()
    orc.binary("mul", ma, mb, 32, M)
    cpu["mul"] = M / (time.perf_counter() - t)
    for X in (MA, MB, MC):
        X.destroy()
    # divmod: 2^18 x (2048 / 1024), divisor top bit set
    da = orc.random_limbs(51, M, 64)
    db = orc.random_limbs(52, M, 32)
    db[:, -1] |= np.uint32(0x80000000)
    DA, DB, DQ, DR = h.integers(2048, M, da), h.integers(1024, M, db), h.integers(2048, M), h.integers(1024, M)
    ms = timed(lambda: xmp.divmod_(h, DQ, DR, DA, DB, M, asynchronous=True))
    wq, wr = orc.divmod_(da[:S], db[:S], 64, 32, S)
    row("divmod", ms, 256 + 128 + 256 + 128, M,
        np.array_equal(DQ.export()[:S], wq) and np.array_equal(DR.export()[:S], wr),
        imad_per_op=2 * (64 - 32 + 1) * 32)
    t = time.perf_counter()
    orc.divmod_(da, db, 64, 32, M)
    cpu["divmod"] = M / (time.perf_counter() - t)
    for X in (DA, DB, DQ, DR):
        X.destroy()
    return res, cpu, hbm


def run_elementwise(args):
    """The elementwise and contraction suite (elementwise_suite) as its own JSON line."""
    import torch
    import oracle as orc
    import xmp_b200 as xmp
    torch.cuda.set_device(0)
    h = xmp.Handle()
    stream = torch.cuda.current_stream()
    h.set_stream(stream.cuda_stream)
    imad_peak = probe_imad_peak()["imad"]
    res, cpu, hbm = elementwise_suite(h, stream, args.steps, args.warmup, imad_peak)
    line = {"metric": "elementwise suite HBM GB/s (256-bit add)", "value": res["add"]["gbs"], "unit": "GB/s",
            "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": res["add"]["ms"], "dtype": "u32", "data": "synthetic (seeded splitmix64 limbs)",
            "config": {"workload": "2^22 x 256-bit elementwise ops, 2^18 x 512x512 mul, 2^18 x 2048/1024 divmod",
                       "l2": "flushed before every step (252 MB write, queued ahead of the events)"},
            "roofline": {"bound": "hbm", "peak": hbm, "unit": "GB/s", "peak_source": "MEASURED_PEAKS.json hbm_gbs"},
            "imad_peak_timad_s": imad_peak, "ops": res,
            "cpu_baseline": {"ops_per_s": cpu, "cores": orc.max_threads(), "kind": "port",
                             "sample": "full arrays, GMP mpz under OpenMP"},
            "result_check": all(r["check"] for r in res.values())}
    print(json.dumps(line), flush=True)
    h.destroy()


def run_latency(args):
    """One exponentiation alone per size (the latency suite of the default run, on its own)."""
    import torch
    import xmp_b200 as xmp
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    h = xmp.Handle()
    h.set_stream(stream.cuda_stream)
    sizes = tuple(int(b) for b in args.latency_bits.split(","))
    print(json.dumps({"metric": "one full-exponent modexp alone", "unit": "ms",
                      "sizes": latency_suite(h, stream, sizes=sizes)}), flush=True)
    h.destroy()


def run_crt(args):
    """CRT-RSA private operations (RSA-2048: 1024-bit primes from GMP nextprime on seeded starts,
    e = 65537, messages uniform below n): --count decryptions under --crt-keys keys through the
    fused xmpIntegersPowmCRT, every result checked against its message."""
    import torch
    import oracle as orc
    import xmp_b200 as xmp
    torch.cuda.set_device(0)
    count, nkeys = args.count, args.crt_keys
    keys = _crt_keys(nkeys, 1024, 777)
    rng = np.random.default_rng(778)
    msgs, cts = [], []
    for i in range(count):
        kk = keys[i % nkeys]
        nn = orc.to_int(kk["n"])
        mm = int.from_bytes(rng.bytes(256), "little") % nn
        msgs.append(mm)
        cts.append(pow(mm, 65537, nn))
    h = xmp.Handle()
    stream = torch.cuda.current_stream()
    h.set_stream(stream.cuda_stream)
    C = h.integers(2048, count, np.stack([orc.from_int(c, 64) for c in cts]))
    ka = {f: h.integers(1024, nkeys, np.stack([kk[f] for kk in keys])) for f in ("p", "q", "dp", "dq", "qinv")}
    out = h.integers(2048, count)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device="cuda")
    step = lambda: xmp.powm_crt(h, out, C, ka["p"], ka["q"], ka["dp"], ka["dq"], ka["qinv"], count, asynchronous=True)
    ms = statistics.median(_timed_events(step, stream, flush, args.steps, args.warmup))
    ok = [orc.to_int(r) for r in out.export()] == msgs
    line = {"metric": "CRT-RSA-2048 private operations/s (fused kernel)", "value": count / (ms * 1e-3),
            "unit": "ops/s", "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "dtype": "u32", "data": "synthetic (seeded keys and messages)",
            "config": {"workload": "RSA-2048 decryption by CRT x %d, %d keys" % (count, nkeys)},
            "result_check": ok}
    print(json.dumps(line), flush=True)
    for v in [C, out] + list(ka.values()):
        v.destroy()
    h.destroy()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--bits", type=int, default=2048)
    ap.add_argument("--count", type=int, default=65536)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--ref-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="headline workload only (no config 1/2/3 or reference GPU)")
    ap.add_argument("--force-config", default=None, help="lanes,limbs,window: time this powm kernel configuration")
    ap.add_argument("--workload", default="powm2048",
                    choices=["powm2048", "mixed", "serve", "elementwise", "crt", "latency"])
    ap.add_argument("--latency-bits", default="1024,2048,3072,4096", help="latency workload: modulus sizes")
    ap.add_argument("--serve-seconds", type=float, default=1.0)
    ap.add_argument("--serve-peak-requests", type=int, default=3000)
    ap.add_argument("--serve-sync-requests", type=int, default=40)
    ap.add_argument("--serve-quick", action="store_true",
                    help="serving: floors, peak and the 70%%-of-peak point only (no overload points, no baseline)")
    ap.add_argument("--crt", type=int, default=16384)
    ap.add_argument("--crt-keys", type=int, default=256)
    args = ap.parse_args()
    if args.workload == "mixed":
        run_mixed(args)
        return
    if args.workload == "serve":
        run_serve(args)
        return
    if args.workload == "elementwise":
        run_elementwise(args)
        return
    if args.workload == "crt":
        run_crt(args)
        return
    if args.workload == "latency":
        run_latency(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        try:
            run_ours(args, rank, world, local_rank)
        finally:
            dist.destroy_process_group()
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
