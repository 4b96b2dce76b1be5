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

L2_BYTES = 126 * 1024 * 1024


def imad_per_modexp(bits, ebits):
    n = bits // 32
    return (ebits + math.ceil(ebits / 5)) * (4 * n * n + n)


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


def cpu_gmp_rate(x, e, m, target_s=10.0, threads=0):
    """GMP mpz_powm over a bounded sample on all host threads; returns (ops/s, threads, sample)."""
    import oracle as orc
    count = len(m)
    n0 = min(count, 256)
    t = time.perf_counter()
    _, used = orc.powm(x[:n0], e[:n0], m[:n0], n0, threads=threads)
    dt = time.perf_counter() - t
    rate0 = n0 / max(dt, 1e-9)
    n1 = int(min(count, max(n0, rate0 * target_s)))
    t = time.perf_counter()
    _, used = orc.powm(x[:n1], e[:n1], m[:n1], n1, threads=threads)
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
    x, e, m = make_inputs(bits, count, seed=2048 + 7919 * rank)

    h = xmp.Handle()
    h.set_stream(stream.cuda_stream)
    X, E, M, O = (h.integers(bits, count) for _ in range(4))
    for arr, rows in ((X, x), (E, e), (M, m)):
        arr.import_(rows)

    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device="cuda")
    lib = xmp.lib()

    def step():
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
    total_ms = sum(step_ms)
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * count * args.steps / (total_ms * 1e-3)

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
    e2e_ms = a.elapsed_time(b)
    if dist:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * count * args.steps / (e2e_ms * 1e-3)

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
                "frac": achieved / peaks["imad"], "traffic": None,
                "peak_source": "measured live: libxmpprobe independent mad.lo.u32 chains, all SMs",
                "carry_row_peak": peaks["carry_rows"],
                "algorithmic_imad_per_modexp": imad_per_modexp(bits, bits)}

    cpu = None
    if not args.no_cpu:
        rate, used, sample, dt = cpu_gmp_rate(x, e, m, target_s=args.cpu_seconds)
        cpu = {"value": rate, "unit": "modexp/s", "cores": used, "kind": "port",
               "sample": "%d instances of the same workload (%.1f s, GMP mpz_powm via OpenMP)" % (sample, dt)}

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
    print(json.dumps(line), flush=True)
    for v in (X, E, M, O):
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
    args = ap.parse_args()
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
