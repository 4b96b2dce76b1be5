"""Builds libxmp.so (the C-ABI library) and libxmpprobe.so for sm_100a, in tree.

Every CUDA source under xmp_b200/csrc is compiled by nvcc with
-gencode arch=compute_100a,code=sm_100a into xmp_b200/_build/, in parallel, and
linked into xmp_b200/libxmp.so with the CUDA runtime linked statically.
Run:  python -m xmp_b200.build [--force] [-j N]
"""
import argparse
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libxmp.so")
PROBE_LIB = os.path.join(HERE, "libxmpprobe.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
                 "-I" + os.path.join(ROOT, "include"), "-diag-suppress", "186"]

PROBE_SOURCES = {"probe.cu"}


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src, obj, force, hdr_time):
    if not force and os.path.exists(obj):
        t = os.path.getmtime(obj)
        if t >= os.path.getmtime(src) and t >= hdr_time:
            return src, None
    cmd = [NVCC] + CFLAGS + ["-c", src, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        return src, p.stdout + p.stderr
    return src, None


def build(force=False, jobs=None, verbose=True):
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr = _newest_header()
    jobs = jobs or max(1, os.cpu_count() or 1)
    objs = {s: os.path.join(BUILD, os.path.basename(s)[:-3] + ".o") for s in sources}
    with ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, objs[s], force, hdr), sources))
    errors = [(s, e) for s, e in results if e]
    if errors:
        for s, e in errors:
            sys.stderr.write("nvcc failed for %s:\n%s\n" % (s, e))
        raise RuntimeError("CUDA build failed")
    lib_objs = [objs[s] for s in sources if os.path.basename(s) not in PROBE_SOURCES]
    probe_objs = [objs[s] for s in sources if os.path.basename(s) in PROBE_SOURCES]
    for out, ol in ((LIB, lib_objs), (PROBE_LIB, probe_objs)):
        if not ol:
            continue
        if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(o) for o in ol):
            continue
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-Xcompiler", "-fPIC", "-o", out] + ol
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed for %s:\n%s%s" % (out, p.stdout, p.stderr))
        if verbose:
            print("built", os.path.relpath(out, ROOT))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    build(force=a.force, jobs=a.j)
