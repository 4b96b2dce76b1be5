"""Serving-loop admission logic on the CPU: the slot ring (contiguous,
granule-aligned, never overlapping live ranges, alloc succeeds exactly when
the largest free run fits) and the wave-launch rule, from the same header the
CUDA server compiles, built here with the host compiler."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_slot_ring_and_wave_policy(tmp_path):
    exe = str(tmp_path / "serve_sched_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "xmp_b200", "csrc"),
                    os.path.join(ROOT, "tests", "native", "serve_sched_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
