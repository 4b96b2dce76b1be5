"""The reference's own sample programs as C callers of this library.

oracle/build_ref.sh compiles the reference's samples (sample01, simple_rsa,
crt_rsa, diffie_hellman; samples/*/*.cc) against include/xmp.h and links them
to xmp_b200/libxmp.so.  Each program allocates through xmpHandleCreate /
xmpIntegersCreate, imports host data, runs powm (and, for CRT-RSA, mod, mul,
add and cmp) and validates its own results, exiting non-zero on any mismatch.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SAMPLES = os.path.join(ROOT, "oracle", "_ref", "samples")

pytestmark = pytest.mark.gpu

CASES = [("sample01", "sample01 executed sucessfully"), ("simple_rsa", "simple RSA executed successfully"),
         ("crt_rsa", "CRT RSA executed successfully"), ("diffie_hellman", "Diffie-Hellman executed successfully")]


@pytest.mark.parametrize("name,marker", CASES)
def test_reference_sample_against_libxmp(name, marker):
    exe = os.path.join(SAMPLES, name + ".exe")
    if not os.path.exists(exe):
        pytest.skip("samples not built (oracle/build_ref.sh)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert marker in r.stdout, r.stdout[-2000:]
    assert "Error" not in r.stdout, r.stdout[-2000:]
