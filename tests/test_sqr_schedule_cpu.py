"""The lane-distributed squaring's decomposition and block schedule, checked on the CPU.

xmp_b200/csrc/sqr.cuh squares a number spread over T lanes (L limbs each) by
having every lane form its own square S, the doubled products P_r = 2 A_g A_{g+r}
(r < T/2) and its half Q of 2 A_g A_{g+T/2}, cut into L-word blocks that each
lane adds into its reduction window at the half-block boundary where the block's
T offset meets the window.  Here (1) a big-integer restatement of exactly those
products, with the offsets the header computes, must sum to A^2 for random A;
(2) the header's constexpr offsets and slot counts, compiled for the host with
nvcc, must match the restatement, and every block must land at a boundary the
reduction visits (0 .. 2T) with at most two blocks per lane per boundary.
"""
import os
import random
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def offset(T, L, g, i):
    if i == 0:
        return 2 * g * L
    if i == 1:
        return 2 * g * L + L
    if i < T:
        h = (g + i // 2) % T
        return L * (g + h) + (L if i % 2 else 0)
    h = (g + T // 2) % T
    return L * (g + h) + (L // 2 if g >= T // 2 else 0) + (0 if i == T else L)


@pytest.mark.parametrize("T", [2, 4, 8])
@pytest.mark.parametrize("L", [4, 8, 16])
def test_products_sum_to_the_square(T, L):
    H = L // 2
    rnd = random.Random(T * 100 + L)
    for _ in range(40):
        A = rnd.getrandbits(32 * T * L)
        if _ == 0:
            A = (1 << (32 * T * L)) - 1  # all ones: the largest carries
        blk = [(A >> (32 * L * g)) & ((1 << (32 * L)) - 1) for g in range(T)]
        limb = lambda x, k: (x >> (32 * k)) & 0xFFFFFFFF
        total = 0
        for g in range(T):
            a = blk[g]
            total += (a * a) << (32 * offset(T, L, g, 0))
            for r in range(1, T // 2):
                total += (2 * a * blk[(g + r) % T]) << (32 * offset(T, L, g, 2 * r))
            h = (g + T // 2) % T
            first = g < T // 2
            q = 0
            for p in range(2):
                x = 2 * ((a & ((1 << (32 * H)) - 1)) if (p == 0 or first) else (a >> (32 * H)))
                for k in range(H):
                    w = limb(blk[h], p * H + k) if first else limb(blk[h], H + k)
                    q += (x * w) << (32 * (p * H + k))
            assert q >> (32 * (L + H + 1)) == 0  # Q fits its two blocks (L + H + 1 words)
            total += q << (32 * offset(T, L, g, T))
        assert total == A * A


def _host_schedule(T):
    """Block offsets (L = 2) and slot counts from the header's constexpr functions."""
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    import tempfile
    d = tempfile.mkdtemp()
    src = os.path.join(d, "sched.cu")
    with open(src, "w") as f:
        f.write('#include "sqr.cuh"\n#include <cstdio>\nusing namespace xmpb;\n'
                'int main() { const int T = %d;\n'
                '  for (int g = 0; g < T; g++) for (int id = 0; id < T + 2; id++)\n'
                '    printf("o %%d %%d %%d\\n", g, id, sqr_block_offset(T, 2, g, id));\n'
                '  for (int b = 0; b <= 2 * T; b++) printf("s %%d %%d\\n", b, (int)((sqr_slots_mask(T) >> (2 * b)) & 3));\n'
                '  for (int g = 0; g < T; g++) { SqrPlanBits p = sqr_lane_plan<T>(g);\n'
                '    printf("p %%d %%u %%u %%u\\n", g, p.w[0], p.w[1], p.w[2]); }\n'
                '  return 0; }\n' % T)
    exe = os.path.join(d, "sched")
    p = subprocess.run([nvcc, "-std=c++17", "-I", os.path.join(ROOT, "xmp_b200", "csrc"), "-I",
                        os.path.join(ROOT, "include"), src, "-o", exe], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr[-2000:]
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    offs, slots, plans = {}, {}, {}
    for line in out:
        parts = line.split()
        if parts and parts[0] == "o":
            offs[(int(parts[1]), int(parts[2]))] = int(parts[3])
        elif parts and parts[0] == "s":
            slots[int(parts[1])] = int(parts[2])
        elif parts and parts[0] == "p":
            plans[int(parts[1])] = [int(x) for x in parts[2:5]]
    return offs, slots, plans


@pytest.mark.parametrize("T", [2, 4])
def test_header_schedule_matches(T):
    offs, slots, plans = _host_schedule(T)
    per = {}
    for g in range(T):
        for i in range(T + 2):
            assert offs[(g, i)] == offset(T, 2, g, i)
            b = offs[(g, i)] - 2 * g  # L = 2: one word per half block
            assert 0 <= b <= 2 * T
            per.setdefault(b, {}).setdefault(g, []).append(i)
    for b in range(2 * T + 1):
        most = max((len(per.get(b, {}).get(g, [])) for g in range(T)), default=0)
        assert most <= 2
        assert slots[b] == most
    # each lane's plan names every block once, in a slot at its boundary (nibble 2b + slot; 15 = none)
    for g in range(T):
        w = plans[g]
        nib = [(w[k // 8] >> (4 * (k % 8))) & 15 for k in range(24)]
        placed = {}
        for b in range(2 * T + 1):
            for s in range(2):
                if nib[2 * b + s] != 15:
                    assert s < slots[b]
                    placed[nib[2 * b + s]] = b
        assert placed == {i: offs[(g, i)] - 2 * g for i in range(T + 2)}
