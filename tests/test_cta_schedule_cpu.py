"""CPU check of the one-exponentiation-per-CTA Montgomery product
(xmp_b200/csrc/cta.cuh), step by step with Python integers:

* each multiplication as 4 x 4-limb tiles summed per anti-diagonal word
  (64-bit column sums, no carries) into the kernel's word-linear buffers (low
  and high tile halves apart, four zero words either side, the buffers kept
  from one product to the next as in shared memory, so a schedule that read a
  word its product did not write would read a stale one), with the tile
  subsets the kernel forms (all; the low half for m; the diagonals from
  n/4 - 2 up for m N, T's sums added in by the same jobs);
* the single-warp resolution: 32 lanes x n/32 words, the bits above 32 of the
  two words below folded in, the remaining one-bit carries by the ballot
  lookahead (P + 2G) xor P, and the value above the top word;
* the schedule: T's low half resolved, m = T N' mod R, U = T + m N with T's
  high half entering as raw column sums and U's low half replaced by the carry
  identity hi(s) + (lo(s) != 0) of word n - 1 (entering as the high half of
  that word's sum), then the conditional subtraction of N with the lane-wise
  borrow lookahead;
* N' by Newton's iteration y <- y (2 + N y) from -N^-1 mod 2^32.

Every result is compared with a b R^-1 mod N; moduli of full length, with
top bits clear, small (3) and of the form 2^(32n) - 1 - 2k."""
import random

import pytest

M32 = (1 << 32) - 1


def words(x, n):
    return [(x >> (32 * i)) & M32 for i in range(n)]


def val(w):
    return sum(v << (32 * i) for i, v in enumerate(w))


class Cta:
    def __init__(self, n):
        self.n, self.q = n, n // 4
        self.diag = 2 * self.q - 1
        # column sums, word i at [4 + i] of lo (tile words 0-3) and hi (tile words 4-7)
        self.dsum = ([0] * (2 * n + 8), [0] * (2 * n + 8))
        self.dsumT = ([0] * (2 * n + 8), [0] * (2 * n + 8))

    def columns(self, x, y, mode, out, merge=None):
        q = self.q
        d0 = q - 2 if mode == "high" else 0
        d1 = q if mode == "low" else self.diag
        for d in range(d0, d1):
            lo, hi = max(0, d - (q - 1)), min(d, q - 1)
            tiles = [words(val(x[4 * t:4 * t + 4]) * val(y[4 * (d - t):4 * (d - t) + 4]), 8) for t in range(lo, hi + 1)]
            for w in range(8):
                half = 0 if w < 4 else 1
                v = sum(t[w] for t in tiles)
                if merge is not None:
                    v += merge[half][4 + 4 * d + w]
                out[half][4 + 4 * d + w] = v
        return out

    @staticmethod
    def ws(buf, i):
        assert -4 <= i < len(buf[0]) - 4
        return buf[0][4 + i] + buf[1][4 + i]


def resolve(nwords, sumf):
    """One warp: lane l holds words [lK, lK + K); returns (words, value above the top word)."""
    k = nwords // 32
    lanes = []
    for lane in range(32):
        i0 = lane * k
        sm = [sumf(i0 - 2 + j) for j in range(k + 2)]
        x = [(sm[j + 1] & M32) + (sm[j] >> 32) for j in range(k + 1)]
        limbs, c, ones = [], 0, 1
        for j in range(k):
            z = (x[j + 1] & M32) + (x[j] >> 32) + c
            assert z <= (1 << 33)
            limbs.append(z & M32)
            c = z >> 32
            ones &= int(limbs[-1] == M32)
        lanes.append((sm, x, limbs, c, ones))
    g = sum(lanes[l][3] << l for l in range(32))
    p = sum(lanes[l][4] << l for l in range(32))
    assert g & p == 0  # a lane that generates a carry cannot also propagate one
    cs = p + (g << 1)
    out = []
    for lane in range(32):
        cin = ((cs ^ p) >> lane) & 1
        for v in lanes[lane][2]:
            v2 = (v + cin) & M32
            out.append(v2)
            cin = int(cin and v2 == 0)
    top = (lanes[31][0][k + 1] >> 32) + (lanes[31][1][k] >> 32) + ((cs >> 32) & 1)
    return out, top


def sub_if(u, nw, top):
    """Lane-wise borrow lookahead of u - N; u - N when top or no final borrow."""
    n = len(nw)
    k = n // 32
    per = []
    for lane in range(32):
        d, b, zero = [], 0, 1
        for j in range(k):
            t = u[lane * k + j] - nw[lane * k + j] - b
            d.append(t & M32)
            b = int(t < 0)
            zero &= int((t & M32) == 0)
        per.append((d, b, zero))
    gb = sum(per[l][1] << l for l in range(32))
    pb = sum(per[l][2] << l for l in range(32))
    bs = pb + (gb << 1)
    take = top or not ((bs >> 32) & 1)
    out = []
    for lane in range(32):
        bin_ = ((bs ^ pb) >> lane) & 1
        for j in range(k):
            d = per[lane][0][j]
            out.append(((d - bin_) & M32) if take else u[lane * k + j])
            bin_ = int(bin_ and d == 0)
    return out


def low_carry(v):
    return ((v >> 32) + int((v & M32) != 0)) << 32


def mont(c, a, b, nw, npw):
    n = c.n
    dt = c.columns(a, b, "full", c.dsumT)
    t, _ = resolve(n, lambda i: c.ws(dt, i))
    dm = c.columns(t, npw, "low", c.dsum)
    m, _ = resolve(n, lambda i: c.ws(dm, i))
    du = c.columns(m, nw, "high", c.dsum, merge=dt)
    u, top = resolve(n, lambda j: 0 if j < -1 else low_carry(c.ws(du, n - 1)) if j == -1 else c.ws(du, n + j))
    return sub_if(u, nw, top)


def neg_inverse(c, nw):
    n = c.n
    y = [0] * n
    y[0] = (-pow(nw[0], -1, 1 << 32)) & M32
    w = 1
    while w < n:
        d = c.columns(nw, y, "low", c.dsum)
        m, _ = resolve(n, lambda j: c.ws(d, j) + (2 if j == 0 else 0))
        d = c.columns(y, m, "low", c.dsum)
        y, _ = resolve(n, lambda j: c.ws(d, j))
        w *= 2
    return y


@pytest.mark.parametrize("n", [32, 64, 96, 128])
def test_cta_montgomery_product(n):
    rnd = random.Random(n)
    c = Cta(n)
    r = 1 << (32 * n)
    moduli = [rnd.getrandbits(32 * n) | 1 | (1 << (32 * n - 1)), r - 1 - 2 * rnd.getrandbits(20),
              rnd.getrandbits(32 * n - 77) | 1, 3]
    for mod in moduli:
        nw = words(mod, n)
        npw = neg_inverse(c, nw)
        assert (val(npw) * mod) % r == r - 1
        rinv = pow(r, -1, mod)
        for k in range(3):
            a, b = rnd.randrange(mod), rnd.randrange(mod)
            if k == 0:
                a = b = mod - 1
            assert val(mont(c, words(a, n), words(b, n), nw, npw)) == a * b * rinv % mod
            assert val(mont(c, words(a, n), words(a, n), nw, npw)) == a * a * rinv % mod
        x = rnd.randrange(r)  # any operand below R times R^2 mod N: x R mod N, fully reduced
        assert val(mont(c, words(x, n), words(r * r % mod, n), nw, npw)) == x * r % mod


def tile_tree(x, y):
    """The kernel's tile product (cta_tile): four row products x * y_j as 5-word chains, rows added
    pairwise with one word of shift, then the halves with two; every add a 32-bit add with carry."""
    def row(yj):
        p = [xk * yj for xk in x]
        r, c = [p[0] & M32], 0
        for k in range(1, 4):
            t = (p[k - 1] >> 32) + (p[k] & M32) + c
            r.append(t & M32)
            c = t >> 32
        r.append(((p[3] >> 32) + c) & M32)
        assert (p[3] >> 32) + c <= M32
        return r

    def add_shift(r, q, shift):
        a, c = r[:shift], 0
        for k in range(shift, len(r)):
            t = r[k] + q[k - shift] + c
            a.append(t & M32)
            c = t >> 32
        for k in range(len(r) - shift, len(q)):
            t = q[k] + c
            a.append(t & M32)
            c = t >> 32
        assert c == 0
        return a

    r0, r1, r2, r3 = (row(y[j]) for j in range(4))
    A, B = add_shift(r0, r1, 1), add_shift(r2, r3, 1)
    return add_shift(A, B, 2)


def test_tile_tree_is_the_product():
    rnd = random.Random(7)
    cases = [([M32] * 4, [M32] * 4), ([0] * 4, [M32] * 4), ([1, 0, 0, 0], [M32] * 4)]
    cases += [([rnd.getrandbits(32) for _ in range(4)], [rnd.getrandbits(32) for _ in range(4)]) for _ in range(2000)]
    for x, y in cases:
        v = tile_tree(x, y)
        assert len(v) == 8 and val(v) == val(x) * val(y)
