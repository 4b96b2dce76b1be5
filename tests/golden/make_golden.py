"""Generates tests/golden/golden.json: known-answer vectors for the XMP ops.

Expected values come from Python's own integer arithmetic (pow, divmod,
shifts, bit ops), independent of GMP, of the C oracle and of the CUDA code.
Semantics follow the reference API: results wrap modulo 2^(output
precision); sub is two's complement; shf is floor(a * 2^s); not is the
complement at the output precision; division by zero gives q = a, r = 0.

Also records the reference's own in-tree constants:
  * the 512-bit modular-exponentiation case documented as a rare Montgomery
    carry failure (src/include/regmp/reduce_xmad.h:110-116);
  * the toy CRT-RSA key of samples/crt_rsa/rsa.cc:166-178
    (n = 17460671 = 4931 * 3541, e = 65537, dp = 1063, dq = 113,
    cp = 15212136, cq = 2248536), whose decryption the sample checks
    (rsa.cc:206-233).

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import random

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")


def rnd(r, bits):
    return r.getrandbits(bits)


def case_list():
    r = random.Random(20151015)
    cases = []

    def add_case(op, precs, count, gen, raw_outputs=False):
        ins, outs = gen(count)
        cases.append({"op": op, "precisions": precs, "inputs": [[hex(v) for v in col] for col in ins],
                      "outputs": [[v if raw_outputs else hex(v) for v in col] for col in outs]})

    edge = lambda bits: [0, 1, (1 << bits) - 1, 1 << (bits - 1), (1 << (bits - 1)) - 1]

    for bits_out, bits_a, bits_b in [(64, 32, 32), (288, 256, 256), (160, 160, 160), (544, 512, 512),
                                     (256, 256, 128), (1056, 1024, 1024)]:
        def gen_add(n, ba=bits_a, bb=bits_b, bo=bits_out):
            a = edge(ba) + [rnd(r, ba) for _ in range(n)]
            b = [rnd(r, bb) for _ in range(n)] + edge(bb)
            return [a, b], [[(x + y) % (1 << bo) for x, y in zip(a, b)]]
        add_case("add", [bits_out, bits_a, bits_b], 11, gen_add)

        def gen_sub(n, ba=bits_a, bb=bits_b, bo=bits_out):
            a = edge(ba) + [rnd(r, ba) for _ in range(n)]
            b = [rnd(r, bb) for _ in range(n)] + edge(bb)
            return [a, b], [[(x - y) % (1 << bo) for x, y in zip(a, b)]]
        add_case("sub", [bits_out, bits_a, bits_b], 11, gen_sub)

        for op, f in [("and", lambda x, y: x & y), ("ior", lambda x, y: x | y), ("xor", lambda x, y: x ^ y)]:
            def gen_l(n, ba=bits_a, bb=bits_b, bo=bits_out, f=f):
                a = edge(ba) + [rnd(r, ba) for _ in range(n)]
                b = [rnd(r, bb) for _ in range(n)] + edge(bb)
                return [a, b], [[f(x, y) % (1 << bo) for x, y in zip(a, b)]]
            add_case(op, [bits_out, bits_a, bits_b], 11, gen_l)

        def gen_not(n, ba=bits_a, bo=bits_out):
            a = edge(ba) + [rnd(r, ba) for _ in range(n)]
            return [a], [[((1 << bo) - 1) ^ x for x in a]]
        add_case("not", [bits_out, bits_a], 11, gen_not)

    for bo, ba, bb in [(64, 32, 32), (1024, 512, 512), (512, 512, 512), (256, 256, 64), (2048, 1024, 1024),
                       (192, 160, 96)]:
        def gen_mul(n, ba=ba, bb=bb, bo=bo):
            a = edge(ba) + [rnd(r, ba) for _ in range(n)]
            b = [rnd(r, bb) for _ in range(n)] + edge(bb)
            return [a, b], [[(x * y) % (1 << bo) for x, y in zip(a, b)]]
        add_case("mul", [bo, ba, bb], 11, gen_mul)

    for bq, br, ba, bb in [(64, 32, 64, 32), (2048, 1024, 2048, 1024), (512, 512, 512, 512), (256, 128, 256, 96),
                           (384, 192, 384, 192), (4096, 2080, 4096, 2080)]:
        def gen_dm(n, ba=ba, bb=bb, bq=bq, br=br):
            a = [rnd(r, ba) for _ in range(n)] + [0, 5, (1 << ba) - 1, 12345, rnd(r, ba)]
            b = [rnd(r, bb) | (1 << (bb - 1)) for _ in range(n)] + [7, 0, 1, (1 << bb) - 1, rnd(r, bb // 2) + 1]
            q, m = [], []
            for x, y in zip(a, b):
                if y == 0:
                    q.append(x % (1 << bq))
                    m.append(0)
                else:
                    q.append((x // y) % (1 << bq))
                    m.append(x % y)
            return [a, b], [q, m]
        add_case("divmod", [bq, br, ba, bb], 11, gen_dm)

    for bo, ba in [(256, 256), (288, 256), (128, 256), (64, 32), (1024, 1024)]:
        def gen_shf(n, ba=ba, bo=bo):
            a = edge(ba) + [rnd(r, ba) for _ in range(n)]
            s = [r.randint(-300, 300) for _ in range(len(a) - 4)] + [0, 31, -32, 33]
            res = [((x << k) if k >= 0 else (x >> -k)) % (1 << bo) for x, k in zip(a, s)]
            return [a, s], [res]
        cases.append(None)  # placeholder replaced below
        ins, outs = gen_shf(11)
        cases[-1] = {"op": "shf", "precisions": [bo, ba], "inputs": [[hex(v) for v in ins[0]], ins[1]],
                     "outputs": [[hex(v) for v in outs[0]]]}

    for ba, bb in [(256, 256), (256, 128), (96, 160)]:
        def gen_cmp(n, ba=ba, bb=bb):
            a = [rnd(r, ba) for _ in range(n)] + [0, 1, 5, (1 << min(ba, bb)) - 1]
            b = [rnd(r, bb) for _ in range(n)] + [0, 0, 5, (1 << min(ba, bb)) - 1]
            b[0] = a[0] % (1 << bb)
            return [a, b], [[(x > y) - (x < y) for x, y in zip(a, b)]]
        add_case("cmp", [ba, bb], 12, gen_cmp, raw_outputs=True)

    for ba in [256, 160, 2048]:
        def gen_popc(n, ba=ba):
            a = edge(ba) + [rnd(r, ba) for _ in range(n)]
            return [a], [[bin(x).count("1") for x in a]]
        add_case("popc", [ba], 11, gen_popc, raw_outputs=True)

    for bits, ebits in [(64, 64), (128, 128), (160, 160), (512, 512), (1024, 1024), (1056, 1056), (2048, 2048),
                        (2048, 64), (3072, 3072), (4096, 4096), (544, 544)]:
        def gen_powm(n, bits=bits, ebits=ebits):
            m = [rnd(r, bits) | 1 | (1 << (bits - 1)) for _ in range(n)]
            m += [1, (1 << bits) - 1, 3, rnd(r, bits // 2) | 1]   # m = 1, all-ones, tiny, top bits clear
            x = [rnd(r, bits) for _ in range(len(m))]
            x[0] = 0
            x[1] = m[1] + 0 if m[1] < (1 << bits) else 0   # base == m
            e = [rnd(r, ebits) for _ in range(len(m))]
            e[2] = 0
            e[3] = 1
            return [x, e, m], [[pow(a, k, mm) for a, k, mm in zip(x, e, m)]]
        add_case("powm", [bits, bits, ebits, bits], 8, gen_powm)

    # Reference constants.
    a = int("b1e451f4e5dbbf65e7901088e87820ed3ce644365acfae8f372e42dfb5c24232c4a1bc48ce5471b20dfc1827c1a5545a"
            "19eadbbf7d99579d82b02f036c18d95d", 16)
    b = int("8ddcf087f521bd3df8748641c40e1d8224548611769b9eb4d0cde0c6bdab8cb2845ea8d4a8585ae9b105a3176125895d"
            "30a3d95aba31e458500dd7b7fb665d32", 16)
    c = int("ffdba45c89ec1b188d3c8f549a32ccafd43b06fb42ec7cb0585c4e2ad78fa438d36b7796b9ea4adcc67e2a97823e5f01"
            "adfc2367c241f8e1c83ed4a11a70dde9", 16)
    cases.append({"op": "powm", "precisions": [512, 512, 512, 512], "source": "src/include/regmp/reduce_xmad.h:110-116",
                  "inputs": [[hex(a)], [hex(b)], [hex(c)]], "outputs": [[hex(pow(a, b, c))]]})
    return cases


def crt_toy():
    n, e, p, q, dp, dq, cp, cq = 17460671, 65537, 4931, 3541, 1063, 113, 15212136, 2248536
    r = random.Random(7)
    msgs = [r.randrange(n) for _ in range(32)]
    ct = [pow(m, e, n) for m in msgs]
    return {"source": "samples/crt_rsa/rsa.cc:166-178,206-233", "n": n, "e": e, "p": p, "q": q, "dp": dp, "dq": dq,
            "cp": cp, "cq": cq, "messages": msgs, "ciphertexts": ct}


def main():
    doc = {"generator": "tests/golden/make_golden.py", "cases": case_list(), "crt_toy": crt_toy()}
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=0, separators=(",", ":"))
    print("wrote", OUT, os.path.getsize(OUT), "bytes", len(doc["cases"]), "cases")


if __name__ == "__main__":
    main()
