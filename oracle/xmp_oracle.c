/*
 * xmp_oracle.c -- CPU oracle for the batched multi-precision path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: tests/, the smoke
 * test and bench.py's CPU baseline call it; the product (libxmp.so) never
 * links or calls it.
 *
 * Two parts:
 *  1. The XMP API semantics restated over compact little-endian uint32 limb
 *     rows, with GMP (libgmp.so.10, called through hand-declared prototypes of
 *     its documented mpz ABI because the image ships no gmp.h) doing the
 *     integer arithmetic, exactly as the reference's own unit tests do
 *     (unit_tests/test.cu:1200-1220 powm vs mpz_powm, :2310-2322 sub with the
 *     2^P correction, generic ops :1674-1838, divmod :1840-1999, shf
 *     :1272-1416 vs mpz_mul_2exp / mpz_fdiv_q_2exp, cmp :2001, popc :2116).
 *     Index rules (docs para. 15-16; src/include/implementations.h:63-68):
 *     input element = index[i % index_count] % array_count, output element =
 *     out_index[i].
 *  2. A plain-C restatement of the reference's exponentiation algorithm:
 *     fixed-window (2^w-ary) left-to-right exponentiation over Montgomery
 *     multiplication (src/include/powm/powm.h:39-127, window size rule
 *     src/include/powm_operators.h:15-31, exponent scanned from bit
 *     precision-1), checked against GMP by the CPU tests.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

/* ---- GMP ABI (documented mpz interface, GMP 6.x) ------------------------- */
typedef struct {
  int _mp_alloc;
  int _mp_size;
  unsigned long *_mp_d;
} mpz_struct;
typedef mpz_struct mpz_t[1];

void __gmpz_init(mpz_struct *);
void __gmpz_clear(mpz_struct *);
void __gmpz_set_ui(mpz_struct *, unsigned long);
void __gmpz_set(mpz_struct *, const mpz_struct *);
void __gmpz_import(mpz_struct *, size_t, int, size_t, int, size_t, const void *);
void *__gmpz_export(void *, size_t *, int, size_t, int, size_t, const mpz_struct *);
void __gmpz_add(mpz_struct *, const mpz_struct *, const mpz_struct *);
void __gmpz_sub(mpz_struct *, const mpz_struct *, const mpz_struct *);
void __gmpz_mul(mpz_struct *, const mpz_struct *, const mpz_struct *);
void __gmpz_and(mpz_struct *, const mpz_struct *, const mpz_struct *);
void __gmpz_ior(mpz_struct *, const mpz_struct *, const mpz_struct *);
void __gmpz_xor(mpz_struct *, const mpz_struct *, const mpz_struct *);
void __gmpz_tdiv_qr(mpz_struct *, mpz_struct *, const mpz_struct *, const mpz_struct *);
void __gmpz_tdiv_r_2exp(mpz_struct *, const mpz_struct *, unsigned long);
void __gmpz_mul_2exp(mpz_struct *, const mpz_struct *, unsigned long);
void __gmpz_fdiv_q_2exp(mpz_struct *, const mpz_struct *, unsigned long);
void __gmpz_powm(mpz_struct *, const mpz_struct *, const mpz_struct *, const mpz_struct *);
void __gmpz_powm_sec(mpz_struct *, const mpz_struct *, const mpz_struct *, const mpz_struct *);
unsigned long __gmpz_popcount(const mpz_struct *);
int __gmpz_cmp(const mpz_struct *, const mpz_struct *);
void __gmpz_nextprime(mpz_struct *, const mpz_struct *);
int __gmpz_invert(mpz_struct *, const mpz_struct *, const mpz_struct *);
void __gmpz_lcm(mpz_struct *, const mpz_struct *, const mpz_struct *);
void __gmpz_sub_ui(mpz_struct *, const mpz_struct *, unsigned long);
void __gmpz_mod(mpz_struct *, const mpz_struct *, const mpz_struct *);
void __gmpz_setbit(mpz_struct *, unsigned long);

static int mpz_sign(const mpz_struct *z) { return (z->_mp_size > 0) - (z->_mp_size < 0); }

static void to_mpz(mpz_struct *z, const uint32_t *limbs, uint32_t n) { __gmpz_import(z, n, -1, 4, 0, 0, limbs); }

/* z mod 2^(32n) into n limbs (z >= 0). */
static void from_mpz(uint32_t *limbs, uint32_t n, const mpz_struct *z) {
  mpz_t t;
  size_t cnt = 0;
  __gmpz_init(t);
  __gmpz_tdiv_r_2exp(t, z, 32ul * n);
  memset(limbs, 0, (size_t)n * 4);
  if (mpz_sign(t) != 0) __gmpz_export(limbs, &cnt, -1, 4, 0, 0, t);
  __gmpz_clear(t);
}

static uint32_t in_el(uint32_t i, const uint32_t *idx, uint32_t nidx, uint32_t cnt) {
  uint32_t k = idx ? idx[i % nidx] : i;
  return k % cnt;
}
static uint32_t out_el(uint32_t i, const uint32_t *idx) { return idx ? idx[i] : i; }

/* Operand description shared by the entry points. */
typedef struct {
  const uint32_t *limbs; /* compact rows, count x n */
  uint32_t n;            /* limbs per element */
  uint32_t count;        /* elements */
  const uint32_t *index; /* optional */
  uint32_t index_count;
} orc_in;

typedef struct {
  uint32_t *limbs;
  uint32_t n;
  uint32_t count;
  const uint32_t *index;
} orc_out;

enum { OP_ADD = 0, OP_SUB, OP_AND, OP_IOR, OP_XOR, OP_MUL, OP_DIV, OP_MOD };

/* out = op(a, b) mod 2^(32 out.n) for `count` instances. */
int oracle_binary(int op, orc_out out, orc_in a, orc_in b, uint32_t count, int threads) {
  int bad = 0;
  omp_set_num_threads(threads > 0 ? threads : omp_get_num_procs());
#pragma omp parallel
  {
    mpz_t x, y, r, q;
    __gmpz_init(x);
    __gmpz_init(y);
    __gmpz_init(r);
    __gmpz_init(q);
#pragma omp for schedule(static)
    for (uint32_t i = 0; i < count; i++) {
      uint32_t o = out_el(i, out.index);
      if (o >= out.count) continue;
      to_mpz(x, a.limbs + (size_t)in_el(i, a.index, a.index_count, a.count) * a.n, a.n);
      to_mpz(y, b.limbs + (size_t)in_el(i, b.index, b.index_count, b.count) * b.n, b.n);
      switch (op) {
        case OP_ADD: __gmpz_add(r, x, y); break;
        case OP_SUB:
          __gmpz_sub(r, x, y);
          if (mpz_sign(r) < 0) { /* two's complement wrap: + 2^P */
            __gmpz_set_ui(q, 0);
            __gmpz_setbit(q, 32ul * out.n);
            __gmpz_add(r, r, q);
          }
          break;
        case OP_AND: __gmpz_and(r, x, y); break;
        case OP_IOR: __gmpz_ior(r, x, y); break;
        case OP_XOR: __gmpz_xor(r, x, y); break;
        case OP_MUL: __gmpz_mul(r, x, y); break;
        case OP_DIV:
        case OP_MOD:
          if (mpz_sign(y) == 0) { /* division by zero: q = a, r = 0 */
            if (op == OP_DIV) __gmpz_set(r, x);
            else __gmpz_set_ui(r, 0);
          } else {
            __gmpz_tdiv_qr(q, r, x, y);
            if (op == OP_DIV) __gmpz_set(r, q);
          }
          break;
        default: bad = 1; break;
      }
      from_mpz(out.limbs + (size_t)o * out.n, out.n, r);
    }
    __gmpz_clear(x);
    __gmpz_clear(y);
    __gmpz_clear(r);
    __gmpz_clear(q);
  }
  return bad ? -1 : 0;
}

/* q = floor(a / b), r = a mod b; division by zero gives q = a, r = 0. */
int oracle_divmod(orc_out qo, orc_out ro, orc_in a, orc_in b, uint32_t count, int threads) {
  omp_set_num_threads(threads > 0 ? threads : omp_get_num_procs());
#pragma omp parallel
  {
    mpz_t x, y, q, r;
    __gmpz_init(x);
    __gmpz_init(y);
    __gmpz_init(q);
    __gmpz_init(r);
#pragma omp for schedule(static)
    for (uint32_t i = 0; i < count; i++) {
      uint32_t oq = out_el(i, qo.index), orr = out_el(i, ro.index);
      to_mpz(x, a.limbs + (size_t)in_el(i, a.index, a.index_count, a.count) * a.n, a.n);
      to_mpz(y, b.limbs + (size_t)in_el(i, b.index, b.index_count, b.count) * b.n, b.n);
      if (mpz_sign(y) == 0) {
        __gmpz_set_ui(r, 0);
        __gmpz_set(q, x);
      } else {
        __gmpz_tdiv_qr(q, r, x, y);
      }
      if (oq < qo.count) from_mpz(qo.limbs + (size_t)oq * qo.n, qo.n, q);
      if (orr < ro.count) from_mpz(ro.limbs + (size_t)orr * ro.n, ro.n, r);
    }
    __gmpz_clear(x);
    __gmpz_clear(y);
    __gmpz_clear(q);
    __gmpz_clear(r);
  }
  return 0;
}

/* c = ~a mod 2^(32 c.n) */
int oracle_not(orc_out c, orc_in a, uint32_t count) {
  for (uint32_t i = 0; i < count; i++) {
    uint32_t o = out_el(i, c.index);
    if (o >= c.count) continue;
    const uint32_t *x = a.limbs + (size_t)in_el(i, a.index, a.index_count, a.count) * a.n;
    for (uint32_t j = 0; j < c.n; j++) c.limbs[(size_t)o * c.n + j] = ~(j < a.n ? x[j] : 0u);
  }
  return 0;
}

/* c = floor(a * 2^s) mod 2^(32 c.n), s = shift[i % shift_count] */
int oracle_shf(orc_out c, orc_in a, const int32_t *shift, uint32_t shift_count, uint32_t count) {
  mpz_t x, r;
  __gmpz_init(x);
  __gmpz_init(r);
  uint32_t sc = shift_count < count ? shift_count : count;
  for (uint32_t i = 0; i < count; i++) {
    uint32_t o = out_el(i, c.index);
    if (o >= c.count) continue;
    to_mpz(x, a.limbs + (size_t)in_el(i, a.index, a.index_count, a.count) * a.n, a.n);
    int32_t s = shift[i % sc];
    if (s >= 0) __gmpz_mul_2exp(r, x, (unsigned long)s);
    else __gmpz_fdiv_q_2exp(r, x, (unsigned long)(-(int64_t)s));
    from_mpz(c.limbs + (size_t)o * c.n, c.n, r);
  }
  __gmpz_clear(x);
  __gmpz_clear(r);
  return 0;
}

int oracle_cmp(int32_t *c, orc_in a, orc_in b, uint32_t count) {
  mpz_t x, y;
  __gmpz_init(x);
  __gmpz_init(y);
  for (uint32_t i = 0; i < count; i++) {
    to_mpz(x, a.limbs + (size_t)in_el(i, a.index, a.index_count, a.count) * a.n, a.n);
    to_mpz(y, b.limbs + (size_t)in_el(i, b.index, b.index_count, b.count) * b.n, b.n);
    int v = __gmpz_cmp(x, y);
    c[i] = (v > 0) - (v < 0);
  }
  __gmpz_clear(x);
  __gmpz_clear(y);
  return 0;
}

int oracle_popc(uint32_t *c, orc_in a, uint32_t count) {
  mpz_t x;
  __gmpz_init(x);
  for (uint32_t i = 0; i < count; i++) {
    to_mpz(x, a.limbs + (size_t)in_el(i, a.index, a.index_count, a.count) * a.n, a.n);
    c[i] = (uint32_t)__gmpz_popcount(x);
  }
  __gmpz_clear(x);
  return 0;
}

/* out = base^exp mod mod via GMP (mode 0: mpz_powm, 1: mpz_powm_sec), `threads`
 * OpenMP threads (<= 0: all).  Returns the number of threads used. */
int oracle_powm(orc_out out, orc_in base, orc_in ex, orc_in mod, uint32_t count, int threads, int mode) {
  int used = 1;
  /* the thread count is set on every call: an earlier call's count would otherwise persist */
  omp_set_num_threads(threads > 0 ? threads : omp_get_num_procs());
#pragma omp parallel
  {
#pragma omp single
    used = omp_get_num_threads();
    mpz_t b, e, m, r;
    __gmpz_init(b);
    __gmpz_init(e);
    __gmpz_init(m);
    __gmpz_init(r);
#pragma omp for schedule(dynamic, 16)
    for (uint32_t i = 0; i < count; i++) {
      uint32_t o = out_el(i, out.index);
      if (o >= out.count) continue;
      to_mpz(b, base.limbs + (size_t)in_el(i, base.index, base.index_count, base.count) * base.n, base.n);
      to_mpz(e, ex.limbs + (size_t)in_el(i, ex.index, ex.index_count, ex.count) * ex.n, ex.n);
      to_mpz(m, mod.limbs + (size_t)in_el(i, mod.index, mod.index_count, mod.count) * mod.n, mod.n);
      if (mode == 1 && mpz_sign(e) > 0)
        __gmpz_powm_sec(r, b, e, m);
      else
        __gmpz_powm(r, b, e, m);
      from_mpz(out.limbs + (size_t)o * out.n, out.n, r);
    }
    __gmpz_clear(b);
    __gmpz_clear(e);
    __gmpz_clear(m);
    __gmpz_clear(r);
  }
  return used;
}

/* ---- plain-C restatement of fixed-window Montgomery exponentiation -------- */

/* t = a*b*R^-1 mod N (CIOS, R = 2^(32n)); result fully below 2N, then reduced below N. */
static void mont_mul_c(uint32_t *t, const uint32_t *a, const uint32_t *b, const uint32_t *N, uint32_t np0,
                       uint32_t n, uint32_t *acc /* n+2 words */) {
  memset(acc, 0, (size_t)(n + 2) * 4);
  for (uint32_t i = 0; i < n; i++) {
    uint64_t c = 0;
    for (uint32_t j = 0; j < n; j++) {
      uint64_t s = (uint64_t)a[j] * b[i] + acc[j] + c;
      acc[j] = (uint32_t)s;
      c = s >> 32;
    }
    uint64_t s = (uint64_t)acc[n] + c;
    acc[n] = (uint32_t)s;
    acc[n + 1] += (uint32_t)(s >> 32);
    uint32_t q = acc[0] * np0;
    c = ((uint64_t)q * N[0] + acc[0]) >> 32;
    for (uint32_t j = 1; j < n; j++) {
      s = (uint64_t)q * N[j] + acc[j] + c;
      acc[j - 1] = (uint32_t)s;
      c = s >> 32;
    }
    s = (uint64_t)acc[n] + c;
    acc[n - 1] = (uint32_t)s;
    acc[n] = acc[n + 1] + (uint32_t)(s >> 32);
    acc[n + 1] = 0;
  }
  /* acc < 2N: subtract N when acc >= N */
  int ge = acc[n] != 0;
  if (!ge) {
    ge = 1;
    for (int32_t j = (int32_t)n - 1; j >= 0; j--) {
      if (acc[j] != N[j]) {
        ge = acc[j] > N[j];
        break;
      }
    }
  }
  if (ge) {
    uint64_t br = 0;
    for (uint32_t j = 0; j < n; j++) {
      uint64_t d = (uint64_t)acc[j] - N[j] - br;
      t[j] = (uint32_t)d;
      br = (d >> 63) & 1;
    }
  } else {
    memcpy(t, acc, (size_t)n * 4);
  }
}

static uint32_t neg_inv32_c(uint32_t n) {
  uint32_t x = n;
  for (int k = 0; k < 4; k++) x = x * (2u - n * x);
  return 0u - x;
}

/* Window bits from the exponent precision (src/include/powm_operators.h:15-31). */
static uint32_t ref_window_bits(uint32_t bits) {
  if (bits < 400) return 4;
  if (bits < 800) return 5;
  if (bits < 1600) return 6;
  if (bits <= 4096) return 7;
  return 8;
}

/* x^e mod N for odd N, n-limb operands, exponent of en limbs scanned from its top bit of precision. */
int oracle_powm_mont(orc_out out, orc_in base, orc_in ex, orc_in mod, uint32_t count) {
  uint32_t n = mod.n;
  uint32_t w = ref_window_bits(32 * ex.n);
  uint32_t entries = 1u << w;
  uint32_t *tab = (uint32_t *)malloc((size_t)entries * n * 4);
  uint32_t *acc = (uint32_t *)malloc((size_t)(n + 2) * 4);
  uint32_t *x = (uint32_t *)malloc((size_t)n * 4), *y = (uint32_t *)malloc((size_t)n * 4);
  uint32_t *r2 = (uint32_t *)malloc((size_t)n * 4), *one = (uint32_t *)calloc(n, 4);
  one[0] = 1;
  for (uint32_t i = 0; i < count; i++) {
    uint32_t o = out_el(i, out.index);
    if (o >= out.count) continue;
    const uint32_t *B = base.limbs + (size_t)in_el(i, base.index, base.index_count, base.count) * base.n;
    const uint32_t *E = ex.limbs + (size_t)in_el(i, ex.index, ex.index_count, ex.count) * ex.n;
    const uint32_t *N = mod.limbs + (size_t)in_el(i, mod.index, mod.index_count, mod.count) * mod.n;
    uint32_t np0 = neg_inv32_c(N[0]);
    /* R^2 mod N by 64n modular doublings of 1 */
    memset(r2, 0, (size_t)n * 4);
    r2[0] = 1;
    int n_is_one = N[0] == 1;
    for (uint32_t j = 1; j < n; j++) n_is_one &= N[j] == 0;
    if (n_is_one) r2[0] = 0;
    for (uint32_t d = 0; d < 64u * n && !n_is_one; d++) {
      uint32_t top = r2[n - 1] >> 31;
      for (int32_t j = (int32_t)n - 1; j > 0; j--) r2[j] = (r2[j] << 1) | (r2[j - 1] >> 31);
      r2[0] <<= 1;
      int ge = top;
      if (!ge) {
        ge = 1;
        for (int32_t j = (int32_t)n - 1; j >= 0; j--)
          if (r2[j] != N[j]) {
            ge = r2[j] > N[j];
            break;
          }
      }
      if (ge) {
        uint64_t br = 0;
        for (uint32_t j = 0; j < n; j++) {
          uint64_t dd = (uint64_t)r2[j] - N[j] - br;
          r2[j] = (uint32_t)dd;
          br = (dd >> 63) & 1;
        }
      }
    }
    /* table of Mont(x^k); x is reduced by the first multiply */
    mont_mul_c(tab, one, r2, N, np0, n, acc);                 /* Mont(1) */
    for (uint32_t j = 0; j < n; j++) x[j] = j < base.n ? B[j] : 0;
    mont_mul_c(tab + n, x, r2, N, np0, n, acc);               /* Mont(x) */
    for (uint32_t k = 2; k < entries; k++) mont_mul_c(tab + (size_t)k * n, tab + (size_t)(k - 1) * n, tab + n, N, np0, n, acc);
    /* windows of w bits aligned at bit 0, scanned from the top of the exponent precision */
    uint32_t bits = 32 * ex.n;
    uint32_t nwin = (bits + w - 1) / w;
    for (int32_t k = (int32_t)nwin - 1; k >= 0; k--) {
      uint32_t win = 0;
      for (uint32_t b = 0; b < w; b++) {
        uint32_t bit = (uint32_t)k * w + b;
        if (bit < bits) win |= ((E[bit >> 5] >> (bit & 31)) & 1u) << b;
      }
      if (k == (int32_t)nwin - 1) {
        memcpy(x, tab + (size_t)win * n, (size_t)n * 4);
        continue;
      }
      for (uint32_t s2 = 0; s2 < w; s2++) {
        mont_mul_c(y, x, x, N, np0, n, acc);
        memcpy(x, y, (size_t)n * 4);
      }
      mont_mul_c(y, x, tab + (size_t)win * n, N, np0, n, acc);
      memcpy(x, y, (size_t)n * 4);
    }
    mont_mul_c(y, x, one, N, np0, n, acc);
    uint32_t *dst = out.limbs + (size_t)o * out.n;
    for (uint32_t j = 0; j < out.n; j++) dst[j] = j < n ? y[j] : 0;
  }
  free(tab);
  free(acc);
  free(x);
  free(y);
  free(r2);
  free(one);
  return 0;
}

/* ---- workload generators (GMP for primes and inverses) -------------------- */

/* CRT key material for one 2-prime RSA key from seeded starts p0, q0 (hn limbs each):
 * p = nextprime(p0), q = nextprime(q0), e = 65537, d = e^-1 mod lcm(p-1, q-1),
 * dp = d mod (p-1), dq = d mod (q-1), qinv = q^-1 mod p, n = p q (2 hn limbs).
 * Returns 0 on success, 1 if e is not invertible (caller reseeds). */
int oracle_crt_key(const uint32_t *p0, const uint32_t *q0, uint32_t hn, uint32_t *p, uint32_t *q, uint32_t *dp,
                   uint32_t *dq, uint32_t *qinv, uint32_t *nout) {
  mpz_t P, Q, E, D, L, t1, t2, N;
  __gmpz_init(P); __gmpz_init(Q); __gmpz_init(E); __gmpz_init(D);
  __gmpz_init(L); __gmpz_init(t1); __gmpz_init(t2); __gmpz_init(N);
  to_mpz(t1, p0, hn);
  __gmpz_nextprime(P, t1);
  to_mpz(t1, q0, hn);
  __gmpz_nextprime(Q, t1);
  __gmpz_set_ui(E, 65537);
  __gmpz_sub_ui(t1, P, 1);
  __gmpz_sub_ui(t2, Q, 1);
  __gmpz_lcm(L, t1, t2);
  int ok = __gmpz_invert(D, E, L);
  if (ok) {
    from_mpz(p, hn, P);
    from_mpz(q, hn, Q);
    __gmpz_mod(t2, D, t1);
    from_mpz(dp, hn, t2);
    __gmpz_sub_ui(t1, Q, 1);
    __gmpz_mod(t2, D, t1);
    from_mpz(dq, hn, t2);
    __gmpz_invert(t2, Q, P);
    from_mpz(qinv, hn, t2);
    __gmpz_mul(N, P, Q);
    from_mpz(nout, 2 * hn, N);
  }
  __gmpz_clear(P); __gmpz_clear(Q); __gmpz_clear(E); __gmpz_clear(D);
  __gmpz_clear(L); __gmpz_clear(t1); __gmpz_clear(t2); __gmpz_clear(N);
  return ok ? 0 : 1;
}

int oracle_max_threads(void) { return omp_get_max_threads(); }
