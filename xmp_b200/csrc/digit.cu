// Digit-serial modular exponentiation: one thread per instance, every operand
// resident in the scratch arena and streamed limb by limb, so any precision
// works (replaces internalPowmDigitMP and digitmp_ar/powm/copy_out_kernel,
// src/include/powm_operators.h:144-256, powm_implementations.h:154-286, and
// the DigitMP representation, src/include/digitmp/).
//
// Working arrays are interleaved across the launch's threads (word j of
// thread t at base + j*T + t) so each warp access is one coalesced 128-byte
// line.  Montgomery multiplication is finely integrated product scanning: the
// product columns of A*B and M*N are accumulated into a three-word
// accumulator, column k < n fixes the quotient digit m_k, columns >= n emit
// the result, so no 2n-word intermediate is stored.
#include "powm.h"
#include <algorithm>

namespace xmpb {

struct Strided {
  uint32_t *p;
  uint32_t T;
  __device__ __forceinline__ uint32_t &operator[](uint32_t j) const { return p[(size_t)j * T]; }
};

struct DigitArgs {
  ArrayView base, exp, mod;
  OutView out;
  uint32_t start, count, window, n, T;
  uint32_t *work;  // (6 + 2^W) * n words per thread, interleaved
};

__device__ __forceinline__ void acc_mul(uint32_t &c0, uint32_t &c1, uint32_t &c2, uint32_t x, uint32_t y) {
  c0 = mad_lo_cc(x, y, c0);
  c1 = madc_hi_cc(x, y, c1);
  c2 = addc(c2, 0u);
}

// t = a*b*R^-1 mod N, almost reduced (< R).  t must not alias a or b.
__device__ void fips_mul(const Strided &t, const Strided &a, const Strided &b, const Strided &N, const Strided &m,
                         uint32_t n, uint32_t np0) {
  uint32_t c0 = 0, c1 = 0, c2 = 0;
  for (uint32_t k = 0; k < n; k++) {
    for (uint32_t i = 0; i < k; i++) {
      acc_mul(c0, c1, c2, a[i], b[k - i]);
      acc_mul(c0, c1, c2, m[i], N[k - i]);
    }
    acc_mul(c0, c1, c2, a[k], b[0]);
    uint32_t mk = c0 * np0;
    m[k] = mk;
    acc_mul(c0, c1, c2, mk, N[0]);
    c0 = c1;
    c1 = c2;
    c2 = 0;
  }
  for (uint32_t k = n; k < 2 * n; k++) {
    for (uint32_t i = k - n + 1; i < n; i++) {
      acc_mul(c0, c1, c2, a[i], b[k - i]);
      acc_mul(c0, c1, c2, m[i], N[k - i]);
    }
    t[k - n] = c0;
    c0 = c1;
    c1 = c2;
    c2 = 0;
  }
  if (c0) {  // result >= R: subtract N once (result < R + N)
    uint32_t borrow = 0;
    for (uint32_t j = 0; j < n; j++) {
      uint64_t d = (uint64_t)t[j] - N[j] - borrow;
      t[j] = (uint32_t)d;
      borrow = (uint32_t)(d >> 63);
    }
  }
}

// x <- x - N if x >= N (x < 2N)
__device__ void digit_reduce(const Strided &x, const Strided &N, const Strided &tmp, uint32_t n) {
  uint32_t borrow = 0;
  for (uint32_t j = 0; j < n; j++) {
    uint64_t d = (uint64_t)x[j] - N[j] - borrow;
    tmp[j] = (uint32_t)d;
    borrow = (uint32_t)(d >> 63);
  }
  if (!borrow)
    for (uint32_t j = 0; j < n; j++) x[j] = tmp[j];
}

__global__ void __launch_bounds__(128) powm_digit_kernel(DigitArgs a) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= a.count) return;
  const uint32_t i = a.start + tid;
  const uint32_t eb = in_element(a.base, i), ee = in_element(a.exp, i), em = in_element(a.mod, i);
  const uint32_t n = a.n, T = a.T;
  uint32_t *w = a.work + tid;
  Strided N{w, T}, X{w + (size_t)n * T, T}, Y{w + (size_t)2 * n * T, T}, M{w + (size_t)3 * n * T, T},
      R2{w + (size_t)4 * n * T, T}, U{w + (size_t)5 * n * T, T};
  Strided tab{w + (size_t)6 * n * T, T};  // entry e, word j at tab[e*n + j]
  auto entry = [&](uint32_t e) { return Strided{tab.p + (size_t)e * n * T, T}; };

  uint32_t bits_n = 0;
  for (uint32_t j = 0; j < n; j++) {
    uint32_t v = load_limb(a.mod.limbs, a.mod.nlimbs, a.mod.stride, em, j);
    N[j] = v;
    if (v) bits_n = j * 32 + 32 - __clz(v);
  }
  const uint32_t np0 = neg_inv32(N[0]);

  // R^2 mod N: exact doublings from 2^(b-1) to 2^(32n+s), then j Montgomery squarings.
  const uint32_t bits = 32 * n, jsq = __ffs(bits) - 1, s = bits >> jsq;
  for (uint32_t j = 0; j < n; j++) R2[j] = 0;
  if (bits_n > 1) {
    R2[(bits_n - 1) >> 5] = 1u << ((bits_n - 1) & 31);
    uint32_t doublings = bits - bits_n + 1 + s;
    for (uint32_t d = 0; d < doublings; d++) {
      uint32_t carry = 0;
      for (uint32_t j = 0; j < n; j++) {
        uint32_t v = R2[j];
        R2[j] = (v << 1) | carry;
        carry = v >> 31;
      }
      uint32_t borrow = 0;
      for (uint32_t j = 0; j < n; j++) {
        uint64_t dd = (uint64_t)R2[j] - N[j] - borrow;
        U[j] = (uint32_t)dd;
        borrow = (uint32_t)(dd >> 63);
      }
      if (carry || !borrow)
        for (uint32_t j = 0; j < n; j++) R2[j] = U[j];
    }
    for (uint32_t q = 0; q < jsq; q++) {
      fips_mul(U, R2, R2, N, M, n, np0);
      for (uint32_t j = 0; j < n; j++) R2[j] = U[j];
    }
  }

  // Table: T[0] = R - N, T[1] = Mont(x), T[e] = T[e-1] * T[1].
  {
    Strided t0 = entry(0);
    uint32_t borrow = 0;
    for (uint32_t j = 0; j < n; j++) {
      uint64_t d = (uint64_t)0 - N[j] - borrow;
      t0[j] = (uint32_t)d;
      borrow = (uint32_t)(d >> 63);
    }
    for (uint32_t j = 0; j < n; j++) X[j] = load_limb(a.base.limbs, a.base.nlimbs, a.base.stride, eb, j);
    fips_mul(entry(1), X, R2, N, M, n, np0);
    for (uint32_t e = 2; e < (1u << a.window); e++) fips_mul(entry(e), entry(e - 1), entry(1), N, M, n, np0);
  }

  // Exponent length of this instance (threads are independent here).
  uint32_t ebits = 0;
  for (int32_t j = (int32_t)a.exp.nlimbs - 1; j >= 0; j--) {
    uint32_t v = load_limb(a.exp.limbs, a.exp.nlimbs, a.exp.stride, ee, (uint32_t)j);
    if (v) {
      ebits = (uint32_t)j * 32 + 32 - __clz(v);
      break;
    }
  }
  const uint32_t W = a.window;
  const uint32_t nwin = ebits ? (ebits + W - 1) / W : 1;
  uint32_t win = exp_window(a.exp, ee, (nwin - 1) * W, W);
  {
    Strided src = entry(win);
    for (uint32_t j = 0; j < n; j++) X[j] = src[j];
  }
  for (int32_t wi = (int32_t)nwin - 2; wi >= 0; wi--) {
    win = exp_window(a.exp, ee, (uint32_t)wi * W, W);
    for (uint32_t sq = 0; sq < W; sq++) {
      fips_mul(Y, X, X, N, M, n, np0);
      Strided t = X;
      X = Y;
      Y = t;
    }
    fips_mul(Y, X, entry(win), N, M, n, np0);
    Strided t = X;
    X = Y;
    Y = t;
  }
  // Leave Montgomery form.
  for (uint32_t j = 0; j < n; j++) U[j] = j == 0 ? 1u : 0u;
  fips_mul(Y, X, U, N, M, n, np0);
  digit_reduce(Y, N, U, n);

  uint32_t o = out_element(a.out, i);
  if (o < a.out.count)
    for (uint32_t j = 0; j < a.out.nlimbs; j++) limb_ref(a.out.limbs, a.out.stride, o, j) = j < n ? Y[j] : 0u;
}

xmpError_t powm_digit_run(xmpHandle_t h, const PowmConfig &cfg0, const OutView &out, const ArrayView &base,
                          const ArrayView &exp, const ArrayView &mod, uint32_t count) {
  PowmConfig cfg = cfg0;
  const uint32_t n = mod.nlimbs;
  size_t limit = scratch_limit(h);
  uint32_t chunk = count;
  while (true) {
    size_t per = (((size_t)1 << cfg.window) * n + 6 * ((size_t)n + 2)) * 4;
    uint64_t fit = limit / per / 128 * 128;
    if (fit >= 128) {
      chunk = (uint32_t)std::min<uint64_t>(count, fit);
      break;
    }
    if (cfg.window <= 1) return xmpErrorIncreaseScratchLimit;
    cfg.window--;
  }
  xmpError_t e = ensure_scratch(h, powm_table_bytes(cfg, n, chunk));
  if (e != xmpErrorSuccess) return e;
  DigitArgs a;
  a.base = base;
  a.exp = exp;
  a.mod = mod;
  a.out = out;
  a.window = cfg.window;
  a.n = n;
  a.work = (uint32_t *)h->scratch;
  for (uint32_t start = 0; start < count; start += chunk) {
    a.start = start;
    a.count = std::min(chunk, count - start);
    a.T = round_up(a.count, 128);
    powm_digit_kernel<<<grid_for(a.count, 128), 128, 0, h->stream>>>(a);
  }
  return check_cuda();
}

}  // namespace xmpb
