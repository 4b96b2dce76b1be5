// xmpIntegersDiv/Mod/DivMod[Async] (replaces src/div.cu:26-517 and the
// kernels regmp_/digitmp_div/mod/divmod_kernel, implementations.h:436-763,
// with RegMP div_rem/rem (regmp/div.h:397-686) and DigitMP div
// (digitmp/div.h:109-526)).
//
// q = floor(a / b), r = a mod b.  Division by zero leaves q = a and r = 0
// (the reference's RegMP behaviour, regmp/div.h:594-596).
//
// Algorithm: schoolbook long division (Knuth, TAOCP vol. 2, 4.3.1, algorithm
// D).  The divisor is normalised by S = 32z + s bits so that its top limb has
// its top bit set (z whole limbs, s bits); the normalised divisor lives in
// registers (BN limbs, a compile-time class) together with a BN+1 limb window
// of the partial remainder.  The shifted dividend is never materialised: each
// step pulls its next limb straight from the interleaved input with the
// funnel shift applied.  The quotient digit estimate divides the top two
// window limbs by the top divisor limb with a precomputed reciprocal
// (Moller & Granlund, "Improved division by invariant integers", IEEE TC
// 2011, algorithm 4), refined once against the second divisor limb; the
// multiply-subtract then needs at most one add-back.
// Divisors above the largest register class use the same algorithm with the
// window and divisor in the scratch arena.
#include "internal.h"
#include "carry.cuh"
#include "tune.h"
#include <algorithm>

using namespace xmpb;

namespace xmpb {

struct DivArgs {
  ArrayView a, b;
  OutView q, r;  // q.limbs or r.limbs may be null (Mod / Div)
  uint32_t count;
  uint32_t *scratch;  // large path: (2*nb + 1) words per thread, interleaved
  uint32_t T;
};

// floor((2^64 - 1) / d) - 2^32 for normalised d (top bit set).
__device__ __forceinline__ uint32_t reciprocal_2by1(uint32_t d) {
  return (uint32_t)(0xffffffffffffffffull / d - 0x100000000ull);
}

// (u1:u0) / d with u1 < d, d normalised, v = reciprocal_2by1(d).
__device__ __forceinline__ uint32_t div_2by1(uint32_t u1, uint32_t u0, uint32_t d, uint32_t v, uint32_t *rem) {
  uint64_t q = (uint64_t)v * u1;
  q += ((uint64_t)(u1 + 1) << 32) | u0;
  uint32_t q1 = (uint32_t)(q >> 32), q0 = (uint32_t)q;
  uint32_t r = u0 - q1 * d;
  if (r > q0) {
    q1--;
    r += d;
  }
  if (r >= d) {
    q1++;
    r -= d;
  }
  *rem = r;
  return q1;
}

// Quotient digit estimate from the window top (w2:w1:w0) and divisor top (d1:d0):
// floor((w2:w1)/d1) refined with w0 and d0; at most one too large.
__device__ __forceinline__ uint32_t estimate_q(uint32_t w2, uint32_t w1, uint32_t w0, uint32_t d1, uint32_t d0,
                                               uint32_t v, bool have_d0) {
  uint32_t qhat, rhat;
  bool rhat_big = false;
  if (w2 >= d1) {
    qhat = 0xffffffffu;
    uint64_t rr = (uint64_t)w1 + d1;  // (w2:w1) - qhat*d1 with w2 == d1
    rhat = (uint32_t)rr;
    rhat_big = (rr >> 32) != 0;
  } else {
    qhat = div_2by1(w2, w1, d1, v, &rhat);
  }
  if (have_d0) {
    for (int it = 0; it < 2 && !rhat_big; it++) {
      uint64_t lhs = (uint64_t)qhat * d0;
      uint64_t rhs = ((uint64_t)rhat << 32) | w0;
      if (lhs <= rhs) break;
      qhat--;
      uint64_t rr = (uint64_t)rhat + d1;
      rhat = (uint32_t)rr;
      rhat_big = (rr >> 32) != 0;
    }
  }
  return qhat;
}

struct ShiftedDividend {
  const ArrayView *a;
  uint32_t e;
  int32_t z;
  uint32_t s;
  // limb t of a * 2^(32z + s)
  __device__ __forceinline__ uint32_t operator()(int32_t t) const {
    int32_t j = t - z;
    uint32_t hi = (j >= 0 && j < (int32_t)a->nlimbs) ? load_limb(a->limbs, a->nlimbs, a->stride, e, (uint32_t)j) : 0u;
    if (s == 0) return hi;
    uint32_t lo = (j - 1 >= 0 && j - 1 < (int32_t)a->nlimbs) ? load_limb(a->limbs, a->nlimbs, a->stride, e, (uint32_t)(j - 1)) : 0u;
    return (hi << s) | (lo >> (32 - s));
  }
};

// Limbs of one instance read through a one-group cache: walking the limbs up
// or down loads each 128-bit group once instead of one 4-byte word per limb.
struct LimbCursor {
  const ArrayView *a;
  uint32_t e;
  int32_t g;
  uint4 v;
  __device__ __forceinline__ uint32_t operator()(int32_t j) {
    if (j < 0 || j >= (int32_t)a->nlimbs) return 0u;
    const int32_t gg = j >> 2;
    if (gg != g) {
      v = load_group(a->limbs, a->nlimbs, a->stride, e, (uint32_t)gg);
      g = gg;
    }
    const uint32_t r = j & 3;
    return r == 0 ? v.x : r == 1 ? v.y : r == 2 ? v.z : v.w;
  }
};

// limb t of a * 2^(32z + s), through two cursors (the limb and the one below it)
struct ShiftedCursor {
  LimbCursor hi, lo;
  int32_t z;
  uint32_t s;
  __device__ __forceinline__ uint32_t operator()(int32_t t) {
    const int32_t j = t - z;
    const uint32_t h = hi(j);
    if (s == 0) return h;
    return (h << s) | (lo(j - 1) >> (32 - s));
  }
};

__device__ __forceinline__ void write_limb(const OutView &o, uint32_t e, uint32_t j, uint32_t v) {
  if (j < o.nlimbs) limb_ref(o.limbs, o.stride, e, j) = v;
}
__device__ __forceinline__ void zero_limbs(const OutView &o, uint32_t e, uint32_t from) {
  for (uint32_t j = from; j < o.nlimbs; j++) limb_ref(o.limbs, o.stride, e, j) = 0;
}

// Special cases shared by both paths; returns true when the instance is done.
__device__ __forceinline__ bool div_trivial(const DivArgs &d, uint32_t ea, uint32_t eqo, uint32_t ero, int32_t bt,
                                            int32_t m) {
  if (bt < 0) {  // divisor 0: q = a, r = 0
    if (d.q.limbs) {
      for (uint32_t j = 0; j < d.q.nlimbs; j++)
        limb_ref(d.q.limbs, d.q.stride, eqo, j) = load_limb(d.a.limbs, d.a.nlimbs, d.a.stride, ea, j);
    }
    if (d.r.limbs) zero_limbs(d.r, ero, 0);
    return true;
  }
  if (m < 0) {  // a has fewer limbs than b: q = 0, r = a
    if (d.q.limbs) zero_limbs(d.q, eqo, 0);
    if (d.r.limbs) {
      for (uint32_t j = 0; j < d.r.nlimbs; j++)
        limb_ref(d.r.limbs, d.r.stride, ero, j) = load_limb(d.a.limbs, d.a.nlimbs, d.a.stride, ea, j);
    }
    return true;
  }
  return false;
}

template <int BN>
__global__ void __launch_bounds__(256) divmod_reg_kernel(DivArgs d) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.count) return;
  const uint32_t ea = in_element(d.a, i), eb = in_element(d.b, i);
  const uint32_t eqo = d.q.limbs ? out_element(d.q, i) : 0, ero = d.r.limbs ? out_element(d.r, i) : 0;
  if ((d.q.limbs && eqo >= d.q.count) || (d.r.limbs && ero >= d.r.count)) return;

  // Top nonzero divisor limb.
  int32_t bt = -1;
  for (int32_t j = (int32_t)d.b.nlimbs - 1; j >= 0; j--)
    if (load_limb(d.b.limbs, d.b.nlimbs, d.b.stride, eb, j)) {
      bt = j;
      break;
    }
  const int32_t m = (int32_t)d.a.nlimbs - bt - 1;  // quotient limbs - 1
  if (div_trivial(d, ea, eqo, ero, bt, m)) return;

  const int32_t z = BN - 1 - bt;
  const uint32_t s = __clz(load_limb(d.b.limbs, d.b.nlimbs, d.b.stride, eb, bt));
  uint32_t V[BN];
  {
    ShiftedDividend sb{&d.b, eb, z, s};
#pragma unroll
    for (int k = 0; k < BN; k++) V[k] = sb(k);
  }
  const uint32_t v = reciprocal_2by1(V[BN - 1]);
  ShiftedCursor sa{LimbCursor{&d.a, ea, -1, make_uint4(0, 0, 0, 0)}, LimbCursor{&d.a, ea, -1, make_uint4(0, 0, 0, 0)},
                   z, s};
  uint32_t W[BN + 1];
#pragma unroll
  for (int k = 0; k <= BN; k++) W[k] = sa(m + k);

  // quotient limbs collect in a group buffer and are stored 128 bits at a time
  uint32_t qb0 = 0, qb1 = 0, qb2 = 0, qb3 = 0;
  for (int32_t j = m; j >= 0; j--) {
    uint32_t qh = estimate_q(W[BN], W[BN - 1], BN >= 2 ? W[BN >= 2 ? BN - 2 : 0] : 0u, V[BN - 1],
                             BN >= 2 ? V[BN >= 2 ? BN - 2 : 0] : 0u, v, BN >= 2);
    // W -= qh * V: one mul.wide per limb; low halves at limbs 0..BN-1, high halves at 1..BN.
    uint64_t p[BN];
#pragma unroll
    for (int k = 0; k < BN; k++) p[k] = mul_wide(qh, V[k]);
    W[0] = sub_cc(W[0], (uint32_t)p[0]);
#pragma unroll
    for (int k = 1; k < BN; k++) W[k] = subc_cc(W[k], (uint32_t)p[k]);
    W[BN] = subc(W[BN], 0u);
    W[1] = sub_cc(W[1], (uint32_t)(p[0] >> 32));
#pragma unroll
    for (int k = 2; k <= BN; k++) W[k] = subc_cc(W[k], (uint32_t)(p[k - 1] >> 32));
    if (W[BN] != 0) {  // estimate was one too large: add back
      qh--;
      W[0] = add_cc(W[0], V[0]);
#pragma unroll
      for (int k = 1; k < BN; k++) W[k] = addc_cc(W[k], V[k]);
      W[BN] = addc(W[BN], 0u);
    }
    const uint32_t r4 = (uint32_t)j & 3u;
    qb0 = r4 == 0 ? qh : qb0;
    qb1 = r4 == 1 ? qh : qb1;
    qb2 = r4 == 2 ? qh : qb2;
    qb3 = r4 == 3 ? qh : qb3;
    if (r4 == 0) {
      const uint32_t g = (uint32_t)j >> 2;
      if (d.q.limbs && g * 4 < d.q.nlimbs) store_group(d.q.limbs, d.q.nlimbs, d.q.stride, eqo, g, make_uint4(qb0, qb1, qb2, qb3));
      qb0 = qb1 = qb2 = qb3 = 0;
    }
    if (j > 0) {
#pragma unroll
      for (int k = BN; k > 0; k--) W[k] = W[k - 1];
      W[0] = sa(j - 1);
    }
  }
  // limbs above the quotient's top group
  if (d.q.limbs) zero_limbs(d.q, eqo, (uint32_t)(m / 4 + 1) * 4);
  if (d.r.limbs) {
    // remainder = W >> S
    if (z == 0) {
      const uint32_t rg = div_up(d.r.nlimbs, 4);
#pragma unroll
      for (int g = 0; g < (BN + 3) / 4; g++) {
        uint32_t o[4];
#pragma unroll
        for (int t = 0; t < 4; t++) {
          const int k = 4 * g + t;
          const uint32_t lo = k < BN ? W[k < BN ? k : 0] : 0u;
          const uint32_t hi = (k + 1 < BN) ? W[k + 1 < BN ? k + 1 : 0] : 0u;
          o[t] = s ? ((lo >> s) | (hi << (32 - s))) : lo;
        }
        if ((uint32_t)g < rg) store_group(d.r.limbs, d.r.nlimbs, d.r.stride, ero, g, make_uint4(o[0], o[1], o[2], o[3]));
      }
      for (uint32_t g = (BN + 3) / 4; g < rg; g++)
        store_group(d.r.limbs, d.r.nlimbs, d.r.stride, ero, g, make_uint4(0, 0, 0, 0));
    } else {
#pragma unroll
      for (int k = 0; k < BN; k++) {
        int32_t dst = k - z;
        if (dst >= 0) {
          uint32_t hi = (k + 1 < BN) ? W[k + 1 < BN ? k + 1 : 0] : 0u;
          uint32_t val = s ? ((W[k] >> s) | (hi << (32 - s))) : W[k];
          write_limb(d.r, ero, (uint32_t)dst, val);
        }
      }
      zero_limbs(d.r, ero, (uint32_t)(BN - z));
    }
  }
}

// Same algorithm with the window and divisor in scratch (any divisor size).
__global__ void __launch_bounds__(256) divmod_stream_kernel(DivArgs d) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.count) return;
  const uint32_t ea = in_element(d.a, i), eb = in_element(d.b, i);
  const uint32_t eqo = d.q.limbs ? out_element(d.q, i) : 0, ero = d.r.limbs ? out_element(d.r, i) : 0;
  if ((d.q.limbs && eqo >= d.q.count) || (d.r.limbs && ero >= d.r.count)) return;
  int32_t bt = -1;
  for (int32_t j = (int32_t)d.b.nlimbs - 1; j >= 0; j--)
    if (load_limb(d.b.limbs, d.b.nlimbs, d.b.stride, eb, j)) {
      bt = j;
      break;
    }
  const int32_t m = (int32_t)d.a.nlimbs - bt - 1;
  if (div_trivial(d, ea, eqo, ero, bt, m)) return;
  const int32_t BN = bt + 1;  // exact divisor length: no whole-limb shift needed
  const uint32_t s = __clz(load_limb(d.b.limbs, d.b.nlimbs, d.b.stride, eb, bt));
  const size_t T = d.T;
  uint32_t *V = d.scratch + i;
  uint32_t *W = V + (size_t)d.b.nlimbs * T;
  ShiftedDividend sb{&d.b, eb, 0, s};
  for (int32_t k = 0; k < BN; k++) V[k * T] = sb(k);
  const uint32_t dtop = V[(BN - 1) * T], dnext = BN >= 2 ? V[(BN - 2) * T] : 0u;
  const uint32_t v = reciprocal_2by1(dtop);
  ShiftedDividend sa{&d.a, ea, 0, s};
  // W[k] for k = 0..BN holds window limb k; the window slides by moving its base.
  // Stored as a ring of BN+1 words: limb k at W[((base + k) % (BN+1)) * T].
  const int32_t WN = BN + 1;
  int32_t base = 0;
  auto wref = [&](int32_t k) -> uint32_t & { return W[(size_t)((base + k) % WN) * T]; };
  for (int32_t k = 0; k <= BN; k++) wref(k) = sa(m + k);
  for (int32_t j = m; j >= 0; j--) {
    uint32_t qh = estimate_q(wref(BN), wref(BN - 1), BN >= 2 ? wref(BN - 2) : 0u, dtop, dnext, v, BN >= 2);
    // W -= qh * V with a running borrow and product carry.
    uint32_t borrow = 0, carry = 0;
    for (int32_t k = 0; k < BN; k++) {
      uint64_t p = (uint64_t)qh * V[k * T] + carry;
      carry = (uint32_t)(p >> 32);
      uint64_t t = (uint64_t)wref(k) - (uint32_t)p - borrow;
      wref(k) = (uint32_t)t;
      borrow = (uint32_t)(t >> 63);
    }
    uint64_t t = (uint64_t)wref(BN) - carry - borrow;
    wref(BN) = (uint32_t)t;
    if ((uint32_t)t != 0) {
      qh--;
      uint32_t c = 0;
      for (int32_t k = 0; k < BN; k++) {
        uint64_t s2 = (uint64_t)wref(k) + V[k * T] + c;
        wref(k) = (uint32_t)s2;
        c = (uint32_t)(s2 >> 32);
      }
      wref(BN) += c;
    }
    if (d.q.limbs) write_limb(d.q, eqo, (uint32_t)j, qh);
    if (j > 0) {
      // slide: new limb k = old limb k-1, new limb 0 = next dividend limb
      base = (base + WN - 1) % WN;
      wref(0) = sa(j - 1);
    }
  }
  if (d.q.limbs) zero_limbs(d.q, eqo, (uint32_t)(m + 1));
  if (d.r.limbs) {
    for (int32_t k = 0; k < BN; k++) {
      uint32_t hi = (k + 1 < BN) ? wref(k + 1) : 0u;
      uint32_t val = s ? ((wref(k) >> s) | (hi << (32 - s))) : wref(k);
      write_limb(d.r, ero, (uint32_t)k, val);
    }
    zero_limbs(d.r, ero, (uint32_t)BN);
  }
}

typedef void (*DivLaunch)(const DivArgs &, int, cudaStream_t);
template <int BN>
static void launch_div(const DivArgs &d, int threads, cudaStream_t s) {
  divmod_reg_kernel<BN><<<grid_for(d.count, threads), threads, 0, s>>>(d);
}
static DivLaunch pick_div(uint32_t nb) {
  if (nb <= 1) return launch_div<1>;
  if (nb <= 2) return launch_div<2>;
  if (nb <= 4) return launch_div<4>;
  if (nb <= 6) return launch_div<6>;
  if (nb <= 8) return launch_div<8>;
  if (nb <= 12) return launch_div<12>;
  if (nb <= 16) return launch_div<16>;
  if (nb <= 24) return launch_div<24>;
  if (nb <= 32) return launch_div<32>;
  if (nb <= 48) return launch_div<48>;
  if (nb <= 64) return launch_div<64>;
  return nullptr;
}

bool div_has_register_kernel(uint32_t nb) { return pick_div(nb) != nullptr; }

static xmpError_t divmod_common(xmpHandle_t h, xmpIntegers_t q, xmpIntegers_t r, xmpIntegers_t a, xmpIntegers_t b,
                                uint32_t count, int qi, int ri, int ai, int bi, const ElemConfig *forced) {
  xmpExecutionPolicy_t pol = h->policy;
  DivArgs d;
  d.a = view_in(a, pol->indices[ai], pol->indices_count[ai]);
  d.b = view_in(b, pol->indices[bi], pol->indices_count[bi]);
  d.count = count;
  d.scratch = nullptr;
  d.T = 0;
  DivLaunch launch = pol->algorithm == xmpAlgorithmDigitMP ? nullptr : pick_div(b->nlimbs);
  if (pol->algorithm == xmpAlgorithmRegMP && !launch) return xmpErrorUnsupported;
  ElemConfig cfg;
  if (forced) {
    cfg = *forced;
  } else if (pol->algorithm == xmpAlgorithmDefault) {
    int slot = tuner_lookup(h, xmpTuneDivMod, b->precision, 0, count, nullptr);
    ElemConfig t;
    if (slot >= 0 && elem_candidate(xmpTuneDivMod, b->nlimbs, slot, &t)) cfg = t;
  }
  if (cfg.variant == 1) launch = nullptr;
  else if (!launch && forced) return xmpErrorUnsupported;
  const int threads = cfg.threads;

  OutTarget tq, tr;
  xmpError_t e;
  // Outputs are written digit by digit while the dividend is still being read: stage any alias.
  size_t q_bytes = q ? q->bytes : 0;
  bool q_stage = q && (q == a || q == b), r_stage = r && (r == a || r == b);
  if (q_stage || r_stage) {
    // size the in-place arena once so staging the second output cannot move the first
    e = ensure_tmp_out(h, (q_stage ? q_bytes : 0) + (r_stage ? r->bytes : 0));
    if (e != xmpErrorSuccess) return e;
  }
  if (q) {
    e = begin_output(h, q, q == a || q == b, true, &tq, 0);
    if (e != xmpErrorSuccess) return e;
  }
  if (r) {
    e = begin_output(h, r, r == a || r == b, true, &tr, tq.staged ? q_bytes : 0);
    if (e != xmpErrorSuccess) return e;
  }

  d.q = q ? view_out(q, tq.limbs, qi >= 0 ? pol->indices[qi] : nullptr) : OutView{nullptr, 0, 0, 0, nullptr};
  d.r = r ? view_out(r, tr.limbs, ri >= 0 ? pol->indices[ri] : nullptr) : OutView{nullptr, 0, 0, 0, nullptr};
  if (launch) {
    launch(d, threads, h->stream);
  } else {
    d.T = round_up(count, 256);
    e = ensure_scratch(h, (size_t)(2 * b->nlimbs + 1) * d.T * 4);
    if (e != xmpErrorSuccess) return e;
    d.scratch = (uint32_t *)h->scratch;
    divmod_stream_kernel<<<grid_for(count, threads), threads, 0, h->stream>>>(d);
  }
  if (q) {
    e = end_output(h, q, tq);
    if (e != xmpErrorSuccess) return e;
  }
  if (r) {
    e = end_output(h, r, tr);
    if (e != xmpErrorSuccess) return e;
  }
  return check_cuda();
}

xmpError_t divmod_entry(xmpHandle_t h, xmpIntegers_t q, xmpIntegers_t r, xmpIntegers_t a, xmpIntegers_t b,
                        uint32_t count, const ElemConfig *forced) {
  if (!h || !q || !r || !a || !b) return xmpErrorInvalidParameter;
  int dev = h->device;
  if (q->device != dev || r->device != dev || a->device != dev || b->device != dev) return xmpErrorInvalidDevice;
  if (count == 0) return xmpErrorSuccess;
  DeviceGuard guard(dev);
  xmpExecutionPolicy_t p = h->policy;
  if (r->count < count || q->count < count) return xmpErrorInvalidCount;
  if (p->indices[0] && p->indices_count[0] < count) return xmpErrorInvalidCount;
  if (p->indices[1] && p->indices_count[1] < count) return xmpErrorInvalidCount;
  if (q->precision < a->precision || r->precision < b->precision) return xmpErrorInvalidPrecision;
  if (q == r) return xmpErrorInvalidParameter;
  return divmod_common(h, q, r, a, b, count, 0, 1, 2, 3, forced);
}

static xmpError_t sync_after(xmpHandle_t h, xmpError_t e) {
  if (e != xmpErrorSuccess) return e;
  DeviceGuard guard(h->device);
  cudaStreamSynchronize(h->stream);
  return check_cuda();
}

}  // namespace xmpb

extern "C" {

xmpError_t XMPAPI xmpIntegersDivAsync(xmpHandle_t h, xmpIntegers_t q, const xmpIntegers_t a, const xmpIntegers_t b,
                                       uint32_t count) {
  if (!h || !q || !a || !b) return xmpErrorInvalidParameter;
  if (q->device != h->device || a->device != h->device || b->device != h->device) return xmpErrorInvalidDevice;
  if (count == 0) return xmpErrorSuccess;
  DeviceGuard guard(h->device);
  xmpExecutionPolicy_t p = h->policy;
  if (q->count < count) return xmpErrorInvalidCount;
  if (p->indices[0] && p->indices_count[0] < count) return xmpErrorInvalidCount;
  if (q->precision < a->precision) return xmpErrorInvalidPrecision;
  return divmod_common(h, q, nullptr, a, b, count, 0, -1, 1, 2, nullptr);
}
xmpError_t XMPAPI xmpIntegersDiv(xmpHandle_t h, xmpIntegers_t q, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count) {
  return sync_after(h, xmpIntegersDivAsync(h, q, a, b, count));
}

xmpError_t XMPAPI xmpIntegersModAsync(xmpHandle_t h, xmpIntegers_t m, const xmpIntegers_t a, const xmpIntegers_t b,
                                       uint32_t count) {
  if (!h || !m || !a || !b) return xmpErrorInvalidParameter;
  if (m->device != h->device || a->device != h->device || b->device != h->device) return xmpErrorInvalidDevice;
  if (count == 0) return xmpErrorSuccess;
  DeviceGuard guard(h->device);
  xmpExecutionPolicy_t p = h->policy;
  if (m->count < count) return xmpErrorInvalidCount;
  if (p->indices[0] && p->indices_count[0] < count) return xmpErrorInvalidCount;
  if (m->precision < b->precision) return xmpErrorInvalidPrecision;
  return divmod_common(h, nullptr, m, a, b, count, -1, 0, 1, 2, nullptr);
}
xmpError_t XMPAPI xmpIntegersMod(xmpHandle_t h, xmpIntegers_t m, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count) {
  return sync_after(h, xmpIntegersModAsync(h, m, a, b, count));
}

xmpError_t XMPAPI xmpIntegersDivModAsync(xmpHandle_t h, xmpIntegers_t q, xmpIntegers_t m, const xmpIntegers_t a,
                                          const xmpIntegers_t b, uint32_t count) {
  return divmod_entry(h, q, m, a, b, count, nullptr);
}
xmpError_t XMPAPI xmpIntegersDivMod(xmpHandle_t h, xmpIntegers_t q, xmpIntegers_t m, const xmpIntegers_t a,
                                     const xmpIntegers_t b, uint32_t count) {
  return sync_after(h, xmpIntegersDivModAsync(h, q, m, a, b, count));
}

}  // extern "C"
