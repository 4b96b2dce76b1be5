// Montgomery arithmetic for integers spread over TPI lanes with L limbs per
// lane (TPI = 1 is the per-thread distribution).  Lane g of a group holds limbs
// [g*L, g*L + L) of each operand; capacity n = TPI*L limbs, R = 2^(32n).
//
// Replaces the reference's per-thread reduce/mul (regmp/reduce_imad.h:26-63,
// regmp/mul_imad.h:26-103) and the warp-distributed WarpMP::mulmod
// (warpmp/mulmod_imad.h:24-183).  The algorithm is interleaved CIOS
// (coarsely integrated operand scanning): for each word b_i of B, broadcast
// from its owner lane with shfl, acc += A*b_i; q = acc_0 * (-N^-1 mod 2^32);
// acc += N*q; acc >>= 32 (a one-lane shfl shift).  Each lane keeps two extra
// carry words above its limbs, so no carry ever crosses a lane inside the
// loop; after the last word the pending carries are delivered with one shfl
// and one ballot-based carry-lookahead (generate/propagate masks), and an
// overflow past R is removed by a conditional subtraction of N, also resolved
// by ballot.  Inputs below R give a result below R that is congruent to
// A*B*R^-1 mod N ("almost Montgomery"); a final compare-subtract makes it
// exact.
#pragma once
#include "carry.cuh"

namespace xmpb {

constexpr uint32_t kFull = 0xffffffffu;

template <int TPI>
struct Group {
  uint32_t lane;  // 0..TPI-1 within the group
  uint32_t base;  // warp lane of the group's lane 0
  __device__ __forceinline__ Group() {
    uint32_t l = threadIdx.x & 31;
    lane = l % TPI;
    base = l - lane;
  }
  __device__ __forceinline__ uint32_t bcast(uint32_t v, uint32_t src) const {
    return TPI == 1 ? v : __shfl_sync(kFull, v, src, TPI);
  }
  // v of lane+1 (0 for the top lane)
  __device__ __forceinline__ uint32_t from_next(uint32_t v) const {
    if (TPI == 1) return 0;
    uint32_t t = __shfl_down_sync(kFull, v, 1, TPI);
    return lane == TPI - 1 ? 0u : t;
  }
  // v of lane-1 (0 for lane 0)
  __device__ __forceinline__ uint32_t from_prev(uint32_t v) const {
    if (TPI == 1) return 0;
    uint32_t t = __shfl_up_sync(kFull, v, 1, TPI);
    return lane == 0 ? 0u : t;
  }
  __device__ __forceinline__ uint32_t seg_max(uint32_t v) const {
#pragma unroll
    for (int o = TPI / 2; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(kFull, v, o, TPI));
    return v;
  }
  // One-bit carry (or borrow) lookahead across the group's lanes.
  //   gen : this lane emits a carry into lane+1
  //   prop: this lane passes an incoming carry on (all ones for carries,
  //         all zeros for borrows)
  // Returns the carry entering this lane; *out = carry leaving the top lane.
  // With G and P the group's ballot bits, the incoming carries are the bits of
  // (P + 2G) xor P: adding 2G to P ripples each generated carry through the
  // following run of propagating lanes.
  __device__ __forceinline__ uint32_t lookahead(uint32_t gen, uint32_t prop, uint32_t *out) const {
    if (TPI == 1) {
      *out = gen;
      return 0;
    }
    uint32_t G = __ballot_sync(kFull, gen != 0), P = __ballot_sync(kFull, prop != 0);
    const uint64_t mask = (TPI == 32) ? 0xffffffffull : ((1ull << TPI) - 1);
    uint64_t g = ((uint64_t)G >> base) & mask, p = ((uint64_t)P >> base) & mask;
    uint64_t s = p + (g << 1);
    *out = (uint32_t)(s >> TPI) & 1u;
    return (uint32_t)(((s ^ p) >> lane) & 1u);
  }
};

// r -= x & m over the whole group (m is 0 or ~0); returns the borrow out of
// the top lane (same value in every lane of the group).
template <int TPI, int L>
__device__ __forceinline__ uint32_t dsub(const Group<TPI> &G, uint32_t (&r)[L], const uint32_t (&x)[L], uint32_t m) {
  r[0] = sub_cc(r[0], x[0] & m);
#pragma unroll
  for (int k = 1; k < L; k++) r[k] = subc_cc(r[k], x[k] & m);
  uint32_t bo = subc(0u, 0u) & 1u;
  if (TPI == 1) return bo;
  uint32_t zero = r[0];
#pragma unroll
  for (int k = 1; k < L; k++) zero |= r[k];
  uint32_t out;
  uint32_t bin = G.lookahead(bo, zero == 0u, &out);
  r[0] = sub_cc(r[0], bin);
#pragma unroll
  for (int k = 1; k < L; k++) r[k] = subc_cc(r[k], 0u);
  return out;
}

// Delivers each lane's pending carry word c0 (weight 2^(32L) above the lane)
// into the next lane; returns the total carry leaving the top lane.
template <int TPI, int L>
__device__ __forceinline__ uint32_t dnormalize(const Group<TPI> &G, uint32_t (&r)[L], uint32_t c0) {
  if (TPI == 1) return c0;
  uint32_t cin = G.from_prev(c0);
  uint32_t top = G.bcast(c0, TPI - 1);
  r[0] = add_cc(r[0], cin);
#pragma unroll
  for (int k = 1; k < L; k++) r[k] = addc_cc(r[k], 0u);
  uint32_t co = addc(0u, 0u);
  uint32_t ones = r[0];
#pragma unroll
  for (int k = 1; k < L; k++) ones &= r[k];
  uint32_t out;
  uint32_t ci = G.lookahead(co, ones == kFull, &out);
  r[0] = add_cc(r[0], ci);
#pragma unroll
  for (int k = 1; k < L; k++) r[k] = addc_cc(r[k], 0u);
  return top + out;
}

// A row of a Montgomery multiplication adds a * w (w a word of B) and then
// n * q (q the quotient digit) to the lane's accumulator (r, c0, c1): r has
// L limbs, c0 is the word above them and c1 the word above c0.  Each limb's
// full 32x32 product is one mul.wide.u32 (a single wide multiply on the
// FMA-heavy pipe; a separate mad.hi costs well over twice a mad.lo there, and
// a mad.wide with a 32-bit addend costs two FMA-pipe instructions), and the
// products are independent of each other.  Two add chains on the integer ALU
// pipe fold each row's products in: the low halves into r[0..L-1] (carry
// into c0, c1), then the high halves into r[1..L-1], c0.  The carry-in-only
// tail steps go to the FMA pipe (addc_fma).
template <int L>
__device__ __forceinline__ void row_products(uint64_t (&p)[L], const uint32_t (&a)[L], uint32_t w) {
#pragma unroll
  for (int k = 0; k < L; k++) p[k] = mul_wide(a[k], w);
}

template <int L>
__device__ __forceinline__ void add_low_halves(uint32_t (&r)[L], uint32_t &c0, uint32_t &c1, const uint64_t (&p)[L]) {
  r[0] = add_cc(r[0], (uint32_t)p[0]);
#pragma unroll
  for (int k = 1; k < L; k++) r[k] = addc_cc(r[k], (uint32_t)p[k]);
  c0 = addc_cc(c0, 0u);
  c1 = addc_fma(c1);
}

template <int L>
__device__ __forceinline__ void add_high_halves(uint32_t (&r)[L], uint32_t &c0, uint32_t &c1, const uint64_t (&p)[L]) {
  if (L > 1) {
    r[1] = add_cc(r[1], (uint32_t)(p[0] >> 32));
#pragma unroll
    for (int k = 2; k < L; k++) r[k] = addc_cc(r[k], (uint32_t)(p[k - 1] >> 32));
    c0 = addc_cc(c0, (uint32_t)(p[L - 1] >> 32));
  } else {
    c0 = add_cc(c0, (uint32_t)(p[0] >> 32));
  }
  c1 = addc_fma(c1);
}

// Row schedule per shape.  The shuffles of a row -- the next word of b, the
// quotient digit (lane 0's r[0] once the low halves of a * w are in) and the
// one-word shift (r[0] once the low halves of n * q are in) -- can be issued
// as soon as their inputs exist ("early") or where the chains leave them.
// Which is faster depends on how the scheduler interleaves the chains, so it
// was measured for every registered shape on a B200 (a full wave of
// instances and a single instance, 512- and up to 4096-bit exponents) and is
// fixed here: early where it was faster at a full wave, or where throughput
// stayed within 1.5% and single-instance latency dropped by 3% or more
// (e.g. 32 lanes x 3 limbs, 3072 bits: one exponentiation 20.3 -> 16.3 ms;
// 8 lanes x 4, 1024 bits x 4,096: 3.12 -> 3.01 ms), late elsewhere (e.g.
// 4 lanes x 12 limbs: 10% slower early).
__host__ __device__ constexpr bool row_early_shuffles(int TPI, int L) {
  return (TPI == 2 && (L == 3 || L == 8)) || (TPI == 4 && (L == 1 || L == 3 || L == 5 || L == 6)) ||
         (TPI == 8 && (L == 3 || L == 4 || L == 5 || L == 6)) || (TPI == 16 && (L == 1 || L == 3 || L == 6)) ||
         (TPI == 32 && (L == 1 || L == 3 || L == 8 || L == 12));
}

// r = a * b * R^-1 (mod N), almost reduced (r < R).  a, b < R; r must not alias a or b.
template <int TPI, int L>
__device__ __forceinline__ void mont_mul(const Group<TPI> &G, uint32_t (&r)[L], const uint32_t (&a)[L],
                                         const uint32_t (&b)[L], const uint32_t (&n)[L], uint32_t np0) {
  uint32_t c0 = 0, c1 = 0;
#pragma unroll
  for (int k = 0; k < L; k++) r[k] = 0;
  constexpr bool kEarly = row_early_shuffles(TPI, L);
  uint32_t w_next = kEarly ? G.bcast(b[0], 0) : 0u;
#pragma unroll 1
  for (int src = 0; src < TPI; src++) {
#pragma unroll
    for (int k = 0; k < L; k++) {
      uint32_t w;
      if constexpr (kEarly) {
        // the next row's word of b does not depend on this row: broadcast it now
        w = w_next;
        w_next = (k + 1 < L) ? G.bcast(b[k + 1 < L ? k + 1 : 0], src) : G.bcast(b[0], src + 1 < TPI ? src + 1 : 0);
      } else {
        w = G.bcast(b[k], src);
      }
      uint64_t p[L], s[L];
      row_products<L>(p, a, w);
      uint32_t q, t;
      // The quotient digit needs only the low word (lane 0's r[0]), final
      // once the low halves of a * w are in; forming the n * q products
      // before the high-half chain of a * w gives the scheduler independent
      // multiplies to overlap with that chain (measured: +3% at 2048 bits).
      if constexpr (kEarly) {
        r[0] = add_cc(r[0], (uint32_t)p[0]);
        q = G.bcast(r[0], 0) * np0;
#pragma unroll
        for (int j = 1; j < L; j++) r[j] = addc_cc(r[j], (uint32_t)p[j]);
        c0 = addc_cc(c0, 0u);
        c1 = addc_fma(c1);
        row_products<L>(s, n, q);
        add_high_halves<L>(r, c0, c1, p);
        // r[0] is final after the first low half of n * q: shift it out now
        r[0] = add_cc(r[0], (uint32_t)s[0]);
        t = G.from_next(r[0]);
#pragma unroll
        for (int j = 1; j < L; j++) r[j] = addc_cc(r[j], (uint32_t)s[j]);
        c0 = addc_cc(c0, 0u);
        c1 = addc_fma(c1);
        add_high_halves<L>(r, c0, c1, s);
      } else {
        add_low_halves<L>(r, c0, c1, p);
        q = G.bcast(r[0], 0) * np0;
        row_products<L>(s, n, q);
        add_high_halves<L>(r, c0, c1, p);
        add_low_halves<L>(r, c0, c1, s);
        add_high_halves<L>(r, c0, c1, s);
        t = G.from_next(r[0]);
      }
      // divide by 2^32: lane 0's low limb is zero now; every other lane's low
      // limb moves to the top of the lane below, on top of that lane's c0.
#pragma unroll
      for (int j = 0; j < L - 1; j++) r[j] = r[j + 1];
      r[L - 1] = add_cc(t, c0);
      c0 = addc_fma(c1);
      c1 = 0;
    }
  }
  uint32_t ovf = dnormalize<TPI, L>(G, r, c0);
  dsub<TPI, L>(G, r, n, 0u - ovf);
}

// x <- x mod N for x < 2N.
template <int TPI, int L>
__device__ __forceinline__ void dreduce(const Group<TPI> &G, uint32_t (&x)[L], const uint32_t (&n)[L]) {
  uint32_t d[L];
#pragma unroll
  for (int k = 0; k < L; k++) d[k] = x[k];
  uint32_t borrow = dsub<TPI, L>(G, d, n, kFull);
#pragma unroll
  for (int k = 0; k < L; k++) x[k] = borrow ? x[k] : d[k];
}

// v <- 2v mod N for v < N (exact) when `commit`, else v unchanged.  Every
// lane of the warp executes the shuffles and ballots either way, so groups
// that need fewer doublings than their warp neighbours stay in step.
template <int TPI, int L>
__device__ __forceinline__ void dmod_double(const Group<TPI> &G, uint32_t (&v)[L], const uint32_t (&n)[L],
                                            bool commit) {
  uint32_t top = v[L - 1] >> 31;
  uint32_t in = G.from_prev(top);
  uint32_t ovf = G.bcast(top, TPI - 1);
  uint32_t w[L], d[L];
#pragma unroll
  for (int k = L - 1; k > 0; k--) w[k] = (v[k] << 1) | (v[k - 1] >> 31);
  w[0] = (v[0] << 1) | in;
#pragma unroll
  for (int k = 0; k < L; k++) d[k] = w[k];
  uint32_t borrow = dsub<TPI, L>(G, d, n, kFull);
  bool take = ovf || !borrow;
#pragma unroll
  for (int k = 0; k < L; k++) v[k] = commit ? (take ? d[k] : w[k]) : v[k];
}

// Bit length of the group's integer (0 for zero), same value in every lane.
template <int TPI, int L>
__device__ __forceinline__ uint32_t dbitlen(const Group<TPI> &G, const uint32_t (&x)[L]) {
  uint32_t bl = 0;
#pragma unroll
  for (int k = 0; k < L; k++)
    if (x[k]) bl = (G.lane * L + k) * 32 + 32 - __clz(x[k]);
  return G.seg_max(bl);
}

// r2 <- R^2 mod N (almost reduced, < R), N odd.  Start from 2^(b-1) < N
// (b = bitlen N), double exactly up to 2^(32n + s) mod N = Mont(2^s), then
// Montgomery-square j times: Mont(2^(s 2^j)) = Mont(R) = R^2 mod N, where
// 32n = s * 2^j with s odd.  All loop counts are warp-uniform (the doubling
// count is the warp maximum, with per-group commit), so every shfl and ballot
// sees the whole warp.  N = 1 gives r2 = 0.
template <int TPI, int L>
__device__ __forceinline__ void compute_r2(const Group<TPI> &G, uint32_t (&r2)[L], const uint32_t (&n)[L],
                                           uint32_t np0) {
  const uint32_t bits = 32u * TPI * L;
  const uint32_t j = __ffs(bits) - 1;  // trailing zeros
  const uint32_t s = bits >> j;
  const uint32_t b = dbitlen<TPI, L>(G, n);
  const bool trivial = b <= 1;  // N == 1 (or the undefined N == 0)
  const uint32_t tb = trivial ? 0u : b - 1;
#pragma unroll
  for (int k = 0; k < L; k++) r2[k] = ((G.lane * L + k) == (tb >> 5)) ? (1u << (tb & 31)) : 0u;
  const uint32_t doublings = trivial ? 0u : bits - b + 1 + s;
  const uint32_t dmax = __reduce_max_sync(kFull, doublings);
#pragma unroll 1
  for (uint32_t d = 0; d < dmax; d++) dmod_double<TPI, L>(G, r2, n, d < doublings);
  uint32_t t[L];
#pragma unroll 1
  for (uint32_t q = 0; q < j; q++) {
    mont_mul<TPI, L>(G, t, r2, r2, n, np0);
#pragma unroll
    for (int k = 0; k < L; k++) r2[k] = t[k];
  }
  if (trivial) {
#pragma unroll
    for (int k = 0; k < L; k++) r2[k] = 0;
  }
}

}  // namespace xmpb
