// Fused CRT-RSA private operation, one kernel per batch (no counterpart in the
// reference library; it replaces the op sequence its CRT-RSA sample runs,
// samples/crt_rsa/rsa.cc:206-219: two mods, two powms, two muls, an add and a
// mod, each a separate launch with its own temporary arrays).
//
// Per instance, on a pair of groups of TPI lanes with L limbs each (n = TPI*L
// limbs = the precision of p and q, R = 2^(32n)), the first group working
// mod p and the second mod q:
//   1. Montgomery form of c mod p, for c of up to 2n limbs (c = c_hi R + c_lo):
//      Mont(c_lo, R^2) == c_lo R and Mont(c_hi, R^3) == c_hi R^2, each brought
//      below p, then added mod p.  The second group does the same mod q.
//   2. mp = c^dp mod p and, side by side, mq = c^dq mod q by fixed-window
//      exponentiation over max(precision of dp, dq) bits: the same number of
//      squarings and multiplies for every exponent (a zero window multiplies
//      by Mont(1)), so the schedule does not depend on the private exponent's
//      bits, and both groups of the pair run one instruction stream.
//   3. Garner's recombination on p: h = (mp - mq mod p) * qinv mod p, all in
//      Montgomery form, then m = mq + q*h as one 2n-limb product and sum.
// Nothing is stored between the steps except the window table (2^W entries
// in the scratch arena, as for powm); every intermediate stays in registers.
//
// Reducing a value y < R below an odd modulus N whose top bits may be clear
// uses Mont(Mont(y, R^2 mod N), 1), which is at most N, and one conditional
// subtraction (no division).
#pragma once
#include "powm_kernel.cuh"

namespace xmpb {

struct CrtArgs {
  ArrayView c, p, q, dp, dq, qinv;
  OutView out;
  uint32_t start;   // first op instance of this launch
  uint32_t count;   // op instances in this launch
  uint32_t window;  // fixed-window bits W
  uint32_t *table;  // per warp: 2^W entries x 32 lanes x L words
};

// r += x over the group; returns the carry out of the top lane (same in every lane).
template <int TPI, int L>
__device__ __forceinline__ uint32_t dadd(const Group<TPI> &G, uint32_t (&r)[L], const uint32_t (&x)[L]) {
  r[0] = add_cc(r[0], x[0]);
#pragma unroll
  for (int k = 1; k < L; k++) r[k] = addc_cc(r[k], x[k]);
  uint32_t co = addc(0u, 0u);
  if (TPI == 1) return co;
  uint32_t ones = r[0];
#pragma unroll
  for (int k = 1; k < L; k++) ones &= r[k];
  uint32_t out;
  // a lane that carried out is not all ones (r + x <= 2^(32L+1) - 2), so generate and propagate are exclusive
  uint32_t ci = G.lookahead(co, ones == kFull, &out);
  r[0] = add_cc(r[0], ci);
#pragma unroll
  for (int k = 1; k < L; k++) r[k] = addc_cc(r[k], 0u);
  return out;
}

// r <- (r + x) mod N for r, x < N.
template <int TPI, int L>
__device__ __forceinline__ void dadd_mod(const Group<TPI> &G, uint32_t (&r)[L], const uint32_t (&x)[L],
                                         const uint32_t (&n)[L]) {
  uint32_t co = dadd<TPI, L>(G, r, x);
  uint32_t d[L];
#pragma unroll
  for (int k = 0; k < L; k++) d[k] = r[k];
  uint32_t bo = dsub<TPI, L>(G, d, n, kFull);
  bool take = co || !bo;
#pragma unroll
  for (int k = 0; k < L; k++) r[k] = take ? d[k] : r[k];
}

// r <- (r - x) mod N for r, x < N.
template <int TPI, int L>
__device__ __forceinline__ void dsub_mod(const Group<TPI> &G, uint32_t (&r)[L], const uint32_t (&x)[L],
                                         const uint32_t (&n)[L]) {
  uint32_t bo = dsub<TPI, L>(G, r, x, kFull);
  uint32_t z[L];
#pragma unroll
  for (int k = 0; k < L; k++) z[k] = 0;
  // add N back when the difference went negative (the carry out cancels the borrow)
  uint32_t nm[L];
#pragma unroll
  for (int k = 0; k < L; k++) nm[k] = bo ? n[k] : z[k];
  dadd<TPI, L>(G, r, nm);
}

// y <- y mod N for any y < R: Mont(y, R^2) == y R, Mont(that, 1) <= N, then one conditional subtraction.
template <int TPI, int L>
__device__ __forceinline__ void dcanon(const Group<TPI> &G, uint32_t (&y)[L], const uint32_t (&n)[L], uint32_t np0,
                                       const uint32_t (&r2)[L]) {
  uint32_t t[L], one[L];
  mont_mul<TPI, L>(G, t, y, r2, n, np0);
#pragma unroll
  for (int k = 0; k < L; k++) one[k] = (G.lane == 0 && k == 0) ? 1u : 0u;
  mont_mul<TPI, L>(G, y, t, one, n, np0);
  dreduce<TPI, L>(G, y, n);
}

// Montgomery form (canonical, below N) of c mod N for c = c_hi R + c_lo.
template <int TPI, int L>
__device__ __forceinline__ void crt_reduce(const Group<TPI> &G, uint32_t (&xm)[L], const uint32_t (&clo)[L],
                                           const uint32_t (&chi)[L], const uint32_t (&n)[L], uint32_t np0,
                                           const uint32_t (&r2)[L]) {
  uint32_t r3[L], u[L];
  mont_mul<TPI, L>(G, r3, r2, r2, n, np0);  // R^3 mod N (below R)
  mont_mul<TPI, L>(G, u, chi, r3, n, np0);  // == c_hi R^2
  dcanon<TPI, L>(G, u, n, np0, r2);
  mont_mul<TPI, L>(G, xm, clo, r2, n, np0);  // == c_lo R
  dcanon<TPI, L>(G, xm, n, np0, r2);
  dadd_mod<TPI, L>(G, xm, u, n);
}

// acc <- Mont(x^e) for the exponent element `ee` scanned over its whole precision in W-bit windows;
// xm = Mont(x) below N.  Table slot e holds Mont(x^e), e < 2^W (slot 0 = R - N, Mont(1)).
template <int TPI, int L>
__device__ __forceinline__ void powm_fixed_full(const Group<TPI> &G, uint32_t (&acc)[L], const uint32_t (&xm)[L],
                                                const ArrayView &ex, uint32_t ee, uint32_t nbits,
                                                const uint32_t (&n)[L], uint32_t np0, uint32_t W, uint32_t *slot,
                                                const SqrSmem &sm) {
  const size_t es = (size_t)32 * L;
  uint32_t t[L], y[L];
#pragma unroll
  for (int k = 0; k < L; k++) t[k] = 0;
  dsub<TPI, L>(G, t, n, kFull);
  slot_store<L>(slot, t);
  slot_store<L>(slot + es, xm);
#pragma unroll
  for (int k = 0; k < L; k++) acc[k] = xm[k];
  const uint32_t entries = 1u << W;
#pragma unroll 1
  for (uint32_t e = 2; e < entries; e++) {
    mont_mul<TPI, L>(G, t, acc, xm, n, np0);
#pragma unroll
    for (int k = 0; k < L; k++) acc[k] = t[k];
    slot_store<L>(slot + e * es, acc);
  }
  const uint32_t nwin = (nbits + W - 1) / W;  // bits past the exponent's precision read as zero
  uint32_t win = exp_window(ex, ee, (nwin - 1) * W, W);
  slot_load<L>(slot + win * es, acc);
#pragma unroll 1
  for (int32_t wi = (int32_t)nwin - 2; wi >= 0; wi--) {
    win = exp_window(ex, ee, (uint32_t)wi * W, W);
#pragma unroll 1
    for (uint32_t s = 0; s < W; s++) {
      mont_square<TPI, L>(G, t, acc, n, np0, sm);
#pragma unroll
      for (int k = 0; k < L; k++) acc[k] = t[k];
    }
    slot_load<L>(slot + win * es, y);
    mont_mul<TPI, L>(G, t, acc, y, n, np0);
#pragma unroll
    for (int k = 0; k < L; k++) acc[k] = t[k];
  }
}

// (lo, hi) <- a * b over the group: the 2n-limb product, lane g holding limbs
// [gL, gL + L) of the low half and of the high half.  Rows of a * b_i on a
// shifting accumulator (as in mont_mul, without the reduction): after row i
// the group's lowest word is final product word i and goes to its owner lane.
template <int TPI, int L>
__device__ __forceinline__ void dmul_wide(const Group<TPI> &G, uint32_t (&lo)[L], uint32_t (&hi)[L],
                                          const uint32_t (&a)[L], const uint32_t (&b)[L]) {
  uint32_t r[L], c0 = 0, c1 = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    r[k] = 0;
    lo[k] = 0;
  }
#pragma unroll 1
  for (int src = 0; src < TPI; src++) {
#pragma unroll
    for (int k = 0; k < L; k++) {
      const uint32_t w = G.bcast(b[k], src);
      uint64_t p[L];
      row_products<L>(p, a, w);
      add_low_halves<L>(r, c0, c1, p);
      add_high_halves<L>(r, c0, c1, p);
      const uint32_t fin = G.bcast(r[0], 0);
      if (G.lane == (uint32_t)src) lo[k] = fin;
      const uint32_t t = G.from_next(r[0]);
#pragma unroll
      for (int j = 0; j < L - 1; j++) r[j] = r[j + 1];
      r[L - 1] = add_cc(t, c0);
      c0 = addc_fma(c1);
      c1 = 0;
    }
  }
  dnormalize<TPI, L>(G, r, c0);  // carry out of the top lane is zero: a * b < R^2
#pragma unroll
  for (int k = 0; k < L; k++) hi[k] = r[k];
}

// Limbs [off + lane*L, off + lane*L + L) of element e.
template <int TPI, int L>
__device__ __forceinline__ void load_lane_limbs_at(uint32_t (&x)[L], const ArrayView &v, uint32_t e, uint32_t lane,
                                                   uint32_t off) {
  const uint32_t j0 = off + lane * L;
  if (L % 4 == 0 && off % 4 == 0) {
#pragma unroll
    for (int m = 0; m < L / 4; m++) {
      uint4 g = load_group(v.limbs, v.nlimbs, v.stride, e, j0 / 4 + m);
      x[4 * m] = g.x;
      x[4 * m + 1] = g.y;
      x[4 * m + 2] = g.z;
      x[4 * m + 3] = g.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < L; k++) x[k] = load_limb(v.limbs, v.nlimbs, v.stride, e, j0 + k);
  }
}

template <int TPI, int L>
__device__ __forceinline__ void store_lane_limbs_at(const uint32_t (&x)[L], const OutView &v, uint32_t e,
                                                    uint32_t lane, uint32_t off) {
  const uint32_t j0 = off + lane * L;
  if (L % 4 == 0 && off % 4 == 0) {
#pragma unroll
    for (int m = 0; m < L / 4; m++) {
      uint32_t g = j0 / 4 + m;
      if (g * 4 < v.nlimbs)
        store_group(v.limbs, v.nlimbs, v.stride, e, g, make_uint4(x[4 * m], x[4 * m + 1], x[4 * m + 2], x[4 * m + 3]));
    }
  } else {
#pragma unroll
    for (int k = 0; k < L; k++)
      if (j0 + k < v.nlimbs) limb_ref(v.limbs, v.stride, e, j0 + k) = x[k];
  }
}

// Modulus constants of element e of `mv`: N, n0' and R^2 mod N.
template <int TPI, int L>
__device__ __forceinline__ uint32_t crt_modulus(const Group<TPI> &G, uint32_t (&n)[L], uint32_t (&r2)[L],
                                                const ArrayView &mv, uint32_t e) {
  load_lane_limbs_at<TPI, L>(n, mv, e, G.lane, 0);
  const uint32_t np0 = neg_inv32(G.bcast(n[0], 0));
  compute_r2<TPI, L>(G, r2, n, np0);
  return np0;
}

// The two exponentiations of an instance run side by side on two adjacent
// groups of one warp (lanes [0, TPI) of the pair work mod p, lanes
// [TPI, 2 TPI) mod q), so a batch has twice as many independent groups as
// instances and each group does one exponentiation: measured on B200 at
// 16,384 RSA-2048 operations (4 lanes x 8 limbs), 17.8 ms against 21.6 ms
// with both exponentiations on one group in turn, and at 1,024 operations
// (8 x 4) 2.0 ms against 4.1 ms.  The results meet with one shuffle per limb
// (lane l and l ^ TPI hold the same limbs of mp and mq); both groups then run
// the same Garner steps on their own modulus -- the first group's are
// h = (mp - mq mod p) * qinv mod p and m = mq + q h, which it stores; the
// second group's mirror image is discarded.
template <int TPI, int L>
__global__ void __launch_bounds__(128) crt_kernel(CrtArgs a) {
  static_assert(TPI <= 16, "both groups of a pair sit in one warp");
  const SqrSmem sm = powm_smem_setup<TPI, L>();
  Group<TPI> G;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t local = gtid / (2 * TPI);
  const bool second = ((gtid / TPI) & 1u) != 0;  // this group works mod q
  const bool valid = local < a.count;
  // pairs past the end run a copy of the last instance so every shuffle sees a full warp
  const uint32_t i = a.start + (valid ? local : a.count - 1);
  uint32_t *slot = a.table + (size_t)(gtid >> 5) * ((size_t)32 * L * (1u << a.window)) + (size_t)(threadIdx.x & 31) * L;
  const ArrayView mv = second ? a.q : a.p, ov = second ? a.p : a.q, ev = second ? a.dq : a.dp;
  const uint32_t em = in_element(mv, i);
  const uint32_t nbits = max(a.dp.nlimbs, a.dq.nlimbs) * 32;
  const uint32_t n_limbs = TPI * L;

  uint32_t n[L], r2[L], xm[L];
  uint32_t np0;
  {
    uint32_t clo[L], chi[L];
    const uint32_t ec = in_element(a.c, i);
    load_lane_limbs_at<TPI, L>(clo, a.c, ec, G.lane, 0);
    load_lane_limbs_at<TPI, L>(chi, a.c, ec, G.lane, n_limbs);
    np0 = crt_modulus<TPI, L>(G, n, r2, mv, em);
    crt_reduce<TPI, L>(G, xm, clo, chi, n, np0, r2);
  }
  uint32_t one[L], acc[L], mine[L], other[L];
#pragma unroll
  for (int k = 0; k < L; k++) one[k] = (G.lane == 0 && k == 0) ? 1u : 0u;
  powm_fixed_full<TPI, L>(G, acc, xm, ev, in_element(ev, i), nbits, n, np0, a.window, slot, sm);
  mont_mul<TPI, L>(G, mine, acc, one, n, np0);
  dreduce<TPI, L>(G, mine, n);
#pragma unroll
  for (int k = 0; k < L; k++) other[k] = __shfl_xor_sync(kFull, mine[k], TPI);
  // Garner on this group's modulus (p for the first group)
  uint32_t h[L];
  {
    compute_r2<TPI, L>(G, r2, n, np0);
    uint32_t d[L], t[L], u[L];
#pragma unroll
    for (int k = 0; k < L; k++) d[k] = other[k];
    dcanon<TPI, L>(G, d, n, np0, r2);  // mq mod p
#pragma unroll
    for (int k = 0; k < L; k++) t[k] = mine[k];
    dsub_mod<TPI, L>(G, t, d, n);  // D = (mp - mq) mod p
    mont_mul<TPI, L>(G, d, t, r2, n, np0);  // == D R
    load_lane_limbs_at<TPI, L>(u, a.qinv, in_element(a.qinv, i), G.lane, 0);
    mont_mul<TPI, L>(G, t, u, r2, n, np0);  // == qinv R
    mont_mul<TPI, L>(G, u, d, t, n, np0);   // == D qinv R
    mont_mul<TPI, L>(G, h, u, one, n, np0);  // == D qinv, at most p
    dreduce<TPI, L>(G, h, n);
  }
  // m = mq + q h (below pq)
  uint32_t lo[L], hi[L];
  load_lane_limbs_at<TPI, L>(n, ov, in_element(ov, i), G.lane, 0);
  dmul_wide<TPI, L>(G, lo, hi, n, h);
  uint32_t co = dadd<TPI, L>(G, lo, other);
  uint32_t cw[L];
#pragma unroll
  for (int k = 0; k < L; k++) cw[k] = (G.lane == 0 && k == 0) ? co : 0u;
  dadd<TPI, L>(G, hi, cw);
  if (valid && !second) {
    const uint32_t o = out_element(a.out, i);
    if (o < a.out.count) {
      store_lane_limbs_at<TPI, L>(lo, a.out, o, G.lane, 0);
      store_lane_limbs_at<TPI, L>(hi, a.out, o, G.lane, n_limbs);
    }
  }
}

}  // namespace xmpb
