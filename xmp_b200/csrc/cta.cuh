// Latency distribution: one exponentiation per CTA.
//
// The lane kernels (powm_kernel.cuh) multiply by interleaved CIOS, whose n
// rows per Montgomery product each wait on the previous row's quotient digit:
// a lone 2048-bit exponentiation on one warp (32 lanes x 2 limbs) takes 8 ms,
// the floor under a server's latency.  Here a CTA of (n/4)^2 threads forms a
// Montgomery product as three whole-operand products with no digit-serial
// dependency (separated operand scanning, Montgomery's REDC on the whole low
// half):
//   T = a b,   m = (T mod R) N' mod R   (N' = -N^-1 mod R),   U = T + m N,
//   r = U / R  (< 2N; one conditional subtraction of N makes it < N).
// Each product x y (n words each) is cut into 4 x 4-word tiles, one per thread
// (16 mul.wide; four row chains added as a tree give the tile's exact 8-word
// product); the tiles on one anti-diagonal share a word offset, so thread
// (d, w) sums word w of the tiles of diagonal d (64-bit accumulators, no
// carries yet) into a word-linear array (low and high tile halves apart);
// one warp then resolves n words, K = n/32 per lane: each word's column sum,
// the bits above 32 of the two words below folded in, and the remaining
// one-bit carries by a ballot lookahead (the incoming carries of 32 lanes are
// the bits of (P + 2G + cin) xor P).  Of U only the high half is resolved and
// of T only the low half (the product schedule below).  A product costs 3
// barriers, a Montgomery product 9.  Operands, the window table and all
// intermediates live in the CTA's shared memory.  It does not reach the lane
// kernels' throughput, so it serves small batches.
//
// Supported sizes: n = 32, 64, 96, 128 limbs (1024 .. 4096 bits; (n/4)^2 a
// multiple of 32 threads); smaller precisions are padded up (any R > N works).
#pragma once
#include "powm_kernel.cuh"

namespace xmpb {

template <int N>
struct CtaShape {
  static_assert(N % 32 == 0 && N >= 32 && N <= 128, "CTA distribution: 32, 64, 96 or 128 limbs");
  static constexpr int Q = N / 4;             // tiles per operand
  static constexpr int THREADS = Q * Q;       // one tile per thread
  static constexpr int DIAG = 2 * Q - 1;      // anti-diagonals of the tile grid
  static constexpr int WARPS = THREADS / 32;
};

// Column sums of a product, word i = lo[4 + i] + hi[4 + i]: lo takes the low four words of the
// tiles (anti-diagonal d, word w < 4 -> i = 4 d + w), hi their high four (w >= 4 -> i = 4 d + w);
// four zero words below word 0 and above word 2n - 1 (never written).
template <int N>
struct ColSums {
  unsigned long long lo[2 * N + 8], hi[2 * N + 8];
};

// Shared memory of one CTA (the window table follows it, `entries` x N words).
template <int N>
struct CtaSmem {
  uint32_t tile[CtaShape<N>::THREADS * 8];  // 8 words per tile
  ColSums<N> dsum;   // column sums of the current product
  ColSums<N> dsumT;  // those of T = a b, kept for U = T + m N
  uint32_t flag[2][32];                     // per warp: carry out with no carry in, all-propagate
  uint32_t t[2 * N];                        // T = a b
  uint32_t m[N], u[N];                      // m; the high half of U before its final subtraction
  uint32_t n[N], np[N];                     // modulus, -N^-1 mod R
  uint32_t acc[N], x[N], k[N];              // accumulator, operand, a small constant (1 or 2)
  uint32_t misc[4];
};

template <int N>
__host__ __device__ constexpr uint32_t cta_smem_bytes(uint32_t entries) {
  static_assert(sizeof(CtaSmem<N>) % 16 == 0, "the window table after CtaSmem is read in 16-byte words");
  return (uint32_t)sizeof(CtaSmem<N>) + entries * N * 4;
}

// v (8 words) = x (4 words) * y (4 words): four row products x y_j (5 words, one carry chain
// each, independent), added pairwise (rows 0 + 1, rows 2 + 3), then the two halves: a dependent
// carry path of 4 + 5 + 6 additions instead of one chain through all 16 products.
__device__ __forceinline__ void cta_row(uint32_t (&r)[5], const uint32_t (&x)[4], uint32_t y) {
  const uint64_t p0 = mul_wide(x[0], y), p1 = mul_wide(x[1], y), p2 = mul_wide(x[2], y), p3 = mul_wide(x[3], y);
  r[0] = (uint32_t)p0;
  r[1] = add_cc((uint32_t)(p0 >> 32), (uint32_t)p1);
  r[2] = addc_cc((uint32_t)(p1 >> 32), (uint32_t)p2);
  r[3] = addc_cc((uint32_t)(p2 >> 32), (uint32_t)p3);
  r[4] = addc((uint32_t)(p3 >> 32), 0u);
}

// a (6 words) = r (5 words) + q (5 words) * 2^32.
__device__ __forceinline__ void cta_add_shift(uint32_t (&a)[6], const uint32_t (&r)[5], const uint32_t (&q)[5]) {
  a[0] = r[0];
  a[1] = add_cc(r[1], q[0]);
  a[2] = addc_cc(r[2], q[1]);
  a[3] = addc_cc(r[3], q[2]);
  a[4] = addc_cc(r[4], q[3]);
  a[5] = addc(q[4], 0u);
}

__device__ __forceinline__ void cta_tile(uint32_t (&v)[8], const uint32_t (&x)[4], const uint32_t (&y)[4]) {
  uint32_t r0[5], r1[5], r2[5], r3[5], A[6], B[6];
  cta_row(r0, x, y[0]);
  cta_row(r1, x, y[1]);
  cta_row(r2, x, y[2]);
  cta_row(r3, x, y[3]);
  cta_add_shift(A, r0, r1);
  cta_add_shift(B, r2, r3);
  v[0] = A[0];
  v[1] = A[1];
  v[2] = add_cc(A[2], B[0]);
  v[3] = addc_cc(A[3], B[1]);
  v[4] = addc_cc(A[4], B[2]);
  v[5] = addc_cc(A[5], B[3]);
  v[6] = addc_cc(B[4], 0u);
  v[7] = addc(B[5], 0u);
}

// Carry lookahead over W words held one per thread (threads [0, W)): word
// value z = limb + 2^32 g with g one bit (g = 1 only when limb = 0).  Returns
// this thread's carry in; *out = the carry out of word W - 1 (every thread).
// All threads of the CTA call it (one barrier).
template <int N, int W>
__device__ __forceinline__ uint32_t cta_carries(CtaSmem<N> &s, uint32_t g, uint32_t p, uint32_t *out) {
  static_assert(W % 32 == 0 && W <= CtaShape<N>::THREADS, "whole warps of words");
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int WW = W / 32;
  uint32_t G = 0, P = 0;
  if (warp < WW) {
    G = __ballot_sync(kFull, g != 0);
    P = __ballot_sync(kFull, p != 0);
    if (lane == 0) {
      s.flag[0][warp] = (uint32_t)((((unsigned long long)P + ((unsigned long long)G << 1)) >> 32) & 1ull);
      s.flag[1][warp] = P == kFull;
    }
  }
  __syncthreads();
  uint32_t cin = 0, total = 0;
#pragma unroll
  for (int k = 0; k < WW; k++) {
    if (k == warp) cin = total;
    total = s.flag[0][k] | (s.flag[1][k] & total);
  }
  *out = total;
  const unsigned long long sum = (unsigned long long)P + ((unsigned long long)G << 1) + cin;
  return (uint32_t)(((sum ^ P) >> lane) & 1ull);
}

// r = x - y over n words if `take` says so after the fact: with B the borrow
// out of x - y, r = x - y when force || !B, else r = x.  Returns 1 when it
// subtracted.  r may alias x.
template <int N>
__device__ __forceinline__ uint32_t cta_sub_if(CtaSmem<N> &s, uint32_t *r, const uint32_t *x, const uint32_t *y,
                                               uint32_t force) {
  const int i = threadIdx.x;
  uint32_t xv = 0, d = 0, g = 0, p = 0;
  if (i < N) {
    xv = x[i];
    const uint32_t yv = y[i];
    d = xv - yv;
    g = xv < yv;
    p = xv == yv;
  }
  uint32_t borrow;
  const uint32_t b = cta_carries<N, N>(s, g, p, &borrow);
  const uint32_t take = force | (borrow ^ 1u);
  if (i < N) r[i] = take ? d - b : xv;
  __syncthreads();
  return take;
}

// ---- the product schedule ---------------------------------------------------------
// Montgomery's U = T + m N is 0 mod R, so its low half need not be formed: with
// s_i the column sums of U, the carry out of word i < n - 1 into word i + 1 is
// exactly hi(s_i) + (lo(s_i) != 0) (the word itself must come out 0), so the
// carry into word n is c = hi(s_(n-1)) + (lo(s_(n-1)) != 0) and only the words
// >= n - 1 of U are summed.  T's high half is therefore never resolved either:
// its raw column sums (dsumT) are added into U's by the same jobs that sum
// m N's diagonals; only T's low half is resolved (it is m's operand).
// (Squarings that form only the tiles on and above the tile grid's diagonal,
// counting the others twice, measured slower with the per-diagonal layout: one
// 2048-bit exponentiation 4.76 against 4.42 ms -- the tile phase does not get
// shorter and the diagonal sums pay for the extra predicates.  Sums over a
// warp-uniform range of tiles instead of all n/4 with predicates, 64-bit
// uncarried tile columns, and two-word jobs where one-word jobs fit the CTA
// all measured slower than the form here.)
enum CtaCols : int { kColsFull = 0, kColsLow = 1, kColsHigh = 2 };

template <int N, int MODE>
__device__ __forceinline__ void cta_cols(CtaSmem<N> &s, const uint32_t *x, const uint32_t *y,
                                         ColSums<N> &out) {
  using C = CtaShape<N>;
  const int tid = threadIdx.x, ti = tid / C::Q, tj = tid % C::Q;
  const bool need = MODE == kColsLow ? ti + tj < C::Q : MODE == kColsHigh ? ti + tj >= C::Q - 2 : true;
  uint32_t v[8];
  if (need) {
    const uint4 xa = *reinterpret_cast<const uint4 *>(x + 4 * ti);
    const uint4 yb = *reinterpret_cast<const uint4 *>(y + 4 * tj);
    const uint32_t xw[4] = {xa.x, xa.y, xa.z, xa.w}, yw[4] = {yb.x, yb.y, yb.z, yb.w};
    cta_tile(v, xw, yw);
    uint4 *tp = reinterpret_cast<uint4 *>(&s.tile[tid * 8]);
    tp[0] = make_uint4(v[0], v[1], v[2], v[3]);
    tp[1] = make_uint4(v[4], v[5], v[6], v[7]);
  }
  __syncthreads();
  constexpr int D0 = MODE == kColsHigh ? C::Q - 2 : 0, D1 = MODE == kColsLow ? C::Q : C::DIAG;
  constexpr bool PAIR = (D1 - D0) * 8 > C::THREADS;  // two words per job when one-word jobs outnumber the threads
  constexpr int WPJ = PAIR ? 2 : 1, JOBS = (D1 - D0) * 8 / WPJ;
  for (int j = tid; j < JOBS; j += C::THREADS) {
    const int d = D0 + j / (8 / WPJ), w = (j % (8 / WPJ)) * WPJ;
    const int lo = d > C::Q - 1 ? d - (C::Q - 1) : 0, hi = d < C::Q - 1 ? d : C::Q - 1;
    // all Q loads of the diagonal in flight at once (predicated)
    unsigned long long a0 = 0, a1 = 0;
    unsigned long long *o = &(w < 4 ? out.lo : out.hi)[4 + 4 * d + w];
    const unsigned long long *tt = &(w < 4 ? s.dsumT.lo : s.dsumT.hi)[4 + 4 * d + w];
    if constexpr (PAIR) {
#pragma unroll
      for (int t = 0; t < C::Q; t++) {
        const bool in = t >= lo && t <= hi;
        const uint2 v = *reinterpret_cast<const uint2 *>(&s.tile[in ? (t * C::Q + (d - t)) * 8 + w : w]);
        a0 += in ? v.x : 0u;
        a1 += in ? v.y : 0u;
      }
      if constexpr (MODE == kColsHigh) {  // U = T + m N
        const ulonglong2 t2 = *reinterpret_cast<const ulonglong2 *>(tt);
        a0 += t2.x;
        a1 += t2.y;
      }
      *reinterpret_cast<ulonglong2 *>(o) = make_ulonglong2(a0, a1);
    } else {
      unsigned long long a2 = 0, a3 = 0;  // four accumulators: shorter add chains (4096 bits: 17.9 -> 17.0 ms)
#pragma unroll
      for (int t = 0; t < C::Q; t++) {
        const bool in = t >= lo && t <= hi;
        const uint32_t v0 = s.tile[in ? (t * C::Q + (d - t)) * 8 + w : w];
        const uint32_t add = in ? v0 : 0u;
        if ((t & 3) == 0) a0 += add;
        else if ((t & 3) == 1) a1 += add;
        else if ((t & 3) == 2) a2 += add;
        else a3 += add;
      }
      unsigned long long v = (a0 + a1) + (a2 + a3);
      if constexpr (MODE == kColsHigh) v += *tt;  // U = T + m N
      *o = v;
    }
  }
  __syncthreads();
}

// Column sum of product word i (-4 <= i < 2n + 4; 0 outside [0, 2n)).
template <int N>
__device__ __forceinline__ unsigned long long cta_ws(const ColSums<N> &c, int i) {
  return c.lo[4 + i] + c.hi[4 + i];
}

// Column sums of words i, i + 1 (i even) with two 16-byte loads.
template <int N>
__device__ __forceinline__ void cta_ws2(const ColSums<N> &c, int i, unsigned long long &v0, unsigned long long &v1) {
  const ulonglong2 a = *reinterpret_cast<const ulonglong2 *>(&c.lo[4 + i]);
  const ulonglong2 b = *reinterpret_cast<const ulonglong2 *>(&c.hi[4 + i]);
  v0 = a.x + b.x;
  v1 = a.y + b.y;
}

// One warp resolves n words whose column sums sum(j) (j = 0 .. n-1; 0 below)
// are given, lane l words [lK, lK + K), K = n / 32 (as cta_resolve_warp).
// SUB: then r = value - N if the value above word n - 1 is set or value >= N.
template <int N, bool SUB, class Sum, class Sum2>
__device__ __forceinline__ void cta_resolve_n(CtaSmem<N> &s, Sum sum, Sum2 sum2, uint32_t *out) {
  constexpr int K = N / 32;
  if (threadIdx.x < 32) {
    const int l = threadIdx.x, i0 = l * K;
    unsigned long long sm[K + 2];
    if constexpr (K % 2 == 0) {
#pragma unroll
      for (int k = 0; k < K + 2; k += 2) sum2(i0 - 2 + k, sm[k], sm[k + 1]);
    } else {
#pragma unroll
      for (int k = 0; k < K + 2; k++) sm[k] = sum(i0 - 2 + k);
    }
    unsigned long long x[K + 1];
#pragma unroll
    for (int k = 0; k <= K; k++) x[k] = (sm[k + 1] & 0xffffffffull) + (sm[k] >> 32);
    uint32_t limb[K], c = 0, all_ones = 1;
#pragma unroll
    for (int k = 0; k < K; k++) {
      const unsigned long long z = (x[k + 1] & 0xffffffffull) + (x[k] >> 32) + c;
      limb[k] = (uint32_t)z;
      c = (uint32_t)(z >> 32);
      all_ones &= limb[k] == kFull;
    }
    const uint32_t G = __ballot_sync(kFull, c != 0), P = __ballot_sync(kFull, all_ones != 0);
    const unsigned long long cs = (unsigned long long)P + ((unsigned long long)G << 1);
    uint32_t cin = (uint32_t)(((cs ^ P) >> l) & 1ull);
#pragma unroll
    for (int k = 0; k < K; k++) {
      limb[k] += cin;
      cin = cin && limb[k] == 0u;
    }
    if constexpr (SUB) {
      const uint32_t top_l = (uint32_t)(sm[K + 1] >> 32) + (uint32_t)(x[K] >> 32);
      const uint32_t top = __shfl_sync(kFull, top_l, 31) + (uint32_t)((cs >> 32) & 1ull);
      uint32_t d[K], b = 0, all_zero = 1;
#pragma unroll
      for (int k = 0; k < K; k++) {
        const unsigned long long t = (unsigned long long)limb[k] - s.n[i0 + k] - b;
        d[k] = (uint32_t)t;
        b = (uint32_t)(t >> 63);
        all_zero &= d[k] == 0u;
      }
      const uint32_t GB = __ballot_sync(kFull, b != 0), PB = __ballot_sync(kFull, all_zero != 0);
      const unsigned long long bs = (unsigned long long)PB + ((unsigned long long)GB << 1);
      uint32_t bin = (uint32_t)(((bs ^ PB) >> l) & 1ull);
      const bool take = top || !((bs >> 32) & 1ull);
#pragma unroll
      for (int k = 0; k < K; k++) {
        const uint32_t v = d[k] - bin;
        bin = bin && d[k] == 0u;
        out[i0 + k] = take ? v : limb[k];
      }
    } else {
#pragma unroll
      for (int k = 0; k < K; k++) out[i0 + k] = limb[k];
    }
  }
  __syncthreads();
}

// r = a b R^-1 mod N (a, b < N; or a, b < R with a b < R N).  r may alias a or b.
template <int N>
__device__ __forceinline__ void mont_cta(CtaSmem<N> &s, uint32_t *r, const uint32_t *a, const uint32_t *b) {
  cta_cols<N, kColsFull>(s, a, b, s.dsumT);
  cta_resolve_n<N, false>(
      s, [&](int i) { return cta_ws<N>(s.dsumT, i); },
      [&](int i, unsigned long long &v0, unsigned long long &v1) { cta_ws2<N>(s.dsumT, i, v0, v1); }, s.t);  // T mod R
  cta_cols<N, kColsLow>(s, s.t, s.np, s.dsum);
  cta_resolve_n<N, false>(
      s, [&](int i) { return cta_ws<N>(s.dsum, i); },
      [&](int i, unsigned long long &v0, unsigned long long &v1) { cta_ws2<N>(s.dsum, i, v0, v1); }, s.m);  // m
  cta_cols<N, kColsHigh>(s, s.m, s.n, s.dsum);  // column sums of U from word n - 1 up
  // Word n - 1 enters as its carry into word n, hi(s) + (lo(s) != 0) (U's low half is 0 mod R),
  // placed in the high half of a sum whose low half is 0; words below it are 0.
  const auto low_carry = [](unsigned long long v) {
    return ((v >> 32) + ((v & 0xffffffffull) != 0ull)) << 32;
  };
  cta_resolve_n<N, true>(
      s,
      [&](int j) {
        const unsigned long long v = cta_ws<N>(s.dsum, N + j);
        return j < -1 ? 0ull : j == -1 ? low_carry(v) : v;
      },
      [&](int j, unsigned long long &v0, unsigned long long &v1) {
        cta_ws2<N>(s.dsum, N + j, v0, v1);
        if (j < 0) {  // j = -2: words n - 2, n - 1
          v0 = 0ull;
          v1 = low_carry(v1);
        }
      },
      r);
}

// The same as a call: at 4096 bits the constant-schedule kernel's main loop, inlined, overflows
// the instruction cache (one exponentiation 19.9 ms inlined, 18.5 ms as a call; everywhere else
// the call measured slower: 2048 bits 3.46 -> 4.00 ms constant-schedule, 3.06 -> 3.95 sliding).
template <int N>
__device__ __noinline__ void mont_cta_call(CtaSmem<N> &s, uint32_t *r, const uint32_t *a, const uint32_t *b) {
  mont_cta<N>(s, r, a, b);
}

// s.np = -N^-1 mod R by Newton's iteration y <- y (2 + N y), which doubles the
// correct low words of y = -N^-1 each time (from -N^-1 mod 2^32).
template <int N>
__device__ __forceinline__ void cta_neg_inverse(CtaSmem<N> &s) {
  const int i = threadIdx.x;
  if (i < N) s.np[i] = i == 0 ? neg_inv32(s.n[0]) : 0u;
  __syncthreads();
#pragma unroll 1
  for (int words = 1; words < N; words *= 2) {
    cta_cols<N, kColsLow>(s, s.n, s.np, s.dsum);
    cta_resolve_n<N, false>(
        s, [&](int j) { return cta_ws<N>(s.dsum, j) + (j == 0 ? 2ull : 0ull); },
        [&](int j, unsigned long long &v0, unsigned long long &v1) {
          cta_ws2<N>(s.dsum, j, v0, v1);
          v0 += j == 0 ? 2ull : 0ull;
        },
        s.m);
    cta_cols<N, kColsLow>(s, s.np, s.m, s.dsum);
    cta_resolve_n<N, false>(
        s, [&](int j) { return cta_ws<N>(s.dsum, j); },
        [&](int j, unsigned long long &v0, unsigned long long &v1) { cta_ws2<N>(s.dsum, j, v0, v1); }, s.np);
  }
}

// Bit length of s.n (every thread).
template <int N>
__device__ __forceinline__ uint32_t cta_bitlen(CtaSmem<N> &s) {
  const int i = threadIdx.x, lane = i & 31, warp = i >> 5;
  uint32_t b = 0;
  if (i < N && s.n[i]) b = (uint32_t)i * 32 + 32 - __clz(s.n[i]);
  if (warp < N / 32) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(kFull, b, o));
    if (lane == 0) s.flag[0][warp] = b;
  }
  __syncthreads();
  uint32_t m = 0;
  for (int k = 0; k < N / 32; k++) m = max(m, s.flag[0][k]);
  __syncthreads();
  return m;
}

// v <- 2 v mod N for v < N.
template <int N>
__device__ __forceinline__ void cta_double(CtaSmem<N> &s, uint32_t *v) {
  const int i = threadIdx.x;
  uint32_t w = 0, top = 0;
  if (i < N) {
    w = (v[i] << 1) | (i ? v[i - 1] >> 31 : 0u);
    top = v[N - 1] >> 31;
  }
  __syncthreads();
  if (i < N) v[i] = w;
  __syncthreads();
  cta_sub_if<N>(s, v, v, s.n, top);
}

// acc = R^2 mod N (R = 2^(32 n)): 2^(bitlen N - 1) doubled up to 2^(32n + e)
// with 32n = e 2^j (e odd), then j Montgomery squarings, each doubling the
// exponent above R.  N = 1 gives 0.
template <int N>
__device__ __forceinline__ void cta_r2(CtaSmem<N> &s, uint32_t *acc) {
  constexpr uint32_t bits = 32u * N;
  constexpr uint32_t j = bits == 1024 ? 10 : bits == 2048 ? 11 : bits == 3072 ? 10 : 12;
  constexpr uint32_t e = bits >> j;
  const uint32_t b = cta_bitlen<N>(s);
  const int i = threadIdx.x;
  const uint32_t tb = b > 1 ? b - 1 : 0;
  if (i < N) acc[i] = (b > 1 && (uint32_t)i == (tb >> 5)) ? (1u << (tb & 31)) : 0u;
  __syncthreads();
  if (b <= 1) return;
#pragma unroll 1
  for (uint32_t d = 0; d < bits + e - tb; d++) cta_double<N>(s, acc);
#pragma unroll 1
  for (uint32_t q = 0; q < j; q++) mont_cta<N>(s, acc, acc, acc);
}

// Copies n words within shared memory (every thread calls it).
template <int N>
__device__ __forceinline__ void cta_copy(uint32_t *dst, const uint32_t *src) {
  if (threadIdx.x < N) dst[threadIdx.x] = src[threadIdx.x];
  __syncthreads();
}

// One exponentiation per CTA.  Sliding window over the exponent's own bits
// (public exponents), or CT: the fixed window over the exponent's whole
// precision (the same schedule for every exponent).  The window table
// (sliding: slot 0 = Mont(1), slot j = Mont(x^(2j - 1)); fixed: slot e =
// Mont(x^e)) is in shared memory after the CtaSmem block.
template <int N, bool CT>
__global__ void __launch_bounds__(CtaShape<N>::THREADS) powm_cta_kernel(PowmArgs a) {
  extern __shared__ uint4 cta_dyn_smem[];
  CtaSmem<N> &s = *reinterpret_cast<CtaSmem<N> *>(cta_dyn_smem);
  uint32_t *table = reinterpret_cast<uint32_t *>(cta_dyn_smem) + sizeof(CtaSmem<N>) / 4;
  const uint32_t inst = a.start + blockIdx.x;
  const int i = threadIdx.x;
  const uint32_t eb = in_element(a.base, inst), ee = in_element(a.exp, inst), em = in_element(a.mod, inst);
  if (i < N) {
    s.n[i] = load_limb(a.mod.limbs, a.mod.nlimbs, a.mod.stride, em, (uint32_t)i);
    s.x[i] = load_limb(a.base.limbs, a.base.nlimbs, a.base.stride, eb, (uint32_t)i);
    s.k[i] = i == 0 ? 1u : 0u;
  }
  {
    unsigned long long *z = &s.dsum.lo[0];  // dsum and dsumT: 4 arrays of 2n + 8 words, contiguous
    for (int w = i; w < 4 * (2 * N + 8); w += CtaShape<N>::THREADS) z[w] = 0ull;
  }
  __syncthreads();
  // x may be >= N (any base below R): x mod N comes out of Mont(x, R^2) = x R mod N
  cta_neg_inverse<N>(s);
  cta_r2<N>(s, s.acc);
  uint32_t *const one = s.k;  // cta_neg_inverse left 2 in word 0: reset below
  if (i < N) one[i] = i == 0 ? 1u : 0u;
  __syncthreads();
  const uint32_t W = a.window;
  const bool sliding = !CT;
  // table
  uint32_t *t1 = table + N;
  mont_cta<N>(s, t1, s.x, s.acc);  // Mont(x)
  mont_cta<N>(s, table, s.acc, one);  // Mont(1) = R mod N
  if (sliding) {
    mont_cta<N>(s, s.x, t1, t1);  // Mont(x^2)
    for (uint32_t j = 2; j <= (1u << (W - 1)); j++) mont_cta<N>(s, table + j * N, table + (j - 1) * N, s.x);
  } else {
    for (uint32_t j = 2; j < (1u << W); j++) mont_cta<N>(s, table + j * N, table + (j - 1) * N, t1);
  }
  if (sliding) {
    // scan from the exponent's top bit
    int32_t top = -1;
    for (int32_t j = (int32_t)a.exp.nlimbs - 1; j >= 0; j--) {
      const uint32_t v = load_limb(a.exp.limbs, a.exp.nlimbs, a.exp.stride, ee, (uint32_t)j);
      if (v) {
        top = j * 32 + 31 - (int32_t)__clz(v);
        break;
      }
    }
    cta_copy<N>(s.acc, table);  // Mont(1)
    ExpCursor cur;
    cursor_init(cur, a.exp, ee, top);
    uint32_t sq, idx;
    bool first = true;
    while (true) {
      const bool more = next_window(a.exp, ee, cur, W, &sq, &idx);
      if (first && more) {
        // the accumulator is Mont(1): skip the squarings and take the first window's entry
        cta_copy<N>(s.acc, table + idx * N);
        first = false;
        continue;
      }
      for (uint32_t q = 0; q < sq; q++) mont_cta<N>(s, s.acc, s.acc, s.acc);
      if (!more) break;
      mont_cta<N>(s, s.acc, s.acc, table + idx * N);
    }
  } else {
    const uint32_t nwin = (a.exp.nlimbs * 32 + W - 1) / W;
    cta_copy<N>(s.acc, table + exp_window(a.exp, ee, (nwin - 1) * W, W) * N);
#pragma unroll 1
    for (int32_t wi = (int32_t)nwin - 2; wi >= 0; wi--) {
      const uint32_t win = exp_window(a.exp, ee, (uint32_t)wi * W, W);
#pragma unroll 1
      for (uint32_t q = 0; q < W; q++) {
        if constexpr (N == 128) mont_cta_call<N>(s, s.acc, s.acc, s.acc);
        else mont_cta<N>(s, s.acc, s.acc, s.acc);
      }
      if constexpr (N == 128) mont_cta_call<N>(s, s.acc, s.acc, table + win * N);
      else mont_cta<N>(s, s.acc, s.acc, table + win * N);
    }
  }
  mont_cta<N>(s, s.acc, s.acc, one);
  const uint32_t o = out_element(a.out, inst);
  if (o < a.out.count && i < N && (uint32_t)i < a.out.nlimbs) limb_ref(a.out.limbs, a.out.stride, o, (uint32_t)i) = s.acc[i];
  // output words above n (a wider output array) are zero
  for (uint32_t w = N + i; w < a.out.nlimbs && o < a.out.count; w += CtaShape<N>::THREADS)
    limb_ref(a.out.limbs, a.out.stride, o, w) = 0u;
}

}  // namespace xmpb
