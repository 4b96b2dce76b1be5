// Squaring-specialised Montgomery product: r = a^2 R^-1 mod N, almost reduced
// (r < R), for the exponentiation's squarings (the reference's per-thread
// sqr, regmp/sqr_imad.h:25-78, used by its powm model powm/three_n.h; here
// also for the four-lane distribution).
//
// Separated operand scanning: the square T = a^2 is formed first with each
// cross product a_i a_j (i < j) computed once and doubled, then reduced by the
// same quotient rows as mont_mul (acc += N q, shift one word) with the words
// of T fed into the accumulator as the rows reach them.  A 2n-limb square
// costs n(n+1)/2 products instead of n^2, so a Montgomery squaring costs about
// 3n^2/2 + n products instead of 2n^2 + n.
//
// Per-thread (TPI = 1): T is formed in registers; the reduction takes T's low
// half as the accumulator and shifts T's high words in at the top.
//
// Four lanes (TPI = 4, lane g holding block A_g of L limbs): every lane
// computes the same three products, each with a partner lane chosen by its
// own index, so the lanes run one instruction stream and the work is even:
//   S = A_g^2 (lane-local, doubled cross products plus the squares of the
//       limbs), at word offset 2gL of T;
//   P = 2 A_g A_h, h = g + 1 mod 4 (the partner's words arrive by shuffle), at
//       offset L(g + h): the adjacent block pairs (0,1) (1,2) (2,3) (3,0);
//   Q = half of 2 A_g A_h, h = g + 2 mod 4: the pairs (0,2) and (1,3) are
//       split between their two lanes -- lanes 0, 1 take their own low half
//       against all of the partner's words, lanes 2, 3 all of their own words
//       against the partner's high half (two passes of L/2 x L/2) -- at offset
//       L(g + h) (+ L/2 for lanes 2, 3).
// Together these are every block pair (g, h), g <= h, once, cross pairs
// doubled.  Each product is cut into L-word blocks kept in this thread's
// shared memory.  A block at T offset o belongs in lane g's accumulator window
// when the reduction reaches row o - gL; every such row is a multiple of L/2,
// so at each half-block boundary every lane adds the (at most two) blocks the
// schedule gives it -- the same instructions in every lane, a shared zero
// block where a lane has none.  The words of T thus enter exactly where the
// reduction of mont_mul would have added the products of a * a, and no block
// is exchanged between lanes.
#pragma once
#include "mont.cuh"

namespace xmpb {

// s = a^2 (2L words), one lane.
template <int L>
__device__ __forceinline__ void lane_square(uint32_t (&s)[2 * L], const uint32_t (&a)[L]) {
#pragma unroll
  for (int k = 0; k < 2 * L; k++) s[k] = 0;
#pragma unroll
  for (int i = 0; i < L - 1; i++) {
    uint64_t p[L];
#pragma unroll
    for (int j = i + 1; j < L; j++) p[j] = mul_wide(a[i], a[j]);
    // low halves at i + j, carry through s[i + L] into s[i + L + 1]
    s[2 * i + 1] = add_cc(s[2 * i + 1], (uint32_t)p[i + 1]);
#pragma unroll
    for (int j = i + 2; j < L; j++) s[i + j] = addc_cc(s[i + j], (uint32_t)p[j]);
    s[i + L] = addc_cc(s[i + L], 0u);
    s[i + L + 1] = addc(s[i + L + 1], 0u);
    // high halves at i + j + 1
    s[2 * i + 2] = add_cc(s[2 * i + 2], (uint32_t)(p[i + 1] >> 32));
#pragma unroll
    for (int j = i + 2; j < L; j++) s[i + j + 1] = addc_cc(s[i + j + 1], (uint32_t)(p[j] >> 32));
    s[i + L + 1] = addc(s[i + L + 1], 0u);
  }
  // double the cross products (their sum is below 2^(64L - 1)) and add the squares of the limbs
#pragma unroll
  for (int k = 2 * L - 1; k > 0; k--) s[k] = __funnelshift_l(s[k - 1], s[k], 1);
  s[0] <<= 1;
  uint64_t d[L];
#pragma unroll
  for (int i = 0; i < L; i++) d[i] = mul_wide(a[i], a[i]);
  s[0] = add_cc(s[0], (uint32_t)d[0]);
  s[1] = addc_cc(s[1], (uint32_t)(d[0] >> 32));
#pragma unroll
  for (int i = 1; i < L; i++) {
    s[2 * i] = addc_cc(s[2 * i], (uint32_t)d[i]);
    s[2 * i + 1] = addc_cc(s[2 * i + 1], (uint32_t)(d[i] >> 32));
  }
}

// One quotient row of the reduction: acc += N q (q from the group's lowest word), then the
// accumulator shifts down one word with `in` (a word of T, or zero) entering at the top of the top lane.
template <int TPI, int L>
__device__ __forceinline__ void redc_row(const Group<TPI> &G, uint32_t (&r)[L], uint32_t &c0, uint32_t &c1,
                                         const uint32_t (&n)[L], uint32_t np0, uint32_t in) {
  const uint32_t q = G.bcast(r[0], 0) * np0;
  uint64_t s[L];
  row_products<L>(s, n, q);
  add_low_halves<L>(r, c0, c1, s);
  add_high_halves<L>(r, c0, c1, s);
  uint32_t t = TPI == 1 ? in : G.from_next(r[0]);
  if (TPI > 1 && G.lane == TPI - 1) t = in;
#pragma unroll
  for (int j = 0; j < L - 1; j++) r[j] = r[j + 1];
  r[L - 1] = add_cc(t, c0);
  c0 = addc_fma(c1);
  c1 = 0;
}

// Per-thread Montgomery squaring (TPI = 1).  r must not alias a.
template <int L>
__device__ __forceinline__ void mont_sqr1(const Group<1> &G, uint32_t (&r)[L], const uint32_t (&a)[L],
                                          const uint32_t (&n)[L], uint32_t np0) {
  uint32_t s[2 * L];
  lane_square<L>(s, a);
  uint32_t c0 = 0, c1 = 0;
#pragma unroll
  for (int k = 0; k < L; k++) r[k] = s[k];
#pragma unroll
  for (int i = 0; i < L; i++) redc_row<1, L>(G, r, c0, c1, n, np0, s[L + i]);
  // (r, c0) = (T + QN) / R < 2R: an overflow past R is removed by subtracting N
  dsub<1, L>(G, r, n, 0u - c0);
}

// ---- several lanes -----------------------------------------------------------------
//
// T lanes (T = 2, 4), lane g holding block A_g of L limbs.  Every lane
// computes, in one instruction stream, its own square S, the products
// P_r = 2 A_g A_{g+r mod T} for r = 1 .. T/2 - 1, and Q, the half of
// 2 A_g A_{g+T/2 mod T} that falls to it (lanes g < T/2 take their own low half
// against all of the partner's words, lanes g >= T/2 all of their own words
// against the partner's high half).  Block ids per lane: 0 S lo, 1 S hi,
// 2r and 2r + 1 the low and high blocks of P_r, T and T + 1 those of Q.
// The offsets and boundaries below are defined for any even T; the lane plan
// (two 4-bit block ids at each of the 2T + 1 boundaries, 24 nibbles) holds
// T <= 4.  Eight lanes would need a wider plan and measured no faster (8 x 4
// limbs at 1024 bits: 21% slower than mont_mul), so they are not offered.

// T-word offset of block `id` of lane g (T lanes, L limbs each).
__host__ __device__ constexpr int sqr_block_offset(int T, int L, int g, int id) {
  if (id == 0) return 2 * g * L;
  if (id == 1) return 2 * g * L + L;
  if (id < T) {
    const int r = id / 2, h = (g + r) % T;
    return L * (g + h) + (id % 2 ? L : 0);
  }
  const int h = (g + T / 2) % T;
  return L * (g + h) + (g >= T / 2 ? L / 2 : 0) + (id == T ? 0 : L);
}

// The half-block boundary (row / (L/2)) at which lane g adds block `id` (independent of L).
__host__ __device__ constexpr int sqr_block_boundary(int T, int g, int id) {
  return (sqr_block_offset(T, 2, g, id) - 2 * g) / 1;
}

// This lane's schedule: nibble 2b + s = the id of its s-th block at boundary b (15: none).
struct SqrPlanBits {
  uint32_t w[3];  // 2 * (2T + 1) <= 18 nibbles for T <= 4
};

template <int T>
__host__ __device__ __forceinline__ SqrPlanBits sqr_lane_plan(uint32_t g) {
  static_assert(T == 2 || T == 4, "the lane plan holds 24 nibbles: two blocks at each of 2T + 1 boundaries");
  SqrPlanBits p;
  p.w[0] = p.w[1] = p.w[2] = 0xffffffffu;
  uint32_t used[2 * T + 1];
#pragma unroll
  for (int b = 0; b <= 2 * T; b++) used[b] = 0;
#pragma unroll
  for (int id = 0; id < T + 2; id++) {
    const uint32_t b = (uint32_t)sqr_block_boundary(T, (int)g, id);
    // slot = blocks already placed at this boundary (at most 2)
    uint32_t slot = 0;
#pragma unroll
    for (int bb = 0; bb <= 2 * T; bb++)
      if ((uint32_t)bb == b) slot = used[bb]++;
    const uint32_t nib = 2 * b + slot;
    const uint32_t word = nib / 8, sh = 4 * (nib % 8);
#pragma unroll
    for (int k = 0; k < 3; k++)
      if ((uint32_t)k == word) p.w[k] = (p.w[k] & ~(15u << sh)) | ((uint32_t)id << sh);
  }
  return p;
}

// Number of blocks the busiest lane adds at boundary b (the same in every lane), 2 bits per boundary.
__host__ __device__ constexpr uint64_t sqr_slots_mask(int T) {
  uint64_t mask = 0;
  for (int b = 0; b <= 2 * T; b++) {
    int most = 0;
    for (int g = 0; g < T; g++) {
      int c = 0;
      for (int id = 0; id < T + 2; id++)
        if (sqr_block_boundary(T, g, id) == b) c++;
      most = c > most ? c : most;
    }
    mask |= (uint64_t)most << (2 * b);
  }
  return mask;
}

// This thread's blocks in the kernel's dynamic shared memory.  Block b, group m
// (4 words) of thread t is blocks[(b * L/4 + m) * 128 + t]: a warp moves 512
// contiguous bytes per access.  extra[(r - 1) * 128 + t] holds the word of P_r
// above its high block; zero is one all-zero block shared by the CTA.
struct SqrSmem {
  uint4 *blocks;
  uint32_t *extra;
  const uint4 *zero;
  uint32_t tid;
  SqrPlanBits plan;
};

// Dynamic shared memory of a 128-thread CTA of the T-lane squaring kernels.
__host__ __device__ constexpr uint32_t sqr_smem_bytes(int T, int L) {
  return (uint32_t)((T + 2) * L * 128 * 4 + L * 4 + (T / 2 > 1 ? T / 2 - 1 : 1) * 128 * 4);
}

template <int T, int L>
__device__ __forceinline__ SqrSmem sqr_smem(uint4 *base, uint32_t lane) {
  SqrSmem s;
  s.blocks = base;
  s.zero = base + (T + 2) * (L / 4) * 128;
  s.extra = reinterpret_cast<uint32_t *>(base + (T + 2) * (L / 4) * 128 + L / 4);
  s.tid = threadIdx.x;
  s.plan = sqr_lane_plan<T>(lane);
  return s;
}

// Zeroes the shared zero block; every thread of the CTA calls it before a __syncthreads.
template <int L>
__device__ __forceinline__ void sqr_smem_init(const SqrSmem &s) {
  if (s.tid < (uint32_t)(L / 4)) const_cast<uint4 *>(s.zero)[s.tid] = make_uint4(0, 0, 0, 0);
}

// Stores words [OFF, OFF + L) of x as block b.
template <int L, int OFF, int N>
__device__ __forceinline__ void sqr_store(const SqrSmem &s, int b, const uint32_t (&x)[N]) {
#pragma unroll
  for (int m = 0; m < L / 4; m++) {
    uint4 v;
    v.x = OFF + 4 * m + 0 < N ? x[OFF + 4 * m + 0 < N ? OFF + 4 * m + 0 : 0] : 0u;
    v.y = OFF + 4 * m + 1 < N ? x[OFF + 4 * m + 1 < N ? OFF + 4 * m + 1 : 0] : 0u;
    v.z = OFF + 4 * m + 2 < N ? x[OFF + 4 * m + 2 < N ? OFF + 4 * m + 2 : 0] : 0u;
    v.w = OFF + 4 * m + 3 < N ? x[OFF + 4 * m + 3 < N ? OFF + 4 * m + 3 : 0] : 0u;
    s.blocks[(b * (L / 4) + m) * 128 + s.tid] = v;
  }
}

// Adds this lane's block in slot `slot` of boundary b (none: the zero block) into the window.
template <int T, int L>
__device__ __forceinline__ void sqr_add(const SqrSmem &s, uint32_t b, uint32_t slot, uint32_t (&r)[L], uint32_t &c0,
                                        uint32_t &c1) {
  const uint32_t nib = 2 * b + slot;
  const uint32_t word = nib < 8 ? s.plan.w[0] : (nib < 16 ? s.plan.w[1] : s.plan.w[2]);
  const uint32_t id = (word >> (4 * (nib % 8))) & 15u;
  const bool has = id < (uint32_t)(T + 2);
  const uint4 *p = has ? s.blocks + (size_t)id * (L / 4) * 128 + s.tid : s.zero;
  const uint32_t step = has ? 128u : 1u;
  uint32_t v[L];
#pragma unroll
  for (int m = 0; m < L / 4; m++) {
    uint4 g = p[m * step];
    v[4 * m] = g.x;
    v[4 * m + 1] = g.y;
    v[4 * m + 2] = g.z;
    v[4 * m + 3] = g.w;
  }
  // the high block of P_r (odd id below T) carries one more word, at the lane's carry word
  const bool extra = has && id >= 2 && id < (uint32_t)T && (id & 1u);
  const uint32_t e = extra ? s.extra[(id / 2 - 1) * 128 + s.tid] : 0u;
  r[0] = add_cc(r[0], v[0]);
#pragma unroll
  for (int k = 1; k < L; k++) r[k] = addc_cc(r[k], v[k]);
  c0 = addc_cc(c0, e);
  c1 = addc(c1, 0u);
}

// x (H + 1 words) = 2 * a[lo, lo + H) as a number of its own.
template <int L, int H>
__device__ __forceinline__ void sqr_double_half(uint32_t (&x)[H + 1], const uint32_t (&a)[L], int lo) {
  x[0] = a[lo] << 1;
#pragma unroll
  for (int j = 1; j < H; j++) x[j] = __funnelshift_l(a[lo + j - 1], a[lo + j], 1);
  x[H] = a[lo + H - 1] >> 31;
}

// r = a^2 R^-1 mod N (almost reduced) over T lanes.  r must not alias a.
template <int T, int L>
__device__ __forceinline__ void mont_sqr_lanes(const Group<T> &G, uint32_t (&r)[L], const uint32_t (&a)[L],
                                               const uint32_t (&n)[L], uint32_t np0, const SqrSmem &sm) {
  static_assert(L % 4 == 0 && (T == 2 || T == 4), "lane squaring: T in {2, 4}, L a multiple of 4");
  constexpr int H = L / 2;
  // S = A_g^2
  {
    uint32_t s[2 * L];
    lane_square<L>(s, a);
    sqr_store<L, 0>(sm, 0, s);
    sqr_store<L, L>(sm, 1, s);
  }
  // P_r = 2 A_g A_h, h = g + r mod T
  if constexpr (T > 2) {
    uint32_t d[L + 1];
    d[0] = a[0] << 1;
#pragma unroll
    for (int j = 1; j < L; j++) d[j] = __funnelshift_l(a[j - 1], a[j], 1);
    d[L] = a[L - 1] >> 31;
#pragma unroll
    for (int rr = 1; rr < T / 2; rr++) {
      const uint32_t h = (G.lane + rr) % T;
      uint32_t R[2 * L + 1];
#pragma unroll
      for (int k = 0; k < 2 * L + 1; k++) R[k] = 0;
#pragma unroll
      for (int k = 0; k < L; k++) {
        const uint32_t w = G.bcast(a[k], h);
        uint64_t p[L];
#pragma unroll
        for (int j = 0; j < L; j++) p[j] = mul_wide(d[j], w);
        const uint32_t top = d[L] ? w : 0u;
        R[k] = add_cc(R[k], (uint32_t)p[0]);
#pragma unroll
        for (int j = 1; j < L; j++) R[k + j] = addc_cc(R[k + j], (uint32_t)p[j]);
        R[k + L] = addc_cc(R[k + L], top);
        R[k + L + 1] = addc(R[k + L + 1], 0u);
        R[k + 1] = add_cc(R[k + 1], (uint32_t)(p[0] >> 32));
#pragma unroll
        for (int j = 1; j < L; j++) R[k + 1 + j] = addc_cc(R[k + 1 + j], (uint32_t)(p[j] >> 32));
        R[k + L + 1] = addc(R[k + L + 1], 0u);
      }
      sqr_store<L, 0>(sm, 2 * rr, R);
      sqr_store<L, L>(sm, 2 * rr + 1, R);
      sm.extra[(rr - 1) * 128 + sm.tid] = R[2 * L];
    }
  }
  // Q: the half of 2 A_g A_h, h = g + T/2 mod T, that falls to this lane
  {
    const uint32_t h = (G.lane + T / 2) % T;
    const bool first = G.lane < (uint32_t)(T / 2);
    uint32_t dl[H + 1], dh[H + 1];
    sqr_double_half<L, H>(dl, a, 0);
    sqr_double_half<L, H>(dh, a, H);
    uint32_t Q[L + H + 1];
#pragma unroll
    for (int k = 0; k < L + H + 1; k++) Q[k] = 0;
#pragma unroll
    for (int pass = 0; pass < 2; pass++) {
      uint32_t x[H + 1];
#pragma unroll
      for (int j = 0; j <= H; j++) x[j] = (pass == 0 || first) ? dl[j] : dh[j];
#pragma unroll
      for (int k = 0; k < H; k++) {
        // each lane sends the word its receiver needs: a first lane (the receiver of a second one) takes
        // word pass*H + k, a second lane (the receiver of a first one) word H + k
        const uint32_t send = first ? a[H + k] : a[pass * H + k];
        const uint32_t w = G.bcast(send, h);
        uint64_t p[H];
#pragma unroll
        for (int j = 0; j < H; j++) p[j] = mul_wide(x[j], w);
        const uint32_t top = x[H] ? w : 0u;
        const int o = pass * H + k;
        Q[o] = add_cc(Q[o], (uint32_t)p[0]);
#pragma unroll
        for (int j = 1; j < H; j++) Q[o + j] = addc_cc(Q[o + j], (uint32_t)p[j]);
        Q[o + H] = addc_cc(Q[o + H], top);
        Q[o + H + 1] = addc(Q[o + H + 1], 0u);
        Q[o + 1] = add_cc(Q[o + 1], (uint32_t)(p[0] >> 32));
#pragma unroll
        for (int j = 1; j < H; j++) Q[o + 1 + j] = addc_cc(Q[o + 1 + j], (uint32_t)(p[j] >> 32));
        Q[o + H + 1] = addc(Q[o + H + 1], 0u);
      }
    }
    sqr_store<L, 0>(sm, T, Q);
    sqr_store<L, L>(sm, T + 1, Q);  // words L .. L + H of Q, zeros above
  }
  // reduction, the blocks of T entering at the half-block boundaries
  uint32_t c0 = 0, c1 = 0;
#pragma unroll
  for (int k = 0; k < L; k++) r[k] = 0;
  sqr_add<T, L>(sm, 0, 0, r, c0, c1);
#pragma unroll 1
  for (int src = 0; src < T; src++) {
#pragma unroll
    for (int k = 0; k < L; k++) {
      if (k == 0 || k == H) {
        const uint32_t b = 2 * src + (k == H ? 1 : 0);
        if (b > 0) {
          // blocks at this boundary: the same count for every lane (warp-uniform)
          constexpr uint64_t kSlots = sqr_slots_mask(T);
          const uint32_t slots = (uint32_t)(kSlots >> (2 * b)) & 3u;
          if (slots > 0) sqr_add<T, L>(sm, b, 0, r, c0, c1);
          if (slots > 1) sqr_add<T, L>(sm, b, 1, r, c0, c1);
        }
      }
      redc_row<T, L>(G, r, c0, c1, n, np0, 0u);
    }
  }
  sqr_add<T, L>(sm, 2 * T, 0, r, c0, c1);
  const uint32_t ovf = dnormalize<T, L>(G, r, c0);
  dsub<T, L>(G, r, n, 0u - ovf);
}

}  // namespace xmpb

namespace xmpb {

// Register kernels whose exponentiation squares with the specialised product.  They use the fixed
// window (every instance of a warp squares at the same steps; the sliding window is not combined with
// it).  Measured on B200 against the same kernels squaring with mont_mul (CUDA events, full waves, every
// result checked): per-thread 16 limbs (512 bits) +12.5%, 8 limbs (256 bits) +16%; four lanes x 8
// limbs (1024 bits) +5.7%, but 4 x 12 -2% and 4 x 16 (2048 bits) -25% -- the unrolled square and
// cross products grow with L^2 and the hot loop no longer fits the instruction cache -- so the wider
// four-lane shapes keep mont_mul (and 4 x 16 its sliding window).
__host__ __device__ constexpr bool powm_sqr(int TPI, int L) { return (TPI == 1 && L <= 16) || (TPI == 4 && L == 8); }

// Dynamic shared memory of a 128-thread CTA of the register powm kernels.
__host__ __device__ constexpr uint32_t powm_smem_bytes(int TPI, int L) {
  return (TPI > 1 && powm_sqr(TPI, L)) ? sqr_smem_bytes(TPI, L) : 0u;
}

// r = a^2 R^-1 mod N (almost reduced) with the shape's squaring.  r must not alias a.
template <int TPI, int L>
__device__ __forceinline__ void mont_square(const Group<TPI> &G, uint32_t (&r)[L], const uint32_t (&a)[L],
                                            const uint32_t (&n)[L], uint32_t np0, const SqrSmem &sm) {
  if constexpr (TPI == 1 && powm_sqr(TPI, L)) {
    mont_sqr1<L>(G, r, a, n, np0);
  } else if constexpr (TPI > 1 && powm_sqr(TPI, L)) {
    mont_sqr_lanes<TPI, L>(G, r, a, n, np0, sm);
  } else {
    mont_mul<TPI, L>(G, r, a, a, n, np0);
  }
}

}  // namespace xmpb
