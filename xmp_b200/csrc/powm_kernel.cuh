// Batched modular exponentiation kernel, one template per distribution
// (TPI lanes per instance x L limbs per lane).
//
// Replaces, fused into one launch, the reference's three kernels per chunk
// (powm_operators.h:105-135): the AR kernel (a*R mod N by division,
// powm_implementations.h:3-87 / 289-443), the powm kernel running the
// fixed-window state machine xmp::fwe (powm/powm.h:39-127) and the copy-out
// kernel (powm_implementations.h:122-152 / 480-516).
//
// Per instance:
//   1. N, n0' = -N^-1 mod 2^32, R^2 mod N (exact doublings + Montgomery squarings)
//   2. window table, stored in the scratch arena, one contiguous slot of L
//      limbs per lane so every lane moves its limbs with 128-bit accesses:
//      slot 0 = R - N (Mont(1)), then for the sliding window the odd powers
//      Mont(x^(2j-1)), j = 1 .. 2^(W-1) (one squaring for Mont(x^2), then one
//      multiply per entry), for the fixed window Mont(x^e), e < 2^W
//   3. the exponent, left to right, by the shape's method (powm_sliding):
//      sliding window: a zero bit is one squaring; a window of at most W bits
//      that starts and ends with a one (odd value v, length l) is l squarings
//      and one multiply by slot (v + 1) / 2.  Every step is one Montgomery
//      multiply acc * B with B = acc (square) or B = the table entry, chosen
//      per lane, so the instances of a warp follow their own exponents in one
//      instruction stream; an instance that has consumed its exponent
//      multiplies by Mont(1) until the warp's last instance is done.  The
//      entry is loaded at the multiply step itself (prefetching it into
//      registers or shared memory a step ahead measured slower: every
//      squaring's operand select then waited on the load).
//      fixed window: W squarings and one table multiply per window (value 0
//      multiplies by Mont(1), keeping the control flow independent of the
//      exponent's bits); the next entry is loaded before the squarings
//   4. one Montgomery multiply by 1 and a compare-subtract give x^e mod N
// Against the reference's fixed window (xmp::fwe, powm/powm.h:39-127, 2^W - 2
// table multiplies and one multiply per W bits) the sliding window takes
// about 2^(W-1) + k/(W+1) multiplies: ~2,373 instead of 2,450 Montgomery
// multiplies for a 2048-bit exponent at W = 6 (warp maximum over random
// exponents).  The sliding scan starts at each instance's own top bit, the
// fixed one at the warp's highest window; the reference's scan from the full
// exponent precision (powm_operators.h:55) only squares Mont(1) there, which
// does not change the result.
#pragma once
#include "internal.h"
#include "mont.cuh"
#include "sqr.cuh"

namespace xmpb {

struct PowmArgs {
  ArrayView base, exp, mod;
  ArrayView r2;     // optional (limbs == nullptr: computed per instance): R^2 mod N per modulus element,
                    // R = 2^(32 * TPI * L), indexed like `mod`
  OutView out;
  uint32_t start;   // first op instance of this launch
  uint32_t count;   // op instances in this launch
  uint32_t window;  // window bits W, 1..7
  uint32_t *table;  // scratch: (launch threads / 32) * 32 * L * powm_table_entries(W, powm_sliding(TPI, L)) words
};

// Exponentiation method of the register kernel with TPI lanes x L limbs:
// sliding window (true) or fixed window (false).  Per shape, from a B200
// sweep of every registered kernel with both methods (exponents of
// min(precision, 2048) bits; a batch of 75,776 / TPI instances and a single
// instance): the sliding window does ~3-4% fewer Montgomery multiplies but
// adds per-step control, so it is taken where it is faster at the batch and
// the batch and single-instance gains together are positive -- the 16-limb
// shapes and a few mid-size ones (2048 bits, 4 x 16: +0.8%; 3072 bits,
// 16 x 6: +4.8%; 1280 bits, 8 x 5: +8.1%).  It loses at 12 limbs per lane
// (-7 to -9%: the compiler's schedule of the multiply inside the sliding loop
// is worse there) and at small precisions, where the control is a larger
// share of a step.
__host__ __device__ constexpr bool powm_sliding(int TPI, int L) {
  return !powm_sqr(TPI, L) && (
         (TPI == 1 && (L == 24 || L == 32)) ||
         (TPI == 2 && (L == 8 || L == 16)) ||
         (TPI == 4 && (L == 5 || L == 6 || L == 16)) ||
         (TPI == 8 && (L == 4 || L == 5 || L == 6 || L == 16)) ||
         (TPI == 16 && (L == 2 || L == 4 || L == 6 || L == 16)) ||
         (TPI == 32 && (L == 8 || L == 16)));
}

// Window-table entries for window bits W.  Sliding: slot 0 holds Mont(1) and
// slot j >= 1 Mont(x^(2j-1)), the odd powers a sliding window multiplies by.
// Fixed: slot e holds Mont(x^e), e < 2^W.
__host__ __device__ constexpr uint32_t powm_table_entries(uint32_t W, bool sliding) {
  return sliding ? (W ? (1u << (W - 1)) + 1u : 1u) : (1u << W);
}

template <int TPI, int L>
__device__ __forceinline__ void load_lane_limbs(uint32_t (&x)[L], const uint32_t *limbs, uint32_t nlimbs,
                                                uint32_t stride, uint32_t e, uint32_t lane) {
  const uint32_t j0 = lane * L;
  if (L % 4 == 0) {
#pragma unroll
    for (int m = 0; m < L / 4; m++) {
      uint4 v = load_group(limbs, nlimbs, stride, e, j0 / 4 + m);
      x[4 * m] = v.x;
      x[4 * m + 1] = v.y;
      x[4 * m + 2] = v.z;
      x[4 * m + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < L; k++) x[k] = load_limb(limbs, nlimbs, stride, e, j0 + k);
  }
}

template <int TPI, int L>
__device__ __forceinline__ void store_lane_limbs(const uint32_t (&x)[L], uint32_t *limbs, uint32_t nlimbs,
                                                 uint32_t stride, uint32_t e, uint32_t lane) {
  const uint32_t j0 = lane * L;
  if (L % 4 == 0) {
#pragma unroll
    for (int m = 0; m < L / 4; m++) {
      uint32_t g = j0 / 4 + m;
      if (g * 4 < nlimbs) store_group(limbs, nlimbs, stride, e, g, make_uint4(x[4 * m], x[4 * m + 1], x[4 * m + 2], x[4 * m + 3]));
    }
  } else {
#pragma unroll
    for (int k = 0; k < L; k++)
      if (j0 + k < nlimbs) limb_ref(limbs, stride, e, j0 + k) = x[k];
  }
}

template <int L>
__device__ __forceinline__ void slot_store(uint32_t *p, const uint32_t (&x)[L]) {
  if (L % 4 == 0) {
#pragma unroll
    for (int m = 0; m < L / 4; m++)
      reinterpret_cast<uint4 *>(p)[m] = make_uint4(x[4 * m], x[4 * m + 1], x[4 * m + 2], x[4 * m + 3]);
  } else if (L % 2 == 0) {
#pragma unroll
    for (int m = 0; m < L / 2; m++) reinterpret_cast<uint2 *>(p)[m] = make_uint2(x[2 * m], x[2 * m + 1]);
  } else {
#pragma unroll
    for (int k = 0; k < L; k++) p[k] = x[k];
  }
}

template <int L>
__device__ __forceinline__ void slot_load(const uint32_t *p, uint32_t (&x)[L]) {
  if (L % 4 == 0) {
#pragma unroll
    for (int m = 0; m < L / 4; m++) {
      uint4 v = reinterpret_cast<const uint4 *>(p)[m];
      x[4 * m] = v.x;
      x[4 * m + 1] = v.y;
      x[4 * m + 2] = v.z;
      x[4 * m + 3] = v.w;
    }
  } else if (L % 2 == 0) {
#pragma unroll
    for (int m = 0; m < L / 2; m++) {
      uint2 v = reinterpret_cast<const uint2 *>(p)[m];
      x[2 * m] = v.x;
      x[2 * m + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < L; k++) x[k] = p[k];
  }
}

// Bits [pos, pos + w) of element e (w <= 8).
__device__ __forceinline__ uint32_t exp_window(const ArrayView &ex, uint32_t e, uint32_t pos, uint32_t w) {
  uint32_t j = pos >> 5, sh = pos & 31;
  uint32_t v = load_limb(ex.limbs, ex.nlimbs, ex.stride, e, j) >> sh;
  if (sh + w > 32) v |= load_limb(ex.limbs, ex.nlimbs, ex.stride, e, j + 1) << (32 - sh);
  return v & ((1u << w) - 1u);
}

// Sliding-window scan over one exponent element.  `pos` is the highest bit
// not yet consumed; `cur` holds word pos / 32 and `nxt` the word below it,
// loaded one word ahead, so a scan waits for memory only after a whole zero
// word.
struct ExpCursor {
  int32_t pos;
  uint32_t cur, nxt;
};

__device__ __forceinline__ void cursor_init(ExpCursor &c, const ArrayView &ex, uint32_t e, int32_t pos) {
  c.pos = pos;
  c.cur = c.nxt = 0;
  if (pos >= 0) {
    const uint32_t j = (uint32_t)pos >> 5;
    c.cur = load_limb(ex.limbs, ex.nlimbs, ex.stride, e, j);
    if (j) c.nxt = load_limb(ex.limbs, ex.nlimbs, ex.stride, e, j - 1);
  }
}

// Steps down to word j (the current `nxt`) and loads the word below it.
__device__ __forceinline__ void cursor_down(ExpCursor &c, const ArrayView &ex, uint32_t e, uint32_t j) {
  c.cur = c.nxt;
  c.nxt = j ? load_limb(ex.limbs, ex.nlimbs, ex.stride, e, j - 1) : 0u;
}

// Skips zero bits and takes the next window of at most W bits that starts and
// ends with a one: *sq = the squarings before its multiply (skipped zeros +
// window length), *idx = its table slot ((v + 1) / 2 for the odd window value
// v).  Returns false when no one bit is left (*sq = the trailing zero bits).
__device__ __forceinline__ bool next_window(const ArrayView &ex, uint32_t e, ExpCursor &c, uint32_t W, uint32_t *sq,
                                            uint32_t *idx) {
  uint32_t zeros = 0;
  while (c.pos >= 0) {
    const uint32_t j = (uint32_t)c.pos >> 5, b = (uint32_t)c.pos & 31;
    const uint32_t w = c.cur & ((2u << b) - 1u);  // bits <= pos of this word
    if (w == 0) {
      zeros += b + 1;
      c.pos = (int32_t)(j * 32) - 1;
      if (j) cursor_down(c, ex, e, j - 1);
      continue;
    }
    const uint32_t tb = 31 - __clz(w);  // the window's top bit, within the word
    zeros += b - tb;
    const int32_t top = (int32_t)(j * 32 + tb);
    uint32_t l = min(W, (uint32_t)top + 1);
    // bits [top - l + 1, top]; a window reaching below bit 0 of the word continues in nxt (j >= 1 then)
    uint32_t v = tb + 1 >= l ? c.cur >> (tb + 1 - l) : (c.cur << (l - tb - 1)) | (c.nxt >> (33 - l + tb));
    v &= (1u << l) - 1u;  // top bit set: v != 0
    const uint32_t tz = __ffs(v) - 1;
    v >>= tz;
    l -= tz;
    c.pos = top - (int32_t)l;
    if (c.pos >= 0 && ((uint32_t)c.pos >> 5) != j) cursor_down(c, ex, e, j - 1);
    *sq = zeros + l;
    *idx = (v + 1) >> 1;
    return true;
  }
  *sq = zeros;
  *idx = 0;
  return false;
}

// Bit length of the exponent element, scanned by the group's lanes in parallel.
template <int TPI>
__device__ __forceinline__ uint32_t exp_bitlen(const Group<TPI> &G, const ArrayView &ex, uint32_t e) {
  uint32_t bl = 0;
  for (int32_t j = (int32_t)ex.nlimbs - 1 - (int32_t)G.lane; j >= 0; j -= TPI) {
    uint32_t v = load_limb(ex.limbs, ex.nlimbs, ex.stride, e, (uint32_t)j);
    if (v) {
      bl = (uint32_t)j * 32 + 32 - __clz(v);
      break;
    }
  }
  return G.seg_max(bl);
}

// One instance group: op instance i of `args` (every lane of the warp calls
// this together; `valid` lanes store their result).  `slot` is this lane's
// window-table slot (entry e at slot + e*32*L).
// CT (constant schedule, for secret exponents): the fixed window over the
// exponent's whole precision for every shape -- the same sequence of
// squarings and multiplies whatever the exponent bits, as the reference's fwe
// scans them (powm/powm.h:39-127); the table is the fixed-window table.
template <int TPI, int L, bool CT = false>
__device__ __forceinline__ void powm_instance(const Group<TPI> &G, const PowmArgs &args, uint32_t i, bool valid,
                                              uint32_t *slot, const SqrSmem &sm) {
  const uint32_t eb = in_element(args.base, i), ee = in_element(args.exp, i), em = in_element(args.mod, i);

  uint32_t n[L];
  load_lane_limbs<TPI, L>(n, args.mod.limbs, args.mod.nlimbs, args.mod.stride, em, G.lane);
  const uint32_t np0 = neg_inv32(G.bcast(n[0], 0));

  const uint32_t W = args.window;
  constexpr bool kSliding = powm_sliding(TPI, L) && !CT;
  // sliding: from this instance's own top bit (its lanes agree), instances of a warp scan independently;
  // fixed: from the highest window any instance of the warp needs (warp-uniform); CT: from the top of
  // the exponent's precision
  ExpCursor cur;
  uint32_t nwin = 0;
  if constexpr (kSliding) {
    cursor_init(cur, args.exp, ee, (int32_t)exp_bitlen<TPI>(G, args.exp, ee) - 1);
  } else if constexpr (CT) {
    nwin = (args.exp.nlimbs * 32 + W - 1) / W;
  } else {
    uint32_t ebits = exp_bitlen<TPI>(G, args.exp, ee);
    ebits = __reduce_max_sync(kFull, ebits);
    nwin = ebits ? (ebits + W - 1) / W : 1;
  }

  const size_t entry_stride = (size_t)32 * L;

  uint32_t x[L], t[L], acc[L];
  // slot 0 = R - N, a representative of Mont(1) below R
#pragma unroll
  for (int k = 0; k < L; k++) acc[k] = 0;
  dsub<TPI, L>(G, acc, n, kFull);
  slot_store<L>(slot, acc);
  {
    uint32_t r2[L];
    if (args.r2.limbs)
      load_lane_limbs<TPI, L>(r2, args.r2.limbs, args.r2.nlimbs, args.r2.stride, in_element(args.r2, i), G.lane);
    else
      compute_r2<TPI, L>(G, r2, n, np0);
    load_lane_limbs<TPI, L>(x, args.base.limbs, args.base.nlimbs, args.base.stride, eb, G.lane);
    mont_mul<TPI, L>(G, t, x, r2, n, np0);  // slot 1 = Mont(x)
  }
  slot_store<L>(slot + entry_stride, t);

  if constexpr (kSliding) {
    // slots 2 .. 2^(W-1): Mont(x^3), Mont(x^5), ...
    const uint32_t half = 1u << (W - 1);
    if (half > 1) {
      mont_mul<TPI, L>(G, x, t, t, n, np0);  // Mont(x^2)
#pragma unroll
      for (int k = 0; k < L; k++) {
        acc[k] = t[k];
        t[k] = x[k];
      }
#pragma unroll 1
      for (uint32_t j = 2; j <= half; j++) {
        mont_mul<TPI, L>(G, x, acc, t, n, np0);
#pragma unroll
        for (int k = 0; k < L; k++) acc[k] = x[k];
        slot_store<L>(slot + j * entry_stride, acc);
      }
    }

    // The first window sets acc (Mont(1) for a zero exponent); then each step is
    // one multiply acc * B: B = acc before step mul_at and, from it on, table
    // slot yidx (the next window's entry, or Mont(1) once the exponent is
    // consumed), loaded at the multiply itself -- other warps cover its latency,
    // and nothing waits on it in the squarings.
    uint32_t sq, yidx;
    next_window(args.exp, ee, cur, W, &sq, &yidx);
    slot_load<L>(slot + yidx * entry_stride, acc);
    bool more = next_window(args.exp, ee, cur, W, &sq, &yidx);
    uint32_t mul_at = sq;
#pragma unroll 1
    for (uint32_t step = 0; __any_sync(kFull, more || step < mul_at); step++) {
      const bool use_y = step >= mul_at;
      uint32_t bsel[L];
      if (use_y) {
        slot_load<L>(slot + yidx * entry_stride, bsel);
      } else {
#pragma unroll
        for (int k = 0; k < L; k++) bsel[k] = acc[k];
      }
      mont_mul<TPI, L>(G, x, acc, bsel, n, np0);
#pragma unroll
      for (int k = 0; k < L; k++) acc[k] = x[k];
      if (use_y && more) {
        more = next_window(args.exp, ee, cur, W, &sq, &yidx);
        mul_at = step + 1 + sq;
      }
    }
  } else {
    // slots 2 .. 2^W - 1: Mont(x^e)
#pragma unroll
    for (int k = 0; k < L; k++) acc[k] = t[k];
    const uint32_t entries = 1u << W;
#pragma unroll 1
    for (uint32_t e = 2; e < entries; e++) {
      mont_mul<TPI, L>(G, x, acc, t, n, np0);
#pragma unroll
      for (int k = 0; k < L; k++) acc[k] = x[k];
      slot_store<L>(slot + e * entry_stride, acc);
    }

    // W squarings and one table multiply per window (window value 0 multiplies
    // by Mont(1)); the window's entry is loaded before its squarings, or, where
    // the shape squares with the specialised product, after them.
    uint32_t win = exp_window(args.exp, ee, (nwin - 1) * W, W);
    slot_load<L>(slot + win * entry_stride, acc);
#pragma unroll 1
    for (int32_t wi = (int32_t)nwin - 2; wi >= 0; wi--) {
      win = exp_window(args.exp, ee, (uint32_t)wi * W, W);
      if constexpr (powm_sqr(TPI, L)) {
#pragma unroll 1
        for (uint32_t s = 0; s < W; s++) {
          mont_square<TPI, L>(G, x, acc, n, np0, sm);
#pragma unroll
          for (int k = 0; k < L; k++) acc[k] = x[k];
        }
        uint32_t y[L];
        slot_load<L>(slot + win * entry_stride, y);
        mont_mul<TPI, L>(G, x, acc, y, n, np0);
#pragma unroll
        for (int k = 0; k < L; k++) acc[k] = x[k];
      } else {
        uint32_t y[L];
        slot_load<L>(slot + win * entry_stride, y);
#pragma unroll 1
        for (uint32_t s = 0; s <= W; s++) {
          uint32_t bsel[L];
#pragma unroll
          for (int k = 0; k < L; k++) bsel[k] = (s < W) ? acc[k] : y[k];
          mont_mul<TPI, L>(G, x, acc, bsel, n, np0);
#pragma unroll
          for (int k = 0; k < L; k++) acc[k] = x[k];
        }
      }
    }
  }

  // Leave Montgomery form: acc * 1 * R^-1, then reduce below N.
#pragma unroll
  for (int k = 0; k < L; k++) t[k] = (G.lane == 0 && k == 0) ? 1u : 0u;
  mont_mul<TPI, L>(G, x, acc, t, n, np0);
  dreduce<TPI, L>(G, x, n);

  if (valid) {
    uint32_t o = out_element(args.out, i);
    if (o < args.out.count) store_lane_limbs<TPI, L>(x, args.out.limbs, args.out.nlimbs, args.out.stride, o, G.lane);
  }
}


// Resident CTAs of 128 threads asked of the register allocator for the
// persistent kernel: left alone, its extra loop state made the allocator take
// ~124 registers at 10-12 limbs per lane (4 CTAs/SM) where the one-shot
// kernel needs 96 (5 CTAs/SM).  The one-shot kernel keeps the allocator's own
// choice (a bound equal to its natural count still changed its schedule and
// cost 2.4% at 2048 bits).
constexpr int powm_batch_min_blocks(int TPI, int L) {
  return (L > 8 && L <= 12) ? 5 : (TPI == 4 && L == 8) ? 4 : 1;  // 4 x 8: the squaring's state took 140
}

// The four-lane squaring's blocks (sqr.cuh) live in the kernel's dynamic shared memory.
template <int TPI, int L>
__device__ __forceinline__ SqrSmem powm_smem_setup() {
  extern __shared__ uint4 powm_dyn_smem[];
  SqrSmem sm{};
  if constexpr (powm_smem_bytes(TPI, L) > 0) {
    sm = sqr_smem<TPI, L>(powm_dyn_smem, threadIdx.x % TPI);
    sqr_smem_init<L>(sm);
    __syncthreads();
  }
  return sm;
}

template <int TPI, int L, bool CT = false>
__global__ void __launch_bounds__(128) powm_kernel(PowmArgs args) {
  const SqrSmem sm = powm_smem_setup<TPI, L>();
  Group<TPI> G;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t local = gtid / TPI;
  const bool valid = local < args.count;
  // Lanes past the end run a copy of the last instance so every shfl sees a full warp.
  const uint32_t i = args.start + (valid ? local : args.count - 1);
  uint32_t *slot = args.table +
                   (size_t)(gtid >> 5) * ((size_t)32 * L * powm_table_entries(args.window, powm_sliding(TPI, L) && !CT)) +
                   (size_t)(threadIdx.x & 31) * L;
  powm_instance<TPI, L, CT>(G, args, i, valid, slot, sm);
}

// R^2 mod N (R = 2^(32 * TPI * L)) for elements start .. start+count-1 of
// `args.mod`, written to the same elements of `args.out` (serving set-up:
// Montgomery constants kept on the device).
template <int TPI, int L>
__global__ void __launch_bounds__(128) r2_kernel(PowmArgs args) {
  Group<TPI> G;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t local = gtid / TPI;
  const bool valid = local < args.count;
  const uint32_t i = args.start + (valid ? local : args.count - 1);
  uint32_t n[L], r2[L];
  load_lane_limbs<TPI, L>(n, args.mod.limbs, args.mod.nlimbs, args.mod.stride, i, G.lane);
  const uint32_t np0 = neg_inv32(G.bcast(n[0], 0));
  compute_r2<TPI, L>(G, r2, n, np0);
  // the stored value must be below R and fit the output's limbs: keep it exact (< N)
  dreduce<TPI, L>(G, r2, n);
  if (valid) store_lane_limbs<TPI, L>(r2, args.out.limbs, args.out.nlimbs, args.out.stride, i, G.lane);
}

// Persistent form for batched launches: a fixed grid whose warps pull work
// items (32/TPI consecutive instances) from an atomic queue over up to
// kPowmSegs segments (arrays of the same precision, e.g. plain instances and
// CRT half-exponentiations), so kernels of several precisions can share the
// GPU for their whole duration.  Only the launched warps need table slots.
// The queue is one counter word: every warp only ever increments it, so
// nothing waits on another warp.
constexpr int kPowmSegs = 4;
struct PowmBatchArgs {
  PowmArgs seg[kPowmSegs];  // each seg's start/count select its instances; table is ignored
  uint32_t nseg;
  uint32_t items;            // work items in total
  uint32_t item_start[kPowmSegs + 1];  // prefix sums of items per segment
  uint32_t window;
  uint32_t *table;
  uint32_t *counter;         // zeroed before the launch
};

template <int TPI, int L>
__global__ void __launch_bounds__(128, powm_batch_min_blocks(TPI, L)) powm_batch_kernel(PowmBatchArgs b) {
  const SqrSmem sm = powm_smem_setup<TPI, L>();
  Group<TPI> G;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t *slot = b.table + (size_t)gwarp * ((size_t)32 * L * powm_table_entries(b.window, powm_sliding(TPI, L))) +
                   (size_t)(threadIdx.x & 31) * L;
  constexpr uint32_t per_item = 32 / TPI;
  while (true) {
    uint32_t item = 0;
    if ((threadIdx.x & 31) == 0) item = atomicAdd(b.counter, 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= b.items) break;
    uint32_t s = 0;
    while (s + 1 < b.nseg && item >= b.item_start[s + 1]) s++;
    const PowmArgs &a = b.seg[s];
    const uint32_t local = (item - b.item_start[s]) * per_item + (threadIdx.x & 31) / TPI;
    const bool valid = local < a.count;
    const uint32_t i = a.start + (valid ? local : a.count - 1);
    PowmArgs args = a;
    args.window = b.window;
    powm_instance<TPI, L>(G, args, i, valid, slot, sm);
  }
}

}  // namespace xmpb
