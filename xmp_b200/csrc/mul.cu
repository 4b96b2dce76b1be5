// xmpIntegersMul[Async] (replaces src/mul.cu:26-303 and the kernels
// regmp_mul/sqr_kernel, digitmp_mul/sqr_kernel, implementations.h:250-434,
// with RegMP mul (regmp/mul_imad.h:26-103) and DigitMP mul (digitmp/mul.h)).
//
// p = a * b mod 2^P(p), operands zero-extended; P(p) >= max(P(a), P(b)).
// Register path: the larger operand is held in registers as AL limbs, the
// smaller as BL limbs (AL, BL from a small set of classes), and the AL+BL-limb
// product is formed by operand scanning, one row of two mad chains (low and
// high halves) per limb of the smaller operand.  Large path (either operand
// above 32 limbs): product scanning straight from the interleaved arrays with
// a three-word column accumulator, so nothing has to fit in registers.
// Squaring (a == b without index arrays, src/mul.cu:147-149) takes the same
// kernels.
#include "internal.h"
#include "carry.cuh"
#include "tune.h"
#include <algorithm>

using namespace xmpb;

namespace xmpb {

template <int N>
__device__ __forceinline__ uint32_t at(const uint32_t (&x)[N], int i) {
  return i < N ? x[i < N ? i : 0] : 0u;
}

template <int L>
__device__ __forceinline__ void load_limbs(uint32_t (&x)[L], const ArrayView &v, uint32_t e) {
#pragma unroll
  for (int g = 0; g < (L + 3) / 4; g++) {
    uint4 q = load_group(v.limbs, v.nlimbs, v.stride, e, g);
    if (4 * g + 0 < L) x[(4 * g + 0) < L ? 4 * g + 0 : 0] = q.x;
    if (4 * g + 1 < L) x[(4 * g + 1) < L ? 4 * g + 1 : 0] = q.y;
    if (4 * g + 2 < L) x[(4 * g + 2) < L ? 4 * g + 2 : 0] = q.z;
    if (4 * g + 3 < L) x[(4 * g + 3) < L ? 4 * g + 3 : 0] = q.w;
  }
}

template <int N>
__device__ __forceinline__ void store_limbs(const uint32_t (&x)[N], const OutView &c, uint32_t e) {
  uint32_t groups = div_up(c.nlimbs, 4);
#pragma unroll
  for (int g = 0; g < (N + 3) / 4; g++)
    if ((uint32_t)g < groups)
      store_group(c.limbs, c.nlimbs, c.stride, e, g, make_uint4(at(x, 4 * g), at(x, 4 * g + 1), at(x, 4 * g + 2), at(x, 4 * g + 3)));
  for (uint32_t g = (N + 3) / 4; g < groups; g++) store_group(c.limbs, c.nlimbs, c.stride, e, g, make_uint4(0, 0, 0, 0));
}

// FAST: every operand holds exactly its class's limbs in whole 16-byte groups, no index arrays, no
// broadcast -- instance i reads and writes element i with plain 128-bit accesses (no masking,
// remainders or range checks: a quarter fewer instructions than the general form at 512 x 512).
template <int AL, int BL, bool FAST>
__global__ void __launch_bounds__(256) mul_reg_kernel(ArrayView a, ArrayView b, OutView c, uint32_t count) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint32_t A[AL], B[BL], P[AL + BL];
  uint32_t ec = i;
  if constexpr (FAST) {
    const uint4 *pa = reinterpret_cast<const uint4 *>(a.limbs) + i, *pb = reinterpret_cast<const uint4 *>(b.limbs) + i;
#pragma unroll
    for (int g = 0; g < AL / 4; g++) {
      const uint4 q = pa[(size_t)g * a.stride];
      A[4 * g] = q.x;
      A[4 * g + 1] = q.y;
      A[4 * g + 2] = q.z;
      A[4 * g + 3] = q.w;
    }
#pragma unroll
    for (int g = 0; g < BL / 4; g++) {
      const uint4 q = pb[(size_t)g * b.stride];
      B[4 * g] = q.x;
      B[4 * g + 1] = q.y;
      B[4 * g + 2] = q.z;
      B[4 * g + 3] = q.w;
    }
  } else {
    const uint32_t ea = in_element(a, i), eb = in_element(b, i);
    ec = out_element(c, i);
    if (ec >= c.count) return;
    load_limbs<AL>(A, a, ea);
    load_limbs<BL>(B, b, eb);
  }
#pragma unroll
  for (int k = 0; k < AL + BL; k++) P[k] = 0;
  // Row j adds A * B[j] at word j: the AL products are one mul.wide each (the
  // FMA pipe), folded in by two ALU carry chains -- low halves at j+k, high
  // halves at j+k+1.  The partial product after row j fits in j+AL+1 words,
  // so the chains never carry out of P[j+AL].
#pragma unroll
  for (int j = 0; j < BL; j++) {
    const uint32_t w = B[j];
    uint64_t p[AL];
#pragma unroll
    for (int k = 0; k < AL; k++) p[k] = mul_wide(A[k], w);
    P[j] = add_cc(P[j], (uint32_t)p[0]);
#pragma unroll
    for (int k = 1; k < AL; k++) P[j + k] = addc_cc(P[j + k], (uint32_t)p[k]);
    P[j + AL] = addc(0u, 0u);
    if (AL > 1) {
      P[j + 1] = add_cc(P[j + 1], (uint32_t)(p[0] >> 32));
#pragma unroll
      for (int k = 1; k < AL - 1; k++) P[j + 1 + k] = addc_cc(P[j + 1 + k], (uint32_t)(p[k] >> 32));
      P[j + AL] = addc(P[j + AL], (uint32_t)(p[AL - 1] >> 32));
    } else {
      P[j + AL] += (uint32_t)(p[0] >> 32);
    }
  }
  if constexpr (FAST) {
    uint4 *pc = reinterpret_cast<uint4 *>(c.limbs) + i;
#pragma unroll
    for (int g = 0; g < (AL + BL) / 4; g++)
      pc[(size_t)g * c.stride] = make_uint4(P[4 * g], P[4 * g + 1], P[4 * g + 2], P[4 * g + 3]);
  } else {
    store_limbs<AL + BL>(P, c, ec);
  }
}

// Column k of the product, accumulated from the interleaved arrays.
__global__ void __launch_bounds__(256) mul_stream_kernel(ArrayView a, ArrayView b, OutView c, uint32_t count) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint32_t ea = in_element(a, i), eb = in_element(b, i), ec = out_element(c, i);
  if (ec >= c.count) return;
  const int32_t na = a.nlimbs, nb = b.nlimbs;
  uint32_t c0 = 0, c1 = 0, c2 = 0;
  uint32_t groups = div_up(c.nlimbs, 4);
  for (uint32_t g = 0; g < groups; g++) {
    uint32_t out[4];
    for (int q = 0; q < 4; q++) {
      int32_t k = g * 4 + q;
      int32_t lo = max(0, k - nb + 1), hi = min(k, na - 1);
      for (int32_t t = lo; t <= hi; t++) {
        uint32_t x = load_limb(a.limbs, a.nlimbs, a.stride, ea, t);
        uint32_t y = load_limb(b.limbs, b.nlimbs, b.stride, eb, k - t);
        c0 = mad_lo_cc(x, y, c0);
        c1 = madc_hi_cc(x, y, c1);
        c2 = addc(c2, 0u);
      }
      out[q] = c0;
      c0 = c1;
      c1 = c2;
      c2 = 0;
    }
    store_group(c.limbs, c.nlimbs, c.stride, ec, g, make_uint4(out[0], out[1], out[2], out[3]));
  }
}

typedef void (*MulLaunch)(ArrayView, ArrayView, OutView, uint32_t, int, cudaStream_t);
template <int AL, int BL>
static void launch_mul(ArrayView a, ArrayView b, OutView c, uint32_t count, int threads, cudaStream_t s) {
  if constexpr (AL % 4 == 0 && BL % 4 == 0) {
    if (!a.index && !b.index && !c.index && a.nlimbs == (uint32_t)AL && b.nlimbs == (uint32_t)BL &&
        c.nlimbs == (uint32_t)(AL + BL) && a.count >= count && b.count >= count && c.count >= count) {
      mul_reg_kernel<AL, BL, true><<<grid_for(count, threads), threads, 0, s>>>(a, b, c, count);
      return;
    }
  }
  mul_reg_kernel<AL, BL, false><<<grid_for(count, threads), threads, 0, s>>>(a, b, c, count);
}

static const int kClasses[] = {2, 4, 8, 12, 16, 24, 32};
static int class_of(uint32_t n) {
  for (int c : kClasses)
    if (n <= (uint32_t)c) return c;
  return 0;
}

#define XMPB_MUL_CASE(A, B) \
  if (al == A && bl == B) return launch_mul<A, B>;
static MulLaunch pick_mul(int al, int bl) {
  XMPB_MUL_CASE(2, 2) XMPB_MUL_CASE(4, 2) XMPB_MUL_CASE(4, 4) XMPB_MUL_CASE(8, 2) XMPB_MUL_CASE(8, 4)
  XMPB_MUL_CASE(8, 8) XMPB_MUL_CASE(12, 2) XMPB_MUL_CASE(12, 4) XMPB_MUL_CASE(12, 8) XMPB_MUL_CASE(12, 12)
  XMPB_MUL_CASE(16, 2) XMPB_MUL_CASE(16, 4) XMPB_MUL_CASE(16, 8) XMPB_MUL_CASE(16, 12) XMPB_MUL_CASE(16, 16)
  XMPB_MUL_CASE(24, 2) XMPB_MUL_CASE(24, 4) XMPB_MUL_CASE(24, 8) XMPB_MUL_CASE(24, 12) XMPB_MUL_CASE(24, 16)
  XMPB_MUL_CASE(24, 24) XMPB_MUL_CASE(32, 2) XMPB_MUL_CASE(32, 4) XMPB_MUL_CASE(32, 8) XMPB_MUL_CASE(32, 12)
  XMPB_MUL_CASE(32, 16) XMPB_MUL_CASE(32, 24) XMPB_MUL_CASE(32, 32)
  return nullptr;
}

bool mul_has_register_kernel(uint32_t na, uint32_t nb) {
  int al = class_of(std::max(na, nb)), bl = class_of(std::min(na, nb));
  return al && bl && pick_mul(al, bl) != nullptr;
}

// Register kernel when one exists for the operand classes (else the streamed
// kernel), 128 threads -- unless the tuner or the caller chose otherwise.
xmpError_t mul_entry(xmpHandle_t h, xmpIntegers_t p, xmpIntegers_t a, xmpIntegers_t b, uint32_t count,
                     const ElemConfig *forced) {
  if (!h || !p || !a || !b) return xmpErrorInvalidParameter;
  int dev = h->device;
  if (p->device != dev || a->device != dev || b->device != dev) return xmpErrorInvalidDevice;
  if (count == 0) return xmpErrorSuccess;
  DeviceGuard guard(dev);
  xmpExecutionPolicy_t pol = h->policy;
  if (p->count < count) return xmpErrorInvalidCount;
  if (pol->indices[0] && pol->indices_count[0] < count) return xmpErrorInvalidCount;
  if (p->precision < std::max(a->precision, b->precision)) return xmpErrorInvalidPrecision;

  ArrayView va = view_in(a, pol->indices[1], pol->indices_count[1]);
  ArrayView vb = view_in(b, pol->indices[2], pol->indices_count[2]);
  // Larger operand first (register rows run over the smaller one).
  if (va.nlimbs < vb.nlimbs) std::swap(va, vb);
  int al = class_of(va.nlimbs), bl = class_of(vb.nlimbs);
  MulLaunch launch = nullptr;
  if (al && bl && pol->algorithm != xmpAlgorithmDigitMP) launch = pick_mul(al, bl);
  if (pol->algorithm == xmpAlgorithmRegMP && !launch) return xmpErrorUnsupported;
  ElemConfig cfg;
  if (forced) {
    cfg = *forced;
  } else if (pol->algorithm == xmpAlgorithmDefault) {
    int slot = tuner_lookup(h, xmpTuneMul, std::max(a->precision, b->precision), 0, count, nullptr);
    ElemConfig t;
    if (slot >= 0 && elem_candidate(xmpTuneMul, std::max(a->nlimbs, b->nlimbs), slot, &t)) cfg = t;
  }
  if (cfg.variant == 1) launch = nullptr;
  else if (!launch && forced) return xmpErrorUnsupported;
  const int threads = cfg.threads;
  bool aliased = (p == a || p == b);
  bool indexed = pol->indices[0] || pol->indices[1] || pol->indices[2];
  OutTarget t;
  // The streamed kernel reads inputs while writing the product: stage whenever it aliases.
  xmpError_t e = begin_output(h, p, aliased, indexed || !launch, &t);
  if (e != xmpErrorSuccess) return e;
  OutView vc = view_out(p, t.limbs, pol->indices[0]);
  if (launch)
    launch(va, vb, vc, count, threads, h->stream);
  else
    mul_stream_kernel<<<grid_for(count, threads), threads, 0, h->stream>>>(va, vb, vc, count);
  e = end_output(h, p, t);
  if (e != xmpErrorSuccess) return e;
  return check_cuda();
}

}  // namespace xmpb

extern "C" {

xmpError_t XMPAPI xmpIntegersMulAsync(xmpHandle_t h, xmpIntegers_t p, const xmpIntegers_t a, const xmpIntegers_t b,
                                       uint32_t count) {
  return mul_entry(h, p, a, b, count, nullptr);
}

xmpError_t XMPAPI xmpIntegersMul(xmpHandle_t h, xmpIntegers_t p, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count) {
  xmpError_t e = xmpIntegersMulAsync(h, p, a, b, count);
  if (e != xmpErrorSuccess) return e;
  DeviceGuard guard(h->device);
  cudaStreamSynchronize(h->stream);
  return check_cuda();
}

}  // extern "C"
