// Elementwise (HBM-bound) ops: add, sub, and, ior, xor, not, shf, cmp, popc.
//
// Replaces src/add_sub.cu:26-256 and src/logic.cu:26-605 with their kernels
// regmp/digitmp_add/sub_kernel and strided_*_kernel (implementations.h:36-248,
// 765-1081).  One instance per thread; every operand moves through 16-byte
// limb groups of the interleaved layout, so each warp access is a contiguous
// 512-byte run.  Runtime limb counts: one kernel per op covers every precision
// (the reference's RegMP/DigitMP size ladder is unnecessary here because these
// ops never hold a whole integer in registers).
//
// Semantics (all as the reference):
//   add  s = (a + b) mod 2^P(s)          sub  d = (a - b) mod 2^P(d)
//   and/ior/xor  zero-extended, result truncated to P(c)
//   not  c = ~a mod 2^P(c)  (limbs above a's precision become all ones)
//   shf  c = floor(a * 2^s) mod 2^P(c), s = shift[i % min(shift_count,count)],
//        positive s shifts left, negative shifts right
//   cmp  c[i] = sign(a - b) in {-1,0,1}; popc c[i] = popcount(a)
// Index arrays: out = indices[0], a = indices[1], b = indices[2] (binary ops);
// cmp uses indices[0] for a and indices[1] for b; popc uses indices[0].
#include "internal.h"
#include <algorithm>

using namespace xmpb;

namespace xmpb {

enum class Bin { Add, Sub, And, Ior, Xor };

// Grid-stride loops over instances: the launch covers at most the GPU's
// resident threads (stream_grid), so each thread handles several instances
// instead of the GPU launching and retiring one short-lived CTA per 256.
// Input element of op instance i, as in_element, with each remainder taken only when it changes
// the index: these kernels are light enough that two integer divisions per operand show (2-3 us
// on shf and cmp over 2^22 instances).  The powm kernels keep in_element's plain remainders.
__device__ __forceinline__ uint32_t ew_element(const ArrayView &v, uint32_t i) {
  const uint32_t k = v.index ? v.index[i < v.index_count ? i : i % v.index_count] : i;
  return k < v.count ? k : k % v.count;
}

#define XMPB_FOR_INSTANCES(i, count)                                                              \
  for (uint64_t i##_ = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i##_ < (count);            \
       i##_ += (uint64_t)gridDim.x * blockDim.x)

template <Bin OP>
__global__ void __launch_bounds__(256) binary_kernel(ArrayView a, ArrayView b, OutView c, uint32_t count) {
  XMPB_FOR_INSTANCES(i, count) {
    const uint32_t i = (uint32_t)i_;
    uint32_t ea = ew_element(a, i), eb = ew_element(b, i), ec = out_element(c, i);
    if (ec >= c.count) continue;
    uint32_t groups = div_up(c.nlimbs, 4);
    uint32_t carry = (OP == Bin::Sub) ? 1u : 0u;  // subtraction as a + ~b + 1
    for (uint32_t g = 0; g < groups; g++) {
      uint4 x = load_group(a.limbs, a.nlimbs, a.stride, ea, g);
      uint4 y = load_group(b.limbs, b.nlimbs, b.stride, eb, g);
      uint4 r;
      if (OP == Bin::Add || OP == Bin::Sub) {
        if (OP == Bin::Sub) {
          y.x = ~y.x;
          y.y = ~y.y;
          y.z = ~y.z;
          y.w = ~y.w;
        }
        uint64_t t;
        t = (uint64_t)x.x + y.x + carry; r.x = (uint32_t)t; carry = (uint32_t)(t >> 32);
        t = (uint64_t)x.y + y.y + carry; r.y = (uint32_t)t; carry = (uint32_t)(t >> 32);
        t = (uint64_t)x.z + y.z + carry; r.z = (uint32_t)t; carry = (uint32_t)(t >> 32);
        t = (uint64_t)x.w + y.w + carry; r.w = (uint32_t)t; carry = (uint32_t)(t >> 32);
      } else if (OP == Bin::And) {
        r = make_uint4(x.x & y.x, x.y & y.y, x.z & y.z, x.w & y.w);
      } else if (OP == Bin::Ior) {
        r = make_uint4(x.x | y.x, x.y | y.y, x.z | y.z, x.w | y.w);
      } else {
        r = make_uint4(x.x ^ y.x, x.y ^ y.y, x.z ^ y.z, x.w ^ y.w);
      }
      store_group(c.limbs, c.nlimbs, c.stride, ec, g, r);
    }
  }
}

__global__ void __launch_bounds__(256) not_kernel(ArrayView a, OutView c, uint32_t count) {
  XMPB_FOR_INSTANCES(i, count) {
    const uint32_t i = (uint32_t)i_;
    uint32_t ea = ew_element(a, i), ec = out_element(c, i);
    if (ec >= c.count) continue;
    uint32_t groups = div_up(c.nlimbs, 4);
    for (uint32_t g = 0; g < groups; g++) {
      uint4 x = load_group(a.limbs, a.nlimbs, a.stride, ea, g);
      store_group(c.limbs, c.nlimbs, c.stride, ec, g, make_uint4(~x.x, ~x.y, ~x.z, ~x.w));
    }
  }
}

// Output limb k = input bits [32k + t, 32k + t + 32) with t = -shift (floor semantics).
__global__ void __launch_bounds__(256) shf_kernel(ArrayView a, OutView c, const int32_t *shift, uint32_t shift_count,
                                                  uint32_t count) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint32_t ea = ew_element(a, i), ec = out_element(c, i);
  if (ec >= c.count) return;
  int64_t t = -(int64_t)shift[i % shift_count];
  int64_t q = (t >= 0) ? t / 32 : -((-t + 31) / 32);  // floor(t / 32)
  uint32_t r = (uint32_t)(t - q * 32);
  uint32_t groups = div_up(c.nlimbs, 4);
  auto limb_at = [&](int64_t j) -> uint32_t {
    if (j < 0 || j >= (int64_t)a.nlimbs) return 0u;
    return load_limb(a.limbs, a.nlimbs, a.stride, ea, (uint32_t)j);
  };
  int64_t j0 = q;
  uint32_t low = limb_at(j0);
  for (uint32_t g = 0; g < groups; g++) {
    uint32_t out[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      uint32_t high = limb_at(j0 + (int64_t)(g * 4 + k) + 1);
      out[k] = r ? __funnelshift_r(low, high, r) : low;
      low = high;
    }
    store_group(c.limbs, c.nlimbs, c.stride, ec, g, make_uint4(out[0], out[1], out[2], out[3]));
  }
}

// Same operation for operands of at most kShfSmemGroups limb groups: the
// operand is read with coalesced 128-bit group loads into this thread's
// column of shared memory ([limb][thread], conflict-free), and the shifted
// limbs are read back from there, so a warp whose lanes shift by different
// amounts still touches HBM only with whole groups.
constexpr uint32_t kShfSmemGroups = 8;  // up to 1024-bit operands
__global__ void __launch_bounds__(256) shf_smem_kernel(ArrayView a, OutView c, const int32_t *shift,
                                                       uint32_t shift_count, uint32_t count) {
  extern __shared__ uint32_t col[];  // [4 * groups of a][256]
  const uint32_t tid = threadIdx.x;
  uint32_t i = blockIdx.x * blockDim.x + tid;
  if (i >= count) return;
  uint32_t ea = ew_element(a, i), ec = out_element(c, i);
  if (ec >= c.count) return;
  const uint32_t ag = div_up(a.nlimbs, 4);
  for (uint32_t g = 0; g < ag; g++) {
    uint4 v = load_group(a.limbs, a.nlimbs, a.stride, ea, g);
    col[(4 * g) * 256 + tid] = v.x;
    col[(4 * g + 1) * 256 + tid] = v.y;
    col[(4 * g + 2) * 256 + tid] = v.z;
    col[(4 * g + 3) * 256 + tid] = v.w;
  }
  int64_t t = -(int64_t)shift[i % shift_count];
  int64_t q = (t >= 0) ? t / 32 : -((-t + 31) / 32);  // floor(t / 32)
  const uint32_t r = (uint32_t)(t - q * 32);
  const uint32_t groups = div_up(c.nlimbs, 4);
  // Output limb k reads source limbs q + k and q + k + 1; a window that misses the operand entirely
  // gives zeros.  Otherwise q fits 32 bits and one unsigned compare tests a limb index.
  const int64_t reach = (int64_t)groups * 4 + 1;
  if (q >= (int64_t)a.nlimbs || q + reach <= 0) q = -reach;
  const int32_t q32 = (int32_t)q;
  const uint32_t na = a.nlimbs;
  auto limb_at = [&](int32_t j) -> uint32_t { return (uint32_t)j < na ? col[j * 256 + tid] : 0u; };
  uint32_t low = limb_at(q32);
  for (uint32_t g = 0; g < groups; g++) {
    uint32_t out[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint32_t high = limb_at(q32 + (int32_t)(g * 4 + k) + 1);
      out[k] = __funnelshift_r(low, high, r);  // r = 0 gives low
      low = high;
    }
    store_group(c.limbs, c.nlimbs, c.stride, ec, g, make_uint4(out[0], out[1], out[2], out[3]));
  }
}

// Compares a and b as unsigned integers of their own precisions.  (The
// reference tests the longer operand's extra limbs of instance 0 instead of
// the selected instance, implementations.h:795; here the selected one.)
__global__ void __launch_bounds__(256) cmp_kernel(ArrayView a, ArrayView b, int32_t *out, uint32_t count) {
  XMPB_FOR_INSTANCES(i, count) {
    const uint32_t i = (uint32_t)i_;
    uint32_t ea = ew_element(a, i), eb = ew_element(b, i);
    uint32_t groups = div_up(max(a.nlimbs, b.nlimbs), 4);
    int32_t result = 0;
    for (int32_t g = (int32_t)groups - 1; g >= 0 && result == 0; g--) {
      uint4 x = load_group(a.limbs, a.nlimbs, a.stride, ea, g);
      uint4 y = load_group(b.limbs, b.nlimbs, b.stride, eb, g);
      if (x.w != y.w) result = x.w > y.w ? 1 : -1;
      else if (x.z != y.z) result = x.z > y.z ? 1 : -1;
      else if (x.y != y.y) result = x.y > y.y ? 1 : -1;
      else if (x.x != y.x) result = x.x > y.x ? 1 : -1;
    }
    out[i] = result;
  }
}

__global__ void __launch_bounds__(256) popc_kernel(ArrayView a, uint32_t *out, uint32_t count) {
  XMPB_FOR_INSTANCES(i, count) {
    const uint32_t i = (uint32_t)i_;
    uint32_t ea = ew_element(a, i);
    uint32_t groups = div_up(a.nlimbs, 4), s = 0;
    uint32_t g = 0;
    for (; g + 2 <= groups; g += 2) {  // two independent group loads in flight per thread
      uint4 x = load_group(a.limbs, a.nlimbs, a.stride, ea, g);
      uint4 y = load_group(a.limbs, a.nlimbs, a.stride, ea, g + 1);
      s += __popc(x.x) + __popc(x.y) + __popc(x.z) + __popc(x.w) + __popc(y.x) + __popc(y.y) + __popc(y.z) +
           __popc(y.w);
    }
    if (g < groups) {
      uint4 x = load_group(a.limbs, a.nlimbs, a.stride, ea, g);
      s += __popc(x.x) + __popc(x.y) + __popc(x.z) + __popc(x.w);
    }
    out[i] = s;
  }
}

// Grid for the grid-stride kernels: no more CTAs of 256 threads than the GPU holds at once.
static int stream_grid(xmpHandle_t h, uint32_t count) {
  return std::min(grid_for(count, 256), (int)h->sm_count * 8);
}

static bool any_index(xmpExecutionPolicy_t p) {
  for (uint32_t k = 0; k < kMaxIndexArrays; k++)
    if (p->indices[k]) return true;
  return false;
}

template <Bin OP>
static xmpError_t binary_op(xmpHandle_t h, xmpIntegers_t c, xmpIntegers_t a, xmpIntegers_t b, uint32_t count) {
  if (!h || !c || !a || !b) return xmpErrorInvalidParameter;
  int dev = h->device;
  if (c->device != dev || a->device != dev || b->device != dev) return xmpErrorInvalidDevice;
  if (count == 0) return xmpErrorSuccess;
  DeviceGuard guard(dev);
  xmpExecutionPolicy_t p = h->policy;
  if (c->count < count) return xmpErrorInvalidCount;
  if (p->indices[0] && p->indices_count[0] < count) return xmpErrorInvalidCount;
  if (c->precision < (a->precision > b->precision ? a->precision : b->precision)) return xmpErrorInvalidPrecision;
  OutTarget t;
  xmpError_t e = begin_output(h, c, c == a || c == b, any_index(p), &t);
  if (e != xmpErrorSuccess) return e;
  binary_kernel<OP><<<stream_grid(h, count), 256, 0, h->stream>>>(
      view_in(a, p->indices[1], p->indices_count[1]), view_in(b, p->indices[2], p->indices_count[2]),
      view_out(c, t.limbs, p->indices[0]), count);
  e = end_output(h, c, t);
  if (e != xmpErrorSuccess) return e;
  return check_cuda();
}

static xmpError_t sync_after(xmpHandle_t h, xmpError_t e) {
  if (e != xmpErrorSuccess) return e;
  DeviceGuard guard(h->device);
  cudaStreamSynchronize(h->stream);
  return check_cuda();
}

// Device buffer for a small per-instance result array that may live in host memory.
struct ResultBuffer {
  void *dev = nullptr;
  bool host = false;
};
static xmpError_t result_buffer(xmpHandle_t h, void *user, size_t bytes, size_t scratch_offset, ResultBuffer *r) {
  r->host = is_host_pointer(user);
  r->dev = user;
  if (r->host) {
    xmpError_t e = ensure_scratch(h, scratch_offset + bytes);
    if (e != xmpErrorSuccess) return e;
    r->dev = (char *)h->scratch + scratch_offset;
  }
  return xmpErrorSuccess;
}

}  // namespace xmpb

extern "C" {

xmpError_t XMPAPI xmpIntegersAddAsync(xmpHandle_t h, xmpIntegers_t s, const xmpIntegers_t a, const xmpIntegers_t b,
                                       uint32_t count) {
  return binary_op<Bin::Add>(h, s, a, b, count);
}
xmpError_t XMPAPI xmpIntegersAdd(xmpHandle_t h, xmpIntegers_t s, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count) {
  return sync_after(h, xmpIntegersAddAsync(h, s, a, b, count));
}
xmpError_t XMPAPI xmpIntegersSubAsync(xmpHandle_t h, xmpIntegers_t d, const xmpIntegers_t a, const xmpIntegers_t b,
                                       uint32_t count) {
  return binary_op<Bin::Sub>(h, d, a, b, count);
}
xmpError_t XMPAPI xmpIntegersSub(xmpHandle_t h, xmpIntegers_t d, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count) {
  return sync_after(h, xmpIntegersSubAsync(h, d, a, b, count));
}
xmpError_t XMPAPI xmpIntegersAndAsync(xmpHandle_t h, xmpIntegers_t c, const xmpIntegers_t a, const xmpIntegers_t b,
                                       uint32_t count) {
  return binary_op<Bin::And>(h, c, a, b, count);
}
xmpError_t XMPAPI xmpIntegersAnd(xmpHandle_t h, xmpIntegers_t c, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count) {
  return sync_after(h, xmpIntegersAndAsync(h, c, a, b, count));
}
xmpError_t XMPAPI xmpIntegersIorAsync(xmpHandle_t h, xmpIntegers_t c, const xmpIntegers_t a, const xmpIntegers_t b,
                                       uint32_t count) {
  return binary_op<Bin::Ior>(h, c, a, b, count);
}
xmpError_t XMPAPI xmpIntegersIor(xmpHandle_t h, xmpIntegers_t c, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count) {
  return sync_after(h, xmpIntegersIorAsync(h, c, a, b, count));
}
xmpError_t XMPAPI xmpIntegersXorAsync(xmpHandle_t h, xmpIntegers_t c, const xmpIntegers_t a, const xmpIntegers_t b,
                                       uint32_t count) {
  return binary_op<Bin::Xor>(h, c, a, b, count);
}
xmpError_t XMPAPI xmpIntegersXor(xmpHandle_t h, xmpIntegers_t c, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count) {
  return sync_after(h, xmpIntegersXorAsync(h, c, a, b, count));
}

xmpError_t XMPAPI xmpIntegersNotAsync(xmpHandle_t h, xmpIntegers_t c, const xmpIntegers_t a, uint32_t count) {
  if (!h || !c || !a) return xmpErrorInvalidParameter;
  if (c->device != h->device || a->device != h->device) return xmpErrorInvalidDevice;
  if (count == 0) return xmpErrorSuccess;
  DeviceGuard guard(h->device);
  xmpExecutionPolicy_t p = h->policy;
  if (c->count < count) return xmpErrorInvalidCount;
  if (p->indices[0] && p->indices_count[0] < count) return xmpErrorInvalidCount;
  if (c->precision < a->precision) return xmpErrorInvalidPrecision;
  OutTarget t;
  xmpError_t e = begin_output(h, c, c == a, any_index(p), &t);
  if (e != xmpErrorSuccess) return e;
  not_kernel<<<stream_grid(h, count), 256, 0, h->stream>>>(view_in(a, p->indices[1], p->indices_count[1]),
                                                           view_out(c, t.limbs, p->indices[0]), count);
  e = end_output(h, c, t);
  if (e != xmpErrorSuccess) return e;
  return check_cuda();
}
xmpError_t XMPAPI xmpIntegersNot(xmpHandle_t h, xmpIntegers_t c, const xmpIntegers_t a, uint32_t count) {
  return sync_after(h, xmpIntegersNotAsync(h, c, a, count));
}

xmpError_t XMPAPI xmpIntegersShfAsync(xmpHandle_t h, xmpIntegers_t c, const xmpIntegers_t a, const int32_t *shift,
                                       const uint32_t shift_count, uint32_t count) {
  if (!h || !c || !a || shift == nullptr) return xmpErrorInvalidParameter;
  if (c->device != h->device || a->device != h->device) return xmpErrorInvalidDevice;
  if (count == 0) return xmpErrorSuccess;
  DeviceGuard guard(h->device);
  xmpExecutionPolicy_t p = h->policy;
  if (c->count < count) return xmpErrorInvalidCount;
  if (p->indices[0] && p->indices_count[0] < count) return xmpErrorInvalidCount;
  if (shift_count == 0) return xmpErrorInvalidParameter;
  uint32_t scount = shift_count < count ? shift_count : count;
  const int32_t *dshift = shift;
  if (is_host_pointer(shift)) {
    xmpError_t e = ensure_scratch(h, (size_t)scount * sizeof(int32_t));
    if (e != xmpErrorSuccess) return e;
    if (cudaMemcpyAsync(h->scratch, shift, (size_t)scount * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream) !=
        cudaSuccess)
      return xmpErrorCuda;
    dshift = (const int32_t *)h->scratch;
  }
  // In place always stages: output limb k reads input limbs above and below k.
  OutTarget t;
  xmpError_t e = begin_output(h, c, c == a, true, &t);
  if (e != xmpErrorSuccess) return e;
  if (div_up(a->nlimbs, 4) <= kShfSmemGroups)
    shf_smem_kernel<<<grid_for(count, 256), 256, div_up(a->nlimbs, 4) * 4 * 256 * sizeof(uint32_t), h->stream>>>(
        view_in(a, p->indices[1], p->indices_count[1]),
                                                                  view_out(c, t.limbs, p->indices[0]), dshift,
                                                                  scount, count);
  else
    shf_kernel<<<grid_for(count, 256), 256, 0, h->stream>>>(view_in(a, p->indices[1], p->indices_count[1]),
                                                             view_out(c, t.limbs, p->indices[0]), dshift, scount,
                                                             count);
  e = end_output(h, c, t);
  if (e != xmpErrorSuccess) return e;
  return check_cuda();
}
xmpError_t XMPAPI xmpIntegersShf(xmpHandle_t h, xmpIntegers_t c, const xmpIntegers_t a, const int32_t *shift,
                                  const uint32_t shift_count, uint32_t count) {
  return sync_after(h, xmpIntegersShfAsync(h, c, a, shift, shift_count, count));
}

xmpError_t XMPAPI xmpIntegersCmpAsync(xmpHandle_t h, int32_t *c, const xmpIntegers_t a, const xmpIntegers_t b,
                                       uint32_t count) {
  if (!h || !a || !b || c == nullptr) return xmpErrorInvalidParameter;
  if (a->device != h->device || b->device != h->device) return xmpErrorInvalidDevice;
  if (count == 0) return xmpErrorSuccess;
  DeviceGuard guard(h->device);
  xmpExecutionPolicy_t p = h->policy;
  ResultBuffer rb;
  xmpError_t e = result_buffer(h, c, (size_t)count * sizeof(int32_t), 0, &rb);
  if (e != xmpErrorSuccess) return e;
  cmp_kernel<<<stream_grid(h, count), 256, 0, h->stream>>>(view_in(a, p->indices[0], p->indices_count[0]),
                                                           view_in(b, p->indices[1], p->indices_count[1]),
                                                           (int32_t *)rb.dev, count);
  if (rb.host &&
      cudaMemcpyAsync(c, rb.dev, (size_t)count * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
    return xmpErrorCuda;
  return check_cuda();
}
xmpError_t XMPAPI xmpIntegersCmp(xmpHandle_t h, int32_t *c, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count) {
  return sync_after(h, xmpIntegersCmpAsync(h, c, a, b, count));
}

xmpError_t XMPAPI xmpIntegersPopcAsync(xmpHandle_t h, uint32_t *c, const xmpIntegers_t a, uint32_t count) {
  if (!h || !a || c == nullptr) return xmpErrorInvalidParameter;
  if (a->device != h->device) return xmpErrorInvalidDevice;
  if (count == 0) return xmpErrorSuccess;
  if (a->count < count) return xmpErrorInvalidCount;
  DeviceGuard guard(h->device);
  xmpExecutionPolicy_t p = h->policy;
  ResultBuffer rb;
  xmpError_t e = result_buffer(h, c, (size_t)count * sizeof(uint32_t), 0, &rb);
  if (e != xmpErrorSuccess) return e;
  popc_kernel<<<stream_grid(h, count), 256, 0, h->stream>>>(view_in(a, p->indices[0], p->indices_count[0]),
                                                            (uint32_t *)rb.dev, count);
  if (rb.host &&
      cudaMemcpyAsync(c, rb.dev, (size_t)count * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
    return xmpErrorCuda;
  return check_cuda();
}
xmpError_t XMPAPI xmpIntegersPopc(xmpHandle_t h, uint32_t *c, const xmpIntegers_t a, uint32_t count) {
  return sync_after(h, xmpIntegersPopcAsync(h, c, a, count));
}

}  // extern "C"
