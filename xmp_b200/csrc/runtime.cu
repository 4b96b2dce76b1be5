// Host runtime of the XMP-compatible C API: handles, execution policies,
// integer arrays, import/export and set.
//
// Reference interfaces replaced (all in src/xmp.cu unless noted):
//   handle          39-191    policy          193-314
//   integers        317-388   import/export   461-682 (xmpTransform 461-489)
//   set             685-813   C2S/S2C         817-843, xmp_internal.h:166-239
// Semantics kept: error codes and their order of checks, index gather/scatter
// rules, GMP-style (words, order, size, endian, nails) wire format where nails
// masks the top `nails` bits of every word after the optional byte swap.
#include "internal.h"
#include "tune.h"
#include <stdlib.h>
#include <string.h>

using namespace xmpb;

namespace xmpb {

static void *default_device_malloc(size_t bytes) {
  void *p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}
static void default_device_free(void *p) {
  if (p) cudaFree(p);
}

size_t scratch_limit(xmpHandle_t h) {
  size_t lim = h->policy ? h->policy->scratch_size_limit : 0;
  if (lim == 0) lim = h->memory_size / 4 * 3;
  return lim;
}

xmpError_t ensure_scratch(xmpHandle_t h, size_t bytes) {
  if (bytes > scratch_limit(h)) return xmpErrorIncreaseScratchLimit;
  if (h->scratch_size < bytes || h->scratch == nullptr) {
    if (h->scratch) h->df(h->scratch);
    size_t want = bytes < 4096 ? 4096 : bytes;
    h->scratch = h->da(want);
    h->scratch_size = h->scratch ? want : 0;
    if (!h->scratch) return xmpErrorInvalidCudaMalloc;
  }
  return check_cuda();
}

xmpError_t ensure_tmp_out(xmpHandle_t h, size_t bytes) {
  if (h->tmp_out_size < bytes || h->tmp_out == nullptr) {
    if (h->tmp_out) h->df(h->tmp_out);
    size_t want = bytes < 4096 ? 4096 : bytes;
    h->tmp_out = h->da(want);
    h->tmp_out_size = h->tmp_out ? want : 0;
    if (!h->tmp_out) return xmpErrorInvalidCudaMalloc;
  }
  return check_cuda();
}

bool is_host_pointer(const void *p) {
  cudaPointerAttributes attr;
  cudaError_t e = cudaPointerGetAttributes(&attr, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return !(attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged);
}

xmpError_t begin_output(xmpHandle_t h, xmpIntegers_t out, bool aliased, bool needs_stage, OutTarget *t,
                        size_t offset) {
  t->limbs = out->limbs;
  t->staged = false;
  if (!(aliased && needs_stage)) return xmpErrorSuccess;
  xmpError_t e = ensure_tmp_out(h, offset + out->bytes);
  if (e != xmpErrorSuccess) return e;
  uint32_t *tmp = reinterpret_cast<uint32_t *>(reinterpret_cast<char *>(h->tmp_out) + offset);
  if (cudaMemcpyAsync(tmp, out->limbs, out->bytes, cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess)
    return xmpErrorCuda;
  t->limbs = tmp;
  t->staged = true;
  return xmpErrorSuccess;
}

xmpError_t end_output(xmpHandle_t h, xmpIntegers_t out, const OutTarget &t) {
  if (!t.staged) return xmpErrorSuccess;
  if (cudaMemcpyAsync(out->limbs, t.limbs, out->bytes, cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess)
    return xmpErrorCuda;
  return xmpErrorSuccess;
}

// ---------------------------------------------------------------------------
// Wire-format kernels.
// ---------------------------------------------------------------------------

template <class T>
__device__ __forceinline__ T bswap(T v);
template <>
__device__ __forceinline__ uint8_t bswap(uint8_t v) { return v; }
template <>
__device__ __forceinline__ uint16_t bswap(uint16_t v) { return (uint16_t)__byte_perm(v, 0, 0x3201) & 0xffff; }
template <>
__device__ __forceinline__ uint32_t bswap(uint32_t v) { return __byte_perm(v, 0, 0x0123); }
template <>
__device__ __forceinline__ uint64_t bswap(uint64_t v) {
  uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
  return ((uint64_t)__byte_perm(lo, 0, 0x0123) << 32) | __byte_perm(hi, 0, 0x0123);
}

struct WireArgs {
  uint32_t words;     // words per integer in the wire format
  int32_t order;      // -1 least significant word first, 1 most significant first
  int32_t swap;       // byte-swap every word
  uint32_t nails;     // top bits of each word forced to zero
  uint32_t count;     // instances to move
  const uint32_t *index;  // optional: import gathers wire element index[i % n]; export scatters to index[i % n]
  uint32_t index_count;
  uint32_t rows;      // wire rows addressable through `index` (staged host buffers hold `count` rows)
};

// Import: one thread per (instance, limb).  Limb j of the number is assembled
// from the wire words overlapping bytes [4j, 4j+4).
template <class T>
__global__ void import_kernel(const T *__restrict__ in, uint32_t *__restrict__ limbs, uint32_t nlimbs,
                              uint32_t stride, WireArgs a) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.count || j >= round_up(nlimbs, 4)) return;
  uint32_t src = a.index ? a.index[i % a.index_count] : i;
  const T mask = (T)(~(T)0) >> a.nails;
  uint32_t limb = 0;
  if (j < nlimbs && src < a.rows) {
    if constexpr (sizeof(T) <= 4) {
      constexpr uint32_t per = 4 / sizeof(T);
#pragma unroll
      for (uint32_t q = 0; q < per; q++) {
        uint32_t w = j * per + q;
        if (w < a.words) {
          uint32_t p = a.order == -1 ? w : a.words - 1 - w;
          T raw = in[(size_t)src * a.words + p];
          if (a.swap) raw = bswap<T>(raw);
          raw &= mask;
          limb |= (uint32_t)raw << (q * 8 * sizeof(T));
        }
      }
    } else {
      uint32_t w = j / 2;
      uint32_t p = a.order == -1 ? w : a.words - 1 - w;
      T raw = in[(size_t)src * a.words + p];
      if (a.swap) raw = bswap<T>(raw);
      raw &= mask;
      uint64_t r64 = (uint64_t)raw;
      limb = (j & 1) ? (uint32_t)(r64 >> 32) : (uint32_t)r64;
    }
  }
  limbs[((size_t)(j >> 2) * stride + i) * 4 + (j & 3)] = limb;
}

// Export: one thread per (instance, wire word).
template <class T>
__global__ void export_kernel(const uint32_t *__restrict__ limbs, uint32_t nlimbs, uint32_t stride,
                              T *__restrict__ out, WireArgs a) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t p = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.count || p >= a.words) return;
  uint32_t dst = a.index ? a.index[i % a.index_count] : i;
  if (dst >= a.rows) return;
  uint32_t w = a.order == -1 ? p : a.words - 1 - p;
  T v;
  if constexpr (sizeof(T) == 8) {
    uint64_t lo = load_limb(limbs, nlimbs, stride, i, 2 * w), hi = load_limb(limbs, nlimbs, stride, i, 2 * w + 1);
    v = (T)(lo | (hi << 32));
  } else {
    constexpr uint32_t per = 4 / sizeof(T);
    uint32_t limb = load_limb(limbs, nlimbs, stride, i, w / per);
    v = (T)(limb >> ((w % per) * 8 * sizeof(T)));
  }
  if (a.swap) v = bswap<T>(v);
  v &= (T)(~(T)0) >> a.nails;
  out[(size_t)dst * a.words + p] = v;
}

// Native fast paths: compact uint32 rows <-> interleaved groups, one uint4 per thread.
// `vec` (128-bit row access) requires nlimbs % 4 == 0 and a 16-byte aligned buffer.
__global__ void compact_to_interleaved(const uint32_t *__restrict__ in, uint32_t *__restrict__ limbs,
                                       uint32_t nlimbs, uint32_t stride, uint32_t count, bool vec) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t g = blockIdx.y;
  if (i >= count) return;
  const uint32_t *row = in + (size_t)i * nlimbs;
  uint4 v;
  uint32_t j = g * 4;
  if (vec) {
    v = __ldg(reinterpret_cast<const uint4 *>(row) + g);
  } else {
    v.x = j < nlimbs ? row[j] : 0;
    v.y = j + 1 < nlimbs ? row[j + 1] : 0;
    v.z = j + 2 < nlimbs ? row[j + 2] : 0;
    v.w = j + 3 < nlimbs ? row[j + 3] : 0;
  }
  reinterpret_cast<uint4 *>(limbs)[(size_t)g * stride + i] = v;
}

__global__ void interleaved_to_compact(const uint32_t *__restrict__ limbs, uint32_t nlimbs, uint32_t stride,
                                       uint32_t *__restrict__ out, uint32_t count, bool vec) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t g = blockIdx.y;
  if (i >= count) return;
  uint4 v = __ldg(reinterpret_cast<const uint4 *>(limbs) + (size_t)g * stride + i);
  uint32_t *row = out + (size_t)i * nlimbs;
  uint32_t j = g * 4;
  if (vec) {
    reinterpret_cast<uint4 *>(row)[g] = v;
  } else {
    if (j < nlimbs) row[j] = v.x;
    if (j + 1 < nlimbs) row[j + 1] = v.y;
    if (j + 2 < nlimbs) row[j + 2] = v.z;
    if (j + 3 < nlimbs) row[j + 3] = v.w;
  }
}

// Indexed copy between arrays of equal precision (xmpReorder_compact_kernel, src/xmp.cu:693-716).
__global__ void reorder_kernel(const uint32_t *__restrict__ in, uint32_t in_stride, uint32_t in_count,
                               const uint32_t *in_index, uint32_t in_index_count, uint32_t *__restrict__ out,
                               uint32_t out_stride, uint32_t out_count, const uint32_t *out_index,
                               uint32_t out_index_count, uint32_t ngroups, uint32_t count) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t g = blockIdx.y;
  if (i >= count) return;
  uint32_t s = in_index ? in_index[i % in_index_count] % in_count : i;
  uint32_t d = out_index ? out_index[i % out_index_count] : i;
  if (d >= out_count) return;
  reinterpret_cast<uint4 *>(out)[(size_t)g * out_stride + d] =
      __ldg(reinterpret_cast<const uint4 *>(in) + (size_t)g * in_stride + s);
}

}  // namespace xmpb

// ---------------------------------------------------------------------------
// Handle
// ---------------------------------------------------------------------------
extern "C" {

xmpError_t XMPAPI xmpHandleCreate(xmpHandle_t *handle) {
  return xmpHandleCreateWithMemoryFunctions(handle, malloc, free, default_device_malloc, default_device_free);
}

xmpError_t XMPAPI xmpHandleCreateWithMemoryFunctions(xmpHandle_t *handle, xmpAllocFunc ha, xmpFreeFunc hf,
                                                      xmpAllocFunc da, xmpFreeFunc df) {
  if (handle == nullptr) return xmpErrorInvalidParameter;
  if (!ha) ha = malloc;
  if (!hf) hf = free;
  if (!da) da = default_device_malloc;
  if (!df) df = default_device_free;
  _xmpHandle_t *h = (_xmpHandle_t *)ha(sizeof(_xmpHandle_t));
  *handle = h;
  if (!h) return xmpErrorInvalidMalloc;
  memset(h, 0, sizeof(*h));
  h->ha = ha;
  h->hf = hf;
  h->da = da;
  h->df = df;
  h->default_policy.algorithm = xmpAlgorithmDefault;
  h->policy = &h->default_policy;
  if (cudaGetDevice(&h->device) != cudaSuccess) return xmpErrorInvalidDevice;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, h->device) != cudaSuccess) return xmpErrorInvalidDevice;
  h->memory_size = prop.totalGlobalMem;
  h->arch = prop.major * 10 + prop.minor;
  h->sm_count = prop.multiProcessorCount;
  // Configuration choices start from the compiled-in learned selector; if it cannot be
  // loaded (e.g. the caller's allocator refuses), the built-in heuristic stays in charge.
  int members = 0;
  if (const float *params = xmpb::default_selector_params(&members)) {
    if (xmpSelectorLoadEnsemble(h, params, members) != xmpErrorSuccess) {
      xmpTuneClear(h);
      cudaGetLastError();  // a refused allocation is not an error of this call
    }
  }
  return check_cuda();
}

xmpError_t XMPAPI xmpHandleDestroy(xmpHandle_t handle) {
  if (!handle) return xmpErrorInvalidParameter;
  DeviceGuard g(handle->device);
  cudaStreamSynchronize(handle->stream);
  if (handle->scratch) handle->df(handle->scratch);
  if (handle->tmp_out) handle->df(handle->tmp_out);
  tuner_destroy(handle);
  xmpFreeFunc hf = handle->hf;
  hf(handle);
  return check_cuda();
}

xmpError_t XMPAPI xmpHandleSetStream(xmpHandle_t handle, cudaStream_t stream) {
  if (!handle) return xmpErrorInvalidParameter;
  handle->stream = stream;
  return check_cuda();
}

xmpError_t XMPAPI xmpHandleGetStream(xmpHandle_t handle, cudaStream_t *stream) {
  if (!handle || !stream) return xmpErrorInvalidParameter;
  *stream = handle->stream;
  return check_cuda();
}

xmpError_t XMPAPI xmpHandleSetCudaStream(xmpHandle_t handle, cudaStream_t stream) {
  return xmpHandleSetStream(handle, stream);
}

xmpError_t XMPAPI xmpHandleGetCudaStream(xmpHandle_t handle, cudaStream_t *stream) {
  return xmpHandleGetStream(handle, stream);
}

xmpError_t XMPAPI xmpHandleGetDevice(xmpHandle_t handle, int32_t *device) {
  if (!handle || !device) return xmpErrorInvalidParameter;
  *device = handle->device;
  return check_cuda();
}

xmpError_t XMPAPI xmpHandleSetExecutionPolicy(xmpHandle_t handle, xmpExecutionPolicy_t policy) {
  if (!handle) return xmpErrorInvalidParameter;
  handle->policy = policy ? policy : &handle->default_policy;
  return xmpErrorSuccess;
}

// The reference assigns *df only when hf is non-NULL (src/xmp.cu:155); here
// each output pointer is filled when it is non-NULL.
xmpError_t XMPAPI xmpHandleGetMemoryFunctions(xmpHandle_t handle, xmpAllocFunc *ha, xmpFreeFunc *hf,
                                               xmpAllocFunc *da, xmpFreeFunc *df) {
  if (!handle) return xmpErrorInvalidParameter;
  if (ha) *ha = handle->ha;
  if (hf) *hf = handle->hf;
  if (da) *da = handle->da;
  if (df) *df = handle->df;
  return check_cuda();
}

// ---------------------------------------------------------------------------
// Execution policy
// ---------------------------------------------------------------------------
xmpError_t XMPAPI xmpExecutionPolicyCreate(xmpHandle_t handle, xmpExecutionPolicy_t *policy) {
  if (!handle || !policy) return xmpErrorInvalidParameter;
  DeviceGuard g(handle->device);
  _xmpExecutionPolicy_t *p = (_xmpExecutionPolicy_t *)handle->ha(sizeof(_xmpExecutionPolicy_t));
  *policy = p;
  if (!p) return xmpErrorInvalidMalloc;
  memset(p, 0, sizeof(*p));
  p->algorithm = xmpAlgorithmDefault;
  return xmpErrorSuccess;
}

xmpError_t XMPAPI xmpExecutionPolicyDestroy(xmpHandle_t handle, xmpExecutionPolicy_t policy) {
  if (!handle || !policy) return xmpErrorInvalidParameter;
  DeviceGuard g(handle->device);
  if (handle->policy == policy) handle->policy = &handle->default_policy;
  cudaStreamSynchronize(handle->stream);
  for (uint32_t i = 0; i < kMaxIndexArrays; i++)
    if (policy->indices[i]) handle->df(policy->indices[i]);
  handle->hf(policy);
  return check_cuda();
}

xmpError_t XMPAPI xmpExecutionPolicySetIndicesAsync(xmpHandle_t handle, xmpExecutionPolicy_t policy,
                                                     uint32_t which_integer, uint32_t *indices, uint32_t count) {
  if (!handle || !policy) return xmpErrorInvalidParameter;
  DeviceGuard g(handle->device);
  if (which_integer >= kMaxIndexArrays) return xmpErrorInvalidParameter;
  uint32_t **slot = &policy->indices[which_integer];
  if (indices == nullptr) {
    if (*slot) {
      cudaStreamSynchronize(handle->stream);
      handle->df(*slot);
      *slot = nullptr;
    }
    policy->indices_count[which_integer] = 0;
    policy->indices_capacity[which_integer] = 0;
    return xmpErrorSuccess;
  }
  if (count == 0) return xmpErrorInvalidCount;
  if (*slot && policy->indices_capacity[which_integer] < count) {
    cudaStreamSynchronize(handle->stream);
    handle->df(*slot);
    *slot = nullptr;
  }
  if (!*slot) {
    *slot = (uint32_t *)handle->da(sizeof(uint32_t) * count);
    if (!*slot) return xmpErrorInvalidCudaMalloc;
    policy->indices_capacity[which_integer] = count;
  }
  if (cudaMemcpyAsync(*slot, indices, sizeof(uint32_t) * count, cudaMemcpyDefault, handle->stream) != cudaSuccess)
    return xmpErrorCuda;
  policy->indices_count[which_integer] = count;
  return check_cuda();
}

xmpError_t XMPAPI xmpExecutionPolicySetIndices(xmpHandle_t handle, xmpExecutionPolicy_t policy,
                                                uint32_t which_integer, uint32_t *indices, uint32_t count) {
  xmpError_t e = xmpExecutionPolicySetIndicesAsync(handle, policy, which_integer, indices, count);
  if (e != xmpErrorSuccess) return e;
  DeviceGuard g(handle->device);
  return cudaStreamSynchronize(handle->stream) == cudaSuccess ? xmpErrorSuccess : xmpErrorCuda;
}

xmpError_t XMPAPI xmpExecutionPolicySetParameter(xmpHandle_t handle, xmpExecutionPolicy_t policy,
                                                  xmpExecutionPolicyParam_t param, xmpExecutionPolicyValue_t val) {
  if (!policy) return xmpErrorInvalidParameter;
  switch (param) {
    case xmpAlgorithm:
      if ((int)val.algorithm < (int)xmpAlgorithmDefault || (int)val.algorithm > (int)xmpAlgorithmDistributedMP)
        return xmpErrorInvalidParameter;
      policy->algorithm = val.algorithm;
      return xmpErrorSuccess;
    case xmpScratchSizeLimit:
      policy->scratch_size_limit = val.size;
      return xmpErrorSuccess;
    default:
      return xmpErrorInvalidParameter;
  }
}

xmpError_t XMPAPI xmpExecutionPolicyGetParameter(xmpHandle_t handle, xmpExecutionPolicy_t policy,
                                                  xmpExecutionPolicyParam_t param, xmpExecutionPolicyValue_t &val) {
  if (!policy) return xmpErrorInvalidParameter;
  switch (param) {
    case xmpAlgorithm:
      val.size = 0;
      val.algorithm = policy->algorithm;
      return xmpErrorSuccess;
    case xmpScratchSizeLimit:
      val.size = policy->scratch_size_limit;
      return xmpErrorSuccess;
    default:
      return xmpErrorInvalidParameter;
  }
}

// ---------------------------------------------------------------------------
// Integer arrays
// ---------------------------------------------------------------------------
xmpError_t XMPAPI xmpIntegersCreate(xmpHandle_t handle, xmpIntegers_t *x, uint32_t precision, uint32_t count) {
  if (!handle || !x) return xmpErrorInvalidParameter;
  DeviceGuard g(handle->device);
  if (count == 0 || count > 0xfffffffcu) return xmpErrorInvalidCount;
  if (precision == 0 || precision % 32 != 0) return xmpErrorUnsupported;
  _xmpIntegers_t *r = (_xmpIntegers_t *)handle->ha(sizeof(_xmpIntegers_t));
  *x = r;
  if (!r) return xmpErrorInvalidMalloc;
  r->precision = precision;
  r->nlimbs = precision / 32;
  r->ngroups = div_up(r->nlimbs, 4);
  r->stride = round_up(count, 32);
  r->count = count;
  r->device = handle->device;
  r->bytes = (size_t)r->ngroups * r->stride * 16;
  r->limbs = (uint32_t *)handle->da(r->bytes);
  if (!r->limbs) {
    handle->hf(r);
    *x = nullptr;
    return xmpErrorInvalidCudaMalloc;
  }
  // Zero so that padding limbs and never-written instances read as 0.
  if (cudaMemsetAsync(r->limbs, 0, r->bytes, handle->stream) != cudaSuccess) return xmpErrorCuda;
  return check_cuda();
}

xmpError_t XMPAPI xmpIntegersDestroy(xmpHandle_t handle, xmpIntegers_t x) {
  if (!handle || !x) return xmpErrorInvalidParameter;
  DeviceGuard g(handle->device);
  cudaStreamSynchronize(handle->stream);
  handle->df(x->limbs);
  handle->hf(x);
  return check_cuda();
}

xmpError_t XMPAPI xmpIntegersGetPrecision(xmpHandle_t handle, xmpIntegers_t x, uint32_t *precision) {
  if (!x || !precision) return xmpErrorInvalidParameter;
  *precision = x->precision;
  return check_cuda();
}

xmpError_t XMPAPI xmpIntegersGetCount(xmpHandle_t handle, xmpIntegers_t x, uint32_t *count) {
  if (!x || !count) return xmpErrorInvalidParameter;
  *count = x->count;
  return check_cuda();
}

static int32_t native_endian() {
  int32_t one = 1;
  return *(char *)&one == 1 ? -1 : 1;
}

static xmpError_t import_internal(xmpHandle_t handle, xmpIntegers_t out, uint32_t words, int32_t order, size_t size,
                                  int32_t endian, uint32_t nails, void *in, uint32_t count, bool async) {
  if (!handle || !out || in == nullptr) return xmpErrorInvalidParameter;
  if (out->device != handle->device) return xmpErrorInvalidDevice;
  DeviceGuard g(handle->device);
  xmpExecutionPolicy_t policy = handle->policy;
  if (endian == 0) endian = native_endian();
  if (size != 1 && size != 2 && size != 4 && size != 8) return xmpErrorInvalidParameter;
  if (count == 0 || count > out->count || words == 0 || (order != 1 && order != -1) || (endian != 1 && endian != -1))
    return xmpErrorInvalidParameter;
  if ((uint64_t)words * size * 8 != out->precision) return xmpErrorInvalidPrecision;
  if (nails >= size * 8) return xmpErrorInvalidParameter;

  // Gather indices address rows of the caller's buffer; a host buffer is staged
  // with `count` rows (as the reference does, src/xmp.cu:515-543), so larger
  // indices read as zero instead of reading past the staging copy.
  size_t bytes = (size_t)count * words * size;
  const uint32_t *gather = policy->indices[0];
  uint32_t rows = 0xffffffffu;
  const void *src = in;
  if (is_host_pointer(in)) {
    rows = count;
    xmpError_t e = ensure_scratch(handle, bytes);
    if (e != xmpErrorSuccess) return e;
    if (cudaMemcpyAsync(handle->scratch, in, bytes, cudaMemcpyHostToDevice, handle->stream) != cudaSuccess)
      return xmpErrorCuda;
    src = handle->scratch;
  }
  bool native = (size == 4 && order == -1 && endian == native_endian() && nails == 0 && gather == nullptr);
  if (native) {
    dim3 block(128), grid(grid_for(count, 128), out->ngroups);
    bool vec = (out->nlimbs % 4 == 0) && ((uintptr_t)src % 16 == 0);
    compact_to_interleaved<<<grid, block, 0, handle->stream>>>((const uint32_t *)src, out->limbs, out->nlimbs,
                                                               out->stride, count, vec);
  } else {
    WireArgs a;
    a.words = words;
    a.order = order;
    a.swap = endian != native_endian();
    a.nails = nails;
    a.count = count;
    a.index = gather;
    a.index_count = policy->indices_count[0];
    a.rows = rows;
    uint32_t padded = round_up(out->nlimbs, 4);
    dim3 block(32, 4), grid(grid_for(count, 32), div_up(padded, 4));
    switch (size) {
      case 1: import_kernel<uint8_t><<<grid, block, 0, handle->stream>>>((const uint8_t *)src, out->limbs, out->nlimbs, out->stride, a); break;
      case 2: import_kernel<uint16_t><<<grid, block, 0, handle->stream>>>((const uint16_t *)src, out->limbs, out->nlimbs, out->stride, a); break;
      case 4: import_kernel<uint32_t><<<grid, block, 0, handle->stream>>>((const uint32_t *)src, out->limbs, out->nlimbs, out->stride, a); break;
      default: import_kernel<uint64_t><<<grid, block, 0, handle->stream>>>((const uint64_t *)src, out->limbs, out->nlimbs, out->stride, a); break;
    }
  }
  if (!async) cudaStreamSynchronize(handle->stream);
  return check_cuda();
}

xmpError_t XMPAPI xmpIntegersImport(xmpHandle_t handle, xmpIntegers_t out, uint32_t words, int32_t order, size_t size,
                                     int32_t endian, uint32_t nails, void *in, uint32_t count) {
  return import_internal(handle, out, words, order, size, endian, nails, in, count, false);
}
xmpError_t XMPAPI xmpIntegersImportAsync(xmpHandle_t handle, xmpIntegers_t out, uint32_t words, int32_t order,
                                          size_t size, int32_t endian, uint32_t nails, void *in, uint32_t count) {
  return import_internal(handle, out, words, order, size, endian, nails, in, count, true);
}

static xmpError_t export_internal(xmpHandle_t handle, void *out, uint32_t *words_out, int32_t order, size_t size,
                                  int32_t endian, uint32_t nails, xmpIntegers_t in, uint32_t count, bool async) {
  if (!handle || !in || out == nullptr) return xmpErrorInvalidParameter;
  if (in->device != handle->device) return xmpErrorInvalidDevice;
  DeviceGuard g(handle->device);
  xmpExecutionPolicy_t policy = handle->policy;
  if (endian == 0) endian = native_endian();
  if (size != 1 && size != 2 && size != 4 && size != 8) return xmpErrorInvalidParameter;
  if (count == 0 || count > in->count || (order != 1 && order != -1) || (endian != 1 && endian != -1))
    return xmpErrorInvalidParameter;
  if (nails >= size * 8) return xmpErrorInvalidParameter;
  // Same word count as the reference (src/xmp.cu:610): limbs*4/size, rounded down.
  uint32_t w = (uint32_t)(in->nlimbs * 4 / size);
  const uint32_t *scatter = policy->indices[0];
  size_t bytes = (size_t)count * w * size;
  bool host = is_host_pointer(out);
  void *dst = out;
  uint32_t rows = 0xffffffffu;
  if (host) {
    rows = count;
    xmpError_t e = ensure_scratch(handle, bytes);
    if (e != xmpErrorSuccess) return e;
    dst = handle->scratch;
    if (scatter) {
      // Scattered rows not written by this call keep the caller's contents.
      if (cudaMemcpyAsync(dst, out, bytes, cudaMemcpyHostToDevice, handle->stream) != cudaSuccess) return xmpErrorCuda;
    }
  }
  bool native = (size == 4 && order == -1 && endian == native_endian() && nails == 0 && scatter == nullptr);
  if (native) {
    dim3 block(128), grid(grid_for(count, 128), in->ngroups);
    bool vec = (in->nlimbs % 4 == 0) && ((uintptr_t)dst % 16 == 0);
    interleaved_to_compact<<<grid, block, 0, handle->stream>>>(in->limbs, in->nlimbs, in->stride, (uint32_t *)dst,
                                                               count, vec);
  } else if (w > 0) {
    WireArgs a;
    a.words = w;
    a.order = order;
    a.swap = endian != native_endian();
    a.nails = nails;
    a.count = count;
    a.index = scatter;
    a.index_count = policy->indices_count[0];
    a.rows = rows;
    dim3 block(32, 4), grid(grid_for(count, 32), div_up(w, 4));
    switch (size) {
      case 1: export_kernel<uint8_t><<<grid, block, 0, handle->stream>>>(in->limbs, in->nlimbs, in->stride, (uint8_t *)dst, a); break;
      case 2: export_kernel<uint16_t><<<grid, block, 0, handle->stream>>>(in->limbs, in->nlimbs, in->stride, (uint16_t *)dst, a); break;
      case 4: export_kernel<uint32_t><<<grid, block, 0, handle->stream>>>(in->limbs, in->nlimbs, in->stride, (uint32_t *)dst, a); break;
      default: export_kernel<uint64_t><<<grid, block, 0, handle->stream>>>(in->limbs, in->nlimbs, in->stride, (uint64_t *)dst, a); break;
    }
  }
  if (host) {
    if (cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToHost, handle->stream) != cudaSuccess) return xmpErrorCuda;
  }
  if (words_out) *words_out = w;
  if (!async) cudaStreamSynchronize(handle->stream);
  return check_cuda();
}

xmpError_t XMPAPI xmpIntegersExport(xmpHandle_t handle, void *out, uint32_t *words, int32_t order, size_t size,
                                     int32_t endian, uint32_t nails, xmpIntegers_t in, uint32_t count) {
  return export_internal(handle, out, words, order, size, endian, nails, in, count, false);
}
xmpError_t XMPAPI xmpIntegersExportAsync(xmpHandle_t handle, void *out, uint32_t *words, int32_t order, size_t size,
                                          int32_t endian, uint32_t nails, xmpIntegers_t in, uint32_t count) {
  return export_internal(handle, out, words, order, size, endian, nails, in, count, true);
}

xmpError_t XMPAPI xmpIntegersSetAsync(xmpHandle_t handle, xmpIntegers_t out, xmpIntegers_t in, uint32_t count) {
  if (!handle || !out || !in) return xmpErrorInvalidParameter;
  if (in->device != handle->device && out->device != handle->device) return xmpErrorInvalidDevice;
  DeviceGuard g(handle->device);
  if (in->precision != out->precision) return xmpErrorInvalidPrecision;
  if (out->count < count || in->count < count) return xmpErrorInvalidCount;
  if (count == 0) return xmpErrorSuccess;
  xmpExecutionPolicy_t policy = handle->policy;
  if (!policy->indices[0] && !policy->indices[1] && in->count == out->count) {
    // Equal counts and no indices: the whole array is copied (src/xmp.cu:750-771).
    if (in != out &&
        cudaMemcpyAsync(out->limbs, in->limbs, in->bytes, cudaMemcpyDefault, handle->stream) != cudaSuccess)
      return xmpErrorCuda;
    return check_cuda();
  }
  // Indexed or partial copy: stage the source so aliasing and cross-device sources are safe.
  xmpError_t e = ensure_scratch(handle, in->bytes);
  if (e != xmpErrorSuccess) return e;
  if (cudaMemcpyAsync(handle->scratch, in->limbs, in->bytes, cudaMemcpyDefault, handle->stream) != cudaSuccess)
    return xmpErrorCuda;
  dim3 block(128), grid(grid_for(count, 128), out->ngroups);
  reorder_kernel<<<grid, block, 0, handle->stream>>>((const uint32_t *)handle->scratch, in->stride, in->count,
                                                     policy->indices[1], policy->indices_count[1], out->limbs,
                                                     out->stride, out->count, policy->indices[0], policy->indices_count[0],
                                                     out->ngroups, count);
  return check_cuda();
}

xmpError_t XMPAPI xmpIntegersSet(xmpHandle_t handle, xmpIntegers_t out, xmpIntegers_t in, uint32_t count) {
  xmpError_t e = xmpIntegersSetAsync(handle, out, in, count);
  if (e != xmpErrorSuccess) return e;
  DeviceGuard g(handle->device);
  return cudaStreamSynchronize(handle->stream) == cudaSuccess ? xmpErrorSuccess : xmpErrorCuda;
}

}  // extern "C"
