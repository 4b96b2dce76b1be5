// Internal runtime types of the B200-native XMP-compatible library.
//
// Device layout of an integer array ("limb-group interleaved"):
//   limb j of instance i lives at uint32 offset ((j/4)*stride + i)*4 + j%4,
//   stride = count rounded up to 32.  Each 4-limb group of an instance is one
//   16-byte aligned uint4, so a thread moves its group with one 128-bit access
//   and a warp touches 512 contiguous bytes per group.  Limbs at positions
//   >= nlimbs inside the last group are padding: every kernel writes them as
//   zero and masks them on load.
// This replaces the reference's pair of device copies (compact + 32-bit
// strided, src/include/xmp_internal.h:194-239; src/xmp.cu:347-348): compact
// data only exists as the import/export wire format.
#pragma once

#include "../../include/xmp.h"
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

namespace xmpb {

constexpr uint32_t kMaxIndexArrays = 4;  // src/include/xmp_internal.h:59

__host__ __device__ inline uint32_t div_up(uint32_t n, uint32_t d) { return (n + d - 1) / d; }
__host__ __device__ inline uint32_t round_up(uint32_t n, uint32_t d) { return div_up(n, d) * d; }

// Read-only description of one operand as seen by a kernel.
struct ArrayView {
  uint32_t *limbs = nullptr;    // interleaved storage
  uint32_t nlimbs = 0;          // precision / 32
  uint32_t stride = 0;          // instances per limb-group row
  uint32_t count = 0;           // array count (for broadcast modulo)
  const uint32_t *index = nullptr;  // optional gather index array (device)
  uint32_t index_count = 0;
};

// Output description: scatter index is out_index[i] (no modulo), as in the
// reference kernels (implementations.h:66).
struct OutView {
  uint32_t *limbs = nullptr;
  uint32_t nlimbs = 0;
  uint32_t stride = 0;
  uint32_t count = 0;     // writes to elements >= count are dropped (bad scatter index)
  const uint32_t *index = nullptr;
};

// Input element selected by op instance i (docs 15-16; implementations.h:63-68).  (Taking the
// remainders only when they change the index saved 2-3 us on shf and cmp over 2^22 instances but
// moved the headline powm kernel's schedule: 240.1 against 237.8 ms per 65,536 x 2048-bit batch on
// the same GPU; the elementwise kernels use their own such form, ew_element, and the multiply's
// whole-group path skips this function.)
__device__ __forceinline__ uint32_t in_element(const ArrayView &v, uint32_t i) {
  uint32_t k = v.index ? v.index[i % v.index_count] : i;
  return k % v.count;
}
__device__ __forceinline__ uint32_t out_element(const OutView &v, uint32_t i) { return v.index ? v.index[i] : i; }

// Load limb group g of element e, masking padding limbs and groups beyond the precision.
__device__ __forceinline__ uint4 load_group(const uint32_t *limbs, uint32_t nlimbs, uint32_t stride, uint32_t e,
                                            uint32_t g) {
  uint4 v = make_uint4(0, 0, 0, 0);
  if (g * 4 < nlimbs) {
    v = __ldg(reinterpret_cast<const uint4 *>(limbs) + (size_t)g * stride + e);
    uint32_t rem = nlimbs - g * 4;
    if (rem < 4) {
      if (rem < 2) v.y = 0;
      if (rem < 3) v.z = 0;
      v.w = 0;
    }
  }
  return v;
}
__device__ __forceinline__ void store_group(uint32_t *limbs, uint32_t nlimbs, uint32_t stride, uint32_t e, uint32_t g,
                                            uint4 v) {
  uint32_t rem = nlimbs - g * 4;
  if (rem < 4) {
    if (rem < 2) v.y = 0;
    if (rem < 3) v.z = 0;
    v.w = 0;
  }
  reinterpret_cast<uint4 *>(limbs)[(size_t)g * stride + e] = v;
}
__device__ __forceinline__ uint32_t load_limb(const uint32_t *limbs, uint32_t nlimbs, uint32_t stride, uint32_t e,
                                              uint32_t j) {
  if (j >= nlimbs) return 0;
  return __ldg(limbs + ((size_t)(j >> 2) * stride + e) * 4 + (j & 3));
}
__device__ __forceinline__ uint32_t &limb_ref(uint32_t *limbs, uint32_t stride, uint32_t e, uint32_t j) {
  return limbs[((size_t)(j >> 2) * stride + e) * 4 + (j & 3)];
}
__device__ __forceinline__ uint32_t u4get(const uint4 &v, int k) {
  return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}

}  // namespace xmpb

// Execution policy (src/include/xmp_internal.h:59-73).
struct _xmpExecutionPolicy_t {
  size_t scratch_size_limit;
  uint32_t *indices[xmpb::kMaxIndexArrays];
  uint32_t indices_count[xmpb::kMaxIndexArrays];
  uint32_t indices_capacity[xmpb::kMaxIndexArrays];
  xmpAlgorithm_t algorithm;
};

// Handle (src/include/xmp_internal.h:75-88).  Owns a grow-only device scratch
// arena, a second arena for in-place outputs and the tuner state.
struct _xmpHandle_t {
  cudaStream_t stream;
  int32_t device;
  xmpAllocFunc ha, da;
  xmpFreeFunc hf, df;
  void *scratch;
  size_t scratch_size;
  void *tmp_out;
  size_t tmp_out_size;
  size_t memory_size;
  uint32_t arch;
  uint32_t sm_count;
  xmpExecutionPolicy_t policy;
  _xmpExecutionPolicy_t default_policy;
  void *tuner;  // xmpb::TunerState*, created lazily
};

// Integer array: only the interleaved layout is kept on the device.
struct _xmpIntegers_t {
  uint32_t *limbs;
  uint32_t precision;
  uint32_t nlimbs;
  uint32_t ngroups;
  uint32_t stride;
  uint32_t count;
  int32_t device;
  size_t bytes;
};

namespace xmpb {

// Saves the current device, switches to the handle's device, restores on exit
// (src/include/xmp_internal.h:50-53,241-253).
class DeviceGuard {
 public:
  explicit DeviceGuard(int device) {
    cudaGetDevice(&old_);
    if (old_ != device) cudaSetDevice(device);
    dev_ = device;
  }
  ~DeviceGuard() {
    if (old_ != dev_) cudaSetDevice(old_);
  }

 private:
  int old_ = 0, dev_ = 0;
};

inline xmpError_t check_cuda() { return cudaPeekAtLastError() == cudaSuccess ? xmpErrorSuccess : xmpErrorCuda; }

// Grow-only scratch; limit = policy limit or 3/4 of device memory (src/xmp.cu:105-129).
xmpError_t ensure_scratch(xmpHandle_t h, size_t bytes);
xmpError_t ensure_tmp_out(xmpHandle_t h, size_t bytes);
size_t scratch_limit(xmpHandle_t h);

// True when `p` is host memory the device cannot address directly (pageable or unknown).
bool is_host_pointer(const void *p);

inline ArrayView view_in(xmpIntegers_t x, const uint32_t *index = nullptr, uint32_t index_count = 0) {
  ArrayView v;
  v.limbs = x->limbs;
  v.nlimbs = x->nlimbs;
  v.stride = x->stride;
  v.count = x->count;
  v.index = index;
  v.index_count = index_count;
  return v;
}
inline OutView view_out(xmpIntegers_t x, uint32_t *limbs, const uint32_t *index) {
  OutView v;
  v.limbs = limbs;
  v.nlimbs = x->nlimbs;
  v.stride = x->stride;
  v.count = x->count;
  v.index = index;
  return v;
}

// In-place support: when an output aliases an input and the op reads other
// instances than the one it writes (index arrays or broadcast), the kernel
// writes into a temporary copy of the output which is copied back afterwards.
struct OutTarget {
  uint32_t *limbs = nullptr;
  bool staged = false;
};
xmpError_t begin_output(xmpHandle_t h, xmpIntegers_t out, bool aliased, bool needs_stage, OutTarget *t,
                        size_t offset = 0);
xmpError_t end_output(xmpHandle_t h, xmpIntegers_t out, const OutTarget &t);

// Releases the handle's tuner state (tables, selector weights).
void tuner_destroy(xmpHandle_t h);

inline int grid_for(uint64_t threads, int block) {
  uint64_t b = (threads + block - 1) / block;
  if (b == 0) b = 1;
  if (b > 0x7fffffffULL) b = 0x7fffffffULL;
  return (int)b;
}

}  // namespace xmpb
