/*
 * xmp.h -- C API of the B200-native batched multi-precision integer library.
 *
 * This header declares the same 54 entry points, types and error codes as the
 * reference library's public header (src/include/xmp.h:40-226), so code written
 * against the reference links against libxmp.so from this project unchanged.
 * Differences from the reference header, all source compatible:
 *   - the header is valid C as well as C++: the C++ constructors of
 *     xmpExecutionPolicyValue_t (xmp.h:72-73) are only declared under
 *     __cplusplus, and xmpExecutionPolicyGetParameter takes its value argument
 *     by reference in C++ (xmp.h:152) and by pointer in C (the same ABI);
 *   - xmpHandleSetCudaStream / xmpHandleGetCudaStream (xmp.h:135,138) are
 *     declared by the reference but never defined there; here they are defined
 *     as aliases of xmpHandleSetStream / xmpHandleGetStream.
 *
 * Integer semantics (reference docs and kernels, implementations.h:36-1081):
 *   - integers are unsigned, precision is a multiple of 32 bits;
 *   - every op processes `count` instances; input instance i reads element
 *     index[i % index_count] % array_count of each input when the execution
 *     policy holds an index array for it, else element i % array_count;
 *     output instance i writes element out_index[i] (or i);
 *   - results wrap modulo 2^(output precision);
 *   - in-place operation (an output aliasing an input) is allowed;
 *   - every *Async call only enqueues work on the handle's stream; the
 *     synchronous forms also wait for the stream.
 */
#ifndef XMP_B200_XMP_H
#define XMP_B200_XMP_H

#include <stdint.h>
#include <stddef.h>
#include <cuda_runtime_api.h>

#if defined(_WIN32) || defined(_WIN64)
#define XMPAPI __declspec(dllexport) __stdcall
#else
#define XMPAPI __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes: same names, order and values as src/include/xmp.h:40-54. */
typedef enum {
  xmpErrorSuccess,
  xmpErrorInvalidDispatchTable,
  xmpErrorInvalidParameter,
  xmpErrorInvalidMalloc,
  xmpErrorInvalidCudaMalloc,
  xmpErrorInvalidCount,
  xmpErrorInvalidDevice,
  xmpErrorInvalidFormat,
  xmpErrorInvalidPrecision,
  xmpErrorIncreaseScratchLimit,
  xmpErrorUnsupported,
  xmpErrorUnspecified,
  xmpErrorCuda
} xmpError_t;

/* Execution policy parameters (src/include/xmp.h:57-60). */
typedef enum {
  xmpAlgorithm,
  xmpScratchSizeLimit
} xmpExecutionPolicyParam_t;

/* Algorithm override (src/include/xmp.h:62-67).  Here RegMP selects the
 * per-thread register distribution, DistributedMP the warp-distributed one
 * and DigitMP the digit-serial (memory-streamed) one. */
typedef enum {
  xmpAlgorithmDefault,
  xmpAlgorithmRegMP,
  xmpAlgorithmDigitMP,
  xmpAlgorithmDistributedMP
} xmpAlgorithm_t;

/* 8-byte value passed by value (src/include/xmp.h:69-74). */
#ifdef __cplusplus
union xmpExecutionPolicyValue_t {
  xmpAlgorithm_t algorithm;
  size_t size;
  xmpExecutionPolicyValue_t() { size = 0; }
  xmpExecutionPolicyValue_t(xmpAlgorithm_t a) { size = 0; algorithm = a; }
  xmpExecutionPolicyValue_t(size_t s) { size = s; }
};
#define XMP_VALUE_OUT(v) xmpExecutionPolicyValue_t &v
#else
typedef union xmpExecutionPolicyValue_t {
  xmpAlgorithm_t algorithm;
  size_t size;
} xmpExecutionPolicyValue_t;
#define XMP_VALUE_OUT(v) xmpExecutionPolicyValue_t *v
#endif

/* Same strings as src/include/xmp.h:76-108. */
static inline const char *xmpGetErrorString(xmpError_t error) {
  switch (error) {
    case xmpErrorSuccess: return "xmpErrorSuccess";
    case xmpErrorInvalidDispatchTable: return "xmpErrorInvalidDispatchTable";
    case xmpErrorInvalidParameter: return "xmpErrorInvalidParameter";
    case xmpErrorInvalidMalloc: return "xmpErrorInvalidMalloc";
    case xmpErrorInvalidCudaMalloc: return "xmpErrorInvalidCudaMalloc";
    case xmpErrorInvalidCount: return "xmpErrorInvalidCount";
    case xmpErrorInvalidDevice: return "xmpErrorInvalidDevice";
    case xmpErrorInvalidFormat: return "xmpErrorInvalidFormat";
    case xmpErrorInvalidPrecision: return "xmpErrorPrecision";
    case xmpErrorIncreaseScratchLimit: return "xmpIncreaseScratchLimit";
    case xmpErrorUnsupported: return "xmpErrorUnsupported";
    case xmpErrorUnspecified: return "xmpErrorUnspecified";
    case xmpErrorCuda: return "xmpErrorCuda";
    default: return "xmpErrorUnknown";
  }
}

typedef struct _xmpHandle_t *xmpHandle_t;
typedef struct _xmpIntegers_t *xmpIntegers_t;
typedef struct _xmpExecutionPolicy_t *xmpExecutionPolicy_t;

typedef void *(*xmpAllocFunc)(size_t);
typedef void (*xmpFreeFunc)(void *);

/* ---- handle (replaces src/xmp.cu:39-191) ---------------------------------- */
xmpError_t XMPAPI xmpHandleCreate(xmpHandle_t *handle);
xmpError_t XMPAPI xmpHandleCreateWithMemoryFunctions(xmpHandle_t *handle, xmpAllocFunc ha, xmpFreeFunc hf,
                                                      xmpAllocFunc da, xmpFreeFunc df);
xmpError_t XMPAPI xmpHandleDestroy(xmpHandle_t handle);
xmpError_t XMPAPI xmpHandleSetStream(xmpHandle_t handle, cudaStream_t stream);
xmpError_t XMPAPI xmpHandleGetStream(xmpHandle_t handle, cudaStream_t *stream);
xmpError_t XMPAPI xmpHandleSetExecutionPolicy(xmpHandle_t handle, xmpExecutionPolicy_t policy);
xmpError_t XMPAPI xmpHandleGetMemoryFunctions(xmpHandle_t handle, xmpAllocFunc *ha, xmpFreeFunc *hf,
                                               xmpAllocFunc *da, xmpFreeFunc *df);
xmpError_t XMPAPI xmpHandleSetCudaStream(xmpHandle_t handle, cudaStream_t stream);
xmpError_t XMPAPI xmpHandleGetCudaStream(xmpHandle_t handle, cudaStream_t *stream);
xmpError_t XMPAPI xmpHandleGetDevice(xmpHandle_t handle, int32_t *device);

/* ---- execution policy (replaces src/xmp.cu:193-314) ------------------------ */
xmpError_t XMPAPI xmpExecutionPolicyCreate(xmpHandle_t handle, xmpExecutionPolicy_t *policy);
xmpError_t XMPAPI xmpExecutionPolicyDestroy(xmpHandle_t handle, xmpExecutionPolicy_t policy);
xmpError_t XMPAPI xmpExecutionPolicySetIndices(xmpHandle_t handle, xmpExecutionPolicy_t policy, uint32_t which_integer,
                                                uint32_t *indices, uint32_t count);
xmpError_t XMPAPI xmpExecutionPolicySetIndicesAsync(xmpHandle_t handle, xmpExecutionPolicy_t policy,
                                                     uint32_t which_integer, uint32_t *indices, uint32_t count);
xmpError_t XMPAPI xmpExecutionPolicySetParameter(xmpHandle_t handle, xmpExecutionPolicy_t policy,
                                                  xmpExecutionPolicyParam_t param, xmpExecutionPolicyValue_t val);
xmpError_t XMPAPI xmpExecutionPolicyGetParameter(xmpHandle_t handle, xmpExecutionPolicy_t policy,
                                                  xmpExecutionPolicyParam_t param, XMP_VALUE_OUT(val));

/* ---- integer arrays (replaces src/xmp.cu:317-813) -------------------------- */
xmpError_t XMPAPI xmpIntegersCreate(xmpHandle_t handle, xmpIntegers_t *x, uint32_t precision, uint32_t count);
xmpError_t XMPAPI xmpIntegersDestroy(xmpHandle_t handle, xmpIntegers_t x);
xmpError_t XMPAPI xmpIntegersGetPrecision(xmpHandle_t handle, xmpIntegers_t x, uint32_t *precision);
xmpError_t XMPAPI xmpIntegersGetCount(xmpHandle_t handle, xmpIntegers_t x, uint32_t *count);
xmpError_t XMPAPI xmpIntegersImport(xmpHandle_t handle, xmpIntegers_t out, uint32_t words, int32_t order, size_t size,
                                     int32_t endian, uint32_t nails, void *in, uint32_t count);
xmpError_t XMPAPI xmpIntegersImportAsync(xmpHandle_t handle, xmpIntegers_t out, uint32_t words, int32_t order,
                                          size_t size, int32_t endian, uint32_t nails, void *in, uint32_t count);
xmpError_t XMPAPI xmpIntegersExport(xmpHandle_t handle, void *out, uint32_t *words, int32_t order, size_t size,
                                     int32_t endian, uint32_t nails, xmpIntegers_t in, uint32_t count);
xmpError_t XMPAPI xmpIntegersExportAsync(xmpHandle_t handle, void *out, uint32_t *words, int32_t order, size_t size,
                                          int32_t endian, uint32_t nails, xmpIntegers_t in, uint32_t count);
xmpError_t XMPAPI xmpIntegersSet(xmpHandle_t handle, xmpIntegers_t out, xmpIntegers_t in, uint32_t count);
xmpError_t XMPAPI xmpIntegersSetAsync(xmpHandle_t handle, xmpIntegers_t out, xmpIntegers_t in, uint32_t count);

/* ---- arithmetic (replaces src/add_sub.cu, mul.cu, div.cu, powm.cu) --------- */
xmpError_t XMPAPI xmpIntegersAdd(xmpHandle_t handle, xmpIntegers_t s, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count);
xmpError_t XMPAPI xmpIntegersAddAsync(xmpHandle_t handle, xmpIntegers_t s, const xmpIntegers_t a,
                                       const xmpIntegers_t b, uint32_t count);
xmpError_t XMPAPI xmpIntegersSub(xmpHandle_t handle, xmpIntegers_t d, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count);
xmpError_t XMPAPI xmpIntegersSubAsync(xmpHandle_t handle, xmpIntegers_t d, const xmpIntegers_t a,
                                       const xmpIntegers_t b, uint32_t count);
xmpError_t XMPAPI xmpIntegersMul(xmpHandle_t handle, xmpIntegers_t p, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count);
xmpError_t XMPAPI xmpIntegersMulAsync(xmpHandle_t handle, xmpIntegers_t p, const xmpIntegers_t a,
                                       const xmpIntegers_t b, uint32_t count);
xmpError_t XMPAPI xmpIntegersDiv(xmpHandle_t handle, xmpIntegers_t q, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count);
xmpError_t XMPAPI xmpIntegersDivAsync(xmpHandle_t handle, xmpIntegers_t q, const xmpIntegers_t a,
                                       const xmpIntegers_t b, uint32_t count);
xmpError_t XMPAPI xmpIntegersMod(xmpHandle_t handle, xmpIntegers_t m, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count);
xmpError_t XMPAPI xmpIntegersModAsync(xmpHandle_t handle, xmpIntegers_t m, const xmpIntegers_t a,
                                       const xmpIntegers_t b, uint32_t count);
xmpError_t XMPAPI xmpIntegersDivMod(xmpHandle_t handle, xmpIntegers_t q, xmpIntegers_t m, const xmpIntegers_t a,
                                     const xmpIntegers_t b, uint32_t count);
xmpError_t XMPAPI xmpIntegersDivModAsync(xmpHandle_t handle, xmpIntegers_t q, xmpIntegers_t m, const xmpIntegers_t a,
                                          const xmpIntegers_t b, uint32_t count);
xmpError_t XMPAPI xmpIntegersPowm(xmpHandle_t handle, xmpIntegers_t out, const xmpIntegers_t base,
                                   const xmpIntegers_t exp, const xmpIntegers_t mod, uint32_t count);
xmpError_t XMPAPI xmpIntegersPowmAsync(xmpHandle_t handle, xmpIntegers_t out, const xmpIntegers_t base,
                                        const xmpIntegers_t exp, const xmpIntegers_t mod, uint32_t count);

/* Allocation-free modular exponentiation (no counterpart in the reference).
 * For callers that cannot allocate device memory: a latency-critical path
 * where cudaMalloc/cudaFree would synchronise the device, or a process whose
 * device memory belongs to another allocator that only hands out the operand
 * buffers.  out[i] = base[i]^exp[i] mod mod[i] for i < count, enqueued on
 * `stream` of the current device; no handle, no cudaMalloc/cudaFree.
 * Operands are device pointers (16-byte aligned) in this library's device
 * layout: limb j of instance i at uint32 offset ((j/4)*stride + i)*4 + j%4,
 * stride >= count; base/mod/out have `precision` bits, exp `exp_precision`
 * bits (multiples of 32); moduli odd; out may alias an input.  Limbs move in
 * whole groups of four, so each buffer must hold ceil(bits/128)*stride*16
 * bytes (bits = precision, or exp_precision for exp); the padding limbs of
 * the last group are read as zero and written as zero.
 * Window tables live in a fixed 16 MiB device array that every GPU loading the
 * library holds until exit; batches whose tables do not fit even with the
 * smallest window return xmpErrorIncreaseScratchLimit (split the batch), and
 * precisions above 16,384 bits return xmpErrorUnsupported.  All calls share
 * that array: calls that overlap on the GPU race, so serialise them.  The
 * first call in each CUDA context looks up the array's device address; make
 * it before any stream capture. */
xmpError_t XMPAPI xmpIntegersPowmNoAlloc(cudaStream_t stream, uint32_t *out, const uint32_t *base,
                                          const uint32_t *exp, const uint32_t *mod, uint32_t precision,
                                          uint32_t exp_precision, uint32_t stride, uint32_t count);

/* ---- bitwise (replaces src/logic.cu) ---------------------------------------- */
xmpError_t XMPAPI xmpIntegersShf(xmpHandle_t handle, xmpIntegers_t c, const xmpIntegers_t a, const int32_t *shift,
                                  const uint32_t shift_count, uint32_t count);
xmpError_t XMPAPI xmpIntegersShfAsync(xmpHandle_t handle, xmpIntegers_t c, const xmpIntegers_t a,
                                       const int32_t *shift, const uint32_t shift_count, uint32_t count);
xmpError_t XMPAPI xmpIntegersIor(xmpHandle_t handle, xmpIntegers_t c, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count);
xmpError_t XMPAPI xmpIntegersIorAsync(xmpHandle_t handle, xmpIntegers_t c, const xmpIntegers_t a,
                                       const xmpIntegers_t b, uint32_t count);
xmpError_t XMPAPI xmpIntegersAnd(xmpHandle_t handle, xmpIntegers_t c, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count);
xmpError_t XMPAPI xmpIntegersAndAsync(xmpHandle_t handle, xmpIntegers_t c, const xmpIntegers_t a,
                                       const xmpIntegers_t b, uint32_t count);
xmpError_t XMPAPI xmpIntegersXor(xmpHandle_t handle, xmpIntegers_t c, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count);
xmpError_t XMPAPI xmpIntegersXorAsync(xmpHandle_t handle, xmpIntegers_t c, const xmpIntegers_t a,
                                       const xmpIntegers_t b, uint32_t count);
xmpError_t XMPAPI xmpIntegersNot(xmpHandle_t handle, xmpIntegers_t c, const xmpIntegers_t a, uint32_t count);
xmpError_t XMPAPI xmpIntegersNotAsync(xmpHandle_t handle, xmpIntegers_t c, const xmpIntegers_t a, uint32_t count);
xmpError_t XMPAPI xmpIntegersPopc(xmpHandle_t handle, uint32_t *c, const xmpIntegers_t a, uint32_t count);
xmpError_t XMPAPI xmpIntegersPopcAsync(xmpHandle_t handle, uint32_t *c, const xmpIntegers_t a, uint32_t count);
xmpError_t XMPAPI xmpIntegersCmp(xmpHandle_t handle, int32_t *c, const xmpIntegers_t a, const xmpIntegers_t b,
                                  uint32_t count);
xmpError_t XMPAPI xmpIntegersCmpAsync(xmpHandle_t handle, int32_t *c, const xmpIntegers_t a, const xmpIntegers_t b,
                                       uint32_t count);

#ifdef __cplusplus
}
#endif

#endif /* XMP_B200_XMP_H */
