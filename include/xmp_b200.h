/*
 * xmp_b200.h -- extensions of the B200-native library beyond the reference API.
 *
 * None of these entry points has a counterpart in the reference's public
 * header; they replace its offline tuning step (src/tune/tune.cu writing the
 * static tables src/tune/tune_*.h that src/powm.cu:120-236 reads) with a
 * runtime autotuner, and expose the kernel configurations it chooses among.
 * All are C ABI, plain pointers and sizes.
 */
#ifndef XMP_B200_EXT_H
#define XMP_B200_EXT_H

#include "xmp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One powm kernel configuration.
 *   distribution: 0 = register kernel with `lanes` threads per instance and
 *                 `limbs` 32-bit limbs per thread (lanes = 1 is the per-thread
 *                 distribution), 1 = digit-serial (lanes/limbs ignored);
 *   window:       fixed-window exponent bits, 1..7. */
typedef struct {
  int32_t distribution;
  int32_t lanes;
  int32_t limbs;
  int32_t window;
} xmpPowmConfig_t;

/* Number of register kernels compiled into the library, and the i-th one's shape. */
xmpError_t XMPAPI xmpPowmKernelCount(int32_t *count);
xmpError_t XMPAPI xmpPowmKernelGet(int32_t index, int32_t *lanes, int32_t *limbs);

/* The configuration xmpIntegersPowm would use now for this problem shape
 * (tuned entry if the handle's tuner has one, else the built-in heuristic). */
xmpError_t XMPAPI xmpPowmGetConfig(xmpHandle_t handle, uint32_t precision, uint32_t exp_precision, uint32_t count,
                                   xmpPowmConfig_t *config);

/* xmpIntegersPowmAsync with an explicit configuration (same validation, index
 * policy and semantics); xmpErrorUnsupported if the configuration cannot hold
 * the modulus precision. */
xmpError_t XMPAPI xmpIntegersPowmWithConfigAsync(xmpHandle_t handle, xmpIntegers_t out, const xmpIntegers_t base,
                                                  const xmpIntegers_t exp, const xmpIntegers_t mod, uint32_t count,
                                                  const xmpPowmConfig_t *config);

#ifdef __cplusplus
}
#endif

#endif /* XMP_B200_EXT_H */
