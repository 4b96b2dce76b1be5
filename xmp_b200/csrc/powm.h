// Host-side interface of the powm kernels shared by the dispatcher, the
// autotuner and the batched (mixed-size) launcher.
#pragma once
#include "internal.h"
#include "powm_kernel.cuh"
#include <vector>

namespace xmpb {

enum PowmDist : int { kDistLanes = 0, kDistDigit = 1, kDistCta = 2 };

struct PowmConfig {
  int dist = kDistLanes;  // lanes: TPI x L register kernel; digit: digit-serial kernel; cta: one instance per CTA
  int tpi = 0;            // threads per instance (1 = per-thread; cta: 0)
  int limbs = 0;          // limbs per lane (cta: limbs of the CTA's operands, 32 / 64 / 96 / 128)
  int window = 0;         // window bits
};

// CTA distribution (cta.cuh): operand size in limbs for an n-limb modulus (0: larger than 4096 bits).
uint32_t powm_cta_limbs(uint32_t nlimbs);
// Launches `count` instances from a.start, one CTA each (ct: the constant-schedule fixed window);
// false if the size or window is not supported.  No scratch: the window table is in shared memory.
bool powm_cta_launch(uint32_t limbs, bool ct, const PowmArgs &a, uint32_t count, cudaStream_t s);
// Whether a batch this small runs faster one instance per CTA than on the lane kernels.
bool powm_cta_preferred(uint32_t nlimbs, uint32_t count, uint32_t sm_count);

typedef void (*PowmLauncher)(const PowmArgs &args, int grid, cudaStream_t stream);
typedef void (*PowmBatchLauncher)(const PowmBatchArgs &args, int grid, cudaStream_t stream);

struct PowmKernelEntry {
  int tpi;
  int limbs;
  PowmLauncher launch;
  const void *fn;
  PowmBatchLauncher launch_batch;
  const void *batch_fn;
  PowmLauncher launch_r2;
  PowmLauncher launch_ct;  // constant schedule (fixed window over the exponent precision), for secret exponents
  uint32_t smem;           // dynamic shared memory per 128-thread CTA (the four-lane squaring's blocks)
};

std::vector<PowmKernelEntry> &powm_registry();
const PowmKernelEntry *powm_find(int tpi, int limbs);

struct PowmKernelRegistrar {
  PowmKernelRegistrar(int tpi, int limbs, PowmLauncher l, const void *fn, PowmBatchLauncher lb, const void *bfn,
                      PowmLauncher lr2, PowmLauncher lct, uint32_t smem) {
    powm_registry().push_back(PowmKernelEntry{tpi, limbs, l, fn, lb, bfn, lr2, lct, smem});
  }
};

// Raises a kernel's dynamic shared memory limit above the 48 KB default once (needs a current device).
template <class F>
inline void powm_smem_attr(F *fn, uint32_t bytes, bool &done) {
  if (!done && bytes > 48 * 1024) {
    cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    done = true;
  }
}

#define XMPB_REGISTER_POWM(TPI, L)                                                                   \
  static void powm_launch_##TPI##_##L(const PowmArgs &a, int grid, cudaStream_t s) {                \
    static bool attr = false;                                                                         \
    powm_smem_attr(powm_kernel<TPI, L>, powm_smem_bytes(TPI, L), attr);                              \
    powm_kernel<TPI, L><<<grid, 128, powm_smem_bytes(TPI, L), s>>>(a);                              \
  }                                                                                                   \
  static void powm_launch_batch_##TPI##_##L(const PowmBatchArgs &a, int grid, cudaStream_t s) {     \
    static bool attr = false;                                                                         \
    powm_smem_attr(powm_batch_kernel<TPI, L>, powm_smem_bytes(TPI, L), attr);                        \
    powm_batch_kernel<TPI, L><<<grid, 128, powm_smem_bytes(TPI, L), s>>>(a);                        \
  }                                                                                                   \
  static void powm_launch_r2_##TPI##_##L(const PowmArgs &a, int grid, cudaStream_t s) {             \
    r2_kernel<TPI, L><<<grid, 128, 0, s>>>(a);                                                       \
  }                                                                                                   \
  static void powm_launch_ct_##TPI##_##L(const PowmArgs &a, int grid, cudaStream_t s) {             \
    static bool attr = false;                                                                         \
    powm_smem_attr(powm_kernel<TPI, L, true>, powm_smem_bytes(TPI, L), attr);                        \
    powm_kernel<TPI, L, true><<<grid, 128, powm_smem_bytes(TPI, L), s>>>(a);                        \
  }                                                                                                   \
  static PowmKernelRegistrar powm_reg_##TPI##_##L(TPI, L, powm_launch_##TPI##_##L,                  \
                                                  (const void *)powm_kernel<TPI, L>,                 \
                                                  powm_launch_batch_##TPI##_##L,                     \
                                                  (const void *)powm_batch_kernel<TPI, L>,           \
                                                  powm_launch_r2_##TPI##_##L, powm_launch_ct_##TPI##_##L, \
                                                  powm_smem_bytes(TPI, L));

// Window bits for a k-bit exponent.  Sliding window (register kernels with
// powm_sliding): minimises the table build (2^(W-1) multiplies, weighted 5/4)
// plus one multiply per window, k/(W+1) on average.  Fixed window (the other
// register kernels, digit-serial kernel): 2^W - 2 plus k/W.  The two agree at
// every 32-bit multiple of the standard sizes (128 .. 16,384 bits).
int window_for_bits(uint32_t exp_bits, bool sliding = true);

// Heuristic configuration for n-limb moduli (used when no tuned entry exists).
// A nonzero `cap` admits only kernels with exactly cap = lanes x limbs (the
// Montgomery radix R = 2^(32 cap) of precomputed constants).
PowmConfig powm_default_config(uint32_t nlimbs, uint32_t exp_bits, uint32_t count, xmpAlgorithm_t alg,
                               uint32_t sm_count, uint32_t cap = 0);
bool powm_config_valid(const PowmConfig &c, uint32_t nlimbs);

// Runs out = base^exp mod mod for `count` op instances starting at 0 with the
// given configuration (validation already done).  Chunks the launch so the
// window tables fit the scratch limit.
xmpError_t powm_run(xmpHandle_t h, const PowmConfig &cfg, const OutView &out, const ArrayView &base,
                    const ArrayView &exp, const ArrayView &mod, uint32_t count);

// Scratch bytes one launch of `count` instances needs.
size_t powm_table_bytes(const PowmConfig &cfg, uint32_t nlimbs, uint32_t count);

// Digit-serial kernel launcher (any precision).
xmpError_t powm_digit_run(xmpHandle_t h, const PowmConfig &cfg, const OutView &out, const ArrayView &base,
                          const ArrayView &exp, const ArrayView &mod, uint32_t count);

// Configuration chosen by the handle's tuner (selector / exhaustive table), if any.
// *source (optional): 1 = a choice set for the exact shape, 2 = the selector.
bool tuner_lookup_powm(xmpHandle_t h, uint32_t nlimbs, uint32_t exp_bits, uint32_t count, PowmConfig *cfg,
                       int *source = nullptr);

}  // namespace xmpb
