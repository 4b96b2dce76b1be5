// Host-side interface of the fused CRT-RSA kernels (crt.cuh), shared by
// xmpIntegersPowmCRT and the batch plans.
#pragma once
#include "powm.h"
#include "crt.cuh"
#include <vector>

namespace xmpb {

typedef void (*CrtLauncher)(const CrtArgs &args, int grid, cudaStream_t stream);

struct CrtKernelEntry {
  int tpi;
  int limbs;
  CrtLauncher launch;
};

std::vector<CrtKernelEntry> &crt_registry();

struct CrtKernelRegistrar {
  CrtKernelRegistrar(int tpi, int limbs, CrtLauncher l) { crt_registry().push_back(CrtKernelEntry{tpi, limbs, l}); }
};

struct CrtConfig {
  int tpi = 0, limbs = 0, window = 0;
  CrtLauncher launch = nullptr;  // null: no kernel holds the precision
};

// Kernel shape (lanes x limbs) for halves of `nlimbs` limbs and the fixed window for `exp_bits`.
CrtConfig crt_config(uint32_t nlimbs, uint32_t exp_bits, uint32_t count, uint32_t sm_count);
// Scratch bytes of the window tables of one launch of `count` instances.
size_t crt_table_bytes(const CrtConfig &c, uint32_t count);
// Instances per launch whose window tables fit `limit` bytes, in whole CTAs and at most `count`
// (0: not even one CTA fits).  Capped so that a launch's thread index stays below 2^31.
uint32_t crt_chunk_for(const CrtConfig &c, size_t limit, uint32_t count);
// Launches `count` instances in chunks of at most `chunk` (a.table sized for one chunk).
void crt_launch(const CrtConfig &c, CrtArgs a, uint32_t count, uint32_t chunk, cudaStream_t s);
xmpError_t crt_validate(xmpHandle_t h, xmpIntegers_t out, xmpIntegers_t c, xmpIntegers_t p, xmpIntegers_t q,
                        xmpIntegers_t dp, xmpIntegers_t dq, xmpIntegers_t qinv, uint32_t count);
CrtArgs crt_args(xmpIntegers_t out, uint32_t *out_limbs, xmpIntegers_t c, xmpIntegers_t p, xmpIntegers_t q,
                 xmpIntegers_t dp, xmpIntegers_t dq, xmpIntegers_t qinv);

}  // namespace xmpb
