// Launchers of the CTA distribution (cta.cuh): one exponentiation per CTA, for
// small batches where a lone instance's latency sets the time.
#include "powm.h"
#include "cta.cuh"
#include <algorithm>

namespace xmpb {

template <int N, bool CT>
static void cta_launch(const PowmArgs &a, uint32_t count, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    // room for the largest window table (W = 7) once
    cudaFuncSetAttribute((const void *)powm_cta_kernel<N, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)cta_smem_bytes<N>(powm_table_entries(7, !CT)));
    attr = true;
  }
  const uint32_t bytes = cta_smem_bytes<N>(powm_table_entries(a.window, !CT));
  PowmArgs b = a;
  for (uint32_t start = 0; start < count; start += (1u << 30)) {
    b.start = a.start + start;
    b.count = std::min(count - start, 1u << 30);
    powm_cta_kernel<N, CT><<<b.count, CtaShape<N>::THREADS, bytes, s>>>(b);
  }
}

uint32_t powm_cta_limbs(uint32_t nlimbs) {
  for (uint32_t n : {32u, 64u, 96u, 128u})
    if (nlimbs <= n) return n;
  return 0;
}

bool powm_cta_launch(uint32_t limbs, bool ct, const PowmArgs &a, uint32_t count, cudaStream_t s) {
  if (a.window < 1 || a.window > 7) return false;
  switch (limbs) {
    case 32: ct ? cta_launch<32, true>(a, count, s) : cta_launch<32, false>(a, count, s); return true;
    case 64: ct ? cta_launch<64, true>(a, count, s) : cta_launch<64, false>(a, count, s); return true;
    case 96: ct ? cta_launch<96, true>(a, count, s) : cta_launch<96, false>(a, count, s); return true;
    case 128: ct ? cta_launch<128, true>(a, count, s) : cta_launch<128, false>(a, count, s); return true;
    default: return false;
  }
}

}  // namespace xmpb
