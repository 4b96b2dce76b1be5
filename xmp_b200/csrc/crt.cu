// Host side of the fused CRT-RSA operation (crt.cuh): kernel registry, the
// configuration rule, and xmpIntegersPowmCRT[Async] (declared in
// include/xmp_b200.h; no counterpart in the reference library).
#include "crt.h"
#include "../../include/xmp_b200.h"
#include <algorithm>
#include <vector>

namespace xmpb {

std::vector<CrtKernelEntry> &crt_registry() {
  static std::vector<CrtKernelEntry> r;
  return r;
}

#define XMPB_REGISTER_CRT(TPI, L)                                                                 \
  static void crt_launch_##TPI##_##L(const CrtArgs &a, int grid, cudaStream_t s) {               \
    static bool attr = false;                                                                     \
    powm_smem_attr(crt_kernel<TPI, L>, powm_smem_bytes(TPI, L), attr);                            \
    crt_kernel<TPI, L><<<grid, 128, powm_smem_bytes(TPI, L), s>>>(a);                             \
  }                                                                                               \
  static CrtKernelRegistrar crt_reg_##TPI##_##L(TPI, L, crt_launch_##TPI##_##L);

// Shapes for halves of 256 to 4096 bits (RSA-512 to RSA-8192): two per size.
XMPB_REGISTER_CRT(4, 2)
XMPB_REGISTER_CRT(8, 1)
XMPB_REGISTER_CRT(4, 4)
XMPB_REGISTER_CRT(8, 2)
XMPB_REGISTER_CRT(4, 6)
XMPB_REGISTER_CRT(8, 3)
XMPB_REGISTER_CRT(4, 8)
XMPB_REGISTER_CRT(8, 4)
XMPB_REGISTER_CRT(4, 12)
XMPB_REGISTER_CRT(8, 6)
XMPB_REGISTER_CRT(4, 16)
XMPB_REGISTER_CRT(8, 8)
XMPB_REGISTER_CRT(8, 12)
XMPB_REGISTER_CRT(16, 6)
XMPB_REGISTER_CRT(8, 16)
XMPB_REGISTER_CRT(16, 8)

CrtConfig crt_config(uint32_t nlimbs, uint32_t exp_bits, uint32_t count, uint32_t sm_count) {
  CrtConfig best;
  double best_score = 1e300;
  const double want_threads = (double)sm_count * 4 * 32;
  for (const auto &e : crt_registry()) {
    const uint32_t cap = (uint32_t)(e.tpi * e.limbs);
    if (cap < nlimbs) continue;
    // the powm heuristic's cost model: padding squared, lane overhead, starved SMs below 4 warps each
    const double pad = (double)cap / nlimbs;
    const double work = pad * pad * (4.0 * e.limbs + 12.0) / (4.0 * e.limbs);
    const double threads = (double)count * e.tpi * 2;  // a pair of groups per instance
    const double starve = threads < want_threads ? want_threads / threads : 1.0;
    const double score = work * starve;
    if (score < best_score) {
      best_score = score;
      best.tpi = e.tpi;
      best.limbs = e.limbs;
      best.launch = e.launch;
    }
  }
  best.window = window_for_bits(exp_bits, false);
  return best;
}

size_t crt_table_bytes(const CrtConfig &c, uint32_t count) {
  const size_t threads = round_up((uint32_t)std::min<uint64_t>((uint64_t)count * c.tpi * 2, 0xffffff80ull), 128);
  return threads * (size_t)c.limbs * ((size_t)1 << c.window) * 4;
}

uint32_t crt_chunk_for(const CrtConfig &c, size_t limit, uint32_t count) {
  const uint32_t per_block = 128 / (2 * c.tpi);  // a pair of groups per instance
  const size_t per_inst = (size_t)2 * c.tpi * c.limbs * ((size_t)1 << c.window) * 4;
  const uint64_t fit = std::min<uint64_t>(limit / per_inst, (1ull << 31) / (2 * c.tpi)) / per_block * per_block;
  return fit < per_block ? 0u : (uint32_t)std::min<uint64_t>(count, fit);
}

void crt_launch(const CrtConfig &c, CrtArgs a, uint32_t count, uint32_t chunk, cudaStream_t s) {
  for (uint32_t start = 0; start < count; start += chunk) {
    a.start = start;
    a.count = std::min(chunk, count - start);
    c.launch(a, grid_for((uint64_t)a.count * c.tpi * 2, 128), s);
  }
}

xmpError_t crt_validate(xmpHandle_t h, xmpIntegers_t out, xmpIntegers_t c, xmpIntegers_t p, xmpIntegers_t q,
                        xmpIntegers_t dp, xmpIntegers_t dq, xmpIntegers_t qinv, uint32_t count) {
  if (!h || !out || !c || !p || !q || !dp || !dq || !qinv) return xmpErrorInvalidParameter;
  for (xmpIntegers_t x : {out, c, p, q, dp, dq, qinv})
    if (x->device != h->device) return xmpErrorInvalidDevice;
  if (out->count < count) return xmpErrorInvalidCount;
  const uint32_t hb = p->precision;
  if (q->precision != hb || qinv->precision != hb || out->precision != 2 * hb || c->precision > 2 * hb)
    return xmpErrorInvalidPrecision;
  return xmpErrorSuccess;
}

CrtArgs crt_args(xmpIntegers_t out, uint32_t *out_limbs, xmpIntegers_t c, xmpIntegers_t p, xmpIntegers_t q,
                 xmpIntegers_t dp, xmpIntegers_t dq, xmpIntegers_t qinv) {
  CrtArgs a;
  a.c = view_in(c);
  a.p = view_in(p);
  a.q = view_in(q);
  a.dp = view_in(dp);
  a.dq = view_in(dq);
  a.qinv = view_in(qinv);
  a.out = view_out(out, out_limbs, nullptr);
  a.start = 0;
  a.count = 0;
  a.window = 0;
  a.table = nullptr;
  return a;
}

}  // namespace xmpb

using namespace xmpb;

extern "C" {

xmpError_t XMPAPI xmpIntegersPowmCRTAsync(xmpHandle_t h, xmpIntegers_t out, const xmpIntegers_t c,
                                          const xmpIntegers_t p, const xmpIntegers_t q, const xmpIntegers_t dp,
                                          const xmpIntegers_t dq, const xmpIntegers_t qinv, uint32_t count) {
  xmpError_t e = crt_validate(h, out, c, p, q, dp, dq, qinv, count);
  if (e != xmpErrorSuccess) return e;
  if (count == 0) return xmpErrorSuccess;
  DeviceGuard guard(h->device);
  CrtConfig cfg = crt_config(p->nlimbs, std::max(dp->precision, dq->precision), count, h->sm_count);
  if (!cfg.launch) return xmpErrorUnsupported;
  // chunk so the window tables fit the scratch limit; shrink the window when one block does not fit
  const size_t limit = scratch_limit(h);
  uint32_t chunk;
  while ((chunk = crt_chunk_for(cfg, limit, count)) == 0) {
    if (cfg.window <= 1) return xmpErrorIncreaseScratchLimit;
    cfg.window--;
  }
  // an output that is also an input is written through the handle's temporary output buffer
  const bool aliased = (out == c || out == p || out == q || out == dp || out == dq || out == qinv);
  OutTarget t;
  if ((e = begin_output(h, out, aliased, aliased, &t)) != xmpErrorSuccess) return e;
  if ((e = ensure_scratch(h, crt_table_bytes(cfg, chunk))) != xmpErrorSuccess) return e;
  CrtArgs a = crt_args(out, t.limbs, c, p, q, dp, dq, qinv);
  a.window = (uint32_t)cfg.window;
  a.table = (uint32_t *)h->scratch;
  crt_launch(cfg, a, count, chunk, h->stream);
  if ((e = check_cuda()) != xmpErrorSuccess) return e;
  return end_output(h, out, t);
}

xmpError_t XMPAPI xmpIntegersPowmCRT(xmpHandle_t h, xmpIntegers_t out, const xmpIntegers_t c, const xmpIntegers_t p,
                                     const xmpIntegers_t q, const xmpIntegers_t dp, const xmpIntegers_t dq,
                                     const xmpIntegers_t qinv, uint32_t count) {
  xmpError_t e = xmpIntegersPowmCRTAsync(h, out, c, p, q, dp, dq, qinv, count);
  if (e != xmpErrorSuccess) return e;
  DeviceGuard guard(h->device);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return xmpErrorCuda;
  return check_cuda();
}

}  // extern "C"
