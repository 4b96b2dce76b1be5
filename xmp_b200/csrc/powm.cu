// Host dispatch of xmpIntegersPowm[Async] (replaces src/powm.cu:61-307 and
// src/include/powm_operators.h:15-455).  Validation and index semantics are the
// reference's: out/base/mod precisions equal, exponent precision free, output
// index = indices[0][i], base/exp/mod = indices[1..3][i % n] % array count.
// The configuration (distribution, lanes per instance, limbs per lane, window)
// comes from the handle's tuner when it has an entry for the size class,
// otherwise from a register/occupancy heuristic; the reference's static
// Maxwell/Kepler latency tables (powm.cu:120-236) have no counterpart.
#include "powm.h"
#include "../../include/xmp_b200.h"
#include <algorithm>
#include <math.h>

using namespace xmpb;

namespace xmpb {

std::vector<PowmKernelEntry> &powm_registry() {
  static std::vector<PowmKernelEntry> r;
  return r;
}

const PowmKernelEntry *powm_find(int tpi, int limbs) {
  for (const auto &e : powm_registry())
    if (e.tpi == tpi && e.limbs == limbs) return &e;
  return nullptr;
}

int window_for_bits(uint32_t exp_bits, bool sliding) {
  if (exp_bits <= 1) return 1;
  int best = 1;
  double best_cost = 1e300;
  for (int w = 1; w <= 7; w++) {
    // sliding: the table build is weighted 5/4 (its entries are also stored; on B200 this puts the
    // 2048-bit choice on W = 6, measured 0.45% faster than W = 7, and keeps 1024 -> 6, 4096 -> 7)
    double cost = sliding ? 1.25 * (double)(1 << (w - 1)) + ceil((double)exp_bits / (w + 1))
                          : (double)((1 << w) - 2) + ceil((double)exp_bits / w);
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best = w;
    }
  }
  return best;
}

bool powm_cta_preferred(uint32_t nlimbs, uint32_t count, uint32_t sm_count) {
  const uint32_t limbs = powm_cta_limbs(nlimbs);
  // Up to 512 bits the smallest CTA (1024-bit operands) pads too much: one instance measured 0.27 /
  // 0.46 / 0.69 ms at 64 / 256 / 512 bits against 0.017 / 0.18 / 0.61 ms on the lane kernels; from
  // 544 bits on it is faster at every measured size (544: 0.72 vs 1.20 ms, 1056: 1.82 vs 2.97,
  // 1536: 2.42 vs 4.20, 2080: 5.54 vs 11.0, 3104: 13.9 vs 23.4, 4096: 17.7 vs 30.5 ms).
  if (!limbs || nlimbs <= 16) return false;
  // A CTA per instance runs it near its lone latency while the SMs hold the batch; the lane kernels
  // need thousands of instances before their throughput beats that.  Measured on B200 through
  // xmpIntegersPowm (full-length exponents), CTA vs the lane kernel at 148 / 296 / 444 / 592 / 888 /
  // 1184 instances: 768 bits -/-/-/1.12/1.36 vs 1.64/1.16 ms; 1024 bits 1.15/1.17/1.36/1.39/1.71/2.10
  // vs 2.13 ms; 1280 bits 2.90 (296), 4.81 (370) vs 3.57 ms; 1536 bits 2.43/3.37/5.60 vs 4.21 ms;
  // 1792 bits 3.84/6.37 (444) vs 7.15 ms; 2048 bits 3.08/4.30/7.15/8.57 vs 8.12 ms; 3072 bits
  // 7.84/15.7 vs 16.0 ms; 4096 bits 17.8/35.6 vs 30.6 ms.
  uint32_t per_sm = 1;
  if (limbs == 32) per_sm = nlimbs > 24 ? 6 : 4;
  else if (limbs == 64) per_sm = nlimbs > 48 ? 3 : 2;
  return count <= per_sm * sm_count;
}

bool powm_config_valid(const PowmConfig &c, uint32_t nlimbs) {
  if (c.window < 1 || c.window > 7) return false;
  if (c.dist == kDistDigit) return true;
  if (c.dist == kDistCta) return powm_cta_limbs(nlimbs) != 0 && (uint32_t)c.limbs == powm_cta_limbs(nlimbs);
  if ((uint64_t)c.tpi * c.limbs < nlimbs) return false;
  return powm_find(c.tpi, c.limbs) != nullptr;
}

PowmConfig powm_default_config(uint32_t nlimbs, uint32_t exp_bits, uint32_t count, xmpAlgorithm_t alg,
                               uint32_t sm_count, uint32_t want_cap) {
  PowmConfig best;
  if (alg == xmpAlgorithmDigitMP) {
    best.window = window_for_bits(exp_bits, false);
    best.dist = kDistDigit;
    return best;
  }
  // Enough lanes to give every SM a few warps; below that, spread instances wider.
  const double want_threads = (double)sm_count * 4 * 32;
  double best_score = 1e300;
  for (const auto &e : powm_registry()) {
    if (alg == xmpAlgorithmRegMP && e.tpi != 1) continue;
    if (alg == xmpAlgorithmDistributedMP && e.tpi == 1) continue;
    uint32_t cap = (uint32_t)e.tpi * e.limbs;
    if (cap < nlimbs || (want_cap && cap != want_cap)) continue;
    // Work per instance grows with capacity^2; lane overhead (shfl, carry
    // bookkeeping) is ~12 instructions per 4L multiply-adds.
    double pad = (double)cap / nlimbs;
    double work = pad * pad * (4.0 * e.limbs + (e.tpi > 1 ? 12.0 : 4.0)) / (4.0 * e.limbs);
    double threads = (double)count * e.tpi;
    double starve = threads < want_threads ? want_threads / threads : 1.0;
    double regs = e.limbs > 16 && e.tpi > 1 ? 1.5 : 1.0;  // register pressure beyond 16 limbs
    double score = work * starve * regs;
    if (score < best_score) {
      best_score = score;
      best.tpi = e.tpi;
      best.limbs = e.limbs;
    }
  }
  // Larger than every register kernel: the digit-serial kernel takes any size,
  // unless the caller forced a register distribution (then Unsupported).
  if (best.tpi == 0 && alg == xmpAlgorithmDefault) best.dist = kDistDigit;
  best.window = window_for_bits(exp_bits, best.dist != kDistDigit && powm_sliding(best.tpi, best.limbs));
  return best;
}

size_t powm_table_bytes(const PowmConfig &cfg, uint32_t nlimbs, uint32_t count) {
  if (cfg.dist == kDistCta) return 0;  // the table is in shared memory
  if (cfg.dist == kDistDigit) {
    // table + N, x, b, m, r, r2 working arrays, all nlimbs+2 words per instance
    size_t words = ((size_t)1 << cfg.window) * nlimbs + 6 * ((size_t)nlimbs + 2);
    return words * 4 * round_up(count, 128);
  }
  size_t threads = round_up((uint32_t)std::min<uint64_t>((uint64_t)count * cfg.tpi, 0xffffff80ull), 128);
  return threads * (size_t)cfg.limbs * powm_table_entries(cfg.window, powm_sliding(cfg.tpi, cfg.limbs)) * 4;
}

xmpError_t powm_run(xmpHandle_t h, const PowmConfig &cfg0, const OutView &out, const ArrayView &base,
                    const ArrayView &exp, const ArrayView &mod, uint32_t count) {
  PowmConfig cfg = cfg0;
  if (cfg.dist == kDistDigit) return powm_digit_run(h, cfg, out, base, exp, mod, count);
  if (cfg.dist == kDistCta) {
    PowmArgs a;
    a.base = base;
    a.exp = exp;
    a.mod = mod;
    a.out = out;
    a.start = 0;
    a.count = count;
    a.window = cfg.window;
    a.table = nullptr;
    if (!powm_cta_launch((uint32_t)cfg.limbs, false, a, count, h->stream)) return xmpErrorUnsupported;
    return check_cuda();
  }
  const PowmKernelEntry *k = powm_find(cfg.tpi, cfg.limbs);
  if (!k) return xmpErrorUnsupported;
  size_t limit = scratch_limit(h);
  // Chunk so the window tables fit; shrink the window if even one block of instances does not fit.
  uint32_t per_block = 128 / cfg.tpi;
  uint32_t chunk = count;
  while (true) {
    size_t per_inst = (size_t)cfg.tpi * cfg.limbs * powm_table_entries(cfg.window, powm_sliding(cfg.tpi, cfg.limbs)) * 4;
    uint64_t fit = limit / per_inst;
    fit = fit / per_block * per_block;
    if (fit >= per_block) {
      chunk = (uint32_t)std::min<uint64_t>(count, fit);
      break;
    }
    if (cfg.window <= 1) return xmpErrorIncreaseScratchLimit;
    cfg.window--;
  }
  xmpError_t e = ensure_scratch(h, powm_table_bytes(cfg, mod.nlimbs, chunk));
  if (e != xmpErrorSuccess) return e;
  PowmArgs a;
  a.base = base;
  a.exp = exp;
  a.mod = mod;
  a.out = out;
  a.window = cfg.window;
  a.table = (uint32_t *)h->scratch;
  for (uint32_t start = 0; start < count; start += chunk) {
    a.start = start;
    a.count = std::min(chunk, count - start);
    int grid = grid_for((uint64_t)a.count * cfg.tpi, 128);
    k->launch(a, grid, h->stream);
  }
  return check_cuda();
}

}  // namespace xmpb

// The configuration for a problem shape under the handle's policy (default algorithm): a choice set
// for the exact shape, else one instance per CTA for small batches, else the selector, else the
// heuristic.  An explicit algorithm takes the heuristic restricted to it.
static PowmConfig powm_choose_config(xmpHandle_t h, uint32_t nlimbs, uint32_t exp_bits, uint32_t count) {
  PowmConfig cfg;
  const xmpAlgorithm_t alg = h->policy->algorithm;
  int src = 0;
  const bool tuned = (alg == xmpAlgorithmDefault) && tuner_lookup_powm(h, nlimbs, exp_bits, count, &cfg, &src);
  if (tuned && src == 1) return cfg;
  if (alg == xmpAlgorithmDefault && powm_cta_preferred(nlimbs, count, h->sm_count)) {
    cfg = PowmConfig();
    cfg.dist = kDistCta;
    cfg.limbs = (int)powm_cta_limbs(nlimbs);
    cfg.window = window_for_bits(exp_bits, true);
    return cfg;
  }
  if (!tuned) cfg = powm_default_config(nlimbs, exp_bits, count, alg, h->sm_count);
  return cfg;
}

static xmpError_t powm_entry(xmpHandle_t h, xmpIntegers_t out, xmpIntegers_t base, xmpIntegers_t exp,
                             xmpIntegers_t mod, uint32_t count, const PowmConfig *forced) {
  if (!h || !out || !base || !exp || !mod) return xmpErrorInvalidParameter;
  int dev = h->device;
  if (out->device != dev || base->device != dev || exp->device != dev || mod->device != dev)
    return xmpErrorInvalidDevice;
  if (count == 0) return xmpErrorSuccess;
  DeviceGuard guard(dev);
  xmpExecutionPolicy_t p = h->policy;
  if (out->count < count) return xmpErrorInvalidCount;
  if (p->indices[0] && p->indices_count[0] < count) return xmpErrorInvalidCount;
  if (base->precision != out->precision || mod->precision != out->precision) return xmpErrorInvalidPrecision;

  PowmConfig cfg;
  if (forced) {
    cfg = *forced;
    if (cfg.dist == kDistCta) cfg.limbs = (int)powm_cta_limbs(mod->nlimbs);
  } else {
    cfg = powm_choose_config(h, mod->nlimbs, exp->precision, count);
  }
  if (!powm_config_valid(cfg, mod->nlimbs)) return xmpErrorUnsupported;

  bool aliased = (out == base || out == exp || out == mod);
  bool indexed = p->indices[0] || p->indices[1] || p->indices[2] || p->indices[3];
  OutTarget t;
  xmpError_t e = begin_output(h, out, aliased, indexed, &t);
  if (e != xmpErrorSuccess) return e;
  e = powm_run(h, cfg, view_out(out, t.limbs, p->indices[0]), view_in(base, p->indices[1], p->indices_count[1]),
               view_in(exp, p->indices[2], p->indices_count[2]), view_in(mod, p->indices[3], p->indices_count[3]),
               count);
  if (e != xmpErrorSuccess) return e;
  e = end_output(h, out, t);
  if (e != xmpErrorSuccess) return e;
  return check_cuda();
}

extern "C" {

xmpError_t XMPAPI xmpIntegersPowmAsync(xmpHandle_t h, xmpIntegers_t out, const xmpIntegers_t base,
                                        const xmpIntegers_t exp, const xmpIntegers_t mod, uint32_t count) {
  return powm_entry(h, out, base, exp, mod, count, nullptr);
}

xmpError_t XMPAPI xmpIntegersPowm(xmpHandle_t h, xmpIntegers_t out, const xmpIntegers_t base, const xmpIntegers_t exp,
                                   const xmpIntegers_t mod, uint32_t count) {
  xmpError_t e = xmpIntegersPowmAsync(h, out, base, exp, mod, count);
  if (e != xmpErrorSuccess) return e;
  DeviceGuard guard(h->device);
  cudaStreamSynchronize(h->stream);
  return check_cuda();
}

xmpError_t XMPAPI xmpIntegersPowmWithConfigAsync(xmpHandle_t h, xmpIntegers_t out, const xmpIntegers_t base,
                                                  const xmpIntegers_t exp, const xmpIntegers_t mod, uint32_t count,
                                                  const xmpPowmConfig_t *config) {
  if (!config) return xmpErrorInvalidParameter;
  PowmConfig c;
  c.dist = config->distribution;
  c.tpi = config->lanes;
  c.limbs = config->limbs;
  c.window = config->window;
  if (c.dist != kDistLanes && c.dist != kDistDigit && c.dist != kDistCta) return xmpErrorInvalidParameter;
  return powm_entry(h, out, base, exp, mod, count, &c);
}

xmpError_t XMPAPI xmpPowmKernelCount(int32_t *count) {
  if (!count) return xmpErrorInvalidParameter;
  *count = (int32_t)powm_registry().size();
  return xmpErrorSuccess;
}

xmpError_t XMPAPI xmpPowmKernelGet(int32_t index, int32_t *lanes, int32_t *limbs) {
  if (index < 0 || index >= (int32_t)powm_registry().size() || !lanes || !limbs) return xmpErrorInvalidParameter;
  *lanes = powm_registry()[index].tpi;
  *limbs = powm_registry()[index].limbs;
  return xmpErrorSuccess;
}

xmpError_t XMPAPI xmpPowmGetConfig(xmpHandle_t h, uint32_t precision, uint32_t exp_precision, uint32_t count,
                                   xmpPowmConfig_t *config) {
  if (!h || !config || precision == 0 || precision % 32 || exp_precision == 0 || exp_precision % 32)
    return xmpErrorInvalidParameter;
  const PowmConfig c = powm_choose_config(h, precision / 32, exp_precision, count);
  config->distribution = c.dist;
  config->lanes = c.tpi;
  config->limbs = c.limbs;
  config->window = c.window;
  return xmpErrorSuccess;
}

}  // extern "C"
