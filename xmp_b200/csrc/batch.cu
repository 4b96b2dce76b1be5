// Batched modular exponentiation over mixed precisions (no counterpart in the
// reference, whose xmpIntegersPowm handles one precision per call through a
// host chunk loop, src/powm.cu:250-307).
//
// A plan bins plain instances by modulus precision.  Each bin is one
// persistent powm_batch_kernel launch: a full grid whose warps pull work items
// from an atomic queue spanning up to kPowmSegs segments (arrays of the same
// precision).  CRT-RSA items run as one fused crt_kernel launch each (c mod p
// and mod q, both half exponentiations and Garner's recombination in one
// kernel, no temporaries; crt.cuh).  Bins and CRT launches are forked onto
// side streams and joined back, so all of them run concurrently.  Everything
// is sized and allocated at plan creation, so the execution can be captured
// into one CUDA graph and replayed.
#include "tune.h"
#include "crt.h"
#include <algorithm>
#include <vector>

using namespace xmpb;

namespace xmpb {

struct BatchSegment {
  xmpIntegers_t out, base, exp, mod;
  uint32_t count;
};

struct BatchBin {
  uint32_t nlimbs = 0, exp_bits = 0, count = 0;
  std::vector<BatchSegment> segs;
  PowmConfig cfg;
  const PowmKernelEntry *k = nullptr;
  int blocks = 0;
  bool serial = false;  // digit-serial fallback, run after the join
  size_t table_offset = 0;
};

struct CrtLaunch {
  xmpPowmCRTItem_t item;
  CrtConfig cfg;
  uint32_t chunk = 0;
  size_t table_offset = 0;
};

}  // namespace xmpb

struct _xmpPowmBatchPlan_t {
  std::vector<BatchBin> bins;
  std::vector<CrtLaunch> crt;
  void *scratch = nullptr;
  size_t scratch_bytes = 0;
  uint32_t *counters = nullptr;
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr;
  cudaStream_t capture = nullptr;
  bool use_graph = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace xmpb {

static void free_plan(xmpHandle_t h, xmpPowmBatchPlan_t p) {
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->scratch) h->df(p->scratch);
  for (auto s : p->side) cudaStreamDestroy(s);
  for (auto e : p->joins) cudaEventDestroy(e);
  if (p->fork) cudaEventDestroy(p->fork);
  if (p->capture) cudaStreamDestroy(p->capture);
  delete p;
}

static PowmArgs seg_args(const BatchSegment &s) {
  PowmArgs a;
  a.base = view_in(s.base);
  a.exp = view_in(s.exp);
  a.mod = view_in(s.mod);
  a.out = view_out(s.out, s.out->limbs, nullptr);
  a.start = 0;
  a.count = s.count;
  a.window = 0;
  a.table = nullptr;
  return a;
}

static xmpError_t launch_bin(xmpHandle_t h, xmpPowmBatchPlan_t p, int b, cudaStream_t stream) {
  BatchBin &bin = p->bins[b];
  PowmBatchArgs a;
  a.nseg = (uint32_t)bin.segs.size();
  a.window = (uint32_t)bin.cfg.window;
  a.table = (uint32_t *)((char *)p->scratch + bin.table_offset);
  a.counter = p->counters + b;
  const uint32_t per_item = 32 / bin.cfg.tpi;
  uint32_t items = 0;
  for (uint32_t s = 0; s < a.nseg; s++) {
    a.seg[s] = seg_args(bin.segs[s]);
    a.item_start[s] = items;
    items += div_up(bin.segs[s].count, per_item);
  }
  a.item_start[a.nseg] = items;
  a.items = items;
  bin.k->launch_batch(a, bin.blocks, stream);
  return check_cuda();
}

// One execution on `main` (the handle's stream, or the capture stream).
static xmpError_t enqueue(xmpHandle_t h, xmpPowmBatchPlan_t p, cudaStream_t main) {
  cudaStream_t saved_stream = h->stream;
  xmpExecutionPolicy_t saved_policy = h->policy;
  h->stream = main;
  h->policy = &h->default_policy;
  xmpError_t e = xmpErrorSuccess;
  auto run = [&]() -> xmpError_t {
    xmpError_t r;
    if (cudaMemsetAsync(p->counters, 0, p->bins.size() * sizeof(uint32_t), main) != cudaSuccess) return xmpErrorCuda;
    if (cudaEventRecord(p->fork, main) != cudaSuccess) return xmpErrorCuda;
    // every bin and every CRT item on its own stream, in launch order (longest instances first)
    int side = 0;
    for (size_t b = 0; b < p->bins.size(); b++) {
      if (p->bins[b].serial) continue;
      cudaStream_t s = p->side[side];
      if (cudaStreamWaitEvent(s, p->fork, 0) != cudaSuccess) return xmpErrorCuda;
      if ((r = launch_bin(h, p, (int)b, s))) return r;
      if (cudaEventRecord(p->joins[side], s) != cudaSuccess) return xmpErrorCuda;
      side++;
    }
    for (const CrtLaunch &c : p->crt) {
      cudaStream_t s = p->side[side];
      if (cudaStreamWaitEvent(s, p->fork, 0) != cudaSuccess) return xmpErrorCuda;
      const xmpPowmCRTItem_t &it = c.item;
      CrtArgs a = crt_args(it.out, it.out->limbs, it.c, it.p, it.q, it.dp, it.dq, it.qinv);
      a.window = (uint32_t)c.cfg.window;
      a.table = (uint32_t *)((char *)p->scratch + c.table_offset);
      crt_launch(c.cfg, a, it.count, c.chunk, s);
      if ((r = check_cuda())) return r;
      if (cudaEventRecord(p->joins[side], s) != cudaSuccess) return xmpErrorCuda;
      side++;
    }
    for (int j = 0; j < side; j++)
      if (cudaStreamWaitEvent(main, p->joins[j], 0) != cudaSuccess) return xmpErrorCuda;
    // bins without a register kernel (precisions above 16,384 bits) run digit-serially after the join
    for (size_t b = 0; b < p->bins.size(); b++) {
      if (!p->bins[b].serial) continue;
      for (const BatchSegment &s : p->bins[b].segs) {
        PowmArgs a = seg_args(s);
        if ((r = powm_digit_run(h, p->bins[b].cfg, a.out, a.base, a.exp, a.mod, s.count))) return r;
      }
    }
    return check_cuda();
  };
  e = run();
  h->stream = saved_stream;
  h->policy = saved_policy;
  return e;
}

}  // namespace xmpb

extern "C" {

xmpError_t XMPAPI xmpPowmBatchPlanCreate(xmpHandle_t h, const xmpPowmBatchItem_t *items, int32_t n_items,
                                         const xmpPowmCRTItem_t *crt, int32_t n_crt, int32_t use_graph,
                                         xmpPowmBatchPlan_t *out_plan) {
  if (!h || !out_plan || n_items < 0 || n_crt < 0 || (n_items && !items) || (n_crt && !crt))
    return xmpErrorInvalidParameter;
  DeviceGuard guard(h->device);
  *out_plan = nullptr;
  xmpPowmBatchPlan_t p = new _xmpPowmBatchPlan_t();
  p->use_graph = use_graph != 0;
  xmpError_t e = xmpErrorSuccess;
  auto fail = [&](xmpError_t err) {
    free_plan(h, p);
    return err;
  };
  // ---- validate and collect segments ----
  std::vector<BatchSegment> segs;
  for (int32_t i = 0; i < n_items; i++) {
    const xmpPowmBatchItem_t &it = items[i];
    if (!it.out || !it.base || !it.exp || !it.mod) return fail(xmpErrorInvalidParameter);
    if (it.count == 0) continue;
    if (it.base->precision != it.out->precision || it.mod->precision != it.out->precision)
      return fail(xmpErrorInvalidPrecision);
    if (it.out->count < it.count) return fail(xmpErrorInvalidCount);
    for (xmpIntegers_t x : {it.out, it.base, it.exp, it.mod})
      if (x->device != h->device) return fail(xmpErrorInvalidDevice);
    segs.push_back(BatchSegment{it.out, it.base, it.exp, it.mod, it.count});
  }
  for (int32_t i = 0; i < n_crt; i++) {
    const xmpPowmCRTItem_t &it = crt[i];
    if (!it.out || !it.c || !it.p || !it.q || !it.dp || !it.dq || !it.qinv) return fail(xmpErrorInvalidParameter);
    if (it.count == 0) continue;
    if ((e = crt_validate(h, it.out, it.c, it.p, it.q, it.dp, it.dq, it.qinv, it.count))) return fail(e);
    CrtLaunch c;
    c.item = it;
    c.cfg = crt_config(it.p->nlimbs, std::max(it.dp->precision, it.dq->precision), it.count, h->sm_count);
    if (!c.cfg.launch) return fail(xmpErrorUnsupported);
    c.chunk = it.count;
    p->crt.push_back(c);
  }
  // ---- bins: one per precision, at most kPowmSegs segments each ----
  {
    for (size_t i = 0; i < segs.size(); i++) {
      const BatchSegment &s = segs[i];
      BatchBin *bin = nullptr;
      for (auto &b : p->bins)
        if (b.nlimbs == s.mod->nlimbs && b.segs.size() < (size_t)kPowmSegs) bin = &b;
      if (!bin) {
        p->bins.emplace_back();
        bin = &p->bins.back();
        bin->nlimbs = s.mod->nlimbs;
      }
      bin->segs.push_back(s);
      bin->count += s.count;
      bin->exp_bits = std::max(bin->exp_bits, s.exp->precision);
    }
  }
  // ---- configurations and grids ----
  // Every bin gets a full persistent grid (SMs x resident CTAs) and all bins
  // are launched at once, longest instances first: the block scheduler runs
  // them back to back at full width and fills each bin's tail with the next
  // bin's CTAs, with no work estimate to get wrong.  Lanes and limbs are the
  // tuner's choice at a saturating batch (an exact tuned entry for the bin's
  // own shape wins); the window follows the exponent length.
  const uint32_t kSaturated = 1u << 16;
  for (auto &b : p->bins) {
    PowmConfig c;
    int src = 0;
    bool exact = tuner_lookup(h, xmpTunePowm, b.nlimbs * 32, b.exp_bits, b.count, &src) >= 0 && src == 1 &&
                 tuner_lookup_powm(h, b.nlimbs, b.exp_bits, b.count, &c) && c.dist == kDistLanes;
    if (!exact) {
      bool tuned = tuner_lookup_powm(h, b.nlimbs, b.exp_bits, std::max(b.count, kSaturated), &c) &&
                   c.dist == kDistLanes;
      if (!tuned)
        c = powm_default_config(b.nlimbs, b.exp_bits, std::max(b.count, kSaturated), xmpAlgorithmDefault,
                                h->sm_count);
      c.window = window_for_bits(b.exp_bits, c.dist != kDistDigit && powm_sliding(c.tpi, c.limbs));
    }
    if (c.dist == kDistDigit) {
      // prefer any register kernel that holds the precision; else digit-serial after the join
      PowmConfig r = powm_default_config(b.nlimbs, b.exp_bits, b.count, xmpAlgorithmDistributedMP, h->sm_count);
      if (r.tpi) c = r;
      else b.serial = true;
    }
    b.cfg = c;
    if (!b.serial) {
      b.k = powm_find(c.tpi, c.limbs);
      if (!b.k) return fail(xmpErrorUnsupported);
    }
  }
  // launch order: longest instances (work per instance) first
  std::stable_sort(p->bins.begin(), p->bins.end(), [](const BatchBin &x, const BatchBin &y) {
    return (uint64_t)x.nlimbs * x.nlimbs * x.exp_bits > (uint64_t)y.nlimbs * y.nlimbs * y.exp_bits;
  });
  size_t bytes = 0;
  for (auto &b : p->bins) {
    if (b.serial) continue;
    int occ = 0;
    if (b.k->smem > 48 * 1024)
      cudaFuncSetAttribute(b.k->batch_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.k->smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, b.k->batch_fn, 128, b.k->smem);
    occ = std::max(occ, 1);
    const uint32_t per_item = 32 / b.cfg.tpi;
    uint64_t items = 0;
    for (const BatchSegment &s : b.segs) items += div_up(s.count, per_item);
    uint64_t blocks = (uint64_t)h->sm_count * occ;
    blocks = std::max<uint64_t>(1, std::min<uint64_t>(blocks, div_up((uint32_t)std::min<uint64_t>(items, 0xffffffffu), 4)));
    b.blocks = (int)blocks;
    // shrink the window if the tables would exceed the scratch limit
    while (b.cfg.window > 1 &&
           (size_t)b.blocks * 128 * b.cfg.limbs * 4 * powm_table_entries(b.cfg.window, powm_sliding(b.cfg.tpi, b.cfg.limbs)) >
               scratch_limit(h) / 2)
      b.cfg.window--;
    b.table_offset = bytes;
    bytes += (size_t)b.blocks * 128 * b.cfg.limbs * 4 * powm_table_entries(b.cfg.window, powm_sliding(b.cfg.tpi, b.cfg.limbs));
    bytes = (bytes + 255) & ~(size_t)255;
  }
  // CRT items: window tables for all instances at once, or chunks of what half the scratch limit holds
  for (auto &c : p->crt) {
    while ((c.chunk = crt_chunk_for(c.cfg, scratch_limit(h) / 2, c.item.count)) == 0) {
      if (c.cfg.window <= 1) return fail(xmpErrorIncreaseScratchLimit);
      c.cfg.window--;
    }
    c.table_offset = bytes;
    bytes += crt_table_bytes(c.cfg, c.chunk);
    bytes = (bytes + 255) & ~(size_t)255;
  }
  size_t counter_offset = bytes;
  bytes += 256;
  p->scratch = h->da(bytes);
  if (!p->scratch) return fail(xmpErrorInvalidCudaMalloc);
  p->scratch_bytes = bytes;
  p->counters = (uint32_t *)((char *)p->scratch + counter_offset);
  if (p->bins.size() > 64) return fail(xmpErrorUnsupported);
  // ---- streams and events ----
  if (cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming) != cudaSuccess) return fail(xmpErrorCuda);
  for (size_t b = 0; b < p->bins.size() + p->crt.size(); b++) {
    if (b < p->bins.size() && p->bins[b].serial) continue;
    cudaStream_t s;
    cudaEvent_t ev;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return fail(xmpErrorCuda);
    p->side.push_back(s);
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return fail(xmpErrorCuda);
    p->joins.push_back(ev);
  }
  if (p->use_graph) {
    if (cudaStreamCreateWithFlags(&p->capture, cudaStreamNonBlocking) != cudaSuccess) return fail(xmpErrorCuda);
    // Run once eagerly so every lazily-sized buffer is in place before capture.
    if ((e = enqueue(h, p, p->capture))) return fail(e);
    if (cudaStreamSynchronize(p->capture) != cudaSuccess) return fail(xmpErrorCuda);
    if (cudaStreamBeginCapture(p->capture, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return fail(xmpErrorCuda);
    e = enqueue(h, p, p->capture);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(p->capture, &g);
    p->graph = g;
    if (e) return fail(e);
    if (ce != cudaSuccess || !g) return fail(xmpErrorCuda);
    if (cudaGraphInstantiate(&p->exec, g, 0) != cudaSuccess) return fail(xmpErrorCuda);
  }
  *out_plan = p;
  return check_cuda();
}

xmpError_t XMPAPI xmpPowmBatchPlanExecute(xmpHandle_t h, xmpPowmBatchPlan_t p) {
  if (!h || !p) return xmpErrorInvalidParameter;
  DeviceGuard guard(h->device);
  if (p->use_graph) return cudaGraphLaunch(p->exec, h->stream) == cudaSuccess ? check_cuda() : xmpErrorCuda;
  return enqueue(h, p, h->stream);
}

xmpError_t XMPAPI xmpPowmBatchPlanDestroy(xmpHandle_t h, xmpPowmBatchPlan_t p) {
  if (!h || !p) return xmpErrorInvalidParameter;
  DeviceGuard guard(h->device);
  cudaStreamSynchronize(h->stream);
  for (auto s : p->side) cudaStreamSynchronize(s);
  free_plan(h, p);
  return check_cuda();
}

xmpError_t XMPAPI xmpPowmBatchPlanInfo(xmpPowmBatchPlan_t p, int32_t *bins, uint32_t *precision, uint32_t *count,
                                       xmpPowmConfig_t *config, int32_t *blocks, int32_t max_bins) {
  if (!p || !bins) return xmpErrorInvalidParameter;
  *bins = (int32_t)p->bins.size();
  for (int32_t b = 0; b < *bins && b < max_bins; b++) {
    const BatchBin &x = p->bins[b];
    if (precision) precision[b] = x.nlimbs * 32;
    if (count) count[b] = x.count;
    if (config) config[b] = xmpPowmConfig_t{x.serial ? kDistDigit : x.cfg.dist, x.cfg.tpi, x.cfg.limbs, x.cfg.window};
    if (blocks) blocks[b] = x.blocks;
  }
  return xmpErrorSuccess;
}

}  // extern "C"
