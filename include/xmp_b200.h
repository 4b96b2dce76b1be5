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
 *                 distribution), 1 = digit-serial (lanes/limbs ignored),
 *                 2 = one instance per CTA (moduli up to 4096 bits; the library
 *                 sets limbs to the CTA's operand size, 32/64/96/128, and
 *                 ignores lanes) -- the lowest latency for a small batch of
 *                 moduli above 512 bits, and the default choice there for
 *                 batches of up to 4-6 (1024-bit and smaller moduli), 2-3
 *                 (up to 2048 bits) or one (larger) instances per SM;
 *   window:       exponent window bits, 1..7. */
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

/* ---- batched powm over mixed precisions ------------------------------------
 * A plan takes plain items (out = base^exp mod mod for `count` instances of
 * one precision) and CRT items (out = c^d mod pq from the half-size key
 * material: cp = c mod p, cq = c mod q, mp = cp^dp mod p, mq = cq^dq mod q,
 * out = mq + q * ((mp - mq) * qinv mod p), Garner recombination; p and q
 * have their top bit set).  Instances are binned by modulus precision (CRT
 * halves join the bin of their precision); every bin runs as one persistent
 * kernel whose warps pull work from an atomic queue, with its configuration
 * from the handle's tuner, and all bins run concurrently (forked onto side
 * streams and joined back to the handle's stream).  With `use_graph` the
 * whole execution is captured once into a CUDA graph and each execute is one
 * graph launch.  All device memory a plan needs (window tables, CRT
 * temporaries) is allocated when it is created.  Index policies do not apply;
 * no item's output may alias another item's input; the arrays must outlive
 * the plan. */
typedef struct {
  xmpIntegers_t out, base, exp, mod;
  uint32_t count;
} xmpPowmBatchItem_t;

typedef struct {
  xmpIntegers_t out;              /* 2h bits */
  xmpIntegers_t c;                /* 2h bits, c < pq */
  xmpIntegers_t p, q, dp, dq, qinv; /* h bits */
  uint32_t count;
} xmpPowmCRTItem_t;

typedef struct _xmpPowmBatchPlan_t *xmpPowmBatchPlan_t;

/* ---- fused CRT-RSA private operation -----------------------------------------
 * (no counterpart in the reference library; replaces the op sequence of its
 * CRT-RSA sample, samples/crt_rsa/rsa.cc:206-219: c mod p, c mod q, two powm,
 * two mul, add, mod.)  out[i] = c[i]^d mod p*q for i < count, computed from
 * p, q, dp = d mod (p-1), dq = d mod (q-1) and qinv = q^-1 mod p in one
 * kernel launch: Montgomery reductions of c, the two half-size
 * exponentiations with a fixed window over the whole precision of dp and dq
 * (the same sequence of multiplications whatever the exponent bits), and
 * Garner's recombination mq + q*((mp - mq)*qinv mod p).  p, q and qinv have
 * one precision h (p and q odd, qinv < p); out has 2h bits; c at most 2h bits
 * and below p*q; dp and dq any precision.  Every input is broadcast like an
 * XMP operand (element i % its count); the handle's index policy is not used.
 * The window tables use the handle's scratch arena (the batch is chunked to
 * its limit). */
xmpError_t XMPAPI xmpIntegersPowmCRT(xmpHandle_t handle, xmpIntegers_t out, const xmpIntegers_t c,
                                     const xmpIntegers_t p, const xmpIntegers_t q, const xmpIntegers_t dp,
                                     const xmpIntegers_t dq, const xmpIntegers_t qinv, uint32_t count);
xmpError_t XMPAPI xmpIntegersPowmCRTAsync(xmpHandle_t handle, xmpIntegers_t out, const xmpIntegers_t c,
                                          const xmpIntegers_t p, const xmpIntegers_t q, const xmpIntegers_t dp,
                                          const xmpIntegers_t dq, const xmpIntegers_t qinv, uint32_t count);


xmpError_t XMPAPI xmpPowmBatchPlanCreate(xmpHandle_t handle, const xmpPowmBatchItem_t *items, int32_t n_items,
                                         const xmpPowmCRTItem_t *crt, int32_t n_crt, int32_t use_graph,
                                         xmpPowmBatchPlan_t *plan);
/* Enqueues one execution on the handle's stream. */
xmpError_t XMPAPI xmpPowmBatchPlanExecute(xmpHandle_t handle, xmpPowmBatchPlan_t plan);
xmpError_t XMPAPI xmpPowmBatchPlanDestroy(xmpHandle_t handle, xmpPowmBatchPlan_t plan);
/* Number of bins (concurrent persistent kernels) and each bin's precision, instances and configuration. */
xmpError_t XMPAPI xmpPowmBatchPlanInfo(xmpPowmBatchPlan_t plan, int32_t *bins, uint32_t *precision, uint32_t *count,
                                       xmpPowmConfig_t *config, int32_t *blocks, int32_t max_bins);

/* ---- autotuner --------------------------------------------------------------
 * A problem shape is (op, bits, exp_bits, count).  Each op has candidate
 * kernel configurations in XMP_TUNE_CANDIDATES slots:
 *   powm:   slot = 6*d + (W-1), d in {per-thread, 2, 4, 8, 16, 32 lanes,
 *           digit-serial}, W = window bits 1..6 (42 slots; each lane count uses
 *           the fewest limbs per lane that hold the precision);
 *   mul, divmod: slot = 4*v + t, v in {register kernel, streamed kernel},
 *           t -> 32, 64, 128, 256 threads per block (8 slots).
 * Slots a shape cannot use are invalid. */
enum { xmpTuneMul = 0, xmpTuneDivMod = 1, xmpTunePowm = 2 };
#define XMP_TUNE_CANDIDATES 48

typedef struct {
  int32_t op;        /* xmpTuneMul, xmpTuneDivMod, xmpTunePowm */
  uint32_t bits;     /* modulus / operand precision (divmod: dividend = 2*bits, divisor = bits) */
  uint32_t exp_bits; /* powm exponent length in bits (0 otherwise) */
  uint32_t count;    /* instances */
} xmpTuneShape_t;

/* Whether `slot` is a valid candidate for (op, bits) and the configuration it
 * stands for (powm: all four fields; mul/divmod: distribution = 0 register /
 * 1 streamed, lanes = threads per block). */
xmpError_t XMPAPI xmpTuneCandidate(int32_t op, uint32_t bits, int32_t slot, int32_t *valid,
                                   xmpPowmConfig_t *config);

/* Exhaustive tuner: times every valid candidate of `shape` on seeded synthetic
 * data (CUDA events on the handle's stream, best of `reps`); ms[slot] is the
 * time in milliseconds, a negative value for invalid slots, or NaN for valid
 * slots of a distribution whose first timing was already over 20x the best
 * (not worth timing its other windows). */
xmpError_t XMPAPI xmpTuneMeasure(xmpHandle_t handle, const xmpTuneShape_t *shape, int32_t reps, float *ms);

/* Records / queries the handle's choice for a shape.  Lookup order: a choice
 * set for the exact shape, else the loaded selector's table, else the
 * built-in heuristic (source 1, 2, 0).  A new handle starts with the
 * selector compiled into the library (trained on this library's B200
 * timings) loaded; xmpTuneClear drops every choice and the selector, leaving
 * the heuristic. */
xmpError_t XMPAPI xmpTuneSetChoice(xmpHandle_t handle, const xmpTuneShape_t *shape, int32_t slot);
xmpError_t XMPAPI xmpTuneGetChoice(xmpHandle_t handle, const xmpTuneShape_t *shape, int32_t *slot, int32_t *source);
xmpError_t XMPAPI xmpTuneClear(xmpHandle_t handle);

/* ---- learned selector ------------------------------------------------------
 * MLP with 4 inputs (op, log2 bits, log2 count, log2 exp_bits, scaled), two
 * hidden layers of 64 FP32 ReLU units and one predicted log2(time) per
 * candidate slot.  Parameters are XMP_SELECTOR_PARAMS floats laid out as
 * W1[4][64], b1[64], W2[64][64], b2[64], W3[64][48], b3[48].  Training,
 * gradients and inference run in this library's own CUDA kernels. */
#define XMP_SELECTOR_HIDDEN 64
#define XMP_SELECTOR_PARAMS (4 * 64 + 64 + 64 * 64 + 64 + 64 * 48 + 48)

/* Trains from measured times ms[n][48] (negative = invalid) with Adam for
 * `epochs` full-batch steps; params is read as the initial value when
 * `init_from_params` is nonzero, else initialised from `seed`; final loss out. */
xmpError_t XMPAPI xmpSelectorTrain(xmpHandle_t handle, const xmpTuneShape_t *shapes, const float *ms, int32_t n,
                                   int32_t epochs, float learning_rate, uint64_t seed, int32_t init_from_params,
                                   float *params, float *final_loss);
/* Loss and its gradient with respect to every parameter (for checking). */
xmpError_t XMPAPI xmpSelectorGradients(xmpHandle_t handle, const float *params, const xmpTuneShape_t *shapes,
                                       const float *ms, int32_t n, float *loss, float *grads);
/* Predicted log2(ms) for every slot of n shapes (pred[n][48]). */
xmpError_t XMPAPI xmpSelectorPredict(xmpHandle_t handle, const float *params, const xmpTuneShape_t *shapes,
                                     int32_t n, float *pred);
/* Installs a trained selector in the handle: a CUDA kernel evaluates it over
 * the lookup grid (every 32-bit precision up to 16,384 bits x log2 count x
 * log2 exponent length) and the per-call choice becomes a table lookup. */
xmpError_t XMPAPI xmpSelectorLoad(xmpHandle_t handle, const float *params);
/* The same from an ensemble: `members` parameter sets back to back; a cell's
 * predicted time per slot is the members' mean (independently seeded networks
 * averaged generalise to untimed precisions better than one). */
xmpError_t XMPAPI xmpSelectorLoadEnsemble(xmpHandle_t handle, const float *params, int32_t members);

/* ---- serving loop ----------------------------------------------------------
 * No counterpart in the reference.  A server admits modular-exponentiation
 * requests (1 .. max_wave_ops ops under one registered key) from any thread
 * and serves them with continuous batching: whenever one of its launch
 * streams is idle, a scheduler thread launches the pending requests of a
 * precision class (oldest first) as one wave, so requests that arrive while
 * others run start as soon as a stream and op slots free up and overlap with
 * them on the device, and waves grow with the load.  Each wave's kernel
 * configuration follows the class's ops in flight: latency-optimal when the
 * GPU is quiet, throughput-optimal when it is full.  Keys (odd moduli) and their
 * Montgomery constants stay on the device; op slots and window tables come
 * from a fixed device arena sized by the HBM budget, which is the admission
 * limit.  Operands and results are host rows of precision/32 little-endian
 * 32-bit limbs per op (exponents have the modulus's precision); results are
 * bit-identical to xmpIntegersPowm on the same operands. */
typedef struct _xmpServer_t *xmpServer_t;

typedef struct {
  size_t hbm_budget;      /* device bytes for keys, op slots and window tables (0: 8 GiB) */
  uint32_t max_wave_ops;  /* ops per launch wave, and per request (0: 4096) */
  uint32_t streams;       /* launch streams, i.e. waves in flight at most (0: 32; give the process
                             CUDA_DEVICE_MAX_CONNECTIONS >= streams so they map to separate
                             hardware queues) */
  uint32_t max_keys;      /* key capacity per precision class (0: 4096) */
  uint32_t max_slots;     /* op slots per class, at most (0: 262144; fewer if the budget says so) */
} xmpServerConfig_t;

typedef struct {
  uint64_t requests_submitted;
  uint64_t requests_completed;
  uint64_t ops_completed;
  uint64_t waves;             /* launch waves */
  uint64_t admission_stalls;  /* times a class had ready work but no free op slots */
  uint32_t max_inflight_ops;
  uint32_t classes;
  size_t device_bytes;        /* device memory the server holds */
} xmpServerStats_t;

/* One precision class per entry of `precisions` (multiples of 32 bits).  The
 * handle provides the device, allocators and tuner (choices are fixed at
 * creation); it must outlive the server. */
xmpError_t XMPAPI xmpServerCreate(xmpHandle_t handle, const uint32_t *precisions, uint32_t n_classes,
                                  const xmpServerConfig_t *config, xmpServer_t *server);
xmpError_t XMPAPI xmpServerDestroy(xmpServer_t server);
/* Registers `count` odd moduli (host rows) and computes R^2 mod m on the
 * device; key ids are first_key .. first_key+count-1. */
xmpError_t XMPAPI xmpServerAddKeys(xmpServer_t server, uint32_t precision, const uint32_t *moduli, uint32_t count,
                                   uint32_t *first_key);
/* Queues out[i] = bases[i]^exps[i] mod key for i < nops.  The buffers must
 * stay valid until the request is reported done. */
xmpError_t XMPAPI xmpServerSubmit(xmpServer_t server, uint32_t key, uint32_t nops, const uint32_t *bases,
                                  const uint32_t *exps, uint32_t *out, uint64_t *request);
/* Waits up to timeout_us (0: poll) for a request; *done = 1 once its results
 * are in `out` (the request id is then retired). */
xmpError_t XMPAPI xmpServerWait(xmpServer_t server, uint64_t request, uint32_t timeout_us, int32_t *done);
xmpError_t XMPAPI xmpServerStats(xmpServer_t server, xmpServerStats_t *stats);
/* Open-loop replay of n requests arriving at arrival_ns (non-decreasing, from
 * the start): mode 0 through the server, mode 1 as plain synchronous
 * per-request calls (Import, xmpIntegersPowm, Export) on the calling thread.
 * latency_ns[i] = completion - scheduled arrival; seconds = last completion
 * - start.  The server must be idle. */
xmpError_t XMPAPI xmpServerReplay(xmpServer_t server, uint32_t n, const uint32_t *keys, const uint32_t *nops,
                                  const uint64_t *arrival_ns, const uint32_t *const *bases,
                                  const uint32_t *const *exps, uint32_t *const *outs, int32_t mode,
                                  uint64_t *latency_ns, double *seconds);

#ifdef __cplusplus
}
#endif

#endif /* XMP_B200_EXT_H */
