// Autotuner internals shared by the op dispatchers, the exhaustive tuner and
// the learned selector.  Replaces the reference's offline tuning tables
// (src/tune/tune.cu:70-275, src/tune/tune_*.h) read by getFastestPowmLaunch
// (src/powm.cu:120-236).
#pragma once
#include "powm.h"
#include "../../include/xmp_b200.h"
#include <stdint.h>
#include <unordered_map>
#include <vector>

namespace xmpb {

constexpr int kCand = XMP_TUNE_CANDIDATES;
constexpr int kPowmDists = 7;          // per-thread, 2, 4, 8, 16, 32 lanes, digit-serial
constexpr int kPowmWindows = 6;        // W = 1..6
constexpr int kElemSlots = 8;          // {register, streamed} x {32, 64, 128, 256} threads
constexpr int kGridMaxLimbs = 512;     // selector lookup grid: precisions 32..16384 bits
constexpr int kGridCountBuckets = 27;  // floor(log2 count), 0..26
constexpr int kGridExpBuckets = 15;    // floor(log2 exp_bits), 0..14 (powm only)
constexpr int kSelectorMinCountLog2 = 6;  // smallest batch the tuner times (2^6); smaller batches use its cell

struct ElemConfig {
  int variant = 0;   // 0 register kernel, 1 streamed kernel
  int threads = 128;
};

// Candidate interpretation (valid = can run the shape).
bool powm_candidate(uint32_t nlimbs, int slot, PowmConfig *cfg);
bool elem_candidate(int op, uint32_t nlimbs, int slot, ElemConfig *cfg);
int elem_threads(int slot);

// Whether a register kernel exists for the operand classes (mul.cu / div.cu).
bool mul_has_register_kernel(uint32_t na, uint32_t nb);
bool div_has_register_kernel(uint32_t nb);

struct TunerState {
  std::unordered_map<uint64_t, int> choices;  // exact shapes set by the exhaustive tuner
  std::vector<uint8_t> table;                 // selector grid: op x limbs x count bucket x exp bucket
  bool has_table = false;
};

TunerState *tuner_state(xmpHandle_t h);
uint64_t shape_key(int op, uint32_t bits, uint32_t exp_bits, uint32_t count);
// Slot for a shape from the handle's tuner (-1: none) and where it came from (1 exact, 2 selector).
int tuner_lookup(xmpHandle_t h, int op, uint32_t bits, uint32_t exp_bits, uint32_t count, int *source);

// Internal op entry points with an explicit configuration (nullptr: usual selection).
xmpError_t mul_entry(xmpHandle_t h, xmpIntegers_t p, xmpIntegers_t a, xmpIntegers_t b, uint32_t count,
                     const ElemConfig *forced);
xmpError_t divmod_entry(xmpHandle_t h, xmpIntegers_t q, xmpIntegers_t r, xmpIntegers_t a, xmpIntegers_t b,
                        uint32_t count, const ElemConfig *forced);

// Selector grid evaluation (selector.cu): fills table[op][limbs-1][cb][eb] with argmin slots.
xmpError_t selector_fill_table(xmpHandle_t h, const float *params, int members, std::vector<uint8_t> *table);
// The compiled-in selector: `*members` networks' parameters back to back (nullptr, 0 when the
// library was built without them).
const float *default_selector_params(int *members);
size_t grid_index(int op, uint32_t nlimbs, int count_bucket, int exp_bucket);
int count_bucket(uint32_t count);
int exp_bucket(uint32_t exp_bits);

}  // namespace xmpb
