// Autotuner state attached to a handle (placeholder until the tuner lands).
#include "powm.h"

namespace xmpb {
bool tuner_lookup_powm(xmpHandle_t h, uint32_t nlimbs, uint32_t exp_bits, uint32_t count, PowmConfig *cfg) {
  (void)h; (void)nlimbs; (void)exp_bits; (void)count; (void)cfg;
  return false;
}
void tuner_destroy(xmpHandle_t h) { (void)h; }
}  // namespace xmpb
