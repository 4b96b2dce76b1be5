// Powm kernel instantiations with 32 lane(s) per instance; registered for the dispatcher and the autotuner.
#include "powm.h"
namespace xmpb {
XMPB_REGISTER_POWM(32, 1)
XMPB_REGISTER_POWM(32, 2)
XMPB_REGISTER_POWM(32, 3)
XMPB_REGISTER_POWM(32, 4)
XMPB_REGISTER_POWM(32, 6)
XMPB_REGISTER_POWM(32, 8)
XMPB_REGISTER_POWM(32, 12)
XMPB_REGISTER_POWM(32, 16)
}  // namespace xmpb
