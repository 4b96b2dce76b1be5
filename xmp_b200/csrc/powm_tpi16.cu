// Powm kernel instantiations with 16 lane(s) per instance; registered for the dispatcher and the autotuner.
#include "powm.h"
namespace xmpb {
XMPB_REGISTER_POWM(16, 1)
XMPB_REGISTER_POWM(16, 2)
XMPB_REGISTER_POWM(16, 3)
XMPB_REGISTER_POWM(16, 4)
XMPB_REGISTER_POWM(16, 6)
XMPB_REGISTER_POWM(16, 8)
XMPB_REGISTER_POWM(16, 12)
XMPB_REGISTER_POWM(16, 16)
}  // namespace xmpb
