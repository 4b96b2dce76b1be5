// Powm kernel instantiations with 1 lane(s) per instance; registered for the dispatcher and the autotuner.
#include "powm.h"
namespace xmpb {
XMPB_REGISTER_POWM(1, 1)
XMPB_REGISTER_POWM(1, 2)
XMPB_REGISTER_POWM(1, 3)
XMPB_REGISTER_POWM(1, 4)
XMPB_REGISTER_POWM(1, 5)
XMPB_REGISTER_POWM(1, 6)
XMPB_REGISTER_POWM(1, 7)
XMPB_REGISTER_POWM(1, 8)
XMPB_REGISTER_POWM(1, 10)
XMPB_REGISTER_POWM(1, 12)
XMPB_REGISTER_POWM(1, 16)
XMPB_REGISTER_POWM(1, 24)
XMPB_REGISTER_POWM(1, 32)
}  // namespace xmpb
