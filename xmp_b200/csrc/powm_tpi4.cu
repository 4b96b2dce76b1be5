// Powm kernel instantiations with 4 lane(s) per instance; registered for the dispatcher and the autotuner.
#include "powm.h"
namespace xmpb {
XMPB_REGISTER_POWM(4, 1)
XMPB_REGISTER_POWM(4, 2)
XMPB_REGISTER_POWM(4, 3)
XMPB_REGISTER_POWM(4, 4)
XMPB_REGISTER_POWM(4, 5)
XMPB_REGISTER_POWM(4, 6)
XMPB_REGISTER_POWM(4, 8)
XMPB_REGISTER_POWM(4, 10)
XMPB_REGISTER_POWM(4, 12)
XMPB_REGISTER_POWM(4, 16)
}  // namespace xmpb
