// Powm kernel instantiations with 2 lane(s) per instance; registered for the dispatcher and the autotuner.
#include "powm.h"
namespace xmpb {
XMPB_REGISTER_POWM(2, 2)
XMPB_REGISTER_POWM(2, 3)
XMPB_REGISTER_POWM(2, 4)
XMPB_REGISTER_POWM(2, 6)
XMPB_REGISTER_POWM(2, 8)
XMPB_REGISTER_POWM(2, 12)
XMPB_REGISTER_POWM(2, 16)
}  // namespace xmpb
