// Powm kernel instantiations with 8 lane(s) per instance; registered for the dispatcher and the autotuner.
#include "powm.h"
namespace xmpb {
XMPB_REGISTER_POWM(8, 1)
XMPB_REGISTER_POWM(8, 2)
XMPB_REGISTER_POWM(8, 3)
XMPB_REGISTER_POWM(8, 4)
XMPB_REGISTER_POWM(8, 5)
XMPB_REGISTER_POWM(8, 6)
XMPB_REGISTER_POWM(8, 8)
XMPB_REGISTER_POWM(8, 10)
XMPB_REGISTER_POWM(8, 12)
XMPB_REGISTER_POWM(8, 16)
}  // namespace xmpb
