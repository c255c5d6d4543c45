/*
 * Type policy override for the FP64 test oracle build of the reference CPU path.
 * Placed ahead of the reference include directories so that `#include "sph/types.hpp"` resolves here:
 * every hydro, mass and x_m1 field becomes double (the reference default is float; sph/types.hpp:39-46).
 * Compiled only when SPHB_ORACLE_MIXED is not defined; the mixed build uses the reference's own header.
 */
#pragma once

#include <cstdint>

namespace sph
{

struct SphTypes
{
    using KeyType        = uint64_t;
    using CoordinateType = double;
    using HydroType      = double;
    using XM1Type        = double;
    using Tmass          = double;
};

} // namespace sph
