// Project-written stand-in for the ISQ quantity kinds the Lucid reference
// uses (see ../framework.h): tags only, no arithmetic of their own.
#pragma once
#include "../framework.h"

namespace mp_units::isq {
#define LUCID_SHIM_KIND(name) \
    inline constexpr struct name final : ::mp_units::quantity_spec_base<name> { } name
LUCID_SHIM_KIND(length);
LUCID_SHIM_KIND(area);
LUCID_SHIM_KIND(volume);
LUCID_SHIM_KIND(displacement);
LUCID_SHIM_KIND(velocity);
LUCID_SHIM_KIND(angular_measure);
LUCID_SHIM_KIND(solid_angular_measure);
LUCID_SHIM_KIND(radiance);
LUCID_SHIM_KIND(power);
#undef LUCID_SHIM_KIND
}  // namespace mp_units::isq
