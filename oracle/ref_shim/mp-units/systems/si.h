// Project-written stand-in for the SI units the Lucid reference uses (see
// ../framework.h): every one has magnitude 1.
#pragma once
#include "../framework.h"

namespace mp_units::si {
inline constexpr unit_dims<1, 0, 0, 0> metre{};
inline constexpr unit_dims<0, 1, 0, 0> watt{};
inline constexpr unit_dims<0, 0, 1, 0> radian{};
inline constexpr unit_dims<0, 0, 0, 1> steradian{};
}  // namespace mp_units::si
