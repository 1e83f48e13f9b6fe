// Project-written stand-in for mp-units' QUANTITY_SPEC macro (see framework.h).
#pragma once
#include "framework.h"

#define QUANTITY_SPEC(name, ...) \
    inline constexpr struct name final : ::mp_units::quantity_spec<name, __VA_ARGS__> { } name
