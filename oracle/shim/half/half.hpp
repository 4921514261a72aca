// Host-only stand-in for the `half` library header that the reference's
// libVLR/shared/shared.h:6-8 includes (the ext/half submodule is empty).
// TEST INFRASTRUCTURE ONLY: the oracle never converts half values; it only
// needs the type name to exist.
#pragma once
#include <cstdint>
namespace half_float {
    struct half {
        uint16_t bits;
        half() : bits(0) {}
        explicit half(float) : bits(0) {}
        operator float() const { return 0.0f; }
    };
}
