// Internal interfaces between the libhoms translation units (not part of the
// C ABI).
#pragma once

#include <stdint.h>

#include "../../include/homs.h"

namespace homs {

// Shape of a device-resident phantom, for the serving loop's admission
// estimate (homs_server.cu) without knowing its layout.
struct ResidentShape {
    int64_t nspins;
    int32_t ncoils;
    homs_dtype compute;  // precision its arrays are kept in
    homs_mode mode;
    int device;
};
bool resident_shape(const homs_resident *r, ResidentShape *out);

}  // namespace homs
