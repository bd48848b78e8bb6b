// Library-internal entry points shared between the C API files: the
// thread-local error message returned by gcs_last_error and the device
// context bound to a host grid.
#pragma once

#include <cstddef>

#include "gamera_cs_types.h"

struct gcs_context;

namespace gcs {
struct Context;
void set_api_error(const char *msg);
// The context of a host grid (created on first use, shared with the
// drop-in step calls on the same grid).
Context *context_for_grid(const gamera_no_grid grid[6], const size_t active[3],
                          size_t ghost);
Context *context_of(gcs_context *ctx);
}  // namespace gcs
