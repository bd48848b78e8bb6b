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
struct Opts;
// The checks and options of gcs_context_run (advance and time-step options,
// dt fraction) for a context with a background.
bool driver_opts(const gamera_no_advance_options *options,
                 const gamera_no_timestep_options *t, double fraction, Opts *O);
// Enqueue one driver-mode step (the body of gcs_context_run's graph) on the
// context's stream; no synchronisation.
int enqueue_driver_step(gcs_context *ctx, const Opts &O);
}  // namespace gcs
