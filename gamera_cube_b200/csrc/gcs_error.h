// Thread-local error message shared by every C entry point of the library
// (returned by gcs_last_error).
#pragma once

namespace gcs {
void set_api_error(const char *msg);
}  // namespace gcs
