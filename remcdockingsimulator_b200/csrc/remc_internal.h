// Internal helpers shared by the library's translation units (not part of the ABI).
#pragma once

namespace remc {
// Records the message returned by remc_last_error_string() for this thread.
void record_error(const char* message);
}  // namespace remc
