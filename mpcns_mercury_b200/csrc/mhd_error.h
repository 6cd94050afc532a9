// The library's error reporting, shared by its translation units: records a
// formatted message for mhd_last_error (per host thread) and returns `code`.
#pragma once

namespace mhd {
int set_error(int code, const char *fmt, ...);
}  // namespace mhd
