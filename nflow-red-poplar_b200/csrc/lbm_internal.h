// lbm_internal.h — declarations shared by the host-side translation units.
#pragma once
namespace lbm {
// Record a formatted message for lbm_last_error() and return `code`.
int set_error(int code, const char* fmt, ...);
void clear_error();
}  // namespace lbm
