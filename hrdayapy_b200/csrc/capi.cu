// Library-wide C entry points: error reporting and version.
#include "hp_common.cuh"

namespace hp {
static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
}  // namespace hp

extern "C" const char* hp_last_error(void) { return hp::g_err; }
extern "C" const char* hp_version(void) { return "hrdaya_b200 0.1.0 (sm_100a)"; }
