// Library-wide entry points: version and last-error string.
#include "tpf_common.cuh"

#include <string>

namespace tpf {

namespace {
thread_local std::string g_last_error;
}

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

const char* last_error() { return g_last_error.c_str(); }

}  // namespace tpf

extern "C" {

int tpf_version(void) { return 10000; }

const char* tpf_last_error(void) { return tpf::last_error(); }

}  // extern "C"
