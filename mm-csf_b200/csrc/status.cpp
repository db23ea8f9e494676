// Status codes and the thread-local last-error message.
#include <cstdio>

#include "common.h"

namespace {
thread_local std::string g_last_error;
}

namespace mmcsf {
int set_error(int status, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}
void clear_error() { g_last_error.clear(); }
}  // namespace mmcsf

extern "C" const char* mmcsf_status_string(int s) {
  switch (s) {
    case MMCSF_OK: return "ok";
    case MMCSF_ERR_INVALID: return "invalid argument";
    case MMCSF_ERR_CUDA: return "CUDA error";
    case MMCSF_ERR_NOMEM: return "out of memory";
    case MMCSF_ERR_IO: return "I/O error";
    case MMCSF_ERR_UNSUPPORTED: return "unsupported";
    case MMCSF_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
  }
}

extern "C" const char* mmcsf_last_error(void) { return g_last_error.c_str(); }

extern "C" int mmcsf_version(void) { return 100; }
