// psg_api.cu -- error reporting and library information of the C API.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "psg_common.cuh"
#include "psgpu_internal.h"

static thread_local char g_err[1024];

extern "C" void psg_set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}

extern "C" const char* psg_last_error(void) { return g_err; }

extern "C" void psg_clear_error(void) { g_err[0] = 0; }

extern "C" int psg_version(void) { return PSG_VERSION; }
