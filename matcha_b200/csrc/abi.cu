// Error reporting and version of the matcha_b200 C ABI.
#include <stdio.h>
#include <string.h>
#include "common.cuh"

namespace {
thread_local char g_last_error[512] = {0};
}

void mtb_set_last_error(const char* msg, const char* file, int line) {
  const char* base = strrchr(file, '/');
  snprintf(g_last_error, sizeof(g_last_error), "%s (%s:%d)", msg, base ? base + 1 : file, line);
}

extern "C" int mtb_version(void) { return 100; }

extern "C" const char* mtb_last_error(void) { return g_last_error; }
