// Library-wide host utilities: version, per-thread error message, launch checks.
#include <cstdarg>
#include <cstdio>

#include "hp_common.cuh"

namespace hp {

static thread_local char g_err[512] = {0};

int32_t set_error(int32_t code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int32_t check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(HP_ERR_CUDA, "%s launch failed: %s", what, cudaGetErrorString(e));
  return HP_OK;
}

}  // namespace hp

extern "C" int32_t hp_version(void) { return 100; }

extern "C" const char* hp_last_error(void) { return hp::g_err; }
