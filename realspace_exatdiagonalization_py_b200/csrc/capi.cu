// C ABI plumbing: version string and per-thread last-error message.
#include <cstdarg>
#include <cstdio>
#include <string>
#include "rsed_internal.cuh"

#include <atomic>

namespace {
thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};
}

void rsed_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

extern "C" long long rsed_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int rsed_set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

extern "C" const char* rsed_version(void) { return "rsed-b200 0.1.0 (sm_100a)"; }

extern "C" const char* rsed_last_error(void) { return g_last_error.c_str(); }

extern "C" int rsed_device_sync(void* stream) {
  RSED_TRY_CUDA(cudaStreamSynchronize(as_stream(stream)));
  return RSED_OK;
}
