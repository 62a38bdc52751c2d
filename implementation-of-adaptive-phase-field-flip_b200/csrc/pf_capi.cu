// Error state, version and launch accounting of libpfflip.
#include <cstdarg>
#include <cstring>

#include "pf_common.cuh"

namespace pf {

static thread_local char g_msg[512] = "";
static thread_local int g_cuda_err = 0;
static std::atomic<uint64_t> g_launches{0};
static thread_local bool g_suppress = false;

void set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int n = std::snprintf(g_msg, sizeof(g_msg), "pfflip error %d: ", code);
  if (n < 0) n = 0;
  std::vsnprintf(g_msg + n, sizeof(g_msg) - (size_t)n, fmt, ap);
  va_end(ap);
}

void set_cuda_error(cudaError_t e, const char* where) {
  g_cuda_err = (int)e;
  set_error(PF_ERR_CUDA, "%s: %s (%s)", where, cudaGetErrorName(e), cudaGetErrorString(e));
}

void count_launch(uint64_t n) {
  if (!g_suppress) g_launches.fetch_add(n, std::memory_order_relaxed);
}

// while a CUDA graph is being captured, launches are counted at replay instead
void count_suppress(bool on) { g_suppress = on; }

}  // namespace pf

extern "C" {

const char* pf_version(void) { return "pfflip-b200 0.1 (sm_100a)"; }
const char* pf_last_error(void) { return pf::g_msg; }
int pf_last_cuda_error(void) { return pf::g_cuda_err; }
uint64_t pf_launch_count(void) { return pf::g_launches.load(); }

}  // extern "C"
