// Process-wide pieces of the C ABI: last-error message and the kernel launch counter.
#include "common.cuh"

#include <atomic>
#include <cstring>
#include <string>

namespace {
thread_local std::string g_last_error;
std::atomic<int64_t> g_launches{0};
}  // namespace

void lica_set_last_error(const char* what, const char* msg, const char* file, int line) {
    g_last_error = std::string(what) + ": " + msg + " (" + file + ":" + std::to_string(line) + ")";
}

extern "C" {

void lica_count_launches(int64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int64_t lica_kernel_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

const char* lica_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"
