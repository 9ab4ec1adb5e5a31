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

namespace {

// Fills the block's whole dynamic shared memory with one value.
__global__ void k_poison_shared(double value, int n) {
    extern __shared__ double buf[];
    for (int i = threadIdx.x; i < n; i += blockDim.x) buf[i] = value;
}

}  // namespace

extern "C" {

int lica_debug_poison_shared(double value, void* stream) {
    int dev = 0, sms = 0, bytes = 0;
    LICA_CUDA_TRY(cudaGetDevice(&dev));
    LICA_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    LICA_CUDA_TRY(cudaDeviceGetAttribute(&bytes, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    LICA_CUDA_TRY(cudaFuncSetAttribute(k_poison_shared, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    LICA_CUDA_TRY(cudaFuncSetAttribute(k_poison_shared, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    // one block per SM at a time (the whole shared memory each); four waves
    k_poison_shared<<<4 * sms, 1024, (size_t)bytes, (cudaStream_t)stream>>>(value, bytes / (int)sizeof(double));
    LICA_CUDA_TRY(cudaGetLastError());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return LICA_OK;
}

void lica_count_launches(int64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int64_t lica_kernel_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

const char* lica_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"
