// Error reporting and version entry points of the C-ABI.
#include <stdarg.h>
#include <stdio.h>
#include <atomic>
#include "common.cuh"

namespace {
thread_local char g_message[512] = "";
std::atomic<long long> g_launches{0};
}

namespace afsi {

int32_t fail(int32_t code, const char* fmt, ...) {
    va_list args;
    va_start(args, fmt);
    vsnprintf(g_message, sizeof g_message, fmt, args);
    va_end(args);
    return code;
}

int32_t launched(const char* what) {
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess)
        return fail(AFSI_ERR_CUDA, "%s: %s", what, cudaGetErrorString(err));
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return AFSI_OK;
}

}  // namespace afsi

extern "C" const char* afsi_b200_last_error(void) { return g_message; }

extern "C" int32_t afsi_b200_version(void) { return 100; }

extern "C" int64_t afsi_b200_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }
