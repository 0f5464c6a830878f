// Library-level entry points: version, thread-local error text, device info.
#include <cstdarg>
#include <mutex>

#include "common.cuh"

namespace qs {

namespace {
thread_local char g_err[512] = "";
}

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int sm_count() {
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cache[dev] == 0) {
        int c = 0;
        if (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || c <= 0) c = 148;
        cache[dev] = c;
    }
    return cache[dev];
}

}  // namespace qs

extern "C" int qs_version(void) { return 1; }

extern "C" const char* qs_last_error(void) { return qs::g_err; }

extern "C" int qs_device_sm_count(void) { return qs::sm_count(); }
