// Thread-local error message and the library-wide entry points of opensol_fdtd.h.
#include "common.cuh"

#include <cstring>

namespace os {

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...) {
    char buf[1024];
    va_list args;
    va_start(args, fmt);
    vsnprintf(buf, sizeof(buf), fmt, args);
    va_end(args);
    g_last_error = buf;
}

const std::string &last_error() { return g_last_error; }

int cuda_status(cudaError_t err, const char *what) {
    set_error("%s failed: %s (%s)", what, cudaGetErrorName(err), cudaGetErrorString(err));
    if (err == cudaErrorMemoryAllocation) return OS_ERR_NO_MEMORY;
    return OS_ERR_CUDA;
}

}  // namespace os

extern "C" int os_fdtd_last_error(char *buf, size_t n) {
    const std::string &msg = os::last_error();
    if (buf && n) {
        size_t len = msg.size() < n - 1 ? msg.size() : n - 1;
        memcpy(buf, msg.data(), len);
        buf[len] = '\0';
    }
    return (int)msg.size();
}

extern "C" int os_fdtd_version(void) { return 100; }

extern "C" int os_fdtd_host_alloc(size_t bytes, void **out) {
    OS_CHECK(out, OS_ERR_INVALID, "os_fdtd_host_alloc: null argument");
    *out = nullptr;
    if (bytes == 0) return OS_OK;
    OS_CUDA(cudaHostAlloc(out, bytes, cudaHostAllocPortable));
    return OS_OK;
}

extern "C" int os_fdtd_host_free(void *ptr) {
    if (ptr) OS_CUDA(cudaFreeHost(ptr));
    return OS_OK;
}
