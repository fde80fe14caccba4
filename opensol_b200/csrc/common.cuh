// Shared host-side plumbing of libopensol_fdtd.so: status codes, the thread-local last-error message, CUDA call
// checks that turn a failure into a status (never an abort), and small device buffers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <cstdio>
#include <cstdarg>

#include "../../include/opensol_fdtd.h"

namespace os {

void set_error(const char *fmt, ...);
const std::string &last_error();

// Returns the status for a CUDA result and records its message.
int cuda_status(cudaError_t err, const char *what);

#define OS_CUDA(call)                                                                                          \
    do {                                                                                                         \
        cudaError_t os_err_ = (call);                                                                            \
        if (os_err_ != cudaSuccess) return ::os::cuda_status(os_err_, #call);                                    \
    } while (0)

#define OS_CHECK(cond, code, ...)                                                                                \
    do {                                                                                                         \
        if (!(cond)) {                                                                                           \
            ::os::set_error(__VA_ARGS__);                                                                        \
            return (code);                                                                                       \
        }                                                                                                        \
    } while (0)

#define OS_TRY(call)                                                                                             \
    do {                                                                                                         \
        int os_rc_ = (call);                                                                                     \
        if (os_rc_ != OS_OK) return os_rc_;                                                                      \
    } while (0)

// A device allocation that frees itself; alloc() returns a status.
// Grow-only: a request that fits the current capacity reuses the allocation (no free while earlier launches on the
// stream may still read it); a larger one frees (cudaFree waits for the device) and allocates anew.
template <typename T>
struct DeviceArray {
    T *ptr = nullptr;
    size_t count = 0;
    size_t capacity = 0;
    DeviceArray() = default;
    DeviceArray(const DeviceArray &) = delete;
    DeviceArray &operator=(const DeviceArray &) = delete;
    ~DeviceArray() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
        capacity = 0;
    }
    int alloc(size_t n) {
        if (ptr && n <= capacity) {
            count = n;
            return OS_OK;
        }
        release();
        if (n == 0) return OS_OK;
        cudaError_t err = cudaMalloc((void **)&ptr, n * sizeof(T));
        if (err != cudaSuccess) {
            ptr = nullptr;
            set_error("cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(err));
            return err == cudaErrorMemoryAllocation ? OS_ERR_NO_MEMORY : OS_ERR_CUDA;
        }
        count = n;
        capacity = n;
        return OS_OK;
    }
    size_t bytes() const { return count * sizeof(T); }
};

// Host-to-device copy of `n` elements on `stream` (the host buffer may be reused on return).
template <typename T>
int upload(DeviceArray<T> &dst, const T *src, size_t n, cudaStream_t stream) {
    OS_TRY(dst.alloc(n));
    if (n) OS_CUDA(cudaMemcpyAsync(dst.ptr, src, n * sizeof(T), cudaMemcpyHostToDevice, stream));
    return OS_OK;
}

}  // namespace os
