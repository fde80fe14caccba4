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

// Device memory pool.  cudaMalloc maps memory and cudaFree waits for the whole device, so engines that come and go
// while others run (a serving loop) stall everyone.  An engine being destroyed instead gives its arrays to this
// process-wide pool together with events recorded on the streams it used; a new allocation of the same size class
// (1/8 octave) takes a pooled block once those events have fired (normally long before), else calls cudaMalloc.
// os_fdtd_pool_trim frees the pooled blocks.
struct PoolEvents;   // the events a released block waits for (shared by the blocks of one release)
size_t pool_class(size_t bytes);
void *pool_take(int device, size_t cls);                                  // nullptr: none of that class
void pool_give(int device, void *ptr, size_t cls, PoolEvents *events);    // events: from pool_events, or null
PoolEvents *pool_events(const cudaStream_t *streams, int n);              // records one event per stream
void pool_events_done(PoolEvents *events);                                // the releaser's reference, dropped
int pool_trim();

// A device allocation that frees itself; alloc() returns a status.
// Grow-only: a request that fits the current capacity reuses the allocation (no free while earlier launches on the
// stream may still read it); a larger one frees (cudaFree waits for the device) and allocates anew.  New blocks come
// from the pool when it holds one of their size class.  give_to_pool() hands the block to the pool instead of freeing
// it (the caller supplies the events that order its last uses).
template <typename T>
struct DeviceArray {
    T *ptr = nullptr;
    size_t count = 0;
    size_t capacity = 0;
    size_t cls = 0;   // allocated bytes (a pool size class)
    DeviceArray() = default;
    DeviceArray(const DeviceArray &) = delete;
    DeviceArray &operator=(const DeviceArray &) = delete;
    ~DeviceArray() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
        capacity = 0;
        cls = 0;
    }
    void give_to_pool(PoolEvents *events) {
        if (!ptr) return;
        int device = 0;
        cudaGetDevice(&device);
        pool_give(device, ptr, cls, events);
        ptr = nullptr;
        count = 0;
        capacity = 0;
        cls = 0;
    }
    // Room for n elements; a block that is too small is freed first (cudaFree, which waits for the whole device).
    int alloc(size_t n) {
        if (ptr && n <= capacity) {
            count = n;
            return OS_OK;
        }
        release();
        return take(n);
    }
    // The same for an array whose uses are all ordered on `stream`: a block that is too small goes to the pool, to be
    // handed out again once the work queued so far on `stream` has finished, so growing waits for nothing.
    int alloc(size_t n, cudaStream_t stream) {
        if (ptr && n <= capacity) {
            count = n;
            return OS_OK;
        }
        if (ptr) {
            PoolEvents *ev = pool_events(&stream, 1);
            give_to_pool(ev);
            pool_events_done(ev);
        }
        return take(n);
    }
    int take(size_t n) {   // ptr is null here
        if (n == 0) return OS_OK;
        // 256 bytes of slack past the last element: a 16-byte-rounded bulk copy of a row window that ends at the last
        // element of the array stays inside the allocation
        const size_t want = pool_class(n * sizeof(T) + 256);
        int device = 0;
        cudaGetDevice(&device);
        ptr = static_cast<T *>(pool_take(device, want));
        if (!ptr) {
            cudaError_t err = cudaMalloc((void **)&ptr, want);
            if (err != cudaSuccess) {
                ptr = nullptr;
                set_error("cudaMalloc of %zu bytes failed: %s", want, cudaGetErrorString(err));
                return err == cudaErrorMemoryAllocation ? OS_ERR_NO_MEMORY : OS_ERR_CUDA;
            }
        }
        cls = want;
        count = n;
        capacity = (want - 256) / sizeof(T);
        return OS_OK;
    }
    size_t bytes() const { return count * sizeof(T); }
};

// Staging arrays whose last uses are queued on `stream` go to the pool (no host wait, no cudaFree).
template <typename... A>
void give_after(cudaStream_t stream, A &...arrays) {
    PoolEvents *ev = pool_events(&stream, 1);
    (arrays.give_to_pool(ev), ...);
    pool_events_done(ev);
}

// Host-to-device copy of `n` elements on `stream` (the host buffer may be reused on return).
template <typename T>
int upload(DeviceArray<T> &dst, const T *src, size_t n, cudaStream_t stream) {
    OS_TRY(dst.alloc(n, stream));
    if (n) OS_CUDA(cudaMemcpyAsync(dst.ptr, src, n * sizeof(T), cudaMemcpyHostToDevice, stream));
    return OS_OK;
}

}  // namespace os
