// Thread-local error message and the library-wide entry points of opensol_fdtd.h.
#include "common.cuh"

#include <cstring>
#include <map>
#include <mutex>
#include <vector>

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

// ---- device memory pool

struct PoolEvents {
    std::vector<cudaEvent_t> events;
    int refs = 0;   // pooled blocks still waiting on them, plus the releaser until pool_events_done
};

namespace {
struct PoolBlock {
    void *ptr;
    PoolEvents *events;
};
std::mutex g_pool_mutex;
std::map<std::pair<int, size_t>, std::vector<PoolBlock>> g_pool;   // (device, class) -> blocks, last in first out
size_t g_pool_bytes = 0;
constexpr size_t kPoolLimit = (size_t)16 << 30;   // bytes kept per process; beyond it a released block is freed

// drop one reference (g_pool_mutex held); the last one destroys the events
void unref(PoolEvents *e) {
    if (e && --e->refs == 0) {
        for (cudaEvent_t ev : e->events) cudaEventDestroy(ev);
        delete e;
    }
}
}  // namespace

size_t pool_class(size_t bytes) {
    // 1/8-octave classes above 2 KiB (at most 12.5 % slack), multiples of 256 bytes below
    if (bytes <= 2048) return (bytes + 255) / 256 * 256;
    size_t p = 2048;
    while (p * 2 <= bytes) p *= 2;   // p <= bytes < 2 p
    const size_t step = p / 8;
    return (bytes + step - 1) / step * step;
}

PoolEvents *pool_events(const cudaStream_t *streams, int n) {
    PoolEvents *e = new PoolEvents();
    for (int k = 0; k < n; ++k) {
        cudaEvent_t ev;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) continue;
        if (cudaEventRecord(ev, streams[k]) != cudaSuccess) {
            cudaEventDestroy(ev);
            continue;
        }
        e->events.push_back(ev);
    }
    e->refs = 1;
    return e;
}

void pool_events_done(PoolEvents *events) {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    unref(events);
}

void pool_give(int device, void *ptr, size_t cls, PoolEvents *events) {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (g_pool_bytes + cls > kPoolLimit) {
        // over the limit: free it (cudaFree orders itself after the device's work)
        cudaFree(ptr);
        return;
    }
    if (events) ++events->refs;
    g_pool[{device, cls}].push_back(PoolBlock{ptr, events});
    g_pool_bytes += cls;
}

void *pool_take(int device, size_t cls) {
    PoolBlock b{nullptr, nullptr};
    {
        std::lock_guard<std::mutex> lock(g_pool_mutex);
        auto it = g_pool.find({device, cls});
        if (it == g_pool.end() || it->second.empty()) return nullptr;
        b = it->second.back();
        it->second.pop_back();
        g_pool_bytes -= cls;
    }
    // the previous owner's last work on the block has finished before it is handed out again
    if (b.events)
        for (cudaEvent_t ev : b.events->events) cudaEventSynchronize(ev);
    {
        std::lock_guard<std::mutex> lock(g_pool_mutex);
        unref(b.events);
    }
    return b.ptr;
}

int pool_trim() {
    std::vector<PoolBlock> blocks;
    {
        std::lock_guard<std::mutex> lock(g_pool_mutex);
        for (auto &kv : g_pool)
            for (auto &b : kv.second) blocks.push_back(b);
        g_pool.clear();
        g_pool_bytes = 0;
    }
    for (auto &b : blocks) {
        if (b.events)
            for (cudaEvent_t ev : b.events->events) cudaEventSynchronize(ev);
        cudaFree(b.ptr);
    }
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    for (auto &b : blocks) unref(b.events);
    return OS_OK;
}

}  // namespace os

extern "C" int os_fdtd_pool_trim(void) { return os::pool_trim(); }

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
