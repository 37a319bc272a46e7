// Device memory pools and the pinned host cache behind workspaces.
#include "pool.h"

#include <cstdint>
#include <map>
#include <mutex>

namespace fpb {
namespace {

struct DevicePool {
    std::mutex mu;
    bool ready = false;
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;  // allocations, set-up work and frees, in order
};

constexpr int kMaxDevices = 64;
DevicePool g_pools[kMaxDevices];

std::mutex g_pin_mu;
std::multimap<size_t, void *> g_pin_free;  // size class -> cached block
size_t g_pin_cached = 0;
constexpr size_t kPinKeep = size_t(1) << 30;  // pinned bytes kept for reuse

struct Current {
    int prev = -1;
    explicit Current(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~Current() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// Creates the device's pool (memory kept across synchronisations) and its
// stream; the caller holds dp.mu with `device` current.
cudaError_t ensure(DevicePool &dp, int device) {
    if (dp.ready) return cudaSuccess;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaError_t e = cudaMemPoolCreate(&dp.pool, &props);
    if (e != cudaSuccess) {
        dp.pool = nullptr;
        return e;
    }
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(dp.pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&dp.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        if (dp.stream) cudaStreamDestroy(dp.stream);
        cudaMemPoolDestroy(dp.pool);
        dp.stream = nullptr;
        dp.pool = nullptr;
        return e;
    }
    dp.ready = true;
    return cudaSuccess;
}

size_t pin_class(size_t bytes) {
    size_t c = 4096;
    while (c < bytes) c <<= 1;
    return c;
}

}  // namespace

cudaError_t pool_alloc(int device, size_t bytes, void **p, const std::function<cudaError_t(cudaStream_t)> &init) {
    *p = nullptr;
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    Current cur(device);
    DevicePool &dp = g_pools[device];
    std::lock_guard<std::mutex> lk(dp.mu);
    cudaError_t e = ensure(dp, device);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(p, bytes ? bytes : 256, dp.pool, dp.stream);
    if (e != cudaSuccess) *p = nullptr;
    if (e == cudaSuccess && init) e = init(dp.stream);
    if (dp.ready) {
        const cudaError_t e2 = cudaStreamSynchronize(dp.stream);
        if (e == cudaSuccess) e = e2;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (*p) {
            cudaFreeAsync(*p, dp.stream);
            cudaStreamSynchronize(dp.stream);
            *p = nullptr;
        }
    }
    return e;
}

void pool_free(int device, void *p) {
    if (!p || device < 0 || device >= kMaxDevices) return;
    Current cur(device);
    DevicePool &dp = g_pools[device];
    std::lock_guard<std::mutex> lk(dp.mu);
    if (!dp.ready) return;
    cudaFreeAsync(p, dp.stream);
    cudaGetLastError();
}

void *pinned_take(size_t bytes) {
    const size_t c = pin_class(bytes);
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        auto it = g_pin_free.find(c);
        if (it != g_pin_free.end()) {
            void *p = it->second;
            g_pin_free.erase(it);
            g_pin_cached -= c;
            return p;
        }
    }
    void *p = nullptr;
    if (cudaHostAlloc(&p, c, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void pinned_give(void *p, size_t bytes) {
    if (!p) return;
    const size_t c = pin_class(bytes);
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        if (g_pin_cached + c <= kPinKeep) {
            g_pin_free.emplace(c, p);
            g_pin_cached += c;
            return;
        }
    }
    cudaFreeHost(p);
}

void pool_release_cached() {
    for (int d = 0; d < kMaxDevices; ++d) {
        DevicePool &dp = g_pools[d];
        std::lock_guard<std::mutex> lk(dp.mu);
        if (!dp.ready) continue;
        Current cur(d);
        cudaStreamSynchronize(dp.stream);
        cudaMemPoolTrimTo(dp.pool, 0);
    }
    std::multimap<size_t, void *> blocks;
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        blocks.swap(g_pin_free);
        g_pin_cached = 0;
    }
    for (auto &kv : blocks) cudaFreeHost(kv.second);
    cudaGetLastError();
}

}  // namespace fpb
