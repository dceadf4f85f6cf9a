// sm_pool.cu -- cache of the handles' large device arrays and of pinned host
// staging buffers (no counterpart in the reference, which allocates and
// frees every array once per program run).
//
// A request loop or a caller that runs shot after shot creates and destroys
// handles of the same sizes over and over; cudaMalloc / cudaFree of a
// gigabyte of wavefields each time costs tens of milliseconds and
// synchronises the device.  The state arrays of a handle (wavefields, CPML
// memory variables, split parts, materials) are therefore taken from and
// given back to a per-device cache of blocks, matched by size rounded up to
// 2 MiB.  A block is given back only when its handle is destroyed, after the
// handle's streams have finished, so no work in flight can still use it.
// The cache keeps at most a set number of bytes per device (sm_pool_set_limit;
// 32 GiB by default) and is emptied by sm_pool_trim, or when an allocation
// fails (then the allocation is tried once more).
#include <map>
#include <mutex>

#include "sm_common.cuh"

namespace sm {
namespace {

constexpr size_t kGran = (size_t)2 << 20;
constexpr int kMaxDev = 64;

struct DevicePool {
    std::multimap<size_t, void *> free_blocks;
    size_t cached = 0;
    size_t limit = (size_t)32 << 30;
};

std::mutex g_mu;
DevicePool g_pools[kMaxDev];
std::multimap<size_t, void *> g_pinned;   // pinned host blocks by size
size_t g_pinned_cached = 0;
constexpr size_t kPinnedLimit = (size_t)4 << 30;

size_t trim_locked(int device) {
    DevicePool &p = g_pools[device];
    size_t freed = 0;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != device) cudaSetDevice(device);
    for (auto &kv : p.free_blocks) {
        cudaFree(kv.second);
        freed += kv.first;
    }
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    p.free_blocks.clear();
    p.cached = 0;
    return freed;
}

}  // namespace

size_t pool_round(size_t bytes) { return (bytes + kGran - 1) / kGran * kGran; }

int pool_get(int device, size_t bytes, void **out) {
    *out = nullptr;
    if (device < 0 || device >= kMaxDev) return sm_fail(SM_EINVAL, "pool: device %d", device);
    bytes = pool_round(bytes);
    {
        std::lock_guard<std::mutex> lk(g_mu);
        DevicePool &p = g_pools[device];
        auto it = p.free_blocks.find(bytes);
        if (it != p.free_blocks.end()) {
            *out = it->second;
            p.cached -= bytes;
            p.free_blocks.erase(it);
            return SM_OK;
        }
    }
    cudaError_t e = cudaMalloc(out, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        {
            std::lock_guard<std::mutex> lk(g_mu);
            trim_locked(device);
        }
        e = cudaMalloc(out, bytes);
        if (e != cudaSuccess) {
            *out = nullptr;
            cudaGetLastError();
            return sm_fail(SM_ENOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes,
                           cudaGetErrorString(e));
        }
    }
    return SM_OK;
}

void pool_put(int device, void *ptr, size_t bytes) {
    if (!ptr) return;
    bytes = pool_round(bytes);
    std::lock_guard<std::mutex> lk(g_mu);
    DevicePool &p = g_pools[device];
    if (p.cached + bytes > p.limit) {
        int prev = -1;
        cudaGetDevice(&prev);
        if (prev != device) cudaSetDevice(device);
        cudaFree(ptr);
        if (prev >= 0 && prev != device) cudaSetDevice(prev);
        return;
    }
    p.free_blocks.emplace(bytes, ptr);
    p.cached += bytes;
}

int pinned_get(size_t bytes, void **out) {
    bytes = pool_round(bytes);
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_pinned.lower_bound(bytes);
        if (it != g_pinned.end() && it->first <= 2 * bytes) {
            *out = it->second;
            g_pinned_cached -= it->first;
            g_pinned.erase(it);
            return SM_OK;
        }
    }
    if (cudaMallocHost(out, bytes) != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return sm_fail(SM_ENOMEM, "cudaMallocHost(%zu bytes) failed", bytes);
    }
    return SM_OK;
}

void pinned_put(void *ptr, size_t bytes) {
    if (!ptr) return;
    bytes = pool_round(bytes);
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_pinned_cached + bytes > kPinnedLimit) {
        cudaFreeHost(ptr);
        return;
    }
    g_pinned.emplace(bytes, ptr);
    g_pinned_cached += bytes;
}

}  // namespace sm

extern "C" int sm_pool_trim(int device, size_t *freed) {
    if (device < 0 || device >= sm::kMaxDev) return sm_fail(SM_EINVAL, "sm_pool_trim: device %d", device);
    std::lock_guard<std::mutex> lk(sm::g_mu);
    const size_t f = sm::trim_locked(device);
    if (freed) *freed = f;
    return SM_OK;
}

extern "C" int sm_pool_set_limit(int device, size_t bytes) {
    if (device < 0 || device >= sm::kMaxDev)
        return sm_fail(SM_EINVAL, "sm_pool_set_limit: device %d", device);
    std::lock_guard<std::mutex> lk(sm::g_mu);
    sm::g_pools[device].limit = bytes;
    if (sm::g_pools[device].cached > bytes) sm::trim_locked(device);
    return SM_OK;
}

extern "C" int sm_pool_cached(int device, size_t *bytes) {
    if (device < 0 || device >= sm::kMaxDev || !bytes)
        return sm_fail(SM_EINVAL, "sm_pool_cached: bad argument");
    std::lock_guard<std::mutex> lk(sm::g_mu);
    *bytes = sm::g_pools[device].cached;
    return SM_OK;
}
