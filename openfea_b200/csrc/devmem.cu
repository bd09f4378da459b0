// Device-memory cache behind every DevBuf of the library.
//
// A context allocates a few dozen buffers (solver vectors, the coarse levels'
// matrices, the learned level, batch vectors) the first time it needs them;
// cudaMalloc / cudaFree of each cost up to milliseconds, which dominated the
// first solve of a fresh context.  Freed blocks are therefore kept per device
// (up to a quarter of the device's memory, at most 32 GB) and handed to
// later requests of a fitting size;
// a block is cached only after the device has finished every queued use of it
// (cudaDeviceSynchronize, the wait cudaFree itself implies).  Sizes are
// rounded (256 B, or 2 MB from 1 MB up) so that contexts of the same problem
// reuse each other's blocks exactly.  ofea_trim_device_memory returns the
// cached blocks to the driver.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <new>

#include "host_pool.cuh"
#include "ofea_internal.cuh"

namespace ofea {
namespace {

// Bytes cached per device: a quarter of the device's memory, at most 32 GB
// (two contexts of a 1.6M-DOF problem and the blocks of earlier ones fit;
// with 8 GB a fresh context of that size found part of its blocks freed).
size_t cache_cap(int dev) {
    size_t fr = 0, total = 0;
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess || (cur != dev && cudaSetDevice(dev) != cudaSuccess) ||
        cudaMemGetInfo(&fr, &total) != cudaSuccess) {
        cudaGetLastError();
        total = size_t(32) << 30;
    }
    if (cur != dev) cudaSetDevice(cur);
    return std::min(size_t(32) << 30, total / 4);
}

struct DeviceCache {
    std::multimap<size_t, void *> free;  // size -> block
    size_t cached = 0;
    size_t cap = 0;  // 0: not yet queried
};

// never destroyed: contexts may be freed during process teardown
struct State {
    std::mutex mu;
    std::map<int, DeviceCache> cache;
};
State &state() {
    static State *s = new State();
    return *s;
}

size_t round_size(size_t bytes) {
    const size_t big = size_t(1) << 20, step = bytes >= big ? (size_t(2) << 20) : 256;
    return (bytes + step - 1) / step * step;
}

}  // namespace

void *dev_alloc(size_t bytes, size_t *got, int *device) {
    const size_t want = round_size(bytes == 0 ? 1 : bytes);
    int dev = 0;
    OFEA_CUDA(cudaGetDevice(&dev));
    *device = dev;
    {
        std::lock_guard<std::mutex> lock(state().mu);
        DeviceCache &c = state().cache[dev];
        auto it = c.free.lower_bound(want);
        if (it != c.free.end() && it->first <= 2 * want) {
            void *p = it->second;
            *got = it->first;
            c.cached -= it->first;
            c.free.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        // give the cached blocks back and try once more
        dev_trim();
        e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            fail(OFEA_ERR_OOM, "cudaMalloc of " + std::to_string(want) + " bytes failed");
        }
    }
    *got = want;
    return p;
}

void dev_free(void *p, size_t bytes, int dev) {
    if (!p) return;
    // the block belongs to `dev`: wait for that device, whichever is current
    int cur = 0;
    const bool have_cur = cudaGetDevice(&cur) == cudaSuccess;
    const bool ok = cudaSetDevice(dev) == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        cudaFree(p);
        if (have_cur) cudaSetDevice(cur);
        return;
    }
    if (have_cur) cudaSetDevice(cur);
    std::lock_guard<std::mutex> lock(state().mu);
    DeviceCache &c = state().cache[dev];
    if (c.cap == 0) c.cap = cache_cap(dev);
    if (c.cached + bytes > c.cap) {
        cudaSetDevice(dev);
        cudaFree(p);
        if (have_cur) cudaSetDevice(cur);
        return;
    }
    c.free.emplace(bytes, p);
    c.cached += bytes;
}

void dev_trim() {
    std::lock_guard<std::mutex> lock(state().mu);
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto &kv : state().cache) {
        if (cudaSetDevice(kv.first) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        cudaDeviceSynchronize();
        for (auto &b : kv.second.free) cudaFree(b.second);
        kv.second.free.clear();
        kv.second.cached = 0;
    }
    cudaSetDevice(cur);
}

}  // namespace ofea

// ------------------------------------------------------ host block cache --
// Large host blocks (host_pool.cuh): kept by rounded size, never returned to
// the allocator until host_cache_trim(), so that the next context's vectors
// land on pages that are already mapped.  Each block is also page-locked
// (cudaHostRegister) when it is first allocated, so the device copies made
// from it (mesh connectivity, coordinates, moduli) run as direct DMA at full
// bus speed instead of through the driver's pageable staging; a block that
// cannot be registered is used as it is.
namespace ofea {
namespace {

constexpr std::size_t kHostSmall = 256u << 10, kHostGrain = 64u << 10, kHostCap = 1ull << 30;

struct HostBlock {
    void *p;
    bool pinned;
};

struct HostCache {
    std::mutex mu;
    std::multimap<std::size_t, HostBlock> free;
    std::map<void *, bool> pinned;  // every large block handed out: registered or not
    std::size_t cached = 0;
};

HostCache &host_cache() {
    static HostCache *h = new HostCache();  // never destroyed: blocks may be freed during exit
    return *h;
}

std::size_t host_round(std::size_t bytes) { return (bytes + kHostGrain - 1) / kHostGrain * kHostGrain; }

void release_block(void *p, bool pinned) {
    if (pinned && cudaHostUnregister(p) != cudaSuccess) cudaGetLastError();
    std::free(p);
}

}  // namespace

void *host_cache_take(std::size_t bytes) {
    if (bytes < kHostSmall) {
        void *p = std::malloc(bytes ? bytes : 1);
        if (!p) throw std::bad_alloc();
        return p;
    }
    const std::size_t r = host_round(bytes);
    HostCache &h = host_cache();
    {
        std::lock_guard<std::mutex> lock(h.mu);
        auto it = h.free.find(r);
        if (it != h.free.end()) {
            HostBlock b = it->second;
            h.free.erase(it);
            h.cached -= r;
            h.pinned[b.p] = b.pinned;
            return b.p;
        }
    }
    void *p = std::aligned_alloc(4096, r);  // r is a multiple of 64 KB
    if (!p) throw std::bad_alloc();
    bool pinned = cudaHostRegister(p, r, cudaHostRegisterDefault) == cudaSuccess;
    if (!pinned) cudaGetLastError();
    std::lock_guard<std::mutex> lock(h.mu);
    h.pinned[p] = pinned;
    return p;
}

void host_cache_give(void *p, std::size_t bytes) {
    if (!p) return;
    if (bytes < kHostSmall) {
        std::free(p);
        return;
    }
    const std::size_t r = host_round(bytes);
    HostCache &h = host_cache();
    std::lock_guard<std::mutex> lock(h.mu);
    bool pinned = false;
    auto it = h.pinned.find(p);
    if (it != h.pinned.end()) {
        pinned = it->second;
        h.pinned.erase(it);
    }
    if (h.cached + r > kHostCap) {
        release_block(p, pinned);
        return;
    }
    h.free.emplace(r, HostBlock{p, pinned});
    h.cached += r;
}

namespace {
struct PinnedCache {
    std::mutex mu;
    std::multimap<std::size_t, void *> free;
};
PinnedCache &pinned_cache() {
    static PinnedCache *c = new PinnedCache();  // never destroyed: blocks may be freed during exit
    return *c;
}
constexpr std::size_t kPinnedGrain = 4096;
}  // namespace

// Small page-locked blocks (flag and scalar buffers of contexts) kept by
// rounded size and handed out again; host_cache_trim() frees them.
void *pinned_take(std::size_t bytes) {
    const std::size_t r = (std::max<std::size_t>(bytes, 1) + kPinnedGrain - 1) / kPinnedGrain * kPinnedGrain;
    PinnedCache &c = pinned_cache();
    {
        std::lock_guard<std::mutex> lock(c.mu);
        auto it = c.free.find(r);
        if (it != c.free.end()) {
            void *p = it->second;
            c.free.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    OFEA_CUDA(cudaMallocHost(&p, r));
    return p;
}

void pinned_give(void *p, std::size_t bytes) {
    if (!p) return;
    const std::size_t r = (std::max<std::size_t>(bytes, 1) + kPinnedGrain - 1) / kPinnedGrain * kPinnedGrain;
    PinnedCache &c = pinned_cache();
    std::lock_guard<std::mutex> lock(c.mu);
    c.free.emplace(r, p);
}

void host_cache_trim() {
    {
        PinnedCache &c = pinned_cache();
        std::lock_guard<std::mutex> lock(c.mu);
        for (auto &kv : c.free)
            if (cudaFreeHost(kv.second) != cudaSuccess) cudaGetLastError();
        c.free.clear();
    }
    HostCache &h = host_cache();
    std::lock_guard<std::mutex> lock(h.mu);
    for (auto &kv : h.free) release_block(kv.second.p, kv.second.pinned);
    h.free.clear();
    h.cached = 0;
}

}  // namespace ofea
