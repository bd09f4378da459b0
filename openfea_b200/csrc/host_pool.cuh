// Host-side parallel loops of the library's set-up code (mesh upload checks,
// coarse-level geometry): kHostChunks fixed chunks run on a persistent pool
// of worker threads plus the caller.  Work is split by chunk, never by
// thread, and callers combine per-chunk results in chunk order, so results do
// not depend on the number of cores.
#pragma once
#include <functional>

namespace ofea {

constexpr int kHostChunks = 16;

// Calls f(k) for k = 0 .. kHostChunks-1 and returns when all calls returned.
// f must not throw; calls from several host threads are serialised.
void host_for_chunks(const std::function<void(int)> &f);

// First index of chunk k of [0, n).
inline long chunk_begin(long n, int k) { return n * k / kHostChunks; }

}  // namespace ofea

#include <cstddef>
#include <new>
#include <vector>

namespace ofea {

// Host blocks of 256 KB and more that the library frees are kept (by size,
// rounded up to 64 KB; 1 GB at most) and handed out again, so a new context
// of the same mesh writes to pages already mapped instead of faulting in
// fresh ones.  host_cache_trim() gives them back.
void *host_cache_take(std::size_t bytes);
void host_cache_give(void *p, std::size_t bytes);
void host_cache_trim();

// HVec<T>(n) and resize(n) default-initialize the new elements (no zero
// fill of tens of MB on the caller's thread): every user writes them all.
template <class T>
struct CachedAlloc {
    using value_type = T;
    CachedAlloc() = default;
    template <class U>
    CachedAlloc(const CachedAlloc<U> &) {}
    T *allocate(std::size_t n) { return static_cast<T *>(host_cache_take(n * sizeof(T))); }
    void deallocate(T *p, std::size_t n) { host_cache_give(p, n * sizeof(T)); }
    template <class U>
    void construct(U *p) {
        ::new (static_cast<void *>(p)) U;
    }
    template <class U, class... Args>
    void construct(U *p, Args &&...args) {
        ::new (static_cast<void *>(p)) U(static_cast<Args &&>(args)...);
    }
    template <class U>
    bool operator==(const CachedAlloc<U> &) const { return true; }
    template <class U>
    bool operator!=(const CachedAlloc<U> &) const { return false; }
};

template <class T>
using HVec = std::vector<T, CachedAlloc<T>>;

}  // namespace ofea
