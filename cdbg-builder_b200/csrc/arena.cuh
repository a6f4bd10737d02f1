// Device memory arena: bump allocation over cached chunks that come from the
// device's stream-ordered memory pool (cudaMallocAsync / cudaFreeAsync).
//
// One pair of arenas lives in each engine.  A build allocates everything from
// them and resets them at the end, so steady-state builds allocate nothing.
// mark()/release() give stack-scoped temporaries inside a build.  Chunks that
// an arena gives back (trim, or a memory limit) return to the pool, which
// keeps them (release threshold = unlimited), so another engine on the same
// device takes them again without a device-wide synchronization -- cudaFree
// would synchronize the whole device and stall every other engine.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"

namespace cdbg {

// The device's default memory pool, set once per device to keep freed memory
// cached (a per-process setting: it ends with the process).
inline cudaMemPool_t device_pool(int device) {
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)pools.size() <= device) pools.resize(device + 1, nullptr);
    if (!pools[device]) {
        cudaMemPool_t p = nullptr;
        CDBG_CUDA(cudaDeviceGetDefaultMemPool(&p, device));
        uint64_t keep = UINT64_MAX;
        CDBG_CUDA(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep));
        pools[device] = p;
    }
    return pools[device];
}

// Bytes the pool holds but has not handed out (free for any stream).
inline size_t pool_cached_free(int device) {
    cudaMemPool_t p = device_pool(device);
    uint64_t reserved = 0, used = 0;
    CDBG_CUDA(cudaMemPoolGetAttribute(p, cudaMemPoolAttrReservedMemCurrent, &reserved));
    CDBG_CUDA(cudaMemPoolGetAttribute(p, cudaMemPoolAttrUsedMemCurrent, &used));
    return reserved > used ? (size_t)(reserved - used) : 0;
}

// Device memory a new allocation can still get: free device memory plus what
// the pool caches.
inline size_t device_available(int device) {
    size_t fr = 0, tot = 0;
    CDBG_CUDA(cudaMemGetInfo(&fr, &tot));
    return fr + pool_cached_free(device);
}

class dev_arena {
public:
    dev_arena() = default;
    ~dev_arena() { free_all(); }
    dev_arena(dev_arena const&) = delete;
    dev_arena& operator=(dev_arena const&) = delete;

    struct mark_t {
        size_t chunk;
        size_t used;
    };

    // Stream that chunk allocations and frees are ordered on (the engine's).
    void set_stream(cudaStream_t st) { m_st = st; }

    template <typename T>
    T* alloc(size_t count) {
        return static_cast<T*>(alloc_bytes(count * sizeof(T)));
    }

    void* alloc_bytes(size_t bytes) {
        bytes = (bytes + 255) & ~size_t(255);
        if (bytes == 0) bytes = 256;
        // 1. the current chunk
        if (m_cur < m_chunks.size()) {
            chunk& c = m_chunks[m_cur];
            if (c.used + bytes <= c.size) {
                void* p = static_cast<char*>(c.ptr) + c.used;
                c.used += bytes;
                track_();
                return p;
            }
        }
        // 2. a later chunk that fits (every chunk after the current one is free);
        //    move it right after the current one so no free chunk is skipped
        const size_t next = m_chunks.empty() ? 0 : m_cur + 1;
        for (size_t i = next; i < m_chunks.size(); ++i) {
            if (m_chunks[i].size >= bytes) {
                std::swap(m_chunks[i], m_chunks[next]);
                m_cur = next;
                m_chunks[m_cur].used = bytes;
                track_();
                return m_chunks[m_cur].ptr;
            }
        }
        // 3. a new chunk; within a memory limit, or when the device is short,
        //    the free chunks go back to the pool first and the request is exact
        size_t sz = bytes > m_chunk_bytes ? bytes : m_chunk_bytes;
        if (m_limit && committed_() + sz > m_limit) {
            drop_free_chunks_(next);
            sz = bytes;
            if (committed_() + sz > m_limit)
                throw std::runtime_error("device memory limit exceeded: request " + std::to_string(bytes >> 20) +
                                         " MiB, engine holds " + std::to_string(committed_() >> 20) +
                                         " MiB of a " + std::to_string(m_limit >> 20) + " MiB limit");
        }
        void* p = nullptr;
        cudaError_t e = cudaMallocAsync(&p, sz, m_st);
        if (e != cudaSuccess) {
            cudaGetLastError();
            drop_free_chunks_(next);
            sz = bytes;
            e = cudaMallocAsync(&p, sz, m_st);
            if (e != cudaSuccess) {
                cudaGetLastError();
                size_t fr = 0, tot = 0;
                cudaMemGetInfo(&fr, &tot);
                throw std::runtime_error("device out of memory: request " + std::to_string(bytes >> 20) +
                                         " MiB, free " + std::to_string(fr >> 20) + " MiB of " +
                                         std::to_string(tot >> 20) + " MiB, arena holds " +
                                         std::to_string(reserved_bytes() >> 20) + " MiB");
            }
        }
        m_chunks.insert(m_chunks.begin() + next, chunk{p, sz, bytes});
        m_cur = next;
        track_();
        return p;
    }

    mark_t mark() const {
        if (m_chunks.empty()) return {0, 0};
        return {m_cur, m_chunks[m_cur].used};
    }
    void release(mark_t m) {
        if (m_chunks.empty()) return;
        m_cur = m.chunk;
        m_chunks[m_cur].used = m.used;
        for (size_t i = m_cur + 1; i < m_chunks.size(); ++i) m_chunks[i].used = 0;
    }
    void reset() {
        for (auto& c : m_chunks) c.used = 0;
        m_cur = 0;
    }
    // Return every chunk to the pool (stream-ordered after the work queued on
    // the arena's stream; nothing queued later may use them).
    void free_all() {
        for (auto& c : m_chunks) cudaFreeAsync(c.ptr, m_st);
        m_chunks.clear();
        m_cur = 0;
    }
    // After reset(): give every chunk back to the pool.
    void trim() { free_all(); }
    size_t reserved_bytes() const {
        size_t s = 0;
        for (auto const& c : m_chunks) s += c.size;
        return s;
    }
    size_t peak_bytes() const { return m_peak; }
    void reset_peak() { m_peak = 0; }
    // Bytes held in cached chunks but not handed out (reusable without allocating).
    size_t cached_free() const {
        size_t s = 0;
        for (size_t i = 0; i < m_chunks.size(); ++i) {
            if (i < m_cur) continue;
            s += m_chunks[i].size - (i == m_cur ? m_chunks[i].used : 0);
        }
        return s;
    }
    void set_chunk_bytes(size_t b) { m_chunk_bytes = b; }
    // Cap (0 = none) on the device memory of this arena, a sibling arena and
    // `external` bytes held elsewhere; allocations beyond it throw.
    void set_limit(size_t limit, dev_arena const* sibling = nullptr, size_t external = 0) {
        m_limit = limit;
        m_sibling = sibling;
        m_external = external;
    }
    size_t limit() const { return m_limit; }
    // Bytes that can still be handed out without exceeding the limit.
    size_t headroom() const {
        if (!m_limit) return SIZE_MAX;
        const size_t r = committed_();
        return cached_free() + (m_limit > r ? m_limit - r : 0);
    }

private:
    struct chunk {
        void* ptr;
        size_t size;
        size_t used;
    };
    void drop_free_chunks_(size_t first_free) {
        while (m_chunks.size() > first_free) {
            cudaFreeAsync(m_chunks.back().ptr, m_st);
            m_chunks.pop_back();
        }
    }
    size_t committed_() const {
        return reserved_bytes() + (m_sibling ? m_sibling->reserved_bytes() : 0) + m_external;
    }
    void track_() {
        size_t s = 0;
        for (size_t i = 0; i <= m_cur && i < m_chunks.size(); ++i)
            s += (i < m_cur) ? m_chunks[i].size : m_chunks[i].used;
        if (s > m_peak) m_peak = s;
    }
    std::vector<chunk> m_chunks;
    size_t m_cur = 0;
    size_t m_chunk_bytes = size_t(4) << 30;
    size_t m_peak = 0;
    size_t m_limit = 0;
    dev_arena const* m_sibling = nullptr;
    size_t m_external = 0;
    cudaStream_t m_st = nullptr;
};

// Growable device array (storage that outlives arena resets: the class
// dictionary across bucket batches, device-resident outputs of a build),
// also from the stream-ordered pool.
template <typename T>
struct dvec {
    T* p = nullptr;
    size_t n = 0, cap = 0;
    cudaStream_t st_last = nullptr;
    dvec() = default;
    dvec(dvec const&) = delete;
    ~dvec() { release(); }
    size_t bytes() const { return cap * sizeof(T); }
    void release() {
        if (p) cudaFreeAsync(p, st_last);
        p = nullptr;
        n = cap = 0;
    }
    void reserve(size_t c, cudaStream_t st, bool zero_new = false) {
        if (c <= cap) return;
        size_t nc = std::max<size_t>(c, std::max<size_t>(cap * 2, 1024));
        T* q = nullptr;
        CDBG_CUDA(cudaMallocAsync(&q, nc * sizeof(T), st));
        if (n) CDBG_CUDA(cudaMemcpyAsync(q, p, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
        if (zero_new) CDBG_CUDA(cudaMemsetAsync(q + n, 0, (nc - n) * sizeof(T), st));
        if (p) CDBG_CUDA(cudaFreeAsync(p, st));
        p = q;
        cap = nc;
        st_last = st;
    }
};

}  // namespace cdbg
