// Device memory arena: bump allocation over cached cudaMalloc chunks.
//
// One arena lives in each engine.  A build allocates everything from it and
// resets it at the end, so steady-state builds do no cudaMalloc at all.
// mark()/release() give stack-scoped temporaries inside a build.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "common.cuh"

namespace cdbg {

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

    template <typename T>
    T* alloc(size_t count) {
        return static_cast<T*>(alloc_bytes(count * sizeof(T)));
    }

    void* alloc_bytes(size_t bytes) {
        bytes = (bytes + 255) & ~size_t(255);
        if (bytes == 0) bytes = 256;
        while (m_cur < m_chunks.size()) {
            chunk& c = m_chunks[m_cur];
            if (c.used + bytes <= c.size) {
                void* p = static_cast<char*>(c.ptr) + c.used;
                c.used += bytes;
                track_();
                return p;
            }
            ++m_cur;
            if (m_cur < m_chunks.size()) m_chunks[m_cur].used = 0;
        }
        size_t sz = bytes > m_chunk_bytes ? bytes : m_chunk_bytes;
        void* p = nullptr;
        CDBG_CUDA(cudaMalloc(&p, sz));
        m_chunks.push_back({p, sz, bytes});
        m_cur = m_chunks.size() - 1;
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
    void free_all() {
        for (auto& c : m_chunks) cudaFree(c.ptr);
        m_chunks.clear();
        m_cur = 0;
    }
    size_t reserved_bytes() const {
        size_t s = 0;
        for (auto const& c : m_chunks) s += c.size;
        return s;
    }
    size_t peak_bytes() const { return m_peak; }
    // Bytes held in cached chunks but not handed out (reusable without cudaMalloc).
    size_t cached_free() const {
        size_t s = 0;
        for (size_t i = 0; i < m_chunks.size(); ++i) {
            if (i < m_cur) continue;
            s += m_chunks[i].size - (i == m_cur ? m_chunks[i].used : 0);
        }
        return s;
    }
    void set_chunk_bytes(size_t b) { m_chunk_bytes = b; }

private:
    struct chunk {
        void* ptr;
        size_t size;
        size_t used;
    };
    void track_() {
        size_t s = 0;
        for (size_t i = 0; i <= m_cur && i < m_chunks.size(); ++i)
            s += (i < m_cur) ? m_chunks[i].size : m_chunks[i].used;
        if (s > m_peak) m_peak = s;
    }
    std::vector<chunk> m_chunks;
    size_t m_cur = 0;
    size_t m_chunk_bytes = size_t(1) << 30;
    size_t m_peak = 0;
};

// Growable device array (storage that outlives arena resets: the class
// dictionary across bucket batches, device-resident outputs of a build).
template <typename T>
struct dvec {
    T* p = nullptr;
    size_t n = 0, cap = 0;
    dvec() = default;
    dvec(dvec const&) = delete;
    ~dvec() {
        if (p) cudaFree(p);
    }
    void reserve(size_t c, cudaStream_t st, bool zero_new = false) {
        if (c <= cap) return;
        size_t nc = std::max<size_t>(c, std::max<size_t>(cap * 2, 1024));
        T* q = nullptr;
        CDBG_CUDA(cudaMalloc(&q, nc * sizeof(T)));
        if (n) CDBG_CUDA(cudaMemcpyAsync(q, p, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
        if (zero_new) CDBG_CUDA(cudaMemsetAsync(q + n, 0, (nc - n) * sizeof(T), st));
        CDBG_CUDA(cudaStreamSynchronize(st));
        if (p) cudaFree(p);
        p = q;
        cap = nc;
    }
};

}  // namespace cdbg
