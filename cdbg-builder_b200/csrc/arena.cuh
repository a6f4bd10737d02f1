// Device memory arena: bump allocation over cached cudaMalloc chunks.
//
// One arena lives in each engine.  A build allocates everything from it and
// resets it at the end, so steady-state builds do no cudaMalloc at all.
// mark()/release() give stack-scoped temporaries inside a build.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <utility>
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
        // 3. a new chunk; on failure give back the free chunks and retry exact
        size_t sz = bytes > m_chunk_bytes ? bytes : m_chunk_bytes;
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, sz);
        if (e != cudaSuccess) {
            cudaGetLastError();
            while (m_chunks.size() > next) {
                cudaFree(m_chunks.back().ptr);
                m_chunks.pop_back();
            }
            sz = bytes;
            e = cudaMalloc(&p, sz);
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
    size_t m_chunk_bytes = size_t(4) << 30;
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
