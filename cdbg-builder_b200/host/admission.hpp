// Admission gate of the build server: device-memory reservations against a
// budget, after the reference's bucket-process gate
// (phase2_bucket_process/bucket_walker.hpp:631-671): a unit of work is
// admitted while the reserved total plus its own estimate stays within the
// budget, and one unit is always admitted when nothing runs, so a request
// larger than the budget still makes progress (alone).
//
// Requests are taken in arrival order; a request that does not fit yet waits
// and blocks the ones behind it (no overtaking), so every request's wait is
// bounded by the work ahead of it.  Pure host code, no CUDA.
#pragma once

#include <algorithm>
#include <cstdint>
#include <deque>

namespace cdbg::serve {

// Device bytes a build of `seq_bytes` input bases needs: phase 1 holds the
// input, its 2-bit packing, the super-k-mer list and its sort buffers
// (`per_base` bytes per base); phase 2 sizes its bucket batches from what
// is left, with at least `floor` bytes to work in.
struct memory_model {
    double per_base = 24.0;
    uint64_t floor = uint64_t(2) << 30;
    uint64_t need(uint64_t seq_bytes) const { return (uint64_t)(per_base * (double)seq_bytes) + floor; }
};

class admission_gate {
public:
    admission_gate(uint64_t budget, uint32_t slots) : m_budget(budget), m_slots(slots ? slots : 1) {}

    // Enqueue request `id` needing `need` bytes.
    void arrive(uint64_t id, uint64_t need) { m_queue.push_back({id, need}); }

    // Next request to start, if the head of the queue fits now: sets `id`
    // and `grant` (the bytes it may use: its need, or the whole budget when
    // it runs alone above the budget) and reserves them.
    bool admit(uint64_t& id, uint64_t& grant) {
        if (m_queue.empty() || m_running >= m_slots) return false;
        const item h = m_queue.front();
        const uint64_t n = std::min(h.need, m_budget);
        if (m_running > 0 && m_reserved + n > m_budget) return false;
        if (m_running == 0 && h.need > m_budget) {
            grant = m_budget;
        } else {
            grant = n;
        }
        m_queue.pop_front();
        m_reserved += grant;
        ++m_running;
        id = h.id;
        return true;
    }

    // A started request finished and returns its grant.
    void finish(uint64_t grant) {
        m_reserved -= std::min(grant, m_reserved);
        if (m_running) --m_running;
    }

    uint64_t reserved() const { return m_reserved; }
    uint32_t running() const { return m_running; }
    size_t waiting() const { return m_queue.size(); }
    uint64_t budget() const { return m_budget; }

private:
    struct item {
        uint64_t id, need;
    };
    std::deque<item> m_queue;
    uint64_t m_budget;
    uint32_t m_slots;
    uint64_t m_reserved = 0;
    uint32_t m_running = 0;
};

}  // namespace cdbg::serve
