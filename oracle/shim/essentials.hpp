#pragma once
// Clean-room stand-in for the few `essentials` names the reference uses
// (test infrastructure only; the submodule nested in external/bits is absent):
//   timer<clock, duration>: start / stop / elapsed / reset  (util.hpp:82-101,
//                           builder.hpp:127-163, stitch_extmem.hpp:848-915)
//   clock_type
//   generic_saver(std::ostream&).visit(x)   (streaming_color_set_dict.hpp:267)
//   generic_loader, save, load               (declared for completeness)
// Serialization writes PODs as raw bytes, vectors as a u64 length followed by
// the raw elements, and anything else through its own visit(visitor).

#include <chrono>
#include <cstdint>
#include <fstream>
#include <istream>
#include <ostream>
#include <string>
#include <type_traits>
#include <vector>

namespace essentials {

using clock_type = std::chrono::high_resolution_clock;

template <typename ClockType, typename DurationType>
struct timer {
    void start() {
        m_start = ClockType::now();
        m_running = true;
    }
    void stop() {
        if (!m_running) return;
        m_acc += std::chrono::duration_cast<DurationType>(ClockType::now() - m_start);
        m_running = false;
    }
    void reset() {
        m_acc = DurationType::zero();
        m_running = false;
    }
    double elapsed() const {
        DurationType d = m_acc;
        if (m_running) d += std::chrono::duration_cast<DurationType>(ClockType::now() - m_start);
        return (double)d.count();
    }
    double average() const { return elapsed(); }

private:
    typename ClockType::time_point m_start{};
    DurationType m_acc = DurationType::zero();
    bool m_running = false;
};

struct generic_saver {
    explicit generic_saver(std::ostream& os) : m_os(os) {}

    template <typename T>
    void visit(T const& x) {
        if constexpr (std::is_trivially_copyable<T>::value) {
            m_os.write(reinterpret_cast<char const*>(&x), sizeof(T));
        } else {
            const_cast<T&>(x).visit(*this);
        }
    }
    template <typename T, typename A>
    void visit(std::vector<T, A> const& v) {
        const uint64_t n = v.size();
        m_os.write(reinterpret_cast<char const*>(&n), sizeof(n));
        if constexpr (std::is_trivially_copyable<T>::value) {
            if (n) m_os.write(reinterpret_cast<char const*>(v.data()), (std::streamsize)(n * sizeof(T)));
        } else {
            for (auto const& e : v) visit(e);
        }
    }

private:
    std::ostream& m_os;
};

struct generic_loader {
    explicit generic_loader(std::istream& is) : m_is(is) {}

    template <typename T>
    void visit(T& x) {
        if constexpr (std::is_trivially_copyable<T>::value) {
            m_is.read(reinterpret_cast<char*>(&x), sizeof(T));
        } else {
            x.visit(*this);
        }
    }
    template <typename T, typename A>
    void visit(std::vector<T, A>& v) {
        uint64_t n = 0;
        m_is.read(reinterpret_cast<char*>(&n), sizeof(n));
        v.resize(n);
        if constexpr (std::is_trivially_copyable<T>::value) {
            if (n) m_is.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(T)));
        } else {
            for (auto& e : v) visit(e);
        }
    }

private:
    std::istream& m_is;
};

template <typename T>
void save(T& x, char const* filename) {
    std::ofstream os(filename, std::ios::binary);
    generic_saver s(os);
    s.visit(x);
}

template <typename T>
void load(T& x, char const* filename) {
    std::ifstream is(filename, std::ios::binary);
    generic_loader l(is);
    l.visit(x);
}

}  // namespace essentials
