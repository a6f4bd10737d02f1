// C-ABI entry points (include/cdbg_gpu.h): engine lifetime, the two
// drop-in phases over files, and the in-memory whole path.

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <functional>
#include <mutex>
#include <map>
#include <memory>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../host/io.hpp"
#include "cdbg_gpu.h"
#include "engine.cuh"
#include "inflate.cuh"
#include "phase1.cuh"
#include "phase2.cuh"
#include "primitives.cuh"
#include "seed.cuh"

namespace {

thread_local std::string g_last_error;
std::map<const uint64_t*, cdbg::io::seq_batch*> g_owned_batches;  // cdbg_read_sequences buffers

int fail(std::exception const& e) {
    g_last_error = e.what();
    return -1;
}

uint32_t best_m(uint32_t k) {  // minimizer.hpp:65-73
    if (k <= 13) return (k / 2 > k - 4) ? (k / 2) : (k > 4 ? (k - 4) : 1);
    if (k <= 15) return 9;
    if (k <= 21) return 10;
    if (k <= 30) return 11;
    if (k <= 37) return 12;
    if (k <= 42) return 13;
    if (k <= 64) return 14;
    return (k + 2) / 4;
}

uint32_t host_threads(uint32_t t) {
    if (t) return t;
    unsigned h = std::thread::hardware_concurrency();
    return h ? h : 8;
}

void validate(uint32_t k, uint32_t m, uint32_t B) {
    if (k < 2 || k > 63) throw std::runtime_error("k must be in [2, 63]");
    if (m == 0 || m >= k || m > 32 || k - m > 62) throw std::runtime_error("invalid minimizer length m");
    if (B == 0) throw std::runtime_error("num_buckets must be > 0");
}

struct dev_batch {
    cdbg::seq_input in;
};

// Upload (or wrap) a sequence batch.
cdbg::seq_input stage_batch(cdbg_engine* e, cdbg_seq_batch const* b, uint64_t* h2d) {
    cdbg::seq_input in;
    in.nbytes = b->seq_bytes;
    in.num_seqs = b->num_seqs;
    if (b->on_device) {
        in.ascii = reinterpret_cast<uint8_t const*>(b->seq);
        in.seq_off = b->seq_off;
        in.seq_color = b->seq_color;
        return in;
    }
    uint8_t* a = e->A.alloc<uint8_t>(b->seq_bytes + 16);
    uint64_t* so = e->A.alloc<uint64_t>((uint64_t)b->num_seqs + 1);
    uint32_t* sc = e->A.alloc<uint32_t>((uint64_t)b->num_seqs + 1);
    if (b->seq_bytes) CDBG_CUDA(cudaMemcpyAsync(a, b->seq, b->seq_bytes, cudaMemcpyHostToDevice, e->st));
    CDBG_CUDA(cudaMemcpyAsync(so, b->seq_off, 8ull * (b->num_seqs + 1), cudaMemcpyHostToDevice, e->st));
    if (b->num_seqs)
        CDBG_CUDA(cudaMemcpyAsync(sc, b->seq_color, 4ull * b->num_seqs, cudaMemcpyHostToDevice, e->st));
    if (h2d) *h2d += b->seq_bytes + 8ull * (b->num_seqs + 1) + 4ull * b->num_seqs;
    in.ascii = a;
    in.seq_off = so;
    in.seq_color = sc;
    return in;
}

// Apply the engine's memory limit to both arenas for the coming call (after
// their reset): cached memory above the limit is returned first.
void apply_limit(cdbg_engine* e) {
    if (!e->mem_limit) {
        e->A.set_limit(0);
        e->P.set_limit(0);
        return;
    }
    const size_t lim = e->mem_limit;
    if (e->p2.bytes() > lim / 4) e->p2.release();
    const size_t ext = e->p2.bytes();
    if (e->A.reserved_bytes() + e->P.reserved_bytes() + ext > lim) {
        e->A.trim();
        e->P.trim();
    }
    const size_t chunk = std::max<size_t>(size_t(256) << 20, std::min<size_t>(size_t(4) << 30, lim / 8));
    e->A.set_chunk_bytes(chunk);
    e->P.set_chunk_bytes(chunk);
    e->A.set_limit(lim, &e->P, ext);
    e->P.set_limit(lim, &e->A, ext);
}

// Per-call scope: route kernel timing to this engine's profiler and small
// device reads to its mailbox, and fold the recorded launches into its totals
// when the call returns.
struct call_scope {
    cdbg_engine* e;
    cdbg::kernel_profiler* prev_prof;
    cdbg::host_mailbox* prev_mailbox;
    int prev_bits;
    explicit call_scope(cdbg_engine* en)
        : e(en), prev_prof(cdbg::g_prof), prev_mailbox(cdbg::g_mailbox), prev_bits(cdbg::g_radix_bits) {
        cdbg::g_prof = &e->prof;
        cdbg::g_mailbox = &e->mailbox;
        cdbg::g_radix_bits = e->tune.radix_bits == 11 ? 11 : 8;
    }
    ~call_scope() {
        if (e->prof.on) e->prof.resolve();
        cdbg::g_prof = prev_prof;  // calls nest (the autotuner builds through the public entry)
        cdbg::g_mailbox = prev_mailbox;
        cdbg::g_radix_bits = prev_bits;
    }
};

// Host inverse of the hybrid encoder (compact_color_set_dict.hpp:176-222)
// with delta(x) = Elias delta of x + 1, LSB-first.
struct bit_reader {
    std::vector<uint64_t> const& w;
    uint64_t p;
    uint64_t bit() {
        const uint64_t i = p >> 6;
        const uint64_t b = i < w.size() ? (w[i] >> (p & 63)) & 1 : 0;
        ++p;
        return b;
    }
    uint64_t take(uint32_t n) {
        uint64_t v = 0;
        for (uint32_t i = 0; i < n; ++i) v |= bit() << i;
        return v;
    }
    uint64_t delta() {
        uint32_t ll = 0;
        while (!bit()) ++ll;
        const uint64_t L1 = (1ull << ll) | take(ll);
        const uint32_t l = (uint32_t)(L1 - 1);
        return ((1ull << l) | take(l)) - 1;
    }
};
void decode_class_host(std::vector<uint64_t> const& words, uint64_t pos, uint32_t C, std::vector<uint32_t>& out) {
    out.clear();
    bit_reader r{words, pos};
    const uint64_t N = r.delta();
    const uint64_t st = (uint64_t)(0.25 * C), dt = (uint64_t)(0.75 * C);
    if (N == 0) return;
    if (N < st) {
        uint64_t v = r.delta();
        out.push_back((uint32_t)v);
        for (uint64_t i = 1; i < N; ++i) {
            v += r.delta() + 1;
            out.push_back((uint32_t)v);
        }
    } else if (N < dt) {
        for (uint32_t i = 0; i < C; ++i)
            if (r.bit()) out.push_back(i);
    } else {
        std::vector<uint32_t> absent;
        if (C > N) {
            uint64_t v = r.delta();
            absent.push_back((uint32_t)v);
            for (uint64_t i = 1; i < C - N; ++i) {
                v += r.delta() + 1;
                absent.push_back((uint32_t)v);
            }
        }
        size_t a = 0;
        for (uint32_t v = 0; v < C; ++v) {
            if (a < absent.size() && absent[a] == v)
                ++a;
            else
                out.push_back(v);
        }
    }
}

inline uint64_t host_bits64(std::vector<uint64_t> const& w, uint64_t pos) {
    const uint64_t i = pos >> 5;
    const uint32_t s = (uint32_t)(pos & 31) * 2;
    uint64_t lo = w[i] >> s;
    if (s && i + 1 < w.size()) lo |= w[i + 1] << (64 - s);
    return lo;
}

}  // namespace

namespace cdbg {
std::atomic<uint64_t> g_launches{0};
void set_last_error(std::string const& msg) { g_last_error = msg; }
thread_local kernel_profiler* g_prof = nullptr;
thread_local host_mailbox* g_mailbox = nullptr;
thread_local int g_radix_bits = 8;

void check_device_error(cdbg_engine* e, char const* stage) {
    uint32_t v = 0;
    read_small(&v, e->d_err, 4, e->st);
    if (v) {
        CDBG_CUDA(cudaMemsetAsync(e->d_err, 0, 4, e->st));
        throw std::runtime_error(std::string("device error ") + std::to_string(v) + " in " + stage);
    }
}
}  // namespace cdbg

extern "C" {

const char* cdbg_last_error(void) { return g_last_error.c_str(); }
int cdbg_gpu_version(void) { return CDBG_GPU_VERSION; }

int cdbg_read_sequences(const char* const* files, uint32_t num_files, uint32_t first_color,
                        uint32_t threads, cdbg_seq_batch* out) {
    try {
        std::vector<std::string> f(files, files + num_files);
        auto* hb = new cdbg::io::seq_batch();
        try {
            cdbg::io::read_files(f, 0, f.size(), first_color, host_threads(threads), *hb);
        } catch (...) {
            delete hb;
            throw;
        }
        out->seq = hb->seq.data();
        out->seq_bytes = hb->seq.size();
        out->seq_off = hb->off.data();
        out->seq_color = hb->color.data();
        out->num_seqs = (uint32_t)hb->color.size();
        out->on_device = 0;
        g_owned_batches[out->seq_off] = hb;
        return 0;
    } catch (std::exception const& ex) {
        return fail(ex);
    }
}

void cdbg_free_sequences(cdbg_seq_batch* b) {
    if (!b) return;
    auto it = g_owned_batches.find(b->seq_off);
    if (it != g_owned_batches.end()) {
        delete it->second;
        g_owned_batches.erase(it);
    }
    b->seq = nullptr;
    b->seq_off = nullptr;
    b->seq_color = nullptr;
    b->seq_bytes = 0;
    b->num_seqs = 0;
}

int cdbg_engine_create(int device, cdbg_engine** out) {
    try {
        if (!out) throw std::runtime_error("null engine pointer");
        int n = 0;
        CDBG_CUDA(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) throw std::runtime_error("no such CUDA device");
        CDBG_CUDA(cudaSetDevice(device));
        auto* e = new cdbg_engine();
        e->device = device;
        cdbg::device_pool(device);  // configure the pool the arenas draw from
        CDBG_CUDA(cudaStreamCreateWithFlags(&e->own_st, cudaStreamNonBlocking));
        CDBG_CUDA(cudaStreamCreateWithFlags(&e->copy_st, cudaStreamNonBlocking));
        CDBG_CUDA(cudaEventCreateWithFlags(&e->copy_ev, cudaEventDisableTiming));
        e->st = e->own_st;
        e->A.set_stream(e->st);
        e->P.set_stream(e->st);
        CDBG_CUDA(cudaMalloc(&e->d_err, 16));
        CDBG_CUDA(cudaMemset(e->d_err, 0, 16));
        e->mailbox.bytes = size_t(256) << 10;
        CDBG_CUDA(cudaHostAlloc(&e->mailbox.h, e->mailbox.bytes, cudaHostAllocMapped));
        CDBG_CUDA(cudaHostGetDevicePointer(&e->mailbox.d, e->mailbox.h, 0));
        *out = e;
        return 0;
    } catch (std::exception const& ex) {
        return fail(ex);
    }
}

void cdbg_engine_destroy(cdbg_engine* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->st);
    e->A.free_all();
    e->P.free_all();
    e->p2.release();
    cudaStreamSynchronize(e->st);
    if (e->d_err) cudaFree(e->d_err);
    e->prof.resolve();
    if (e->copy_st) {
        cudaStreamSynchronize(e->copy_st);
        cudaStreamDestroy(e->copy_st);
    }
    if (e->copy_ev) cudaEventDestroy(e->copy_ev);
    if (e->own_st) cudaStreamDestroy(e->own_st);
    if (e->mailbox.h) cudaFreeHost(e->mailbox.h);
    delete e;
}

int cdbg_engine_set_stream(cdbg_engine* e, void* stream) {
    if (!e) return -1;
    cudaSetDevice(e->device);
    // memory the engine holds was ordered on the old stream
    if (cudaStreamSynchronize(e->st) != cudaSuccess) {
        g_last_error = "stream synchronize failed";
        return -1;
    }
    e->st = stream ? (cudaStream_t)stream : e->own_st;
    e->A.set_stream(e->st);
    e->P.set_stream(e->st);
    e->p2.set_stream(e->st);
    return 0;
}

int cdbg_engine_trim(cdbg_engine* e) {
    if (!e) {
        g_last_error = "null engine";
        return -1;
    }
    cudaSetDevice(e->device);
    e->A.reset();
    e->P.reset();
    e->have_rs = false;
    e->A.trim();
    e->P.trim();
    e->p2.release();
    return 0;
}

uint64_t cdbg_launch_count(void) { return cdbg::g_launches.load(); }

int cdbg_engine_set_memory_limit(cdbg_engine* e, uint64_t bytes) {
    if (!e) {
        g_last_error = "null engine";
        return -1;
    }
    e->mem_limit = bytes;
    return 0;
}

int cdbg_engine_memory(cdbg_engine* e, uint64_t* reserved, uint64_t* peak) {
    if (!e) {
        g_last_error = "null engine";
        return -1;
    }
    if (reserved) *reserved = e->A.reserved_bytes() + e->P.reserved_bytes() + e->p2.bytes();
    if (peak) *peak = e->A.peak_bytes() + e->P.peak_bytes() + e->p2.bytes();
    e->A.reset_peak();
    e->P.reset_peak();
    return 0;
}

int cdbg_engine_copy_out(cdbg_engine* e, const void* device_src, void* host_dst, uint64_t bytes) {
    try {
        if (!e) throw std::runtime_error("null engine");
        if (bytes == 0) return 0;
        CDBG_CUDA(cudaSetDevice(e->device));
        CDBG_CUDA(cudaMemcpyAsync(host_dst, device_src, bytes, cudaMemcpyDeviceToHost, e->st));
        CDBG_CUDA(cudaStreamSynchronize(e->st));
        return 0;
    } catch (std::exception const& ex) {
        return fail(ex);
    }
}

int cdbg_engine_profile(cdbg_engine* e, int32_t enable) {
    if (!e) return -1;
    e->prof.resolve();
    if (enable) {
        e->prof.totals.clear();
        e->prof.bytes.clear();
    }
    e->prof.on = enable != 0;
    return 0;
}

int cdbg_engine_kernel_bytes(cdbg_engine* e, char* names, uint64_t names_cap, double* bytes, uint32_t cap) {
    if (!e) return -1;
    uint32_t i = 0;
    uint64_t used = 0;
    for (auto const& kv : e->prof.bytes) {
        if (i >= cap) break;
        const uint64_t len = kv.first.size() + 1;
        if (names && used + len <= names_cap) std::memcpy(names + used, kv.first.c_str(), len);
        used += len;
        if (bytes) bytes[i] = kv.second;
        ++i;
    }
    return (int)e->prof.bytes.size();
}

int cdbg_engine_kernel_stats(cdbg_engine* e, char* names, uint64_t names_cap, double* ms,
                             uint64_t* launches, uint32_t cap) {
    if (!e) return -1;
    e->prof.resolve();
    uint32_t i = 0;
    uint64_t used = 0;
    for (auto const& kv : e->prof.totals) {
        if (i >= cap) break;
        const uint64_t len = kv.first.size() + 1;
        if (names && used + len <= names_cap) std::memcpy(names + used, kv.first.c_str(), len);
        used += len;
        if (ms) ms[i] = kv.second.first;
        if (launches) launches[i] = kv.second.second;
        ++i;
    }
    return (int)e->prof.totals.size();
}

int cdbg_gpu_gunzip(cdbg_engine* e, const uint8_t* const* streams, const uint64_t* lens, uint32_t n,
                    uint8_t* const* outs, const uint64_t* out_caps, uint64_t* out_lens, uint32_t* status) {
    if (!e || (n && (!streams || !lens || !outs || !out_caps || !out_lens || !status))) {
        g_last_error = "null argument";
        return -1;
    }
    call_scope scope_(e);
    try {
        CDBG_CUDA(cudaSetDevice(e->device));
        cudaStream_t st = e->st;
        std::vector<uint64_t> meta(4 * (size_t)n + 1, 0);
        uint64_t ti = 0, to = 0;
        for (uint32_t i = 0; i < n; ++i) {
            meta[i] = ti;
            meta[n + i] = lens[i];
            meta[2 * (size_t)n + i] = to;
            meta[3 * (size_t)n + 1 + i] = out_caps[i];
            ti += lens[i];
            to += (out_caps[i] + 15) & ~uint64_t(15);
        }
        meta[3 * (size_t)n] = to;
        std::vector<uint8_t> hin(ti + 64, 0), gz(n, 1);
        for (uint32_t i = 0; i < n; ++i)
            if (lens[i]) std::memcpy(hin.data() + meta[i], streams[i], lens[i]);
        auto mk = e->A.mark();
        uint8_t* d_in = e->A.alloc<uint8_t>(ti + 64);
        uint8_t* d_out = e->A.alloc<uint8_t>(to + 64);
        uint64_t* d_meta = e->A.alloc<uint64_t>(meta.size());
        uint8_t* d_gz = e->A.alloc<uint8_t>(n + 1);
        uint64_t* d_olen = e->A.alloc<uint64_t>(n + 1);
        uint32_t* d_st = e->A.alloc<uint32_t>(n + 1);
        CDBG_CUDA(cudaMemcpyAsync(d_in, hin.data(), hin.size(), cudaMemcpyHostToDevice, st));
        CDBG_CUDA(cudaMemcpyAsync(d_meta, meta.data(), 8 * meta.size(), cudaMemcpyHostToDevice, st));
        CDBG_CUDA(cudaMemcpyAsync(d_gz, gz.data(), n, cudaMemcpyHostToDevice, st));
        cdbg::stream_set ss{d_in, d_meta, d_meta + n, d_gz, d_out, d_meta + 2 * (size_t)n,
                            d_meta + 3 * (size_t)n + 1, d_olen, d_st, n};
        cdbg::inflate_streams(ss, st);
        CDBG_CUDA(cudaMemcpyAsync(out_lens, d_olen, 8ull * n, cudaMemcpyDeviceToHost, st));
        CDBG_CUDA(cudaMemcpyAsync(status, d_st, 4ull * n, cudaMemcpyDeviceToHost, st));
        CDBG_CUDA(cudaStreamSynchronize(st));
        for (uint32_t i = 0; i < n; ++i)
            if (status[i] == cdbg::STREAM_OK && out_lens[i])
                CDBG_CUDA(cudaMemcpyAsync(outs[i], d_out + meta[2 * (size_t)n + i], out_lens[i],
                                          cudaMemcpyDeviceToHost, st));
        CDBG_CUDA(cudaStreamSynchronize(st));
        e->A.release(mk);
        return 0;
    } catch (std::exception const& ex) {
        return fail(ex);
    }
}

int cdbg_gpu_sort_pairs_u64(cdbg_engine* e, uint64_t* keys, uint32_t* vals, uint64_t n) {
    if (!e) {
        g_last_error = "null engine";
        return -1;
    }
    call_scope scope_(e);
    try {
        CDBG_CUDA(cudaSetDevice(e->device));
        e->A.reset();
        cdbg::prim::sort_pairs_u64_exact<uint32_t>(keys, vals, n, e->A, e->st, e->d_err);
        CDBG_CUDA(cudaStreamSynchronize(e->st));
        cdbg::check_device_error(e, "sort");
        return 0;
    } catch (std::exception const& ex) {
        return fail(ex);
    }
}

int cdbg_gpu_dump_supers(cdbg_engine* e, const cdbg_seq_batch* b, uint32_t k, uint32_t m,
                         uint32_t num_buckets, const char* dump_path, uint64_t* n_supers) {
    if (!e) {
        g_last_error = "null engine";
        return -1;
    }
    call_scope scope_(e);
    try {
        if (m == 0) m = best_m(k);
        validate(k, m, num_buckets);
        CDBG_CUDA(cudaSetDevice(e->device));
        e->A.reset();
        apply_limit(e);
        cdbg::seq_input in = stage_batch(e, b, nullptr);
        cdbg::run_table rt;
        cdbg::build_runs(in, k, e->A, e->st, rt, e->A);
        cdbg::super_list sl;
        cdbg::find_supers(rt, k, m, num_buckets, e->A, e->st, sl, e->d_err, e->tune.minimizer_tile);
        cdbg::check_device_error(e, "super-k-mers");
        const uint64_t n = sl.n;
        std::vector<uint64_t> start(n), words(rt.nwords);
        std::vector<uint32_t> len(n), color(n), flags(n), bucket(n);
        if (n) {
            CDBG_CUDA(cudaMemcpyAsync(start.data(), sl.start, 8 * n, cudaMemcpyDeviceToHost, e->st));
            CDBG_CUDA(cudaMemcpyAsync(len.data(), sl.len, 4 * n, cudaMemcpyDeviceToHost, e->st));
            CDBG_CUDA(cudaMemcpyAsync(color.data(), sl.color, 4 * n, cudaMemcpyDeviceToHost, e->st));
            CDBG_CUDA(cudaMemcpyAsync(flags.data(), sl.flags, 4 * n, cudaMemcpyDeviceToHost, e->st));
            CDBG_CUDA(cudaMemcpyAsync(bucket.data(), sl.bucket, 4 * n, cudaMemcpyDeviceToHost, e->st));
            CDBG_CUDA(cudaMemcpyAsync(words.data(), rt.words, 8 * rt.nwords, cudaMemcpyDeviceToHost, e->st));
        }
        CDBG_CUDA(cudaStreamSynchronize(e->st));
        std::FILE* f = std::fopen(dump_path, "wb");
        if (!f) throw std::runtime_error(std::string("cannot open ") + dump_path);
        std::fwrite(&n, 8, 1, f);
        std::vector<uint8_t> pk;
        for (uint64_t i = 0; i < n; ++i) {
            const uint8_t fl = (uint8_t)flags[i];
            std::fwrite(&bucket[i], 4, 1, f);
            std::fwrite(&fl, 1, 1, f);
            std::fwrite(&color[i], 4, 1, f);
            std::fwrite(&len[i], 4, 1, f);
            pk.assign((len[i] + 3) / 4, 0);
            for (uint32_t j = 0; j < len[i]; j += 32) {
                uint64_t w = host_bits64(words, start[i] + j);
                const uint32_t nb = std::min<uint32_t>(32, len[i] - j);
                for (uint32_t q = 0; q < (nb + 3) / 4; ++q) {
                    uint8_t byte = (uint8_t)(w >> (8 * q));
                    const uint32_t valid = std::min<uint32_t>(4, nb - 4 * q);
                    if (valid < 4) byte &= (uint8_t)((1u << (2 * valid)) - 1);
                    pk[j / 4 + q] = byte;
                }
            }
            std::fwrite(pk.data(), 1, pk.size(), f);
        }
        std::fclose(f);
        if (n_supers) *n_supers = n;
        e->A.reset();
        return 0;
    } catch (std::exception const& ex) {
        if (e) e->A.reset();
        return fail(ex);
    }
}

namespace {
bool phase1_from_files(cdbg_engine* e, std::vector<std::string> const& files, uint32_t threads, uint32_t k,
                       uint32_t m, uint32_t B, cdbg::run_table& rt_all, cdbg::super_list& sl_all, uint64_t* h2d,
                       uint64_t* input_bytes, uint32_t color_base = 0, bool packed = true,
                       uint64_t* seq_bytes = nullptr);
}  // namespace

int cdbg_gpu_phase1(cdbg_engine* e, const cdbg_phase1_args* a, cdbg_phase1_stats* s) {
    if (!e) {
        g_last_error = "null engine";
        return -1;
    }
    call_scope scope_(e);
    try {
        auto t0 = std::chrono::steady_clock::now();
        const uint32_t k = a->k;
        const uint32_t m = a->m ? a->m : best_m(k);
        validate(k, m, a->num_buckets);
        CDBG_CUDA(cudaSetDevice(e->device));
        e->A.reset();
        e->P.reset();
        e->have_rs = false;
        apply_limit(e);
        const uint32_t T = host_threads(a->host_threads);
        std::vector<std::string> files(a->files, a->files + a->num_files);
        cdbg::io::bucket_file_set out(a->tmp_dir, a->num_buckets);
        cdbg_phase1_stats st{};
        // chunks of whole files by inflated size: one chunk is one device
        // pass (records are deduplicated within a chunk, the reference's own
        // compaction is per 64 KiB window); the default chunk is a share of
        // the device memory this engine may use
        uint64_t chunk = a->chunk_bytes;
        if (chunk == 0) {
            size_t fr = 0, tot = 0;
            CDBG_CUDA(cudaMemGetInfo(&fr, &tot));
            uint64_t avail = fr + e->A.cached_free() + e->P.cached_free();
            if (e->mem_limit) avail = std::min<uint64_t>(avail, e->mem_limit);
            chunk = std::max<uint64_t>(64ull << 20, avail / 24);
        }
        std::vector<uint64_t> hint(files.size());
        for (size_t i = 0; i < files.size(); ++i) hint[i] = cdbg::io::inflated_size_hint(files[i]);
        if ((uint64_t)a->first_color + a->num_files > 0xffffffffull) throw std::runtime_error("colors past 2^32");
        const bool packed = (uint64_t)a->first_color + a->num_files < (1u << 28);
        double dev_s = 0;
        size_t f0 = 0;
        while (f0 < files.size()) {
            // files [f0, f1): whole files until the byte budget is reached
            size_t f1 = f0;
            uint64_t acc = 0;
            while (f1 < files.size()) {
                if (f1 > f0 && acc + hint[f1] > chunk) break;
                acc += hint[f1];
                ++f1;
            }
            auto td = std::chrono::steady_clock::now();
            e->A.reset();
            e->P.reset();
            std::vector<std::string> cf(files.begin() + f0, files.begin() + f1);
            cdbg::run_table rt;
            cdbg::super_list sl;
            uint64_t inb = 0, nseq = 0;
            // the files are read on host threads while the device already
            // runs phase 1 on the ones read before
            if (!phase1_from_files(e, cf, T, k, m, a->num_buckets, rt, sl, nullptr, &inb, a->first_color + (uint32_t)f0, packed,
                                   &nseq)) {
                // a file inflated past its size hint: read the chunk whole
                e->A.reset();
                e->P.reset();
                cdbg::io::seq_batch hb;
                cdbg::io::read_files(files, f0, f1 - f0, a->first_color + (uint32_t)f0, T, hb);
                inb = hb.input_bytes;
                nseq = hb.seq.size();
                cdbg_seq_batch b{hb.seq.data(), hb.seq.size(), hb.off.data(), hb.color.data(),
                                 (uint32_t)hb.color.size(), 0};
                cdbg::seq_input in = stage_batch(e, &b, nullptr);
                cdbg::build_runs(in, k, e->A, e->st, rt, e->P);
                cdbg::find_supers(rt, k, m, a->num_buckets, e->A, e->st, sl, e->d_err, e->tune.minimizer_tile,
                                  packed);
                CDBG_CUDA(cudaStreamSynchronize(e->st));
            }
            st.input_bytes += inb;
            st.seq_bytes += nseq;
            cdbg::record_set rs;
            cdbg::build_records(rt, sl, k, a->num_buckets, e->A, e->st, rs, e->d_err, e->A);
            cdbg::serialized_buckets sb;
            cdbg::serialize_records(rs, e->A, e->st, sb);
            cdbg::check_device_error(e, "phase 1");
            // the serialized records come back in bucket ranges: host threads
            // compress and append one range while the next is still copying
            std::vector<uint64_t> boff(a->num_buckets + 1);
            CDBG_CUDA(cudaMemcpyAsync(boff.data(), sb.bucket_off, 8ull * (a->num_buckets + 1),
                                      cudaMemcpyDeviceToHost, e->st));
            CDBG_CUDA(cudaStreamSynchronize(e->st));
            uint8_t* raw = (uint8_t*)e->h_frag.ensure(sb.nbytes + 64);
            std::vector<uint32_t> rcut{0};
            const uint64_t per = std::max<uint64_t>(16ull << 20, sb.nbytes / 16);
            for (uint32_t b = 1; b < a->num_buckets; ++b)
                if (boff[b] - boff[rcut.back()] >= per) rcut.push_back(b);
            rcut.push_back(a->num_buckets);
            std::vector<cudaEvent_t> rev(rcut.size() - 1);
            for (auto& x : rev) CDBG_CUDA(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
            for (size_t r = 0; r + 1 < rcut.size(); ++r) {
                const uint64_t lo = boff[rcut[r]], hi = boff[rcut[r + 1]];
                if (hi > lo)
                    CDBG_CUDA(cudaMemcpyAsync(raw + lo, sb.bytes + lo, hi - lo, cudaMemcpyDeviceToHost, e->st));
                CDBG_CUDA(cudaEventRecord(rev[r], e->st));
            }
            dev_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - td).count();
            try {
                for (size_t r = 0; r + 1 < rcut.size(); ++r) {
                    CDBG_CUDA(cudaEventSynchronize(rev[r]));
                    out.append_frames_range(raw, boff.data(), rcut[r], rcut[r + 1], T);
                }
            } catch (...) {
                for (auto& x : rev) cudaEventDestroy(x);
                throw;
            }
            for (auto& x : rev) cudaEventDestroy(x);
            st.n_kmers += rt.n_kmers;
            st.n_supers += sl.n;
            st.n_records += rs.n;
            e->A.reset();
            e->P.reset();
            f0 = f1;
        }
        out.close();
        for (uint64_t u : out.unc_bytes()) st.unc_bytes += u;
        st.comp_bytes = out.comp_bytes();
        if (a->bucket_unc_bytes)
            std::memcpy(a->bucket_unc_bytes, out.unc_bytes().data(), 8ull * a->num_buckets);
        st.seconds_device = dev_s;
        st.seconds_total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (s) *s = st;
        return 0;
    } catch (std::exception const& ex) {
        if (e) e->A.reset();
        return fail(ex);
    }
}

int cdbg_gpu_phase2(cdbg_engine* e, const cdbg_phase2_args* a, cdbg_phase2_stats* s) {
    if (!e) {
        g_last_error = "null engine";
        return -1;
    }
    call_scope scope_(e);
    std::thread reader;
    try {
        auto t0 = std::chrono::steady_clock::now();
        CDBG_CUDA(cudaSetDevice(e->device));
        const uint32_t T = host_threads(a->host_threads);
        const uint32_t B = a->num_buckets;
        if (a->k < 2 || a->k > 63) throw std::runtime_error("k must be in [2, 63]");
        if (B == 0) throw std::runtime_error("num_buckets must be > 0");
        e->A.reset();
        apply_limit(e);
        const std::string dir = a->tmp_dir;
        // buckets in consecutive ranges of at most pass_bytes uncompressed
        // bytes (a bucket larger than that is a range of its own), the
        // reference's bucket-at-a-time admission (bucket_walker.hpp:643-672)
        // at range granularity: a range is read and decompressed on host
        // threads while the device processes the range before it
        const std::vector<uint64_t> unc = cdbg::io::bucket_sizes(dir, B, T);
        uint64_t pass = a->pass_bytes;
        if (pass == 0) {
            size_t fr = 0, tot = 0;
            CDBG_CUDA(cudaMemGetInfo(&fr, &tot));
            uint64_t avail = fr + e->A.cached_free();
            if (e->mem_limit) avail = std::min<uint64_t>(avail, e->mem_limit);
            pass = std::max<uint64_t>(64ull << 20, std::min<uint64_t>(16ull << 30, avail / 16));
        }
        std::vector<uint32_t> rb{0};
        {
            uint64_t acc = 0;
            for (uint32_t b = 0; b < B; ++b) {
                if (b > rb.back() && acc + unc[b] > pass) {
                    rb.push_back(b);
                    acc = 0;
                }
                acc += unc[b];
            }
            rb.push_back(B);
        }
        const size_t nr = rb.size() - 1;
        uint64_t maxr = 0;
        for (size_t i = 0; i < nr; ++i) {
            uint64_t r = 0;
            for (uint32_t b = rb[i]; b < rb[i + 1]; ++b) r += unc[b];
            maxr = std::max(maxr, r);
        }
        uint8_t* hbuf[2] = {(uint8_t*)e->h_bk[0].ensure(maxr + 128), (uint8_t*)e->h_bk[1].ensure(maxr + 128)};
        cdbg::io::bucket_bytes bb[2];
        std::exception_ptr rerr;
        auto read_range = [&](size_t i) {
            try {
                cdbg::io::read_bucket_range(dir, B, rb[i], rb[i + 1], T, [&](uint64_t) { return hbuf[i & 1]; },
                                            bb[i & 1]);
            } catch (...) {
                rerr = std::current_exception();
            }
        };
        std::FILE* ff = std::fopen(a->frag_path, "wb");
        if (!ff) throw std::runtime_error(std::string("cannot open frag spill: ") + a->frag_path);
        struct file_closer {
            std::FILE*& f;
            ~file_closer() {
                if (f) std::fclose(f);
            }
        } fc{ff};
        cdbg_phase2_stats st{};
        cdbg::phase2_result res;
        double dev_s = 0;
        read_range(0);
        for (size_t i = 0; i < nr; ++i) {
            if (reader.joinable()) reader.join();
            if (rerr) std::rethrow_exception(rerr);
            if (i + 1 < nr) reader = std::thread(read_range, i + 1);
            auto td = std::chrono::steady_clock::now();
            cdbg::io::bucket_bytes& cb = bb[i & 1];
            e->A.reset();
            uint8_t* dbytes = e->A.alloc<uint8_t>(cb.nbytes + 64);
            CDBG_CUDA(cudaMemcpyAsync(dbytes, cb.data, cb.nbytes + 64, cudaMemcpyHostToDevice, e->st));
            const uint32_t nch = (uint32_t)cb.chunk_bucket.size();
            uint64_t* dco = e->A.alloc<uint64_t>(nch + 1);
            uint32_t* dcb = e->A.alloc<uint32_t>(nch + 1);
            CDBG_CUDA(cudaMemcpyAsync(dco, cb.chunk_off.data(), 8ull * (nch + 1), cudaMemcpyHostToDevice, e->st));
            if (nch)
                CDBG_CUDA(cudaMemcpyAsync(dcb, cb.chunk_bucket.data(), 4ull * nch, cudaMemcpyHostToDevice, e->st));
            cdbg::record_set rs;
            cdbg::parse_records(dbytes, cb.nbytes, dco, dcb, nch, B, e->A, e->st, rs, e->d_err);
            cdbg::check_device_error(e, "bucket record parse");
            cdbg::phase2_params pp;
            pp.k = a->k;
            pp.num_colors = a->num_colors;
            pp.batch_occ = a->batch_occ ? a->batch_occ : e->tune.batch_occ;
            pp.heavy_colors = e->tune.heavy_colors;
            pp.table_slots_q = e->tune.table_slots_q;
            pp.union_bitmaps = e->tune.union_lists == 0;
            pp.group_bytes = e->tune.table_group_mb ? (uint64_t)e->tune.table_group_mb << 20 : ~0ull;
            pp.to_host = true;
            pp.keep_dict = i > 0;
            pp.copy_dict = i + 1 == nr;
            res.state = &e->p2;
            cdbg::run_phase2(rs, pp, e->A, e->st, e->d_err, res);
            dev_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - td).count();
            // this range's fragments, then (only then) its bucket files go
            if (!res.frag.empty() && std::fwrite(res.frag.data(), 1, res.frag.size(), ff) != res.frag.size())
                throw std::runtime_error(std::string("short write to ") + a->frag_path);
            if (a->delete_consumed) {
                if (std::fflush(ff) != 0) throw std::runtime_error(std::string("short write to ") + a->frag_path);
                cdbg::io::delete_bucket_files(dir, rb[i], rb[i + 1]);
            }
            st.n_records += rs.n;
            st.n_kmers += res.n_occ;
            st.n_distinct += res.n_distinct;
            st.n_fragments += res.n_fragments;
            st.total_seq_bytes += res.total_seq_bytes;
        }
        if (std::fclose(ff) != 0) {
            ff = nullptr;
            throw std::runtime_error(std::string("short write to ") + a->frag_path);
        }
        ff = nullptr;
        if (a->color_sets_path) {
            // the Elias-Fano finalize of the class offsets runs on the device,
            // over the offsets the dictionary holds there
            e->A.reset();
            cdbg::ef_encoded ef;
            cdbg::ef_encode(e->p2.bit_off.p, res.n_classes, res.nbits, e->A, e->st, ef);
            std::vector<uint64_t> lh(ef.low_words + ef.high_words + 1);
            if (ef.low_words)
                CDBG_CUDA(cudaMemcpyAsync(lh.data(), ef.low, 8 * ef.low_words, cudaMemcpyDeviceToHost, e->st));
            if (ef.high_words)
                CDBG_CUDA(cudaMemcpyAsync(lh.data() + ef.low_words, ef.high, 8 * ef.high_words,
                                          cudaMemcpyDeviceToHost, e->st));
            CDBG_CUDA(cudaStreamSynchronize(e->st));
            cdbg::io::write_color_sets_ef(a->color_sets_path, a->num_colors, res.words.data(), res.nbits, ef.n,
                                          ef.l, lh.data(), lh.data() + ef.low_words, ef.high_bits);
        }
        if (a->on_class) {
            std::vector<uint32_t> cls;
            for (uint64_t c = 0; c < res.n_classes; ++c) {
                decode_class_host(res.words, res.offsets[c], a->num_colors, cls);
                a->on_class(a->ctx, cls.data(), cls.size());
            }
        }
        if (s) {
            st.n_color_sets = res.n_classes;
            st.total_integers = res.total_integers;
            st.color_bits = res.nbits;
            st.seconds_device = dev_s;
            st.seconds_total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            st.n_passes = nr;
            *s = st;
        }
        e->A.reset();
        return 0;
    } catch (std::exception const& ex) {
        if (reader.joinable()) reader.join();
        if (e) e->A.reset();
        return fail(ex);
    }
}

namespace {

// Phase 1 of an in-memory build from host sequences, overlapped with the
// upload: the sequence bytes go to the device in pieces on the copy stream,
// and the runs and super-k-mers of each piece are found while the later
// pieces are still in flight.  Pieces end at sequence boundaries, so no run
// spans two of them; all pieces pack into one 2-bit stream, and their
// super-k-mer lists are concatenated in input order (the order the single
// pass produces).
void phase1_pipelined(cdbg_engine* e, cdbg_seq_batch const* b, uint32_t k, uint32_t m, uint32_t B,
                      uint32_t pieces, cdbg::run_table& rt_all, cdbg::super_list& sl_all, uint64_t* h2d) {
    const uint64_t N = b->seq_bytes;
    const uint32_t S = b->num_seqs;
    cudaStream_t st = e->st;
    uint8_t* d_ascii = e->A.alloc<uint8_t>(N + 16);
    uint32_t* d_color = e->A.alloc<uint32_t>((uint64_t)S + 1);
    CDBG_CUDA(cudaMemcpyAsync(d_color, b->seq_color, 4ull * S, cudaMemcpyHostToDevice, st));
    // piece boundaries (sequence indices) near equal byte shares
    std::vector<uint32_t> cut{0};
    for (uint32_t s = 1; s < S && cut.size() < pieces; ++s)
        if (b->seq_off[s] >= (N / pieces) * cut.size()) cut.push_back(s);
    cut.push_back(S);
    const size_t np = cut.size() - 1;
    // every piece's offsets rebased to its first byte, uploaded before the
    // sequence bytes (a small upload queued behind them would stall the host)
    std::vector<uint64_t> off((uint64_t)S + np);
    std::vector<uint64_t> off_at(np);
    {
        uint64_t o = 0;
        for (size_t i = 0; i < np; ++i) {
            off_at[i] = o;
            const uint64_t b0 = b->seq_off[cut[i]];
            for (uint32_t s = cut[i]; s <= cut[i + 1]; ++s) off[o++] = b->seq_off[s] - b0;
        }
    }
    uint64_t* d_off = e->A.alloc<uint64_t>(off.size());
    CDBG_CUDA(cudaMemcpyAsync(d_off, off.data(), 8 * off.size(), cudaMemcpyHostToDevice, st));
    // the copies start after this call's allocations and small uploads (ordered on st)
    CDBG_CUDA(cudaEventRecord(e->copy_ev, st));
    CDBG_CUDA(cudaStreamWaitEvent(e->copy_st, e->copy_ev, 0));
    std::vector<cudaEvent_t> ev(np);
    for (auto& x : ev) CDBG_CUDA(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    for (size_t i = 0; i < np; ++i) {
        const uint64_t b0 = b->seq_off[cut[i]], b1 = b->seq_off[cut[i + 1]];
        if (b1 > b0)
            CDBG_CUDA(cudaMemcpyAsync(d_ascii + b0, b->seq + b0, b1 - b0, cudaMemcpyHostToDevice, e->copy_st));
        CDBG_CUDA(cudaEventRecord(ev[i], e->copy_st));
    }
    // every kept run has >= k bases and is padded to whole words
    const uint64_t cap = N / 32 + N / std::max<uint32_t>(k, 1) + 64 * np + 64;
    uint64_t* words = e->P.alloc<uint64_t>(cap);
    uint64_t base = 0, n_kmers = 0, n_bases = 0;
    std::vector<cdbg::super_list> lists;
    for (size_t i = 0; i < np; ++i) {
        const uint64_t b0 = b->seq_off[cut[i]], b1 = b->seq_off[cut[i + 1]];
        const uint32_t ns = cut[i + 1] - cut[i];
        CDBG_CUDA(cudaStreamWaitEvent(st, ev[i], 0));
        cdbg::seq_input in;
        in.ascii = d_ascii + b0;
        in.nbytes = b1 - b0;
        in.seq_off = d_off + off_at[i];
        in.seq_color = d_color + cut[i];
        in.num_seqs = ns;
        cdbg::run_table rt;
        cdbg::build_runs(in, k, e->A, st, rt, e->P, words, base, cap);
        if (rt.n == 0) continue;
        base = rt.nwords - 8;
        n_kmers += rt.n_kmers;
        n_bases += rt.n_bases;
        cdbg::super_list sl;
        cdbg::find_supers(rt, k, m, B, e->A, st, sl, e->d_err, e->tune.minimizer_tile, true);
        if (sl.n) lists.push_back(sl);
    }
    for (auto& x : ev) cudaEventDestroy(x);
    uint64_t n = 0;
    for (auto const& l : lists) n += l.n;
    if (n >= 0xffffffffull) throw std::runtime_error("more than 2^32 super-k-mers in one call");
    sl_all = cdbg::super_list();
    sl_all.n = n;
    sl_all.key = e->A.alloc<uint64_t>(n + 1);
    sl_all.packed = e->A.alloc<uint4>(n + 1);
    uint64_t o = 0;
    for (auto const& l : lists) {
        CDBG_CUDA(cudaMemcpyAsync(sl_all.key + o, l.key, 8 * l.n, cudaMemcpyDeviceToDevice, st));
        CDBG_CUDA(cudaMemcpyAsync(sl_all.packed + o, l.packed, 16 * l.n, cudaMemcpyDeviceToDevice, st));
        o += l.n;
    }
    rt_all = cdbg::run_table();
    rt_all.words = words;
    rt_all.nwords = base + 8;
    rt_all.n_kmers = n_kmers;
    rt_all.n_bases = n_bases;
    if (h2d) *h2d += N + 8ull * (S + 1) + 4ull * S;
}

// Phase 1 of an in-memory build from files: the files are read (inflate +
// parse, host threads) in groups into the engine's pinned input buffer on a
// reader thread, while each group already read is uploaded (copy stream) and
// runs through build_runs / find_supers; the groups' runs pack into one 2-bit
// stream and their super-k-mer lists concatenate in file order, the order a
// single pass produces.  The buffers are sized from the files' inflated-size
// hints; returns false (nothing launched that matters) when a file inflates
// to more than its hint says, and the caller reads the files whole instead.
// Phase 1 from the files with the device reader: the files' bytes as stored
// go to the device; one warp per gzip file inflates it into the file's region
// of HBM (inflate_streams), the FASTA records are cut in place
// (fasta_compact), and the regions -- one sequence per file, records
// separated by a byte that is not a base -- go through build_runs and
// find_supers like the host reader's sequences, with the same runs.
// Returns false, with nothing kept, when the files do not suit it (no gzip
// file, or, with gpu_inflate = 0, one file holding so much of the input that
// a warp per file is slower than the host threads) or when a stream goes
// back to the host reader.
bool phase1_device_reader(cdbg_engine* e, std::vector<std::string> const& files, uint32_t threads, uint32_t k,
                          uint32_t m, uint32_t B, cdbg::run_table& rt_all, cdbg::super_list& sl_all, uint64_t* h2d,
                          uint64_t* input_bytes, uint32_t color_base, bool packed, uint64_t* seq_bytes) {
    if (e->tune.gpu_inflate == 2) return false;
    const size_t nf = files.size();
    if (nf == 0 || nf >= (1u << 31)) return false;
    std::vector<cdbg::io::file_probe> pr;
    cdbg::io::probe_files(files, threads, pr);
    std::vector<uint64_t> ioff(nf + 1, 0), ooff(nf + 1, 0), ocap(nf);
    std::vector<uint8_t> gz(nf);
    uint64_t max_out = 0;
    bool any_gz = false;
    for (size_t i = 0; i < nf; ++i) {
        ioff[i + 1] = ioff[i] + pr[i].size;
        ocap[i] = pr[i].gz ? pr[i].hint : pr[i].size;
        ooff[i + 1] = ooff[i] + ((ocap[i] + 15) & ~uint64_t(15));
        gz[i] = pr[i].gz ? 1 : 0;
        any_gz |= pr[i].gz;
        max_out = std::max(max_out, ocap[i]);
    }
    const uint64_t tot_in = ioff[nf], tot_out = ooff[nf];
    if (!any_gz) return false;
    // a warp inflates a few tens of MB/s, a host thread several times that:
    // the device reader wins while no file holds more than about 1/(6T) of
    // the input
    if (e->tune.gpu_inflate == 0 && (double)max_out * 6.0 * threads > (double)tot_out) return false;
    cudaStream_t st = e->st;
    char* h = (char*)e->h_in.ensure(tot_in + 64);
    cdbg::io::read_raw_files(files, threads, h, ioff.data());
    auto ma = e->A.mark();
    auto mp = e->P.mark();
    uint8_t* d_in = e->A.alloc<uint8_t>(tot_in + 64);
    uint8_t* d_out = e->A.alloc<uint8_t>(tot_out + 64);
    // per-file arrays in one upload: in_off, in_len, out_off (nf + 1), out_cap
    std::vector<uint64_t> meta(4 * nf + 1);
    for (size_t i = 0; i < nf; ++i) {
        meta[i] = ioff[i];
        meta[nf + i] = pr[i].size;
        meta[3 * nf + 1 + i] = ocap[i];
    }
    for (size_t i = 0; i <= nf; ++i) meta[2 * nf + i] = ooff[i];
    uint64_t* d_meta = e->A.alloc<uint64_t>(meta.size());
    uint8_t* d_gz = e->A.alloc<uint8_t>(nf);
    uint64_t* d_olen = e->A.alloc<uint64_t>(nf);
    uint64_t* d_sb = e->A.alloc<uint64_t>(nf);
    uint32_t* d_status = e->A.alloc<uint32_t>(nf);
    uint32_t* d_color = e->A.alloc<uint32_t>(nf);
    std::vector<uint32_t> col(nf);
    for (size_t i = 0; i < nf; ++i) col[i] = color_base + (uint32_t)i;
    CDBG_CUDA(cudaMemcpyAsync(d_in, h, tot_in, cudaMemcpyHostToDevice, st));
    CDBG_CUDA(cudaMemcpyAsync(d_meta, meta.data(), 8 * meta.size(), cudaMemcpyHostToDevice, st));
    CDBG_CUDA(cudaMemcpyAsync(d_gz, gz.data(), nf, cudaMemcpyHostToDevice, st));
    CDBG_CUDA(cudaMemcpyAsync(d_color, col.data(), 4 * nf, cudaMemcpyHostToDevice, st));
    cdbg::stream_set ss{d_in,  d_meta,        d_meta + nf, d_gz,     d_out,
                        d_meta + 2 * nf, d_meta + 3 * nf + 1, d_olen, d_status, (uint32_t)nf};
    {
        CDBG_PROF_BYTES("k_inflate", st, (double)tot_in + (double)tot_out);
        cdbg::inflate_streams(ss, st);
    }
    {
        CDBG_PROF_BYTES("k_fasta_compact", st, 2.0 * (double)tot_out);
        cdbg::fasta_compact(ss, d_sb, st);
    }
    std::vector<uint32_t> status(nf);
    std::vector<uint64_t> sb(nf);
    CDBG_CUDA(cudaMemcpyAsync(status.data(), d_status, 4 * nf, cudaMemcpyDeviceToHost, st));
    CDBG_CUDA(cudaMemcpyAsync(sb.data(), d_sb, 8 * nf, cudaMemcpyDeviceToHost, st));
    CDBG_CUDA(cudaStreamSynchronize(st));
    for (size_t i = 0; i < nf; ++i)
        if (status[i] != cdbg::STREAM_OK) {
            e->A.release(ma);
            e->P.release(mp);
            return false;
        }
    cdbg::seq_input in;
    in.ascii = d_out;
    in.nbytes = tot_out;
    in.seq_off = d_meta + 2 * nf;
    in.seq_color = d_color;
    in.num_seqs = (uint32_t)nf;
    const uint64_t cap = tot_out / 32 + tot_out / std::max<uint32_t>(k, 1) + 128;
    uint64_t* words = e->P.alloc<uint64_t>(cap);
    cdbg::run_table rt;
    cdbg::build_runs(in, k, e->A, st, rt, e->P, words, 0, cap);
    if (rt.n == 0) {  // nothing to build from: the host reader's path handles it
        e->A.release(ma);
        e->P.release(mp);
        return false;
    }
    sl_all = cdbg::super_list();
    cdbg::find_supers(rt, k, m, B, e->A, st, sl_all, e->d_err, e->tune.minimizer_tile, packed);
    rt_all = cdbg::run_table();
    rt_all.words = words;
    rt_all.nwords = rt.nwords;
    rt_all.n_kmers = rt.n_kmers;
    rt_all.n_bases = rt.n_bases;
    if (h2d) *h2d += tot_in + 8 * meta.size() + 5 * nf;
    if (input_bytes) *input_bytes = tot_in;
    if (seq_bytes) {
        uint64_t t = 0;
        for (uint64_t v : sb) t += v;
        *seq_bytes = t;
    }
    return true;
}

bool phase1_from_files(cdbg_engine* e, std::vector<std::string> const& files, uint32_t threads, uint32_t k,
                       uint32_t m, uint32_t B, cdbg::run_table& rt_all, cdbg::super_list& sl_all, uint64_t* h2d,
                       uint64_t* input_bytes, uint32_t color_base, bool packed, uint64_t* seq_bytes) {
    if (phase1_device_reader(e, files, threads, k, m, B, rt_all, sl_all, h2d, input_bytes, color_base, packed,
                             seq_bytes))
        return true;
    cudaStream_t st = e->st;
    const size_t nf = files.size();
    uint64_t N = 0;
    for (auto const& f : files) N += cdbg::io::inflated_size_hint(f);
    char* h_in = (char*)e->h_in.ensure(N + 64);
    // groups of consecutive files: enough of them to overlap reading with
    // the device work, few enough that each keeps the reader threads busy
    const size_t ng = std::max<size_t>(1, std::min<size_t>(nf, std::min<uint64_t>(16, N / (32ull << 20) + 1)));
    std::vector<size_t> gfirst(ng + 1);
    for (size_t g = 0; g <= ng; ++g) gfirst[g] = nf * g / ng;
    struct group {
        cdbg::io::seq_batch meta;
        uint64_t at = 0, nbytes = 0;
        int state = 0;  // 0 pending, 1 ready, 2 too large, 3 failed
        std::string err;
    };
    std::vector<group> G(ng);
    std::mutex mu;
    std::condition_variable cv;
    std::atomic<bool> stop{false};
    std::thread reader([&] {
        uint64_t used = 0;
        for (size_t g = 0; g < ng && !stop; ++g) {
            int stt = 1;
            std::string err;
            uint64_t nb = 0;
            try {
                cdbg::io::seq_batch mb;
                if (cdbg::io::read_files_into(files, gfirst[g], gfirst[g + 1] - gfirst[g],
                                              color_base + (uint32_t)gfirst[g], threads, h_in + used, N - used, mb)) {
                    nb = mb.off.back();
                    G[g].meta = std::move(mb);
                } else {
                    stt = 2;
                }
            } catch (std::exception const& ex) {
                stt = 3;
                err = ex.what();
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                G[g].at = used;
                G[g].nbytes = nb;
                G[g].state = stt;
                G[g].err = err;
            }
            cv.notify_all();
            if (stt != 1) break;
            used += nb;
        }
    });
    struct join_on_exit {
        std::thread& t;
        std::atomic<bool>& s;
        ~join_on_exit() {
            s = true;
            if (t.joinable()) t.join();
        }
    } joiner{reader, stop};
    uint8_t* d_ascii = e->A.alloc<uint8_t>(N + 16);
    const uint64_t cap = N / 32 + N / std::max<uint32_t>(k, 1) + 64 * ng + 64;
    uint64_t* words = e->P.alloc<uint64_t>(cap);
    uint64_t base = 0, n_kmers = 0, n_bases = 0, up = 0, inb = 0;
    std::vector<cdbg::super_list> lists;
    cudaEvent_t ev;
    CDBG_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    for (size_t g = 0; g < ng; ++g) {
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return G[g].state != 0; });
        }
        if (G[g].state == 3) {
            cudaEventDestroy(ev);
            throw std::runtime_error(G[g].err);
        }
        if (G[g].state == 2) {
            cudaEventDestroy(ev);
            return false;
        }
        auto const& mb = G[g].meta;
        const uint32_t ns = (uint32_t)mb.color.size();
        inb += mb.input_bytes;
        if (ns == 0 || G[g].nbytes == 0) continue;
        uint64_t* d_off = e->A.alloc<uint64_t>((uint64_t)ns + 1);
        uint32_t* d_col = e->A.alloc<uint32_t>(ns);
        CDBG_CUDA(cudaMemcpyAsync(d_off, mb.off.data(), 8ull * (ns + 1), cudaMemcpyHostToDevice, st));
        CDBG_CUDA(cudaMemcpyAsync(d_col, mb.color.data(), 4ull * ns, cudaMemcpyHostToDevice, st));
        CDBG_CUDA(cudaEventRecord(e->copy_ev, st));
        CDBG_CUDA(cudaStreamWaitEvent(e->copy_st, e->copy_ev, 0));
        CDBG_CUDA(cudaMemcpyAsync(d_ascii + G[g].at, h_in + G[g].at, G[g].nbytes, cudaMemcpyHostToDevice,
                                  e->copy_st));
        CDBG_CUDA(cudaEventRecord(ev, e->copy_st));
        CDBG_CUDA(cudaStreamWaitEvent(st, ev, 0));
        up += G[g].nbytes + 12ull * ns + 8;
        cdbg::seq_input in;
        in.ascii = d_ascii + G[g].at;
        in.nbytes = G[g].nbytes;
        in.seq_off = d_off;
        in.seq_color = d_col;
        in.num_seqs = ns;
        cdbg::run_table rt;
        cdbg::build_runs(in, k, e->A, st, rt, e->P, words, base, cap);
        if (rt.n == 0) continue;
        base = rt.nwords - 8;
        n_kmers += rt.n_kmers;
        n_bases += rt.n_bases;
        cdbg::super_list sl;
        cdbg::find_supers(rt, k, m, B, e->A, st, sl, e->d_err, e->tune.minimizer_tile, packed);
        if (sl.n) lists.push_back(sl);
    }
    cudaEventDestroy(ev);
    if (seq_bytes) {
        uint64_t tot = 0;
        for (auto const& gr : G) tot += gr.nbytes;
        *seq_bytes = tot;
    }
    uint64_t n = 0;
    for (auto const& l : lists) n += l.n;
    if (n >= 0xffffffffull) throw std::runtime_error("more than 2^32 super-k-mers in one call");
    sl_all = cdbg::super_list();
    sl_all.n = n;
    sl_all.key = e->A.alloc<uint64_t>(n + 1);
    if (packed) {
        sl_all.packed = e->A.alloc<uint4>(n + 1);
    } else {
        sl_all.start = e->A.alloc<uint64_t>(n + 1);
        sl_all.len = e->A.alloc<uint32_t>(n + 1);
        sl_all.color = e->A.alloc<uint32_t>(n + 1);
        sl_all.flags = e->A.alloc<uint32_t>(n + 1);
        sl_all.bucket = e->A.alloc<uint32_t>(n + 1);
    }
    uint64_t o = 0;
    for (auto const& l : lists) {
        CDBG_CUDA(cudaMemcpyAsync(sl_all.key + o, l.key, 8 * l.n, cudaMemcpyDeviceToDevice, st));
        if (packed) {
            CDBG_CUDA(cudaMemcpyAsync(sl_all.packed + o, l.packed, 16 * l.n, cudaMemcpyDeviceToDevice, st));
        } else {
            CDBG_CUDA(cudaMemcpyAsync(sl_all.start + o, l.start, 8 * l.n, cudaMemcpyDeviceToDevice, st));
            CDBG_CUDA(cudaMemcpyAsync(sl_all.len + o, l.len, 4 * l.n, cudaMemcpyDeviceToDevice, st));
            CDBG_CUDA(cudaMemcpyAsync(sl_all.color + o, l.color, 4 * l.n, cudaMemcpyDeviceToDevice, st));
            CDBG_CUDA(cudaMemcpyAsync(sl_all.flags + o, l.flags, 4 * l.n, cudaMemcpyDeviceToDevice, st));
            CDBG_CUDA(cudaMemcpyAsync(sl_all.bucket + o, l.bucket, 4 * l.n, cudaMemcpyDeviceToDevice, st));
        }
        o += l.n;
    }
    rt_all = cdbg::run_table();
    rt_all.words = words;
    rt_all.nwords = base + 8;
    rt_all.n_kmers = n_kmers;
    rt_all.n_bases = n_bases;
    if (h2d) *h2d += up;
    if (input_bytes) *input_bytes = inb;
    return true;
}

// Phase 1 of an in-memory build: fills rt / sl (records come after), adding
// the bytes it uploads to *h2d; returns false to make the build start over
// from a host batch (see phase1_from_files).
using phase1_fn = std::function<bool(cdbg::run_table&, cdbg::super_list&, uint64_t*)>;

// An in-memory build (phases 1 + 2 in HBM) with the given phase 1.
int build_core(cdbg_engine* e, const cdbg_build_params* p, phase1_fn const& phase1, cdbg_build_result* r,
               bool* redo) {
    if (!e) {
        g_last_error = "null engine";
        return -1;
    }
    call_scope scope_(e);
    try {
        const uint32_t k = p->k;
        const uint32_t m = p->m ? p->m : best_m(k);
        validate(k, m, p->num_buckets);
        CDBG_CUDA(cudaSetDevice(e->device));
        e->A.reset();
        e->P.reset();
        e->have_rs = false;
        apply_limit(e);
        cdbg_build_result res{};
        cudaEvent_t ev[4];
        for (auto& x : ev) CDBG_CUDA(cudaEventCreate(&x));
        CDBG_CUDA(cudaEventRecord(ev[0], e->st));
        cdbg::run_table rt;
        cdbg::super_list sl;
        if (!phase1(rt, sl, &res.h2d_bytes)) {
            for (auto& x : ev) cudaEventDestroy(x);
            CDBG_CUDA(cudaStreamSynchronize(e->st));
            CDBG_CUDA(cudaStreamSynchronize(e->copy_st));
            e->A.reset();
            e->P.reset();
            if (redo) *redo = true;
            return 0;
        }
        if (p->bucket_hi > p->bucket_lo) {
            if (p->bucket_hi > p->num_buckets) throw std::runtime_error("bucket range beyond num_buckets");
            cdbg::keep_bucket_range(sl, p->num_buckets, p->bucket_lo, p->bucket_hi, e->A, e->st);
        } else if (p->bucket_lo || p->bucket_hi) {
            throw std::runtime_error("empty bucket range");
        }
        cdbg::record_set rs;
        cdbg::build_records(rt, sl, k, p->num_buckets, e->A, e->st, rs, e->d_err, e->P);
        e->last_rs = rs;  // for cdbg_engine_record_bytes (lives in P until the next call)
        e->have_rs = true;
        cdbg::check_device_error(e, "phase 1");
        const uint64_t n_kmers = rt.n_kmers, n_supers = sl.n, n_bases = rt.n_bases;
        e->A.reset();  // phase-1 scratch (staged input, super-k-mers, sort buffers)
        CDBG_CUDA(cudaEventRecord(ev[1], e->st));
        cdbg::phase2_params pp;
        pp.k = k;
        pp.num_colors = p->num_colors;
        pp.batch_occ = p->batch_occ ? p->batch_occ : e->tune.batch_occ;
        pp.heavy_colors = e->tune.heavy_colors;
        pp.table_slots_q = e->tune.table_slots_q;
        pp.union_bitmaps = e->tune.union_lists == 0;
        pp.group_bytes = e->tune.table_group_mb ? (uint64_t)e->tune.table_group_mb << 20 : ~0ull;
        pp.to_host = false;  // outputs accumulate in HBM
        pp.keep_frag_offsets = e->keep_frag_offsets && !p->outputs_to_host;
        e->frag_sink.streamed = 0;
        if (!p->outputs_to_host && e->frag_sink.fn && e->h_frag.p && e->h_frag.cap) {
            // the caller writes each batch's fragments out while later batches
            // run: stream them into the (already large enough, from earlier
            // builds) pinned buffer and tell it
            pp.frag_host = (uint8_t*)e->h_frag.p;
            pp.frag_host_cap = e->h_frag.cap;
            pp.copy_st = e->copy_st;
            pp.copy_ev = e->copy_ev;
            pp.on_frag = e->frag_sink.fn;
            pp.on_frag_ctx = e->frag_sink.ctx;
        }
        if (p->outputs_to_host && e->h_frag.p && e->h_frag.cap) {
            // stream each batch's fragments into the (already large enough,
            // from earlier builds) pinned buffer while phase 2 goes on
            pp.frag_host = (uint8_t*)e->h_frag.p;
            pp.frag_host_cap = e->h_frag.cap;
            pp.copy_st = e->copy_st;
            pp.copy_ev = e->copy_ev;
            if (e->h_words.p && e->h_offsets.p) {
                pp.words_host = (uint64_t*)e->h_words.p;
                pp.words_host_cap = e->h_words.cap / 8;
                pp.offs_host = (uint64_t*)e->h_offsets.p;
                pp.offs_host_cap = e->h_offsets.cap / 8;
            }
        }
        cdbg::phase2_result out;
        out.state = &e->p2;
        cdbg::run_phase2(rs, pp, e->A, e->st, e->d_err, out);
        if (pp.on_frag) e->frag_sink.streamed = out.frag_host_copied;
        const uint64_t nwords = (out.nbits + 63) / 64;
        if (p->outputs_to_host) {
            const bool streamed = pp.frag_host && out.frag_host_copied == out.frag_nbytes;
            if (pp.copy_st) {
                // the compute stream (and the caller's events on it) wait for the copies
                CDBG_CUDA(cudaEventRecord(e->copy_ev, e->copy_st));
                CDBG_CUDA(cudaStreamWaitEvent(e->st, e->copy_ev, 0));
            }
            // a streamed prefix is kept only if its buffer holds the whole output
            const bool w_ok = pp.words_host && 8 * nwords + 8 <= e->h_words.cap;
            const bool o_ok = pp.offs_host && 8 * out.n_classes + 8 <= e->h_offsets.cap;
            if (!streamed || !w_ok || !o_ok)
                CDBG_CUDA(cudaStreamSynchronize(e->copy_st));  // before a buffer may move
            void* hf = streamed ? e->h_frag.p : e->h_frag.ensure(out.frag_nbytes + 8);
            void* hw = w_ok ? e->h_words.p : e->h_words.ensure(8 * nwords + 8);
            void* ho = o_ok ? e->h_offsets.p : e->h_offsets.ensure(8 * out.n_classes + 8);
            if (out.frag_nbytes && !streamed)
                CDBG_CUDA(cudaMemcpyAsync(hf, out.d_frag, out.frag_nbytes, cudaMemcpyDeviceToHost, e->st));
            const uint64_t wfrom = w_ok ? out.words_host_copied : 0;
            if (nwords > wfrom)
                CDBG_CUDA(cudaMemcpyAsync((uint64_t*)hw + wfrom, out.d_words + wfrom, 8 * (nwords - wfrom),
                                          cudaMemcpyDeviceToHost, e->st));
            const uint64_t ofrom = o_ok ? out.offs_host_copied : 0;
            if (out.n_classes > ofrom)
                CDBG_CUDA(cudaMemcpyAsync((uint64_t*)ho + ofrom, out.d_offsets + ofrom, 8 * (out.n_classes - ofrom),
                                          cudaMemcpyDeviceToHost, e->st));
            res.frag_bytes = (const uint8_t*)hf;
            res.class_words = (const uint64_t*)hw;
            res.class_offsets = (const uint64_t*)ho;
            res.d2h_bytes = out.frag_nbytes + 8 * nwords + 8 * out.n_classes;
        } else {
            res.frag_bytes = out.d_frag;
            res.class_words = out.d_words;
            res.class_offsets = out.d_offsets;
        }
        CDBG_CUDA(cudaEventRecord(ev[2], e->st));
        CDBG_CUDA(cudaEventSynchronize(ev[2]));
        CDBG_CUDA(cudaStreamSynchronize(e->st));
        float ms1 = 0, ms2 = 0;
        CDBG_CUDA(cudaEventElapsedTime(&ms1, ev[0], ev[1]));
        CDBG_CUDA(cudaEventElapsedTime(&ms2, ev[1], ev[2]));
        for (auto& x : ev) cudaEventDestroy(x);
        res.ms_phase1 = ms1;
        res.ms_phase2 = ms2;
        res.ms_total = ms1 + ms2;
        res.n_kmers = n_kmers;
        res.n_supers = n_supers;
        res.n_bases = n_bases;
        res.n_records = rs.n;
        res.n_occ = out.n_occ;
        res.n_distinct = out.n_distinct;
        res.n_fragments = out.n_fragments;
        res.total_seq_bytes = out.total_seq_bytes;
        res.n_color_sets = out.n_classes;
        res.total_integers = out.total_integers;
        res.class_bits = out.nbits;
        res.frag_nbytes = out.frag_nbytes;
        *r = res;
        return 0;
    } catch (std::exception const& ex) {
        if (e) e->A.reset();
        return fail(ex);
    }
}

}  // namespace

int cdbg_gpu_build(cdbg_engine* e, const cdbg_seq_batch* b, const cdbg_build_params* p, cdbg_build_result* r) {
    if (!e || !b || !p || !r) {
        g_last_error = "null argument";
        return -1;
    }
    const uint32_t k = p->k;
    const uint32_t m = p->m ? p->m : best_m(k);
    auto ph1 = [&](cdbg::run_table& rt, cdbg::super_list& sl, uint64_t* h2d) {
        const bool packed = p->num_colors < (1u << 28);
        if (!b->on_device && packed && b->num_seqs >= 8 && b->seq_bytes >= (64ull << 20)) {
            phase1_pipelined(e, b, k, m, p->num_buckets, 4, rt, sl, h2d);
        } else {
            cdbg::seq_input in = stage_batch(e, b, h2d);
            cdbg::build_runs(in, k, e->A, e->st, rt, e->P);
            cdbg::find_supers(rt, k, m, p->num_buckets, e->A, e->st, sl, e->d_err, e->tune.minimizer_tile, packed);
        }
        return true;
    };
    return build_core(e, p, ph1, r, nullptr);
}

namespace {
// Writes the fragment file while phase 2 runs: phase 2 streams each batch's
// fragments to the engine's pinned buffer (engine.frag_sink) and this writer,
// on its own thread, writes each range once its copy has completed.
struct frag_file_writer {
    struct item {
        uint64_t off, n;
        cudaEvent_t ev;
    };
    cdbg_engine* e;
    cdbg::io::range_file file;
    uint32_t threads;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<item> q;
    std::vector<cudaEvent_t> events;
    bool done = false;
    std::exception_ptr err;
    std::thread t;

    frag_file_writer(cdbg_engine* en, std::string const& path, uint32_t th) : e(en), file(path), threads(th) {
        t = std::thread([this] { run(); });
    }
    ~frag_file_writer() {
        try {
            drain();
        } catch (...) {
        }
    }
    // phase 2 queued fragment bytes [off, off + n) to the pinned buffer on the
    // copy stream
    static void hook(void* ctx, uint64_t off, uint64_t n) {
        auto* w = static_cast<frag_file_writer*>(ctx);
        cudaEvent_t ev;
        CDBG_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        {
            std::lock_guard<std::mutex> lk(w->mu);
            w->events.push_back(ev);
        }
        CDBG_CUDA(cudaEventRecord(ev, w->e->copy_st));
        {
            std::lock_guard<std::mutex> lk(w->mu);
            w->q.push_back({off, n, ev});
        }
        w->cv.notify_one();
    }
    void run() {
        cudaSetDevice(e->device);
        for (;;) {
            item it;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return done || !q.empty(); });
                if (q.empty()) return;
                it = q.front();
                q.pop_front();
            }
            if (err) continue;
            try {
                CDBG_CUDA(cudaEventSynchronize(it.ev));
                file.write(static_cast<uint8_t const*>(e->h_frag.p) + it.off, it.off, it.n, threads);
            } catch (...) {
                err = std::current_exception();
            }
        }
    }
    // every queued range written (before the pinned buffer may move)
    void drain() {
        {
            std::lock_guard<std::mutex> lk(mu);
            done = true;
        }
        cv.notify_one();
        if (t.joinable()) t.join();
        for (auto ev : events) cudaEventDestroy(ev);
        events.clear();
        if (err) {
            std::exception_ptr x = err;
            err = nullptr;
            std::rethrow_exception(x);
        }
    }
};
}  // namespace

static void seed_pass(cdbg_engine* e, uint8_t const* dF, uint64_t const* dOff, uint64_t nc, cdbg::seed_config const& c,
                      cdbg::io::round0_store& store, std::FILE* cf, char const* closed_path, uint32_t T,
                      cudaEvent_t* ev, cdbg_seed_stats* s);

int cdbg_gpu_build_files(cdbg_engine* e, const cdbg_build_files_args* a, cdbg_build_result* r) {
    if (!e || !a || !r || (!a->files && a->num_files)) {
        g_last_error = "null argument";
        return -1;
    }
    try {
        if (a->num_files == 0) throw std::runtime_error("no input files");
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<std::string> files(a->files, a->files + a->num_files);
        const uint32_t th = host_threads(a->host_threads);
        cdbg_build_params p{};
        p.k = a->k;
        p.m = a->m;
        p.num_buckets = a->num_buckets;
        p.num_colors = a->num_files;
        p.batch_occ = a->batch_occ;
        const bool seed = a->stitch_dir != nullptr;
        if (a->stitch_kmer_bits != 0 && a->stitch_kmer_bits != 64 && a->stitch_kmer_bits != 128)
            throw std::runtime_error("stitch_kmer_bits must be 0, 64 or 128");
        // the round-0 seed reads the fragments where phase 2 leaves them, in HBM
        p.outputs_to_host = a->frag_path || a->color_sets_path || seed ? 0 : 1;
        const uint32_t m = p.m ? p.m : best_m(p.k);
        uint64_t inb = 0;
        auto ph1 = [&](cdbg::run_table& rt, cdbg::super_list& sl, uint64_t* h2d) {
            if (p.num_colors >= (1u << 28)) return false;
            return phase1_from_files(e, files, th, p.k, m, p.num_buckets, rt, sl, h2d, &inb);
        };
        // the fragment file is written batch by batch while phase 2 runs
        std::unique_ptr<frag_file_writer> fw;
        if (a->frag_path) {
            fw.reset(new frag_file_writer(e, a->frag_path, th));
            e->frag_sink.fn = &frag_file_writer::hook;
            e->frag_sink.ctx = fw.get();
        }
        e->keep_frag_offsets = seed;
        struct unhook {
            cdbg_engine* e;
            ~unhook() {
                e->frag_sink.fn = nullptr;
                e->frag_sink.ctx = nullptr;
                e->keep_frag_offsets = false;
            }
        } unhook_{e};
        bool redo = false;
        int rc = build_core(e, &p, ph1, r, &redo);
        if (rc != 0) return rc;
        if (redo) {
            // a file inflated past its size hint: read everything, then build
            cdbg::io::seq_batch hb;
            cdbg::io::read_files(files, 0, files.size(), 0, th, hb);
            inb = hb.input_bytes;
            cdbg_seq_batch b{hb.seq.data(), hb.seq.size(), hb.off.data(), hb.color.data(),
                             (uint32_t)hb.color.size(), 0};
            rc = cdbg_gpu_build(e, &b, &p, r);
            if (rc != 0) return rc;
        }
        const auto t_built = std::chrono::steady_clock::now();
        const uint64_t streamed = fw ? std::min<uint64_t>(e->frag_sink.streamed, r->frag_nbytes) : 0;
        // the pinned fragment buffer may move below unless it holds them all:
        // then the streamed ranges must be written first
        if (fw && streamed < r->frag_nbytes) fw->drain();
        if (!p.outputs_to_host) {
            // outputs are in HBM: the frag bytes, color-set words and the
            // Elias-Fano encoding of the class offsets (made on the device)
            // come to pinned memory and go to the files
            call_scope scope_(e);
            CDBG_CUDA(cudaSetDevice(e->device));
            cdbg::ef_encoded ef;
            const uint64_t nwords = (r->class_bits + 63) / 64;
            if (a->color_sets_path)
                cdbg::ef_encode(r->class_offsets, r->n_color_sets, r->class_bits, e->A, e->st, ef);
            void* hf_before = e->h_frag.p;
            // the fragments come to the host unless only the seed reads them
            const bool frag_out = !seed || a->frag_path;
            // (a buffer that took every fragment stays where the writer reads it)
            uint8_t* hf = !frag_out ? nullptr
                          : fw && streamed == r->frag_nbytes && r->frag_nbytes
                              ? (uint8_t*)e->h_frag.p
                              : (uint8_t*)e->h_frag.ensure(r->frag_nbytes + 8);
            // bytes of hf already holding the fragments (the streamed prefix,
            // unless the buffer just moved)
            const uint64_t have = (void*)hf == hf_before ? streamed : 0;
            uint64_t* hw = (uint64_t*)e->h_words.ensure(8 * nwords + 8);
            uint64_t* hl = (uint64_t*)e->h_offsets.ensure(
                a->color_sets_path ? 8 * (ef.low_words + ef.high_words) + 16 : 8 * r->n_color_sets + 8);
            if (frag_out && r->frag_nbytes > have)
                CDBG_CUDA(cudaMemcpyAsync(hf + have, r->frag_bytes + have, r->frag_nbytes - have,
                                          cudaMemcpyDeviceToHost, e->st));
            if (!a->color_sets_path) {
                // no .color_sets file: the class words and offsets come back
                if (nwords)
                    CDBG_CUDA(cudaMemcpyAsync(hw, r->class_words, 8 * nwords, cudaMemcpyDeviceToHost, e->st));
                if (r->n_color_sets)
                    CDBG_CUDA(cudaMemcpyAsync(hl, r->class_offsets, 8 * r->n_color_sets, cudaMemcpyDeviceToHost,
                                              e->st));
            }
            if (a->color_sets_path) {
                if (nwords)
                    CDBG_CUDA(cudaMemcpyAsync(hw, r->class_words, 8 * nwords, cudaMemcpyDeviceToHost, e->st));
                if (ef.low_words)
                    CDBG_CUDA(cudaMemcpyAsync(hl, ef.low, 8 * ef.low_words, cudaMemcpyDeviceToHost, e->st));
                if (ef.high_words)
                    CDBG_CUDA(cudaMemcpyAsync(hl + ef.low_words, ef.high, 8 * ef.high_words,
                                              cudaMemcpyDeviceToHost, e->st));
            }
            CDBG_CUDA(cudaStreamSynchronize(e->st));
            r->d2h_bytes = (frag_out ? r->frag_nbytes : 0) +
                           (a->color_sets_path ? 8 * (nwords + ef.low_words + ef.high_words)
                                               : 8 * (nwords + r->n_color_sets));
            std::thread cs_writer;
            std::exception_ptr cs_err;
            if (a->color_sets_path)
                cs_writer = std::thread([&] {
                    try {
                        cdbg::io::write_color_sets_ef(a->color_sets_path, a->num_files, hw, r->class_bits,
                                                      ef.n, ef.l, hl, hl + ef.low_words, ef.high_bits);
                    } catch (...) {
                        cs_err = std::current_exception();
                    }
                });
            if (fw) {
                try {
                    fw->drain();  // the streamed ranges are in the file
                    fw->file.write(hf + streamed, streamed, r->frag_nbytes - streamed, th);
                    fw->file.finish(r->frag_nbytes);
                } catch (...) {
                    if (cs_writer.joinable()) cs_writer.join();
                    throw;
                }
            }
            if (cs_writer.joinable()) cs_writer.join();
            if (cs_err) std::rethrow_exception(cs_err);
            r->frag_bytes = hf;
            r->class_words = hw;
            r->class_offsets = a->color_sets_path ? nullptr : hl;  // else in the file, Elias-Fano coded
            e->A.reset();
        }
        if (seed) {
            // round 0 of the stitch from the fragments and record offsets
            // phase 2 left in HBM
            call_scope scope_(e);
            CDBG_CUDA(cudaSetDevice(e->device));
            const auto ts = std::chrono::steady_clock::now();
            cdbg::seed_config c;
            c.k = p.k;
            c.num_buckets = a->stitch_buckets ? a->stitch_buckets : 1024;
            c.wide = a->stitch_kmer_bits ? a->stitch_kmer_bits == 128 : p.k > 31;
            if (c.k > (c.wide ? 63u : 32u)) throw std::runtime_error("k out of range for the k-mer width");
            const uint64_t n = r->n_fragments;
            if (e->p2.frag_off.n != n || (n && !e->p2.frag_off.p))
                throw std::runtime_error("the build kept no fragment record offsets");
            uint64_t* dOff = n ? e->p2.frag_off.p : e->A.alloc<uint64_t>(1);  // room for n + 1 entries
            const uint64_t end = r->frag_nbytes;
            CDBG_CUDA(cudaMemcpyAsync(dOff + n, &end, 8, cudaMemcpyHostToDevice, e->st));
            cdbg::io::round0_store store(a->stitch_dir, c.num_buckets);
            const std::string cp = a->stitch_closed_path ? std::string(a->stitch_closed_path)
                                                         : std::string(a->stitch_dir) + "/stitch_r0_closed.bin";
            std::FILE* cf = std::fopen(cp.c_str(), "wb");
            if (!cf) throw std::runtime_error("cannot open " + cp);
            std::unique_ptr<std::FILE, int (*)(std::FILE*)> cf_guard(cf, [](std::FILE* f) { return std::fclose(f); });
            cudaEvent_t ev[2];
            CDBG_CUDA(cudaEventCreate(&ev[0]));
            CDBG_CUDA(cudaEventCreate(&ev[1]));
            std::unique_ptr<cudaEvent_t, void (*)(cudaEvent_t*)> ev_guard(ev, [](cudaEvent_t* v) {
                cudaEventDestroy(v[0]);
                cudaEventDestroy(v[1]);
            });
            cdbg_seed_stats ss{};
            // passes of at most 2^31 records (the kernels index records in 32
            // bits); the offsets are absolute, so a pass is a slice of them
            constexpr uint64_t PASS = 1ull << 31;
            for (uint64_t i0 = 0; i0 < n || (n == 0 && i0 == 0); i0 += PASS) {
                seed_pass(e, e->p2.frag.p, dOff + i0, std::min(PASS, n - i0), c, store, cf, cp.c_str(), th, ev,
                          &ss);
                e->A.reset();
                if (n == 0) break;
            }
            store.finish(th);
            if (std::fclose(cf_guard.release()) != 0) throw std::runtime_error("close failed on " + cp);
            e->A.reset();
            r->seed_routed = ss.routed;
            r->seed_closed_unitigs = ss.closed_unitigs;
            r->ms_seed = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ts).count();
        }
        (void)inb;
        const auto t_end = std::chrono::steady_clock::now();
        r->ms_outputs = std::chrono::duration<double, std::milli>(t_end - t_built).count();
        r->ms_total = std::chrono::duration<double, std::milli>(t_end - t0).count();
        return 0;
    } catch (std::exception const& ex) {
        if (e) e->A.reset();
        return fail(ex);
    }
}

// One device pass of the stitch's round-0 seed over n records at dF / dOff
// (device): the tigs come back in bucket ranges of ~1/16 of their bytes and
// host threads compress and write one range while the next still copies; the
// closed unitigs follow and go to cf (or to e->h_closed) on their own thread.
static void seed_pass(cdbg_engine* e, uint8_t const* dF, uint64_t const* dOff, uint64_t nc, cdbg::seed_config const& c,
                      cdbg::io::round0_store& store, std::FILE* cf, char const* closed_path, uint32_t T,
                      cudaEvent_t* ev, cdbg_seed_stats* s) {
    std::vector<uint64_t> boff(c.num_buckets + 1);
    CDBG_CUDA(cudaEventRecord(ev[0], e->st));
    cdbg::seed_device_out out;
    cdbg::seed_fragments(dF, dOff, nc, c, e->A, e->st, e->d_err, out);
    CDBG_CUDA(cudaEventRecord(ev[1], e->st));
    CDBG_CUDA(cudaMemcpyAsync(boff.data(), out.bucket_off, 8 * boff.size(), cudaMemcpyDeviceToHost, e->st));
    CDBG_CUDA(cudaStreamSynchronize(e->st));
    float ms = 0;
    CDBG_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    s->ms_device += ms;
    const auto tf = std::chrono::steady_clock::now();
    // the tigs come back in bucket ranges of ~1/16 of their bytes: host
    // threads compress and write one range while the next still copies;
    // the closed unitigs follow and go out on their own thread
    uint8_t* ht = (uint8_t*)e->h_tigs.ensure(out.tig_bytes + 16);
    uint8_t* hc = (uint8_t*)e->h_unitigs.ensure(out.closed_bytes + 16);
    std::vector<uint32_t> cut{0};
    const uint64_t per = std::max<uint64_t>(64ull << 20, out.tig_bytes / 16);
    for (uint32_t b = 1; b < c.num_buckets; ++b)
        if (boff[b] - boff[cut.back()] >= per) cut.push_back(b);
    cut.push_back(c.num_buckets);
    std::vector<cudaEvent_t> rev(cut.size());  // ranges, then the closed unitigs
    for (auto& x : rev) CDBG_CUDA(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    std::unique_ptr<std::vector<cudaEvent_t>, void (*)(std::vector<cudaEvent_t>*)> rev_guard(
        &rev, [](std::vector<cudaEvent_t>* v) {
            for (auto x : *v) cudaEventDestroy(x);
        });
    for (size_t r = 0; r + 1 < cut.size(); ++r) {
        const uint64_t lo = boff[cut[r]], hi = boff[cut[r + 1]];
        if (hi > lo) CDBG_CUDA(cudaMemcpyAsync(ht + lo, out.tigs + lo, hi - lo, cudaMemcpyDeviceToHost, e->st));
        CDBG_CUDA(cudaEventRecord(rev[r], e->st));
    }
    CDBG_CUDA(cudaMemcpyAsync(hc, out.closed, out.closed_bytes, cudaMemcpyDeviceToHost, e->st));
    CDBG_CUDA(cudaEventRecord(rev.back(), e->st));
    bool closed_ok = true;
    cudaError_t closed_err = cudaSuccess;
    std::thread closed_writer([&] {
        closed_err = cudaSetDevice(e->device);
        if (closed_err == cudaSuccess) closed_err = cudaEventSynchronize(rev.back());
        if (closed_err != cudaSuccess) return;
        if (cf)
            closed_ok = !out.closed_bytes || std::fwrite(hc, 1, out.closed_bytes, cf) == out.closed_bytes;
        else
            e->h_closed.insert(e->h_closed.end(), hc, hc + out.closed_bytes);
    });
    try {
        for (size_t r = 0; r + 1 < cut.size(); ++r) {
            CDBG_CUDA(cudaEventSynchronize(rev[r]));
            store.append_range(ht, boff.data(), cut[r], cut[r + 1], T);
        }
    } catch (...) {
        closed_writer.join();
        throw;
    }
    closed_writer.join();
    CDBG_CUDA(closed_err);
    if (!closed_ok) throw std::runtime_error(std::string("short write to ") + closed_path);
    s->ms_files += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tf).count();
    s->routed += out.n_routed;
    s->closed_fragments += out.n_closed;
    s->closed_unitigs += out.n_pieces;
    s->routed_frag_bytes += out.routed_record_bytes;
    s->closed_nbytes += out.closed_bytes;
    ++s->n_passes;
}

int cdbg_gpu_stitch_seed(cdbg_engine* e, const cdbg_seed_args* a, cdbg_seed_stats* s) {
    if (!e || !a || !s || (!a->frags && a->frag_nbytes) || !a->round_dir) {
        g_last_error = "null argument";
        return -1;
    }
    call_scope scope_(e);
    try {
        using clk = std::chrono::steady_clock;
        const auto t0 = clk::now();
        CDBG_CUDA(cudaSetDevice(e->device));
        *s = cdbg_seed_stats();
        if (a->kmer_bits != 0 && a->kmer_bits != 64 && a->kmer_bits != 128)
            throw std::runtime_error("kmer_bits must be 0, 64 or 128");
        cdbg::seed_config c;
        c.k = a->k;
        c.num_buckets = a->num_buckets ? a->num_buckets : 1024;
        c.wide = a->kmer_bits ? a->kmer_bits == 128 : a->k > 31;
        if (c.k < 2 || c.k > (c.wide ? 63u : 32u)) throw std::runtime_error("k out of range for the k-mer width");
        const uint32_t T = host_threads(a->host_threads);
        e->A.reset();
        // fragment bytes per device pass: a pass holds about 3x its bytes
        // (fragments, tigs, closed unitigs, ~80 bytes per fragment)
        uint64_t chunk = a->chunk_bytes;
        if (!chunk) {
            size_t fr = 0, tot = 0;
            CDBG_CUDA(cudaMemGetInfo(&fr, &tot));
            uint64_t avail = fr + e->A.cached_free();
            if (e->mem_limit && e->mem_limit < avail) avail = e->mem_limit;
            chunk = std::max<uint64_t>(avail / 4, 64ull << 20);
        }
        // One pass: the bytes go up on another thread while the records are
        // found (the copy needs no record boundaries).
        const bool one_pass = a->frag_nbytes <= chunk;
        uint8_t* dF1 = nullptr;
        cudaError_t up_err = cudaSuccess;
        std::thread uploader;
        if (one_pass && a->frag_nbytes) {
            dF1 = e->A.alloc<uint8_t>(a->frag_nbytes + 16);
            uploader = std::thread([&] {
                up_err = cudaSetDevice(e->device);
                if (up_err == cudaSuccess) up_err = cudaMemsetAsync(dF1 + a->frag_nbytes, 0, 16, e->st);
                if (up_err == cudaSuccess)
                    up_err = cudaMemcpyAsync(dF1, a->frags, a->frag_nbytes, cudaMemcpyHostToDevice, e->st);
                if (up_err == cudaSuccess) up_err = cudaStreamSynchronize(e->st);
            });
        }
        // record boundaries: the records are variable-length and back to back
        // (into pinned memory the engine keeps: no page faults on later calls,
        // and the upload is a direct copy)
        uint64_t n = 0;
        try {
            n = cdbg::io::frag_record_offsets(
                a->frags, a->frag_nbytes, T,
                [&](uint64_t m) { return (uint64_t*)e->h_rec_off.ensure(8 * m); }, &e->h_rec_parts);
        } catch (...) {
            if (uploader.joinable()) uploader.join();
            throw;
        }
        if (uploader.joinable()) uploader.join();
        CDBG_CUDA(up_err);
        uint64_t const* off = (uint64_t const*)e->h_rec_off.p;
        s->fragments = n;
        s->ms_scan = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
        cdbg::io::round0_store store(a->round_dir, c.num_buckets);
        std::FILE* cf = nullptr;
        if (a->closed_path) {
            cf = std::fopen(a->closed_path, "wb");
            if (!cf) throw std::runtime_error(std::string("cannot open ") + a->closed_path);
        }
        std::unique_ptr<std::FILE, int (*)(std::FILE*)> cf_guard(cf, [](std::FILE* f) { return f ? std::fclose(f) : 0; });
        e->h_closed.clear();
        cudaEvent_t ev[2];
        CDBG_CUDA(cudaEventCreate(&ev[0]));
        CDBG_CUDA(cudaEventCreate(&ev[1]));
        std::unique_ptr<cudaEvent_t, void (*)(cudaEvent_t*)> ev_guard(ev, [](cudaEvent_t* v) {
            cudaEventDestroy(v[0]);
            cudaEventDestroy(v[1]);
        });
        std::vector<uint64_t> loff;
        for (uint64_t i0 = 0; i0 < n;) {
            uint64_t i1 = i0 + 1;
            while (i1 < n && off[i1 + 1] - off[i0] <= chunk) ++i1;
            const uint64_t nc = i1 - i0, bytes = off[i1] - off[i0];
            auto mk = e->A.mark();
            uint8_t* dF = dF1;
            if (!dF) {
                dF = e->A.alloc<uint8_t>(bytes + 16);
                CDBG_CUDA(cudaMemsetAsync(dF + bytes, 0, 16, e->st));
                CDBG_CUDA(cudaMemcpyAsync(dF, a->frags + off[i0], bytes, cudaMemcpyHostToDevice, e->st));
            }
            uint64_t* dOff = e->A.alloc<uint64_t>(nc + 1);
            if (i0 == 0 && i1 == n) {
                CDBG_CUDA(cudaMemcpyAsync(dOff, off, 8 * (nc + 1), cudaMemcpyHostToDevice, e->st));
            } else {
                loff.resize(nc + 1);
                for (uint64_t i = 0; i <= nc; ++i) loff[i] = off[i0 + i] - off[i0];
                CDBG_CUDA(cudaMemcpyAsync(dOff, loff.data(), 8 * (nc + 1), cudaMemcpyHostToDevice, e->st));
            }
            seed_pass(e, dF, dOff, nc, c, store, cf, a->closed_path, T, ev, s);
            e->A.release(mk);
            i0 = i1;
        }
        const auto tf = clk::now();
        store.finish(T);
        s->ms_files += std::chrono::duration<double, std::milli>(clk::now() - tf).count();
        if (cf && std::fclose(cf_guard.release()) != 0)
            throw std::runtime_error(std::string("close failed on ") + a->closed_path);
        s->closed = cf ? nullptr : e->h_closed.data();
        s->round0_bytes = store.raw_bytes();
        s->round0_file_bytes = store.comp_bytes();
        s->ms_total = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
        return 0;
    } catch (std::exception const& ex) {
        return fail(ex);
    }
}

int cdbg_frag_record_offsets(const uint8_t* frags, uint64_t frag_nbytes, uint32_t threads, uint64_t* offsets,
                             uint64_t cap, uint64_t* n_records) {
    if ((!frags && frag_nbytes) || !n_records || (!offsets && cap)) {
        g_last_error = "null argument";
        return -1;
    }
    try {
        std::vector<uint64_t> off;
        cdbg::io::frag_record_offsets(frags, frag_nbytes, off, host_threads(threads));
        *n_records = off.size() - 1;
        if (off.size() <= cap) std::memcpy(offsets, off.data(), 8 * off.size());
        return 0;
    } catch (std::exception const& ex) {
        return fail(ex);
    }
}

int cdbg_engine_record_bytes(cdbg_engine* e, uint64_t* bytes) {
    if (!e || !bytes) {
        g_last_error = "null argument";
        return -1;
    }
    call_scope scope_(e);
    try {
        if (!e->have_rs) throw std::runtime_error("no in-memory build to measure");
        CDBG_CUDA(cudaSetDevice(e->device));
        unsigned long long* d = e->P.alloc<unsigned long long>(1);
        cdbg::record_bytes_async(e->last_rs, d, e->st);
        unsigned long long v = 0;
        CDBG_CUDA(cudaMemcpyAsync(&v, d, sizeof v, cudaMemcpyDeviceToHost, e->st));
        CDBG_CUDA(cudaStreamSynchronize(e->st));
        *bytes = v;
        return 0;
    } catch (std::exception const& ex) {
        return fail(ex);
    }
}

int cdbg_engine_set_tuning(cdbg_engine* e, const cdbg_tuning* t) {
    if (!e || !t) {
        g_last_error = "null argument";
        return -1;
    }
    cdbg_tuning v = *t;
    if (v.minimizer_tile == 0) v.minimizer_tile = 4096;
    if (v.heavy_colors == 0) v.heavy_colors = 64;
    if (v.table_slots_q == 0) v.table_slots_q = 8;
    if (v.minimizer_tile != 1024 && v.minimizer_tile != 2048 && v.minimizer_tile != 4096) {
        g_last_error = "minimizer_tile must be 1024, 2048 or 4096";
        return -1;
    }
    if (v.table_slots_q < 5 || v.table_slots_q > 16) {
        g_last_error = "table_slots_q must be in [5, 16]";
        return -1;
    }
    if (v.union_lists > 1) {
        g_last_error = "union_lists must be 0 or 1";
        return -1;
    }
    if (v.radix_bits == 0) v.radix_bits = 8;
    if (v.radix_bits != 8 && v.radix_bits != 11) {
        g_last_error = "radix_bits must be 8 or 11";
        return -1;
    }
    if (v.gpu_inflate > 2) {
        g_last_error = "gpu_inflate must be 0, 1 or 2";
        return -1;
    }
    e->tune = v;
    return 0;
}

int cdbg_engine_get_tuning(cdbg_engine* e, cdbg_tuning* t) {
    if (!e || !t) {
        g_last_error = "null argument";
        return -1;
    }
    *t = e->tune;
    return 0;
}

int cdbg_engine_autotune(cdbg_engine* e, const cdbg_seq_batch* b, const cdbg_build_params* p, uint32_t rounds,
                         cdbg_tuning* best, double* best_ms) {
    if (!e || !b || !p) {
        g_last_error = "null argument";
        return -1;
    }
    try {
        if (rounds == 0) rounds = 1;
        cdbg_build_params q = *p;
        q.batch_occ = 0;  // the tuned split threshold applies
        q.outputs_to_host = 0;
        // best of `rounds` device times of one configuration
        auto measure = [&](cdbg_tuning const& t) {
            e->tune = t;
            double v = 1e300;
            for (uint32_t r = 0; r < rounds; ++r) {
                cdbg_build_result res{};
                if (cdbg_gpu_build(e, b, &q, &res) != 0) throw std::runtime_error(g_last_error);
                v = std::min(v, res.ms_total);
            }
            return v;
        };
        cdbg_tuning cur = e->tune;
        if (cur.minimizer_tile == 0) cur.minimizer_tile = 4096;
        if (cur.heavy_colors == 0) cur.heavy_colors = 64;
        if (cur.table_slots_q == 0) cur.table_slots_q = 8;
        if (cur.radix_bits == 0) cur.radix_bits = 8;
        measure(cur);  // warm-up: allocations reach their working sizes
        double cur_ms = measure(cur);
        auto consider = [&](cdbg_tuning const& t) {
            const double ms = measure(t);
            if (ms < cur_ms * 0.99) {  // keep only a clear gain
                cur = t;
                cur_ms = ms;
            }
        };
        for (uint64_t v : {uint64_t(1) << 27, uint64_t(1) << 26, uint64_t(1) << 25, uint64_t(1) << 24}) {
            cdbg_tuning t = cur;
            t.batch_occ = v;
            if (t.batch_occ != cur.batch_occ) consider(t);
        }
        for (uint32_t v : {2048u, 4096u}) {
            cdbg_tuning t = cur;
            t.minimizer_tile = v;
            if (t.minimizer_tile != cur.minimizer_tile) consider(t);
        }
        for (uint32_t v : {16u, 32u, 64u, 128u, 256u}) {
            cdbg_tuning t = cur;
            t.heavy_colors = v;
            if (t.heavy_colors != cur.heavy_colors) consider(t);
        }
        for (uint32_t v : {8u, 6u, 5u}) {
            cdbg_tuning t = cur;
            t.table_slots_q = v;
            if (t.table_slots_q != cur.table_slots_q) consider(t);
        }
        for (uint32_t v : {0u, 64u, 256u}) {
            cdbg_tuning t = cur;
            t.table_group_mb = v;
            if (t.table_group_mb != cur.table_group_mb) consider(t);
        }
        for (uint32_t v : {8u, 11u}) {
            cdbg_tuning t = cur;
            t.radix_bits = v;
            if (t.radix_bits != cur.radix_bits) consider(t);
        }
        e->tune = cur;
        if (best) *best = cur;
        if (best_ms) *best_ms = cur_ms;
        return 0;
    } catch (std::exception const& ex) {
        return fail(ex);
    }
}

}  // extern "C"
