// Device k-mer / hashing helpers shared by the phase-1 and phase-2 kernels.
#pragma once

#include <stdint.h>

#include "common.cuh"

namespace cdbg {

// ntHash per-base seeds (phase1_bucket_write/minimizer.hpp:21-26).
__device__ __forceinline__ uint64_t nt_seed(uint32_t b) {
    // branch-free select of the four 64-bit seeds
    const uint64_t s0 = 0x3c8bfbb395c60474ULL, s1 = 0x3193c18562a02b4cULL;
    const uint64_t s2 = 0x20323ed082572324ULL, s3 = 0x295549f54be24456ULL;
    uint64_t lo = (b & 1) ? s1 : s0;
    uint64_t hi = (b & 1) ? s3 : s2;
    return (b & 2) ? hi : lo;
}

__device__ __forceinline__ uint64_t rol64(uint64_t x, uint32_t r) {
    r &= 63u;
    return r ? (x << r) | (x >> (64u - r)) : x;
}
__device__ __forceinline__ uint64_t ror64(uint64_t x, uint32_t r) {
    r &= 63u;
    return r ? (x >> r) | (x << (64u - r)) : x;
}

// Reverse the order of the 2-bit groups of a 64-bit word.
__host__ __device__ __forceinline__ uint64_t rev2_64(uint64_t x) {
    x = ((x >> 2) & 0x3333333333333333ULL) | ((x & 0x3333333333333333ULL) << 2);
    x = ((x >> 4) & 0x0F0F0F0F0F0F0F0FULL) | ((x & 0x0F0F0F0F0F0F0F0FULL) << 4);
    x = ((x >> 8) & 0x00FF00FF00FF00FFULL) | ((x & 0x00FF00FF00FF00FFULL) << 8);
    x = ((x >> 16) & 0x0000FFFF0000FFFFULL) | ((x & 0x0000FFFF0000FFFFULL) << 16);
    return (x >> 32) | (x << 32);
}

template <typename K>
struct kmer_ops;

// k <= 31: 64-bit k-mer, first base in the highest used 2-bit group
// (kmer.hpp:11-18).
template <>
struct kmer_ops<uint64_t> {
    typedef uint64_t K;
    static __host__ __device__ __forceinline__ K mask(uint32_t k) {
        return (2 * k >= 64) ? ~K(0) : ((K(1) << (2 * k)) - 1);
    }
    static __host__ __device__ __forceinline__ K revcomp(K x, uint32_t k) {
        return rev2_64(~x) >> (64 - 2 * k);
    }
    static __host__ __device__ __forceinline__ K empty() { return ~K(0); }
    static __host__ __device__ __forceinline__ uint64_t hash(K x) { return mix64(x); }
    static __host__ __device__ __forceinline__ uint32_t low2(K x) { return (uint32_t)(x & 3); }
    // k-mer whose bases are the k bases of `x` read LSB-first (base i at bits
    // 2i): forward value and reverse-complement value.
    static __device__ __forceinline__ void from_lsb(uint64_t x, uint32_t k, K& fwd, K& rc) {
        const K m = mask(k);
        x &= m;
        rc = (~x) & m;
        fwd = rev2_64(x) >> (64 - 2 * k);
    }
    // Load the k-mer at stream base position `pos`.
    static __device__ __forceinline__ void load(uint64_t const* __restrict__ words, uint64_t pos,
                                                uint32_t k, K& fwd, K& rc) {
        from_lsb(stream_bits64(words, pos), k, fwd, rc);
    }
};

// k <= 63: 128-bit k-mer.
template <>
struct kmer_ops<u128> {
    typedef u128 K;
    static __host__ __device__ __forceinline__ K mask(uint32_t k) {
        return (2 * k >= 128) ? ~K(0) : ((K(1) << (2 * k)) - 1);
    }
    static __host__ __device__ __forceinline__ K rev2_128(K x) {
        const uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
        return ((K)rev2_64(lo) << 64) | (K)rev2_64(hi);
    }
    static __host__ __device__ __forceinline__ K revcomp(K x, uint32_t k) {
        return rev2_128(~x) >> (128 - 2 * k);
    }
    static __host__ __device__ __forceinline__ K empty() { return ~K(0); }
    static __host__ __device__ __forceinline__ uint64_t hash(K x) {
        const uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
        return mix64(lo) ^ (mix64(hi + 0x9e3779b97f4a7c15ULL) << 1);
    }
    static __host__ __device__ __forceinline__ uint32_t low2(K x) { return (uint32_t)(x & 3); }
    static __device__ __forceinline__ void load(uint64_t const* __restrict__ words, uint64_t pos,
                                                uint32_t k, K& fwd, K& rc) {
        const uint64_t a = stream_bits64(words, pos);
        const uint64_t b = stream_bits64(words, pos + 32);
        K x = ((K)b << 64) | (K)a;
        const K m = mask(k);
        x &= m;
        rc = (~x) & m;
        fwd = rev2_128(x) >> (128 - 2 * k);
    }
};

// 64-bit key hash of a super-k-mer (length + bases 32 at a time), identical
// to oracle::super_hash.
__device__ __forceinline__ uint64_t super_hash_dev(uint64_t const* __restrict__ words, uint64_t pos,
                                                   uint32_t len) {
    uint64_t h = mix64(0x51ed2701f3a5c2b9ULL ^ (uint64_t)len);
    for (uint32_t i = 0; i < len; i += 32) {
        uint64_t w = stream_bits64(words, pos + i);
        const uint32_t n = len - i;
        if (n < 32) w &= (uint64_t(1) << (2 * n)) - 1;
        h = mix64(h ^ w);
    }
    return h;
}

// Hash of a sorted color list (class identity): splitmix chain over the
// length and the elements.
__device__ __forceinline__ uint64_t list_hash_step(uint64_t h, uint32_t c) { return mix64(h ^ c); }
__device__ __forceinline__ uint64_t list_hash_init(uint64_t n) {
    return mix64(0x7f4a7c159e3779b9ULL ^ n);
}

}  // namespace cdbg
