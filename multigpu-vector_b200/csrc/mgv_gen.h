/*
 * mgv_gen.h -- counter-based seeded data generator shared by the CUDA kernels,
 * the host library and the CPU oracle.
 *
 * Every value is a pure function of (seed, stream, row index), so a column can
 * be produced in parallel on the GPU and row-by-row on the CPU with identical
 * results.  The reference draws its inputs from unseeded rand()/mt19937
 * (src/main8.cu:169, src/main9.cu:556-566), which makes its runs
 * unreproducible; this generator replaces that source with fixed seeds.
 *
 * Distributions:
 *   - uniform int32 in [lo, lo + range)            mgv_gen_uniform
 *   - seeded permutation of 0..n-1                 mgv_gen_perm
 *   - join probe keys: p_hit from the build keys,  mgv_gen_probe_key
 *     else uniform in a disjoint miss range
 *   - Zipf(s) over G groups by inverse CDF on a    mgv_gen_zipf
 *     32-bit cumulative table built on the host
 *
 * Plain C99, usable from C, C++ and CUDA (host and device).
 */
#ifndef MGV_GEN_H_
#define MGV_GEN_H_

#include <stdint.h>

#if defined(__CUDACC__)
#define MGV_HD __host__ __device__ __forceinline__
#else
#define MGV_HD static inline
#endif

/* splitmix64 finaliser (Steele, Lea, Flood 2014). */
MGV_HD uint64_t mgv_mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* 64 random bits for row i of stream `stream` under `seed`. */
MGV_HD uint64_t mgv_rand64(uint64_t seed, uint32_t stream, uint64_t i) {
    uint64_t key = mgv_mix64(seed ^ ((uint64_t)stream * 0xD1B54A32D192ED03ull));
    return mgv_mix64(key + i * 0x9E3779B97F4A7C15ull);
}

/* Uniform in [lo, lo + range); range <= 2^32.  Multiply-shift (Lemire)
 * mapping of the top 32 random bits: exact integer arithmetic. */
MGV_HD int32_t mgv_gen_uniform(uint64_t seed, uint32_t stream, uint64_t i,
                               int64_t lo, uint64_t range) {
    uint64_t r = mgv_rand64(seed, stream, i) >> 32;
    return (int32_t)(lo + (int64_t)((r * range) >> 32));
}

/* Number of bits needed to hold n-1 (n >= 1). */
MGV_HD uint32_t mgv_bits_for(uint64_t n) {
    uint32_t b = 0;
    while (b < 63 && ((uint64_t)1 << b) < n) ++b;
    return b;
}

/* One bijective round on k-bit words: add, odd multiply, xorshift. */
MGV_HD uint64_t mgv_perm_round(uint64_t x, uint64_t mask, uint32_t k,
                               uint64_t add, uint64_t mul) {
    x = (x + add) & mask;
    x = (x * (mul | 1ull)) & mask;
    x ^= x >> ((k >> 1) + 1);
    return x;
}

/* Bijection on [0, 2^k), k <= 40. */
MGV_HD uint64_t mgv_perm_pow2(uint64_t seed, uint32_t k, uint64_t x) {
    if (k == 0) return 0;
    uint64_t mask = (k >= 64) ? ~0ull : (((uint64_t)1 << k) - 1);
    uint64_t a0 = mgv_mix64(seed + 1), a1 = mgv_mix64(seed + 2), a2 = mgv_mix64(seed + 3);
    uint64_t m0 = mgv_mix64(seed + 4), m1 = mgv_mix64(seed + 5), m2 = mgv_mix64(seed + 6);
    x = mgv_perm_round(x, mask, k, a0, m0);
    x = mgv_perm_round(x, mask, k, a1, m1);
    x = mgv_perm_round(x, mask, k, a2, m2);
    return x;
}

/* Element i of a seeded permutation of 0..n-1 (cycle walking on the
 * next power of two, so every n >= 1 works; expected < 2 rounds). */
MGV_HD uint32_t mgv_gen_perm(uint64_t seed, uint64_t n, uint64_t i) {
    uint32_t k = mgv_bits_for(n);
    uint64_t x = i;
    do {
        x = mgv_perm_pow2(seed, k, x);
    } while (x >= n);
    return (uint32_t)x;
}

/* Join probe key for probe row i.  With probability hit_num / 2^32 it is
 * a uniformly chosen build key perm(build_seed, nbuild, j); otherwise it
 * is uniform in [miss_lo, miss_lo + miss_range), a range disjoint from the
 * build keys.  `hit` reports which branch was taken (the generator knows
 * the exact match count, a known answer for the join). */
MGV_HD int32_t mgv_gen_probe_key(uint64_t seed, uint64_t build_seed, uint64_t nbuild,
                                 uint32_t hit_num, int64_t miss_lo, uint64_t miss_range,
                                 uint64_t i, int *hit) {
    uint64_t r = mgv_rand64(seed, 7u, i);
    uint32_t coin = (uint32_t)(r >> 32);
    uint32_t pick = (uint32_t)r;
    if (coin < hit_num) {
        uint64_t j = ((uint64_t)pick * nbuild) >> 32;
        if (hit) *hit = 1;
        return (int32_t)mgv_gen_perm(build_seed, nbuild, j);
    }
    if (hit) *hit = 0;
    return (int32_t)(miss_lo + (int64_t)(((uint64_t)pick * miss_range) >> 32));
}

/* Zipf sample: smallest g with u < cdf[g], where cdf is a non-decreasing
 * table of G thresholds in 2^32 units (last entry saturates).  Returns the
 * 0-based rank (0 = most frequent group). */
MGV_HD int32_t mgv_gen_zipf(uint64_t seed, uint32_t stream, uint64_t i,
                            const uint64_t *cdf, uint32_t G) {
    uint64_t u = mgv_rand64(seed, stream, i) >> 32;
    uint32_t lo = 0, hi = G - 1;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (u < cdf[mid]) hi = mid; else lo = mid + 1;
    }
    return (int32_t)lo;
}

#endif /* MGV_GEN_H_ */
