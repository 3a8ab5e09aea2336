// hash_table.cuh -- device logic of the open-addressing join table.
//
// Layout: nbuckets buckets of 32 bytes (one L2 sector), 4 slots each; a
// slot is a 64-bit {key (low word), payload (high word)}.  A table built
// without payloads (key_only) holds 8 slots of a 32-bit key per bucket
// instead: half the bytes per key, every match with payload 0.  The key
// INT32_MIN marks an empty slot (in both layouts every 32-bit word of an
// empty bucket is INT32_MIN); build rows with that key go to a side list.  A key's run starts at bucket_of(key) and continues linearly;
// slots of a run are claimed in order, so a lookup may stop at the first
// empty slot (and, for tables without duplicate keys, at the first match).
//
// Replaces the reference's chained table: first[2^L] + next[2 * max]
// (src/operators/hashjoin.cu:40-75), whose probe walks dependent pointers.
#pragma once

#include "device_common.cuh"
#include "mgv_internal.h"

namespace mgv {

// Home bucket of a key (radix-aware; see TableView).
__device__ __forceinline__ uint32_t home_bucket(int32_t key, const TableView& t) {
    const uint32_t part = ((uint32_t)key >> t.radix_shift) & t.radix_mask;
    return part * t.bpp + __umulhi(murmur32((uint32_t)key), t.bpp);
}

__device__ __forceinline__ void table_insert(const TableView& t, int32_t key, int32_t pay,
                                             uint32_t* err, bool& dup, bool& ok) {
    ok = false;
    if (key == kEmptyKey) {
        unsigned long long i = atomicAdd(t.meta + 0, 1ull);
        atomicAdd(t.meta + 1, (unsigned long long)(long long)pay);
        if (i < t.side_cap) t.side_pay[i] = pay;
        else set_error(err, kDevTableFull, 1);
        return;
    }
    uint32_t b = home_bucket(key, t);
    if (t.key_only) {
        uint32_t* keys = reinterpret_cast<uint32_t*>(t.slots);
        for (uint32_t it = 0; it < t.nbuckets; ++it) {
            unsigned long long s[4];
            ld_bucket_relaxed(t.slots + 4ull * b, s);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                uint32_t cur = (uint32_t)(s[j >> 1] >> (32 * (j & 1)));
                if ((int32_t)cur == kEmptyKey) {
                    const uint32_t old = atomicCAS(keys + 8ull * b + j, (uint32_t)kEmptyKey, (uint32_t)key);
                    if (old == (uint32_t)kEmptyKey) {
                        ok = true;
                        return;
                    }
                    cur = old;
                }
                if ((int32_t)cur == key) dup = true;
            }
            b = (b + 1 == t.nbuckets) ? 0u : b + 1;
        }
        set_error(err, kDevTableFull, 2);
        return;
    }
    const unsigned long long v = ((unsigned long long)(uint32_t)pay << 32) | (uint32_t)key;
    for (uint32_t it = 0; it < t.nbuckets; ++it) {
        unsigned long long s[4];
        ld_bucket_relaxed(t.slots + 4ull * b, s);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            unsigned long long cur = s[j];
            if ((int32_t)(uint32_t)cur == kEmptyKey) {
                unsigned long long old = atomicCAS(t.slots + 4ull * b + j, kEmptySlot, v);
                if (old == kEmptySlot) {
                    ok = true;
                    return;
                }
                cur = old;
            }
            if ((int32_t)(uint32_t)cur == key) dup = true;
        }
        b = (b + 1 == t.nbuckets) ? 0u : b + 1;
    }
    set_error(err, kDevTableFull, 2);
}

// Inserts R rows per thread with their latencies overlapped: the R home
// buckets are loaded together, each row's first empty home slot is claimed
// with one CAS (the R CASes in flight together), and only a row whose home
// bucket is full or whose CAS lost a race takes the scalar path.  Any slot
// read that already holds the row's key marks a duplicate (the row itself
// is not in the table yet).
template <int R>
__device__ __forceinline__ void table_insert_rows(const TableView& t, const int32_t (&key)[R],
                                                  const int32_t (&pay)[R], const bool (&valid)[R],
                                                  uint32_t* err, bool& dup, uint32_t& inserted) {
    if (t.key_only) {  // key-only tables: one 32-bit claim per row (builds under 2^16 rows come here)
#pragma unroll
        for (int j = 0; j < R; ++j) {
            if (!valid[j]) continue;
            bool ok;
            table_insert(t, key[j], pay[j], err, dup, ok);
            inserted += ok;
        }
        return;
    }
    unsigned long long s[R][4];
    uint32_t b[R];
    bool fast[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        fast[j] = valid[j] && key[j] != kEmptyKey;
        b[j] = fast[j] ? home_bucket(key[j], t) : 0u;
        if (fast[j]) ld_bucket_relaxed(t.slots + 4ull * b[j], s[j]);
    }
    int q[R];
    unsigned long long v[R], old[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        q[j] = -1;
        v[j] = ((unsigned long long)(uint32_t)pay[j] << 32) | (uint32_t)key[j];
        if (!fast[j]) continue;
#pragma unroll
        for (int k = 3; k >= 0; --k) {
            const int32_t sk = (int32_t)(uint32_t)s[j][k];
            if (sk == kEmptyKey) q[j] = k;
            if (sk == key[j]) dup = true;
        }
        // slots are claimed in order, so the first empty slot starts the free tail
    }
#pragma unroll
    for (int j = 0; j < R; ++j)
        old[j] = q[j] >= 0 ? atomicCAS(t.slots + 4ull * b[j] + q[j], kEmptySlot, v[j]) : 0ull;
#pragma unroll
    for (int j = 0; j < R; ++j) {
        if (!valid[j]) continue;
        if (q[j] >= 0 && old[j] == kEmptySlot) {
            ++inserted;
            continue;
        }
        if (q[j] >= 0 && (int32_t)(uint32_t)old[j] == key[j]) dup = true;
        bool ok;
        table_insert(t, key[j], pay[j], err, dup, ok);
        inserted += ok;
    }
}

// Matches of `key` inside one bucket w[0..7] = k0 p0 k1 p1 k2 p2 k3 p3
// (KO: eight keys, every payload 0).  more = the probe must continue to the
// next bucket.
template <bool UNIQUE, bool KO = false>
__device__ __forceinline__ void match_bucket(const uint32_t (&w)[8], int32_t key, uint32_t& mc,
                                             long long& ms, bool& more) {
    const uint32_t k = (uint32_t)key;
    if (KO) {
        uint32_t c = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) c += w[q] == k;
        const bool full = w[7] != (uint32_t)kEmptyKey;
        mc = UNIQUE ? (c != 0) : c;
        ms = 0;
        more = UNIQUE ? (c == 0 && full) : full;
        return;
    }
    const bool m0 = w[0] == k, m1 = w[2] == k, m2 = w[4] == k, m3 = w[6] == k;
    const bool full = w[6] != (uint32_t)kEmptyKey;
    if (UNIQUE) {
        const bool f = m0 | m1 | m2 | m3;
        mc = f;
        ms = f ? (long long)(int32_t)(m0 ? w[1] : m1 ? w[3] : m2 ? w[5] : w[7]) : 0ll;
        more = !f && full;
    } else {
        mc = (uint32_t)m0 + m1 + m2 + m3;
        ms = (m0 ? (long long)(int32_t)w[1] : 0ll) + (m1 ? (long long)(int32_t)w[3] : 0ll) +
             (m2 ? (long long)(int32_t)w[5] : 0ll) + (m3 ? (long long)(int32_t)w[7] : 0ll);
        more = full;
    }
}

// Continuation past a full home bucket (rare at the default load factor).
// Returns {matches, payload sum}; kept out of line so the common path of
// the probe loop stays small.
struct Matches {
    unsigned long long sum;
    uint32_t count;
};

template <bool UNIQUE, bool KO = false>
__device__ __forceinline__ Matches probe_rest(const unsigned long long* __restrict__ slots,
                                           uint32_t nbuckets, int32_t key, uint32_t b) {
    Matches r{0ull, 0u};
    for (uint32_t it = 1; it < nbuckets; ++it) {
        b = (b + 1 == nbuckets) ? 0u : b + 1;
        uint32_t w[8];
        ld_bucket(slots + 4ull * b, w);
        uint32_t c;
        long long s;
        bool more;
        match_bucket<UNIQUE, KO>(w, key, c, s, more);
        r.count += c;
        r.sum += (unsigned long long)s;
        if (!more) break;
    }
    return r;
}

}  // namespace mgv
