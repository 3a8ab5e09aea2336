// chain.cu -- the generic fused operator chain:
//
//     [select] -> [hash_probe] -> { aggregate | group-by | sink }
//
// one kernel per consume call.  Warp-ballot select as in
// unstable_select::consume_warp (src/operators/select3.cu:19-85): each warp
// takes 512-row windows (16 filter loads per lane in flight), evaluates the
// predicate and compacts the offsets of the qualifying rows with
// __ballot_sync / __popc into a per-warp shared-memory ring of 1024 entries.
// Every 128 offsets form a vector whose carried columns -- only those the
// rest of the chain reads -- are gathered and handed to the probe and the
// terminal (the reference's parent->consume_warp(x, 128)).
//
// The probe emits one output row per matching build row (all duplicates
// match, src/operators/hashjoin.cu:148-162); the build payload of the match
// is visible to the terminal as column `ncols`.
//
// Shared scans of the query server (k_batch_cells, no reference
// counterpart) run the same chain at the largest of several requests' filter
// bounds and aggregate each matched row into a (filter range, group) cell;
// a prefix over the ranges then gives each request its groups.
//
// Group-by (no reference counterpart): each CTA aggregates into a
// shared-memory hash table with native 32-bit shared atomics (count, and the
// int64 sum as two biased words).  Groups that do not find a shared slot
// within a few probes, or arrive once the table is 5/8 full, go to the global
// table; at the end of the CTA the shared table is merged into the global one.
#include <cuda_runtime.h>

#include "../../include/mgv_device.cuh"
#include "device_common.cuh"
#include "hash_table.cuh"
#include "mgv_internal.h"

#include <algorithm>

namespace mgv {

constexpr int kChainBlock = 512;  // 16 warps: one CTA per SM with the largest group table
constexpr int kChainWarps = kChainBlock / 32;
constexpr int kWinRows = 512;  // rows per warp per select window: 16 loads per lane in flight
constexpr int kIdRing = 1024;  // per-warp ring of qualifying row offsets (>= kWinRows + 127)
constexpr int kMaxTermSlots = 3;  // carried columns of an aggregate / group-by chain: key + 2 references
constexpr size_t kRingBytes = (size_t)kChainWarps * kIdRing * sizeof(uint32_t);


// ---- device buffer pool: pop (swap-on-full for the sink) -------------------

// One pop from the pool's device free stack (include/mgv_device.cuh), or kNil.
__device__ __forceinline__ uint32_t pool_pop(PoolDev* p) {
    mgv_pool_device v;
    v.head = &p->head;
    v.available = &p->available;
    v.producers = &p->producers;
    v.next = p->next;
    uint32_t id;
    return mgv_dev_stack_pop(&v, &id) ? id : kNil;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Buffer id for chunk c of a sink; the warp that owns row c*capacity takes
// a buffer from the pool and publishes it, everyone else waits for it with
// a bounded wait (swap-on-full, src/buffer_manager.cuh:147-176).
__device__ uint32_t sink_chunk(const SinkView& s, uint32_t c, bool opener, uint32_t* err) {
    if (opener) {
        uint32_t id = pool_pop(s.pool);
        if (id == kNil) {
            set_error(err, kDevOverflow, 3);
            id = kNil - 1;  // published "no buffer" marker
        }
        atomicExch(s.chain + c, id);
        return id;
    }
    const unsigned long long t0 = global_ns();
    for (;;) {
        uint32_t id = *((volatile uint32_t*)(s.chain + c));
        if (id != kNil) return id;
        if (global_ns() - t0 > 2000000000ull) {  // 2 s
            set_error(err, kDevTimeout, 4);
            return kNil - 1;
        }
        __nanosleep(64);
    }
}

// Append `my_cnt` rows per lane, reserved warp-wide; row_val(i, col).
template <class RowFn>
__device__ __forceinline__ void sink_emit_warp(const SinkView& s, uint32_t my_cnt, RowFn row_val, uint32_t* err) {
    const uint32_t lane = lane_id();
    uint32_t incl = my_cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) return;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(s.cursor, (unsigned long long)total);
    base = __shfl_sync(0xffffffffu, base, 0);
    const unsigned long long limit = (unsigned long long)s.max_chunks * s.capacity;
    const unsigned long long first_c = base / s.capacity;
    const unsigned long long last_c = (base + total - 1) / s.capacity;
    uint32_t my_chunk_id = kNil - 1;
    const unsigned long long c = first_c + lane;
    if (c <= last_c && c < s.max_chunks) {
        const bool opener = c * s.capacity >= base;  // this warp owns the chunk's first row
        my_chunk_id = sink_chunk(s, (uint32_t)c, opener, err);
    }
    __syncwarp();
    if (lane == 0 && (last_c - first_c >= 32 || base + total > limit)) set_error(err, kDevOverflow, 5);
    const uint32_t maxc = __reduce_max_sync(0xffffffffu, my_cnt);
    const unsigned long long pos0 = base + incl - my_cnt;
    for (uint32_t i = 0; i < maxc; ++i) {
        const bool act = i < my_cnt;
        const unsigned long long pos = pos0 + i;
        const unsigned long long rel = act ? pos / s.capacity - first_c : 0ull;
        const uint32_t id = __shfl_sync(0xffffffffu, my_chunk_id, (int)(rel & 31ull));
        if (!act || pos >= limit || rel >= 32 || id >= s.pool->nbuffers) continue;
        const uint32_t off = (uint32_t)(pos % s.capacity);
        int32_t* base_ptr = s.slab + (size_t)id * s.pool_ncols * s.capacity;
        for (uint32_t col = 0; col < s.ncols; ++col) base_ptr[(size_t)col * s.capacity + off] = row_val(i, col);
    }
}

// ---- group tables ------------------------------------------------------------
//
// Both tables use Fibonacci hashing, (g * 2654435769) >> (32 - log2 cap), and
// linear probing; a slot's key goes from EMPTY (INT32_MIN) to its group once
// (atomicCAS) and never changes until the table is cleared, so a reader that
// sees a stale EMPTY just loses the CAS and reads the winner's key.

__device__ __forceinline__ uint32_t group_hash(int32_t g, uint32_t cap) {
    return ((uint32_t)g * 2654435769u) >> (__clz(cap) + 1);  // cap = 2^k: shift = 32 - k
}

// Adds (sum, cnt) to group g of the global table; the adds are fire-and-forget.
__device__ __forceinline__ void global_group_add(const GroupTableView& gt, int32_t g, unsigned long long sum,
                                                 unsigned long long cnt, uint32_t* err) {
    if (g == kEmptyKey) {  // the reserved key has its own counters
        atomicAdd(gt.special + 0, sum);
        atomicAdd(gt.special + 1, cnt);
        return;
    }
    uint32_t slot = group_hash(g, gt.cap);
    for (uint32_t i = 0; i < gt.cap; ++i) {
        int32_t k = gt.keys[slot];
        if (k == kEmptyKey) k = atomicCAS(gt.keys + slot, kEmptyKey, g);
        if (k == kEmptyKey || k == g) {
            atomicAdd(gt.sums + slot, sum);
            atomicAdd(gt.counts + slot, cnt);
            return;
        }
        slot = (slot + 1) & (gt.cap - 1);
    }
    set_error(err, kDevTableFull, 20);
}

// A CTA's shared group table: cap slots plus one for the reserved group
// INT32_MIN, all 32-bit so that every update is a native shared atomic.
// The int64 sum of a slot is kept biased, as sum + count * 2^31 in two words
// (lo, hi): a value v adds v + 2^31, which lies in [0, 2^32), to lo and a
// carry to hi.
struct SmemGroups {
    int32_t* keys;
    uint32_t* cnt;
    uint32_t* lo;
    uint32_t* hi;
    uint32_t* used;  // slots claimed so far
    uint32_t cap;    // power of two, 0 = no shared table
};

constexpr uint32_t kGroupProbes = 16;  // shared-table probes before a row goes to the global table

// New groups are admitted to the shared table until it is this full; later
// ones go to the global table, so a lookup that misses ends at an empty slot
// after a few probes instead of scanning a crowded table.
__host__ __device__ __forceinline__ uint32_t smem_groups_limit(uint32_t cap) { return cap - cap / 4 - cap / 8; }

__host__ __device__ __forceinline__ size_t smem_groups_bytes(uint32_t cap) {
    return cap ? (size_t)(cap + 1) * 16 + 16 : 0;
}

__device__ __forceinline__ SmemGroups smem_groups_at(unsigned char* base, uint32_t cap) {
    SmemGroups sg;
    sg.keys = reinterpret_cast<int32_t*>(base);
    sg.cnt = reinterpret_cast<uint32_t*>(base) + (cap + 1);
    sg.lo = reinterpret_cast<uint32_t*>(base) + 2 * (cap + 1);
    sg.hi = reinterpret_cast<uint32_t*>(base) + 3 * (cap + 1);
    sg.used = reinterpret_cast<uint32_t*>(base) + 4 * (cap + 1);
    sg.cap = cap;
    return sg;
}

// One row (g, v) of a group-by, per lane.
__device__ __forceinline__ void group_add_row(const SmemGroups& sg, const GroupTableView& gt, int32_t g, int32_t v,
                                              uint32_t* err) {
    if (sg.cap) {
        uint32_t slot = sg.cap;  // the reserved group's slot
        bool hit = g == kEmptyKey;
        if (!hit) {
            slot = group_hash(g, sg.cap);
#pragma unroll 1
            for (uint32_t i = 0; i < kGroupProbes; ++i) {
                int32_t k = *((volatile int32_t*)(sg.keys + slot));
                if (k == kEmptyKey) {
                    if (*(volatile uint32_t*)sg.used >= smem_groups_limit(sg.cap)) break;  // stays global
                    k = atomicCAS(sg.keys + slot, kEmptyKey, g);
                    if (k == kEmptyKey) atomicAdd(sg.used, 1u);
                }
                if (k == kEmptyKey || k == g) {
                    hit = true;
                    break;
                }
                slot = (slot + 1) & (sg.cap - 1);
            }
        }
        if (hit) {
            const uint32_t x = (uint32_t)v ^ 0x80000000u;  // v + 2^31
            atomicAdd(sg.cnt + slot, 1u);
            const uint32_t old = atomicAdd(sg.lo + slot, x);
            if (old + x < old) atomicAdd(sg.hi + slot, 1u);
            return;
        }
    }
    global_group_add(gt, g, (unsigned long long)(long long)v, 1ull, err);
}

__device__ __forceinline__ void smem_groups_init(const SmemGroups& sg) {
    for (uint32_t i = threadIdx.x; i <= sg.cap; i += blockDim.x) {
        sg.keys[i] = kEmptyKey;
        sg.cnt[i] = 0;
        sg.lo[i] = 0;
        sg.hi[i] = 0;
    }
    if (threadIdx.x == 0) *sg.used = 0;
}

// Merges a CTA's shared table into the global one.  A thread takes
// kFlushBatch of its slots at a time and loads the global home slot of each
// of their groups before adding any: a group already at its home slot (the
// common case once one CTA has flushed it; a slot's key never changes after
// it is claimed) is added there directly, so a flush costs about one L2
// round trip per batch instead of one per group.  The rest take the full
// insert.
constexpr int kFlushBatch = 8;
__device__ __forceinline__ void smem_groups_flush(const SmemGroups& sg, const GroupTableView& gt, uint32_t* err) {
    for (uint32_t i0 = threadIdx.x; i0 <= sg.cap; i0 += blockDim.x * kFlushBatch) {
        uint32_t c[kFlushBatch], home[kFlushBatch];
        int32_t g[kFlushBatch], at[kFlushBatch];
#pragma unroll
        for (int u = 0; u < kFlushBatch; ++u) {
            const uint32_t i = i0 + u * blockDim.x;
            c[u] = i <= sg.cap ? sg.cnt[i] : 0u;
            g[u] = i < sg.cap ? sg.keys[i] : kEmptyKey;
            home[u] = group_hash(g[u], gt.cap);
            at[u] = (c[u] && g[u] != kEmptyKey) ? gt.keys[home[u]] : kEmptyKey;
        }
#pragma unroll
        for (int u = 0; u < kFlushBatch; ++u) {
            if (c[u] == 0) continue;
            const uint32_t i = i0 + u * blockDim.x;
            const unsigned long long biased = ((unsigned long long)sg.hi[i] << 32) | sg.lo[i];
            const unsigned long long sum = biased - ((unsigned long long)c[u] << 31);
            if (g[u] != kEmptyKey && at[u] == g[u]) {
                atomicAdd(gt.sums + home[u], sum);
                atomicAdd(gt.counts + home[u], (unsigned long long)c[u]);
            } else {
                global_group_add(gt, g[u], sum, c[u], err);
            }
        }
    }
}

// ---- shared scans: per-(range, group) cells ------------------------------------
//
// A CTA's shared cell table, keyed by (range << 21) | group in 32 bits for
// groups in [0, 2^21 - 1) (EMPTY = ~0, which no such key produces), with a
// count and the biased two-word sum as in SmemGroups: 16 bytes a slot, so
// 8192 slots fit beside the rings.  Cells of other groups, and cells that
// find no shared slot, go to the range's global table, which shares its key
// array (the group directory) with every other range (CellsView).

constexpr uint32_t kCellSlots = 8192;  // shared cells per CTA (128 KiB)
constexpr uint32_t kEmptyCell = 0xFFFFFFFFu;
constexpr uint32_t kCellGroupBits = 21;  // range index above, group below

struct SmemCells {
    uint32_t* keys;
    uint32_t* cnt;
    uint32_t* lo;
    uint32_t* hi;
    uint32_t* used;
    uint32_t cap;  // power of two
};

__host__ __device__ __forceinline__ size_t smem_cells_bytes(uint32_t cap) { return (size_t)cap * 16 + 16; }

__device__ __forceinline__ SmemCells smem_cells_at(unsigned char* base, uint32_t cap) {
    SmemCells c;
    c.keys = reinterpret_cast<uint32_t*>(base);
    c.cnt = c.keys + cap;
    c.lo = c.cnt + cap;
    c.hi = c.lo + cap;
    c.used = c.hi + cap;
    c.cap = cap;
    return c;
}

__device__ __forceinline__ uint32_t cell_hash(uint32_t key, uint32_t cap) {
    return (key * 2654435769u) >> (__clz(cap) + 1);  // cap = 2^k: shift = 32 - k
}

// Range of a filter value that passed the select (f <= b[m-1]): the first j
// with b[j] >= f, by binary search.
__device__ __forceinline__ uint32_t cell_range(const int32_t* b, uint32_t m, int32_t f) {
    uint32_t lo = 0, hi = m - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (b[mid] >= f) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// One matched row (g, v) of range j, per lane.
__device__ __forceinline__ void cells_add_row(const SmemCells& sc, const CellsView& cv, uint32_t j, int32_t g,
                                              int32_t v, uint32_t* err) {
    if ((uint32_t)g < (1u << kCellGroupBits) - 1u) {
        const uint32_t key = (j << kCellGroupBits) | (uint32_t)g;
        uint32_t slot = cell_hash(key, sc.cap);
#pragma unroll 1
        for (uint32_t i = 0; i < kGroupProbes; ++i) {
            uint32_t k = *((volatile uint32_t*)(sc.keys + slot));
            if (k == kEmptyCell) {
                if (*(volatile uint32_t*)sc.used >= smem_groups_limit(sc.cap)) break;  // stays global
                k = atomicCAS(sc.keys + slot, kEmptyCell, key);
                if (k == kEmptyCell) atomicAdd(sc.used, 1u);
            }
            if (k == kEmptyCell || k == key) {
                const uint32_t x = (uint32_t)v ^ 0x80000000u;  // v + 2^31
                atomicAdd(sc.cnt + slot, 1u);
                const uint32_t old = atomicAdd(sc.lo + slot, x);
                if (old + x < old) atomicAdd(sc.hi + slot, 1u);
                return;
            }
            slot = (slot + 1) & (sc.cap - 1);
        }
    }
    global_group_add(cells_range(cv, j), g, (unsigned long long)(long long)v, 1ull, err);
}

__device__ __forceinline__ void smem_cells_init(const SmemCells& sc) {
    for (uint32_t i = threadIdx.x; i < sc.cap; i += blockDim.x) {
        sc.keys[i] = kEmptyCell;
        sc.cnt[i] = 0;
        sc.lo[i] = 0;
        sc.hi[i] = 0;
    }
    if (threadIdx.x == 0) *sc.used = 0;
}

__device__ __forceinline__ void smem_cells_flush(const SmemCells& sc, const CellsView& cv, uint32_t* err) {
    for (uint32_t i = threadIdx.x; i < sc.cap; i += blockDim.x) {
        const uint32_t c = sc.cnt[i];
        if (c == 0) continue;
        const uint32_t key = sc.keys[i];
        const unsigned long long biased = ((unsigned long long)sc.hi[i] << 32) | sc.lo[i];
        global_group_add(cells_range(cv, key >> kCellGroupBits),
                         (int32_t)(key & ((1u << kCellGroupBits) - 1u)),
                         biased - ((unsigned long long)c << 31), (unsigned long long)c, err);
    }
}

// What a shared scan's chain needs besides the descriptor: the CTA's cell
// table, the bounds and the range lookup table, copied to shared memory.
struct CellCtx {
    SmemCells sc;
    const int32_t* bounds;
    const uint16_t* lut;
    uint32_t lut_len;
    int32_t lut_base;
};

// The same from the scan's lookup table when f lies in [lut_base, lut_base +
// lut_len) -- the span of the bounds, when it is short -- else by search.
__device__ __forceinline__ uint32_t cell_range_of(const CellCtx& cc, uint32_t m, int32_t f) {
    const uint32_t d = (uint32_t)f - (uint32_t)cc.lut_base;
    return d < cc.lut_len ? (uint32_t)cc.lut[d] : cell_range(cc.bounds, m, f);
}

// ---- the chain: per-warp processing of a row range ------------------------------

// Value of carried slot `slot` (a run-time index) from the registers of a
// vector; j is a compile-time row position after unrolling.
template <int NS>
__device__ __forceinline__ int32_t pick_slot(const int32_t (&v)[NS][4], int32_t slot, int j) {
    int32_t r = 0;
#pragma unroll
    for (int c = 0; c < NS; ++c)
        if (slot == c) r = v[c][j];
    return r;
}

// Windows of kWinRows rows of [row_lo, row_hi) (fewer than 2^32 rows), this
// warp taking windows win_first, win_first + win_stride, ...
//
// A window is filtered with 16 independent coalesced loads per lane (one
// 128-byte warp load each, all in flight together), and the offsets of its
// qualifying rows are compacted with __ballot_sync / __popc into the warp's
// shared ring, in row order.  Every 128 offsets form a vector: its carried
// columns are gathered into registers (4 rows per lane, all loads
// independent), its keys probed, and its rows handed to the terminal.  Only
// qualifying rows' columns are ever loaded.
template <bool SEL, bool PROBE, int TERM, bool FIXED = false>
__device__ __forceinline__ void chain_windows(const ChainDev& a, bool unique, uint64_t row_lo, uint64_t row_hi,
                                              uint64_t win_first, uint64_t win_stride, uint32_t* ids,
                                              const SmemGroups& sg, unsigned long long& acnt,
                                              unsigned long long& asum, uint32_t* err,
                                              const CellCtx* cc = nullptr) {
    constexpr int NS = TERM == kTermSink ? MGV_MAX_COLS : kMaxTermSlots;
    // A batch query's carried slots are fixed (FIXED): key, group, value from
    // input columns 0, 2, 3, so every slot pick below resolves at compile time.
    const uint32_t nslots = FIXED ? 3u : a.nslots;
    const int32_t probe_slot = FIXED ? 0 : a.probe_slot;
    const int32_t ref0 = FIXED ? 1 : a.ref[0];
    const int32_t ref1 = FIXED ? 2 : a.ref[1];
    auto slot_col = [&](int c) -> const int32_t* { return a.cols[FIXED ? (c == 0 ? 0 : c + 1) : a.slot_src[c]]; };
    const uint32_t lane = lane_id();
    const uint32_t len = (uint32_t)(row_hi - row_lo);
    const uint64_t stream_policy = l2_policy_evict_first();  // columns are read once; the join table stays

    // push `cnt` (<= 128) offsets of the ring starting at `start`
    auto push_vector = [&](uint32_t start, uint32_t cnt) {
        __syncwarp();
        uint32_t rid[4];
        uint32_t rng[4];  // shared scan: each row's filter range
        bool in[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t idx = j * 32 + lane;
            in[j] = idx < cnt;
            rid[j] = ids[(start + idx) & (kIdRing - 1)];
            rng[j] = 0;
            if (TERM == kTermCells) {
                rng[j] = rid[j] >> kCellRowBits;
                rid[j] &= (1u << kCellRowBits) - 1u;
            }
        }
        int32_t v[NS][4];
#pragma unroll
        for (int c = 0; c < NS; ++c) {
            const bool carried = (uint32_t)c < nslots;
            const int32_t* col = carried ? slot_col(c) + row_lo : nullptr;
#pragma unroll
            for (int j = 0; j < 4; ++j) v[c][j] = (carried && in[j]) ? ld_stream1(col + rid[j], stream_policy) : 0;
        }
        // value of terminal reference r for the lane's row j and build payload bp
        auto val = [&](int32_t ref, int j, int32_t bp) -> int32_t {
            return ref == kBP ? bp : pick_slot<NS>(v, ref, j);
        };
        // one output row (warp-collective)
        auto emit = [&](bool active, int j, int32_t bp) {
            if (TERM == kTermAgg) {
                if (active) {
                    long long t = 0;
                    if (ref0 >= 0) t += val(ref0, j, bp);
                    if (ref1 >= 0) t += val(ref1, j, bp);
                    acnt += 1;
                    asum += (unsigned long long)t;
                }
            } else if (TERM == kTermGroupby) {
                if (active) {
                    const int32_t g = val(ref0, j, bp);
                    const int32_t x = ref1 >= 0 ? val(ref1, j, bp) : 0;
                    group_add_row(sg, a.gt, g, x, err);
                }
            } else if (TERM == kTermCells) {
                if (active) cells_add_row(cc->sc, a.cells, rng[j], val(ref0, j, bp), val(ref1, j, bp), err);
            } else {
                sink_emit_warp(
                    a.sink, active ? 1u : 0u, [&](uint32_t, uint32_t col) { return val(a.ref[col], j, bp); }, err);
            }
        };
        if (!PROBE) {
#pragma unroll
            for (int j = 0; j < 4; ++j) emit(in[j], j, 0);
        } else {
            // Rounds over the four rows' runs: every round examines one bucket
            // per row still walking and emits its matches; the rows whose run
            // continues past a full bucket then load their next buckets
            // together, so a round costs one memory latency for all of them.
            const unsigned long long* __restrict__ slots = a.table.slots;
            const uint32_t nbuckets = a.table.nbuckets;
            uint32_t w[4][8];
            uint32_t b[4];
            int32_t key[4];
            bool live[4];
            bool reserved_any = false;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                key[j] = pick_slot<NS>(v, probe_slot, j);
                live[j] = in[j] && key[j] != kEmptyKey;
                reserved_any |= in[j] && key[j] == kEmptyKey;
                b[j] = home_bucket(key[j], a.table);
                if (live[j]) ld_bucket(slots + 4ull * b[j], w[j]);
            }
            if (__any_sync(0xffffffffu, reserved_any)) {  // INT32_MIN keys join every side-list row
                const uint32_t side_n =
                    (uint32_t)min((unsigned long long)a.table.meta[0], (unsigned long long)a.table.side_cap);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const bool r = in[j] && key[j] == kEmptyKey;
                    if (__any_sync(0xffffffffu, r))
                        for (uint32_t i = 0; i < side_n; ++i) emit(r, j, a.table.side_pay[i]);
                }
            }
            const bool ko = a.table.key_only != 0;  // eight keys per bucket, payloads 0
            for (uint32_t round = 0; round <= nbuckets; ++round) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const uint32_t k = (uint32_t)key[j];
                    if (ko) {
                        if (unique) {  // at most one match per run
                            bool f = false;
#pragma unroll
                            for (int q = 0; q < 8; ++q) f |= live[j] && w[j][q] == k;
                            if (__any_sync(0xffffffffu, f)) emit(f, j, 0);
                            live[j] = live[j] && !f && w[j][7] != (uint32_t)kEmptyKey;
                        } else {  // every match of the run
#pragma unroll
                            for (int q = 0; q < 8; ++q) {
                                const bool m = live[j] && w[j][q] == k;
                                if (__any_sync(0xffffffffu, m)) emit(m, j, 0);
                            }
                            live[j] = live[j] && w[j][7] != (uint32_t)kEmptyKey;
                        }
                    } else if (unique) {  // at most one match per run
                        bool f = false;
                        int32_t bp = 0;
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            if (live[j] && !f && w[j][2 * q] == k) {
                                f = true;
                                bp = (int32_t)w[j][2 * q + 1];
                            }
                        if (__any_sync(0xffffffffu, f)) emit(f, j, bp);
                        live[j] = live[j] && !f && w[j][6] != (uint32_t)kEmptyKey;
                    } else {  // every match of the run
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const bool m = live[j] && w[j][2 * q] == k;
                            if (__any_sync(0xffffffffu, m)) emit(m, j, (int32_t)w[j][2 * q + 1]);
                        }
                        live[j] = live[j] && w[j][6] != (uint32_t)kEmptyKey;
                    }
                }
                if (!__any_sync(0xffffffffu, live[0] || live[1] || live[2] || live[3])) break;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (live[j]) {
                        b[j] = (b[j] + 1 == nbuckets) ? 0u : b[j] + 1;
                        ld_bucket(slots + 4ull * b[j], w[j]);
                    }
            }
        }
        __syncwarp();
    };

    const int32_t* __restrict__ fcol = SEL ? a.cols[a.sel_col] + row_lo : nullptr;
    const uint32_t lt = (1u << lane) - 1u;
    const uint64_t nwin = (len + kWinRows - 1) / kWinRows;
    uint32_t head = 0, fill = 0;  // fill < 128 between windows
    for (uint64_t win = win_first; win < nwin; win += win_stride) {
        const uint32_t r0 = (uint32_t)win * kWinRows;
        int32_t f[kWinRows / 32];
        if (SEL) {
#pragma unroll
            for (int k = 0; k < kWinRows / 32; ++k) {
                const uint32_t row = r0 + k * 32 + lane;
                f[k] = row < len ? ld_stream1(fcol + row, stream_policy) : 0;
            }
        }
#pragma unroll
        for (int k = 0; k < kWinRows / 32; ++k) {
            const uint32_t row = r0 + k * 32 + lane;
            const bool pass = row < len && (!SEL || f[k] <= a.sel_bound);
            const unsigned m = __ballot_sync(0xffffffffu, pass);
            if (pass) {
                uint32_t e = row;
                if (TERM == kTermCells) e |= cell_range_of(*cc, a.cells.m, f[k]) << kCellRowBits;
                ids[(head + fill + __popc(m & lt)) & (kIdRing - 1)] = e;
            }
            fill += __popc(m);
        }
        while (fill >= 128) {
            push_vector(head, 128);
            head = (head + 128) & (kIdRing - 1);
            fill -= 128;
        }
    }
    if (fill) push_vector(head, fill);
}

template <bool SEL, bool PROBE, int TERM>
__global__ void __launch_bounds__(kChainBlock, 1) k_chain(ChainDev a, uint32_t* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t warp = threadIdx.x / 32;
    // shared layout: [id rings | group table]
    uint32_t* rings = reinterpret_cast<uint32_t*>(smem_raw);
    SmemGroups sg{nullptr, nullptr, nullptr, nullptr, nullptr, 0};
    if (TERM == kTermGroupby && a.smem_groups) {
        sg = smem_groups_at(smem_raw + kRingBytes, a.smem_groups);
        smem_groups_init(sg);
        __syncthreads();
    }
    unsigned long long acnt = 0, asum = 0;
    chain_windows<SEL, PROBE, TERM>(a, a.unique != 0, 0, a.n, (uint64_t)blockIdx.x * kChainWarps + warp,
                                    (uint64_t)gridDim.x * kChainWarps, rings + (size_t)warp * kIdRing, sg,
                                    acnt, asum, err);
    if (TERM == kTermAgg) block_accumulate2<kChainBlock>(acnt, asum, a.acc);
    if (TERM == kTermGroupby && a.smem_groups) {
        __syncthreads();
        smem_groups_flush(sg, a.gt, err);
    }
}

// ---- batched queries ------------------------------------------------------------

// The work items of this CTA: item_order 0 deals them round-robin, so at any
// moment all CTAs work on neighbouring items (in query order: the same few
// queries, whose tables then stay in L2); 1 gives each CTA one contiguous run.
struct ItemRange {
    uint32_t first, end, step;
};
__device__ __forceinline__ ItemRange item_range(uint32_t nitems, uint32_t item_order) {
    if (item_order == 0) return ItemRange{blockIdx.x, nitems, gridDim.x};
    return ItemRange{(uint32_t)((uint64_t)blockIdx.x * nitems / gridDim.x),
                     (uint32_t)((uint64_t)(blockIdx.x + 1) * nitems / gridDim.x), 1u};
}

// Probe phase of a batch: every CTA takes a contiguous run of (query, rows)
// items in query order, so it stays on one query for many items; each query
// aggregates in the CTA's shared group table (up to kMaxSmemGroups slots;
// rows whose group finds no shared slot go to the query's global table),
// flushed to the global table when the CTA moves to another query.  The
// current query's descriptor is copied to shared memory at each switch, so
// its fields cost a shared load instead of registers or global loads.
__global__ void __launch_bounds__(kChainBlock, 1) k_batch_probe(const ChainDev* __restrict__ qs,
                                                                const BatchItem* __restrict__ items,
                                                                uint32_t nitems, uint32_t item_order, uint32_t* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ ChainDev sq;
    static_assert(sizeof(ChainDev) % 4 == 0, "ChainDev is copied as 32-bit words");
    const uint32_t warp = threadIdx.x / 32;
    uint32_t* rings = reinterpret_cast<uint32_t*>(smem_raw);
    const SmemGroups no_sg{nullptr, nullptr, nullptr, nullptr, nullptr, 0};
    SmemGroups sg = no_sg;

    const ItemRange r = item_range(nitems, item_order);
    int64_t cur = -1;
    unsigned long long acnt = 0, asum = 0;
    for (uint32_t it = r.first; it < r.end; it += r.step) {
        const BatchItem item = items[it];
        if ((int64_t)item.q != cur) {
            __syncthreads();  // every warp is done with the previous query
            if (sg.cap) {
                smem_groups_flush(sg, sq.gt, err);
                __syncthreads();  // the flush is done reading sq and the shared table
            }
            cur = item.q;
            for (uint32_t i = threadIdx.x; i < sizeof(ChainDev) / 4; i += kChainBlock)
                reinterpret_cast<uint32_t*>(&sq)[i] = reinterpret_cast<const uint32_t*>(qs + cur)[i];
            const uint32_t cap = qs[cur].smem_groups;
            sg = cap ? smem_groups_at(smem_raw + kRingBytes, cap) : no_sg;
            if (sg.cap) smem_groups_init(sg);
            __syncthreads();
        }
        const ChainDev& a = sq;
        const bool unique = a.table.meta[3] == 0;
        chain_windows<true, true, kTermGroupby, true>(a, unique, item.lo, item.hi, warp, kChainWarps,
                                                rings + (size_t)warp * kIdRing, sg, acnt, asum, err);
    }
    if (sg.cap) {
        __syncthreads();
        smem_groups_flush(sg, sq.gt, err);
    }
}

// Probe phase of shared scans: the items of every scan dealt round-robin, as
// in k_batch_probe; a scan's matched rows go to their (range, group) cells
// in the CTA's shared cell table, flushed to the scan's global cells when
// the CTA moves to another scan.  The scan's bounds sit in shared memory for
// the range search of every qualifying row.
__global__ void __launch_bounds__(kChainBlock, 1) k_batch_cells(const ChainDev* __restrict__ qs,
                                                                const BatchItem* __restrict__ items,
                                                                uint32_t nitems, uint32_t* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ ChainDev sq;
    const uint32_t warp = threadIdx.x / 32;
    uint32_t* rings = reinterpret_cast<uint32_t*>(smem_raw);
    const SmemGroups no_sg{nullptr, nullptr, nullptr, nullptr, nullptr, 0};
    CellCtx cc;
    cc.sc = smem_cells_at(smem_raw + kRingBytes, kCellSlots);
    int32_t* sb = reinterpret_cast<int32_t*>(smem_raw + kRingBytes + smem_cells_bytes(kCellSlots));
    uint16_t* sl = reinterpret_cast<uint16_t*>(sb + kMaxCellRanges);
    cc.bounds = sb;
    cc.lut = sl;
    cc.lut_len = 0;
    cc.lut_base = 0;

    int64_t cur = -1;
    unsigned long long acnt = 0, asum = 0;
    for (uint32_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        const BatchItem item = items[it];
        if ((int64_t)item.q != cur) {
            __syncthreads();  // every warp is done with the previous scan
            if (cur >= 0) {
                smem_cells_flush(cc.sc, sq.cells, err);
                __syncthreads();  // the flush is done reading sq and the cell table
            }
            cur = item.q;
            for (uint32_t i = threadIdx.x; i < sizeof(ChainDev) / 4; i += kChainBlock)
                reinterpret_cast<uint32_t*>(&sq)[i] = reinterpret_cast<const uint32_t*>(qs + cur)[i];
            const CellsView cv = qs[cur].cells;
            for (uint32_t i = threadIdx.x; i < cv.m; i += kChainBlock) sb[i] = cv.bounds[i];
            for (uint32_t i = threadIdx.x; i < cv.lut_len; i += kChainBlock) sl[i] = cv.lut[i];
            cc.lut_len = cv.lut_len;
            cc.lut_base = cv.lut_base;
            smem_cells_init(cc.sc);
            __syncthreads();
        }
        const ChainDev& a = sq;
        const bool unique = a.table.meta[3] == 0;
        chain_windows<true, true, kTermCells, true>(a, unique, item.lo, item.hi, warp, kChainWarps,
                                                    rings + (size_t)warp * kIdRing, no_sg, acnt, asum, err, &cc);
    }
    if (cur >= 0) {
        __syncthreads();
        smem_cells_flush(cc.sc, sq.cells, err);
    }
}

// Turns a scan's per-range cells into per-bound results: block j becomes the
// sum of blocks 0..j, word by word (sums, counts and the INT32_MIN group's
// pair alike; the directory is shared, so a group has one slot in every block).
__global__ void k_cells_prefix(unsigned long long* __restrict__ vals, uint64_t words, uint32_t m) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < words; x += stride) {
        unsigned long long run = 0;
        for (uint32_t j = 0; j < m; ++j) {
            unsigned long long* p = vals + (size_t)j * words + x;
            run += *p;
            *p = run;
        }
    }
}

cudaError_t launch_cells(const ChainDev* d_scans, const BatchItem* items, uint32_t nitems, cudaStream_t s,
                         Context* ctx) {
    if (nitems == 0) return cudaSuccess;
    const size_t smem = kRingBytes + smem_cells_bytes(kCellSlots) + sizeof(int32_t) * kMaxCellRanges +
                        sizeof(uint16_t) * kCellLut;
    cudaError_t e = cudaFuncSetAttribute(k_batch_cells, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = (int)std::min<uint64_t>((uint64_t)ctx->prop.multiProcessorCount, nitems);
    k_batch_cells<<<grid, kChainBlock, smem, s>>>(d_scans, items, nitems, ctx->d_err);
    ctx->launches++;
    return cudaGetLastError();
}

cudaError_t launch_cells_prefix(const CellsView& c, cudaStream_t s, Context* ctx) {
    if (c.m < 2) return cudaSuccess;
    const uint64_t words = cell_block_words(c.cap);
    const uint64_t want = (words + 255) / 256;
    const uint64_t cap = (uint64_t)ctx->prop.multiProcessorCount * 8;
    k_cells_prefix<<<(int)(want < cap ? want : cap), 256, 0, s>>>(c.vals, words, c.m);
    ctx->launches++;
    return cudaGetLastError();
}

// Packs each query's groups into its output region (unsorted) and counts them;
// one warp-aggregated reservation of output rows per warp (a query's counter
// is one address, and per-row atomics on it serialise in L2).
__global__ void k_batch_compact(const BatchOut* __restrict__ outs, const BatchItem* __restrict__ items,
                                uint32_t nitems, uint32_t* err) {
    const uint32_t lane = lane_id();
    for (uint32_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        const BatchItem item = items[it];
        const BatchOut& o = outs[item.q];
        // whole warps take part in the ballots
        const uint64_t end = item.lo + ((item.hi - item.lo + 31) & ~31ull);
        for (uint64_t i = item.lo + threadIdx.x; i < end; i += blockDim.x) {
            bool keep = false;
            mgv_group_row r{};
            if (i < item.hi) {
                const bool special = i == o.gt.cap;  // one extra index for the group INT32_MIN
                const int32_t k = special ? kEmptyKey : o.gt.keys[i];
                const unsigned long long c = special ? o.gt.special[1] : o.gt.counts[i];
                keep = (special || k != kEmptyKey) && c != 0;
                if (keep) {
                    r.group = k;
                    r.sum = (int64_t)(special ? o.gt.special[0] : o.gt.sums[i]);
                    r.count = (int64_t)c;
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            uint32_t base = 0;
            if (lane == 0 && m) base = atomicAdd(o.count, (uint32_t)__popc(m));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (!keep) continue;
            const uint32_t pos = base + __popc(m & ((1u << lane) - 1u));
            if (pos >= o.capacity) {
                set_error(err, kDevOverflow, 30);
                continue;
            }
            o.rows[pos] = r;
        }
    }
}

// Packs the non-empty groups of a global group table (the group INT32_MIN
// included) into out[0 .. *count); one warp-aggregated reservation per warp.
__global__ void k_group_pack(GroupTableView gt, mgv_group_row* __restrict__ out, uint32_t* count) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t end = ((uint64_t)gt.cap + 1 + 31) & ~31ull;  // whole warps take part in the ballots
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < end; i += stride) {
        const bool special = i == gt.cap;
        bool keep = false;
        mgv_group_row r{};
        if (i <= gt.cap) {
            r.group = special ? kEmptyKey : gt.keys[i];
            const unsigned long long c = special ? gt.special[1] : gt.counts[i];
            keep = c != 0 && (special || r.group != kEmptyKey);
            if (keep) {
                r.sum = (int64_t)(special ? gt.special[0] : gt.sums[i]);
                r.count = (int64_t)c;
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        uint32_t base = 0;
        if (lane_id() == 0 && m) base = atomicAdd(count, (uint32_t)__popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (keep) out[base + __popc(m & ((1u << lane_id()) - 1u))] = r;
    }
}

cudaError_t launch_group_pack(const GroupTableView& gt, mgv_group_row* out, uint32_t* count, cudaStream_t s,
                              Context* ctx) {
    const uint64_t want = ((uint64_t)gt.cap + 1 + 255) / 256;
    const uint64_t cap = (uint64_t)ctx->prop.multiProcessorCount * 8;
    k_group_pack<<<(int)(want < cap ? want : cap), 256, 0, s>>>(gt, out, count);
    ctx->launches++;
    return cudaGetLastError();
}

cudaError_t launch_batch(const ChainDev* d_qs, const BatchOut* d_outs, const BatchItem* probe_items, uint32_t n_probe,
                         const BatchItem* compact_items, uint32_t n_compact, int ctas_per_sm, uint32_t item_order,
                         cudaStream_t s, Context* ctx) {
    const int sms = ctx->prop.multiProcessorCount;
    if (n_probe) {
        const size_t smem = kRingBytes + smem_groups_bytes(kMaxSmemGroups);
        cudaError_t e = cudaFuncSetAttribute(k_batch_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_probe, kChainBlock, smem);
        per_sm = std::max(per_sm, 1);
        if (ctas_per_sm > 0 && ctas_per_sm < per_sm) per_sm = ctas_per_sm;
        const int grid = (int)std::min<uint64_t>((uint64_t)per_sm * sms, n_probe);
        k_batch_probe<<<grid, kChainBlock, smem, s>>>(d_qs, probe_items, n_probe, item_order, ctx->d_err);
        ctx->launches++;
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (n_compact) {
        const int grid = (int)std::min<uint64_t>((uint64_t)sms * 8, n_compact);
        k_batch_compact<<<grid, 256, 0, s>>>(d_outs, compact_items, n_compact, ctx->d_err);
        ctx->launches++;
        return cudaGetLastError();
    }
    return cudaSuccess;
}

template <bool SEL, bool PROBE, int TERM>
static cudaError_t launch_chain_t(const ChainDev& d, size_t smem, uint64_t n, cudaStream_t s, Context* ctx) {
    auto k = k_chain<SEL, PROBE, TERM>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int full = occupancy_grid((const void*)k, kChainBlock, smem, ctx);
    // row offsets inside the kernel are 32-bit: launch at most 2^31 rows at a time
    constexpr uint64_t kChunk = 1ull << 31;
    for (uint64_t base = 0; base < n; base += kChunk) {
        ChainDev c = d;
        c.n = std::min<uint64_t>(kChunk, n - base);
        for (uint32_t i = 0; i < c.ncols; ++i)
            if (c.cols[i]) c.cols[i] += base;
        int grid = full;
        const uint64_t need = ((c.n + kWinRows - 1) / kWinRows + kChainWarps - 1) / kChainWarps;
        if ((uint64_t)grid > need) grid = (int)(need ? need : 1);
        k<<<grid, kChainBlock, smem, s>>>(c, ctx->d_err);
        ctx->launches++;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <int TERM>
static cudaError_t launch_chain_term(const ChainArgs& a, const ChainDev& d, size_t smem, cudaStream_t s, Context* ctx) {
    if (!a.has_probe)
        return a.has_sel ? launch_chain_t<true, false, TERM>(d, smem, a.n, s, ctx)
                         : launch_chain_t<false, false, TERM>(d, smem, a.n, s, ctx);
    return a.has_sel ? launch_chain_t<true, true, TERM>(d, smem, a.n, s, ctx)
                     : launch_chain_t<false, true, TERM>(d, smem, a.n, s, ctx);
}

cudaError_t launch_chain(const ChainArgs& a, cudaStream_t s, Context* ctx) {
    if (a.n == 0) return cudaSuccess;
    ChainDev d{};
    for (uint32_t c = 0; c < a.ncols; ++c) d.cols[c] = a.cols[c];
    d.n = a.n;
    d.ncols = a.ncols;
    d.sel_col = a.sel_col;
    d.sel_bound = a.sel_bound;
    d.table = a.table;
    d.unique = a.unique ? 1u : 0u;
    d.acc = a.acc;
    d.gt = a.gt;
    d.sink = a.sink;
    // carried columns: the probe key and every column the terminal reads
    int32_t slot_of[MGV_MAX_COLS];
    for (int c = 0; c < MGV_MAX_COLS; ++c) slot_of[c] = -1;
    auto carry = [&](int32_t col) -> int32_t {
        if (col < 0) return -1;
        if ((uint32_t)col == a.ncols) return kBP;
        if (slot_of[col] < 0) {
            slot_of[col] = (int32_t)d.nslots;
            d.slot_src[d.nslots++] = col;
        }
        return slot_of[col];
    };
    d.probe_slot = a.has_probe ? carry((int32_t)a.probe_col) : -1;
    d.nref = a.nref;
    for (uint32_t i = 0; i < a.nref; ++i) d.ref[i] = carry(a.ref[i]);
    if (a.term != kTermSink && d.nslots > (uint32_t)kMaxTermSlots) return cudaErrorInvalidValue;
    // the shared group table: as large as the global one (2 x max_groups, a
    // power of two), capped by the tuning's slot limit
    d.smem_groups = a.term == kTermGroupby ? std::min(a.smem_groups, a.gt.cap) : 0;
    const size_t smem = kRingBytes + smem_groups_bytes(d.smem_groups);
    switch (a.term) {
        case kTermAgg: return launch_chain_term<kTermAgg>(a, d, smem, s, ctx);
        case kTermGroupby: return launch_chain_term<kTermGroupby>(a, d, smem, s, ctx);
        default: return launch_chain_term<kTermSink>(a, d, smem, s, ctx);
    }
}

}  // namespace mgv
