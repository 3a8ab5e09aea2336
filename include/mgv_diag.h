/*
 * mgv_diag.h -- measurement probes of the hardware rates the operators are
 * measured against.  Diagnostics only: NOT part of the drop-in operator
 * API of mgv.h and with no counterpart in the reference; bench.py uses them
 * to measure the ceilings that bound a hash probe on this GPU.
 */
#ifndef MGV_DIAG_H_
#define MGV_DIAG_H_

#include "mgv.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Random 32-byte bucket-read ceiling: times `reps` passes of n hashed
 * 32-byte loads into a table of table_bytes (R = 4 loads in flight per
 * thread, ctas_per_sm CTAs of 256 threads per SM) and returns the mean
 * milliseconds per pass. */
mgv_status mgv_diag_random_gather(mgv_ctx *ctx, uint64_t table_bytes, uint64_t n, uint32_t ctas_per_sm,
                                  uint32_t reps, double *ms_per_pass);

/* Random line-read ceiling by width and by path.  Each lookup reads one
 * aligned block of line_bytes (32, 64 or 128) at a hashed position of a
 * table of table_bytes:
 *   method 0: LSU loads (line_bytes / 32 lanes read one block, 32 bytes
 *             each, `inflight` blocks in flight per lane group);
 *   method 1: TMA tile::gather4 (4 blocks per instruction into shared
 *             memory, `inflight` instructions in flight per issuing lane);
 *   method 2: both in one kernel, `tma_share` of the lookups through TMA.
 * CTAs hold lsu_warps LSU warps and tma_warps TMA warps (method 0 uses no
 * TMA warps, method 1 no LSU warps).  Returns ms per pass of `lookups`. */
typedef struct mgv_diag_gather_desc {
    uint64_t table_bytes;
    uint64_t lookups;
    uint32_t line_bytes;
    uint32_t method;
    uint32_t ctas_per_sm;
    uint32_t reps;
    uint32_t inflight;
    uint32_t lsu_warps;
    uint32_t tma_warps;
    float tma_share;
} mgv_diag_gather_desc;

mgv_status mgv_diag_gather(mgv_ctx *ctx, const mgv_diag_gather_desc *d, double *ms_per_pass);

#ifdef __cplusplus
}
#endif

#endif /* MGV_DIAG_H_ */
