/*
 * pcf_bench.h -- measurement helpers of libpcf.so (no counterpart in the
 * reference, which publishes no throughput figures): device peak rates used as
 * roofline denominators, and a count of the library's kernel launches.
 */
#ifndef PCF_BENCH_H
#define PCF_BENCH_H

#include "pcf.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
    PCF_MB_FP32_FMA = 0,
    PCF_MB_SMEM_ATOMIC = 1,
    PCF_MB_SMEM_ATOMIC_F64 = 2,
    PCF_MB_SMEM_ATOMIC_U64 = 3,
    PCF_MB_SMEM_ATOMIC_F32 = 4
};

/* PCF_MB_FP32_FMA: FP32 FMA throughput in TFLOP/s; PCF_MB_SMEM_ATOMIC:
 * conflict-free shared-memory 32-bit atomicAdd throughput in Gop/s; _F64,
 * _U64, _F32: the same for 64-bit float, 64-bit integer and 32-bit float adds. */
pcf_status pcf_microbench(pcf_ctx *ctx, int which, double *result);

/* Context options for tests and tuning.
 *   PCF_OPT_TRIP_FLUSH_BUDGET  adds the isotropic triplet kernel's per-CTA
 *                              u32 histogram absorbs between flushes into the
 *                              u64 global histogram (1 .. 2^31, default 2^31;
 *                              a counter can therefore never wrap).  A small
 *                              budget forces many flushes (a test of them).
 *   PCF_OPT_ABORT_HOST_CHECK   0: calls launch even while an abort is
 *                              requested, so the kernels' own polling is what
 *                              stops them (a test of it); 1 (default): they
 *                              return PCF_ERR_TIMEOUT without launching.
 *   PCF_OPT_PAIR_VARIANT       the weighted one-pass (PCF_BOTH) pair kernel:
 *                              0 (default) four isotropic sub-copies,
 *                              candidates through the L1 path; 1 two
 *                              sub-copies; 2 two sub-copies and candidates
 *                              staged into shared memory by cp.async (the
 *                              measured A/B of staging); 3 the anisotropic
 *                              copy shared by each warp pair, five CTAs per
 *                              SM (single-job launches; others use 0).
 *                              Results are the same in every variant.
 *   PCF_OPT_GRID_BUILD         the grid build: 0 (default) by size (the
 *                              bucketed counting sort from 6M points, the
 *                              per-point one below), 1 per-point, 2
 *                              bucketed wherever its shared arrays allow.
 *                              Grids are the same either way up to the
 *                              order of points inside a cell.
 *   PCF_OPT_GRID_DEFER         0 (default): pcf_grid_build returns a
 *                              complete grid, or the catalog's error.  1:
 *                              it returns once the build is queued; the
 *                              first call that uses the grid completes it
 *                              (waiting only for this build's cell table)
 *                              and reports a catalog error such as
 *                              PCF_ERR_OUT_OF_BOX, as does every later use.
 *                              Building several grids before counting then
 *                              overlaps each build's host work with the next
 *                              build on the device.  Host points passed to a
 *                              deferred build must stay unchanged until that
 *                              first use. */
enum {
    PCF_OPT_TRIP_FLUSH_BUDGET = 1,
    PCF_OPT_ABORT_HOST_CHECK = 2,
    PCF_OPT_PAIR_VARIANT = 3,
    PCF_OPT_GRID_BUILD = 4,
    PCF_OPT_GRID_DEFER = 5
};
pcf_status pcf_ctx_set_option(pcf_ctx *ctx, int option, int64_t value);

/* Kernels this context has launched since it was created. */
int64_t pcf_ctx_launch_count(const pcf_ctx *ctx);

/* Kernel-time log: while enabled, every counting kernel is bracketed by CUDA
 * events on the context stream.  _read synchronises the stream, returns the
 * summed kernel time and the number of logged launches, and clears the log. */
pcf_status pcf_ctx_profile(pcf_ctx *ctx, int enable);
pcf_status pcf_ctx_profile_read(pcf_ctx *ctx, double *total_ms, int64_t *launches);
/* The same log for grid builds (the counting-sort and scatter kernels of
 * each cell structure built while enabled): summed kernel time, number of
 * builds and points gridded; clears that log. */
pcf_status pcf_ctx_profile_read_grid(pcf_ctx *ctx, double *total_ms, int64_t *builds,
                                     int64_t *points);

/* Process-wide allocation counters: device allocations (cudaMalloc) and
 * page-locked host allocations (cudaMallocHost) the library has made, their
 * bytes and the wall time spent in those calls (each of which can stall other
 * threads' work on the device).  out[0..5] = device count, device bytes,
 * device ns, host count, host bytes, host ns. */
pcf_status pcf_alloc_counters(uint64_t out[6]);

#ifdef __cplusplus
}
#endif

#endif
