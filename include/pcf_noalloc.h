/*
 * pcf_noalloc.h -- a pair-histogram entry point of libpcf.so that allocates
 * no device memory.  It has no counterpart in the reference.
 *
 * Some callers cannot call cudaMalloc: plug-in hosts that own the device
 * memory budget and forbid allocations from the libraries they load (a
 * cudaMalloc there fails, or fragments a pool the host manages itself), and
 * processes whose allocator is already at its limit, where a library that
 * allocates per call would fail midway.  pcf_count_pairs_noalloc serves
 * them: its scratch
 * (the cell-sorted copies of both catalogs, the cell and tile tables, the
 * stencil rows and the histogram accumulators) lives in one fixed array of
 * PCF_NOALLOC_SCRATCH_BYTES in the library's device image, which every GPU
 * that loads libpcf.so holds until the process exits.
 */
#ifndef PCF_NOALLOC_H
#define PCF_NOALLOC_H

#include "pcf.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Size of the fixed device scratch array (8 MiB): enough for two catalogs of
 * about 100k points each at the default grid.  Larger inputs are rejected. */
#define PCF_NOALLOC_SCRATCH_BYTES (8u << 20)

/*
 * Same histogram as pcf_count_pairs, computed without allocating:
 *   a, na       device pointer to na points (16-byte aligned, as cudaMalloc gives)
 *   b, nb       device pointer to the second catalog for XY (DR), or NULL for XX
 *   box         periodic / bounding box side; every coordinate in [0, box)
 *   kind        PCF_ISO (bins doubles) or PCF_ANI (bins*bins doubles)
 *   flags       PCF_BPC, PCF_DS_EXACT, PCF_RULE_* as for pcf_count_pairs
 *   hist        device pointer to the output histogram (overwritten)
 *   stream      cudaStream_t to run on (NULL: the legacy default stream)
 * Returns PCF_ERR_UNSUPPORTED when the inputs need more scratch than
 * PCF_NOALLOC_SCRATCH_BYTES, or an anisotropic histogram has more than 2^24
 * bins.  The call waits for `stream` once (it reads the tile count back to
 * size the work queue); hist is complete when `stream` reaches the end of the
 * call's work.  The first call on a device looks up the scratch array's
 * device address; make that first call before any stream capture.  All calls
 * share the one array: calls that overlap on the GPU (other streams, other
 * host threads) race and must be serialised by the caller.
 */
pcf_status pcf_count_pairs_noalloc(const pcf_point *a, int64_t na, const pcf_point *b,
                                   int64_t nb, float box, int kind, int bins, float dmax,
                                   uint32_t flags, double *hist, void *stream);

#ifdef __cplusplus
}
#endif

#endif
