/*
 * pcf_tune.h -- the autotuner of libpcf.so (no counterpart in the reference,
 * which hard-codes 35 partitions per side and one thread per cell pair).
 *
 * The launch shape of a pair histogram is the cell size (cells per dmax,
 * "refine": the default rule, 3, 4, 5, 6 or 8), the histogram privatisation
 * scheme (-1: the library's rule; 0: a u32 column per lane; 1: one copy per
 * warp with shared atomics; 3: per-warp fixed-point limbs of the exact
 * weight products; 4: lane-private fixed-point limbs (isotropic); for
 * PCF_BOTH a scheme >= 0 means one pass over the candidates for both kinds)
 * and the home-tile size (32 or 16 points per warp item).  The best shape
 * depends on the kind, the bins and the point density, so the tuner times
 * candidates on the caller's own catalogs (every refine x scheme at 32-point
 * tiles, then 16-point tiles at the winner) and records the winner for the
 * class (kind, periodic, XX/XY, weighted, bins, expected neighbours per
 * point in half-octave buckets).  Later counting calls of that class in the
 * same context use it.  The table can be saved and loaded as text.
 */
#ifndef PCF_TUNE_H
#define PCF_TUNE_H

#include "pcf.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pcf_tune_result {
    int refine;       /* chosen cells per dmax                      */
    int hist_mode;    /* chosen histogram scheme                    */
    float best_ms;    /* kernel time of the winner                  */
    float default_ms; /* kernel time of the default shape           */
    int tried;        /* candidates timed                           */
    int tile;         /* chosen home points per tile (32 or 16)     */
    int chunk;        /* chosen work items per ticket at most (8, 4 or 1) */
} pcf_tune_result;

/* Times the candidates for one pair histogram (arguments as pcf_count_pairs)
 * and stores the winner in the context's table. */
pcf_status pcf_autotune_pairs(pcf_ctx *ctx, int kind, const pcf_grid *a, const pcf_grid *b,
                              int bins, float dmax, uint32_t flags, pcf_tune_result *res);
/* Text form: one line "key refine hist_mode ms tile chunk" per class (tile
 * and chunk may be omitted: 32 and 8). */
pcf_status pcf_tune_save(const pcf_ctx *ctx, const char *path);
pcf_status pcf_tune_load(pcf_ctx *ctx, const char *path);
/* Number of classes in the table. */
int pcf_tune_size(const pcf_ctx *ctx);

#ifdef __cplusplus
}
#endif

#endif
