/*
 * pcf_tune.h -- the autotuner of libpcf.so (no counterpart in the reference,
 * which hard-codes 35 partitions per side and one thread per cell pair).
 *
 * The launch shape of a pair histogram is the cell size (cells per dmax,
 * "refine") and the histogram privatisation scheme (0: one column per lane,
 * 1: one copy per warp with shared atomics, 2: global atomics).  The best
 * shape depends on the kind, the bins and the point density, so the tuner
 * times candidates on the caller's own catalogs and records the winner for
 * the class (kind, periodic, XX/XY, weighted, bins, expected neighbours per
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
} pcf_tune_result;

/* Times the candidates for one pair histogram (arguments as pcf_count_pairs)
 * and stores the winner in the context's table. */
pcf_status pcf_autotune_pairs(pcf_ctx *ctx, int kind, const pcf_grid *a, const pcf_grid *b,
                              int bins, float dmax, uint32_t flags, pcf_tune_result *res);
/* Text form: one line "key refine hist_mode ms" per class. */
pcf_status pcf_tune_save(const pcf_ctx *ctx, const char *path);
pcf_status pcf_tune_load(pcf_ctx *ctx, const char *path);
/* Number of classes in the table. */
int pcf_tune_size(const pcf_ctx *ctx);

#ifdef __cplusplus
}
#endif

#endif
