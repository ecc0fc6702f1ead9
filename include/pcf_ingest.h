/*
 * pcf_ingest.h -- catalog files.  Replaces open_files
 * (cuda/create_grid.cuh:35-78): text rows "x y z w" (any whitespace), parsed
 * on all host threads, or the binary form ".f4" (raw little-endian float32
 * x, y, z, w per point).
 */
#ifndef PCF_INGEST_H
#define PCF_INGEST_H

#include "pcf.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Reads the first n points of path into out (n entries).  n_read receives
 * the number read; box_candidate (may be NULL) the reference's automatic box
 * ceil(max component + 1).  PCF_ERR_IO if the file is missing, malformed or
 * holds fewer than n points. */
pcf_status pcf_read_catalog(const char *path, int64_t n, pcf_point *out, int64_t *n_read,
                            float *box_candidate);
/* Writes n points in the binary ".f4" form. */
pcf_status pcf_write_catalog_f4(const char *path, const pcf_point *pts, int64_t n);

#ifdef __cplusplus
}
#endif

#endif
