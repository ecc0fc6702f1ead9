/*
 * pcf_estimator.h -- correlation-function estimators on the device, the step
 * the reference performs in its plotting scripts
 * (cpp/2PCFisotropic/normal/graph_2DPF.py:9-10 estim_LS,
 *  cpp/3PCFisotropic/BPC/graph_3PCF.py:5 estim_LS).
 */
#ifndef PCF_ESTIMATOR_H
#define PCF_ESTIMATOR_H

#include "pcf.h"

#ifdef __cplusplus
extern "C" {
#endif

/*
 * npoint 2: h0=DD, h1=DR, h2=RR -> out = (DD - 2DR + RR)/RR (Landy-Szalay);
 *           zero bins are set to 1e-11 first, as the reference script does.
 * npoint 3: h0=DDD, h1=DDR, h2=DRR, h3=RRR -> out = (DDD - 3DDR + 3DRR - RRR)/RRR,
 *           non-finite results set to 0.
 * n_d, n_r > 0 normalise each histogram by its number of point pairs or
 * triples first (catalogs of different sizes); 0 uses raw counts.
 * nb = number of bins (bins, bins^2, bins^3 ...); arrays host or device.
 */
pcf_status pcf_estimate(pcf_ctx *ctx, int npoint, int nb, const double *h0, const double *h1,
                        const double *h2, const double *h3, int64_t n_d, int64_t n_r,
                        double *out);

#ifdef __cplusplus
}
#endif

#endif
