// estimator.cu -- correlation-function estimators from the histograms, on
// the device.
//
// The reference leaves this to its plotting scripts:
//   2-point: xi = (DD - 2 DR + RR) / RR with zero bins of each histogram set
//            to 1e-11 first (cpp/2PCFisotropic/normal/graph_2DPF.py:9-16)
//   3-point: zeta = (DDD - 3 DDR + 3 DRR - RRR) / RRR with NaN / inf -> 0
//            (cpp/3PCFisotropic/BPC/graph_3PCF.py:5-21)
// on raw counts of equal-size catalogs.  With n_d, n_r > 0 every histogram is
// first divided by its number of point pairs / triples (DD: n_d (n_d - 1),
// DR: n_d n_r, ... ), which is the estimator for catalogs of different sizes.
#include <cmath>

#include "../../include/pcf_estimator.h"
#include "pcf_internal.cuh"

namespace {

__global__ void k_ls2(const double *dd, const double *dr, const double *rr, double a, double b,
                      double c, int n, double *xi) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double DD = dd[k], DR = dr[k], RR = rr[k];
    if (DD == 0.0) DD = 1e-11;
    if (DR == 0.0) DR = 1e-11;
    if (RR == 0.0) RR = 1e-11;
    DD *= a;
    DR *= b;
    RR *= c;
    xi[k] = (DD - 2.0 * DR + RR) / RR;
}

__global__ void k_ls3(const double *ddd, const double *ddr, const double *drr, const double *rrr,
                      double a, double b, double c, double d, int n, double *zeta) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double v = (a * ddd[k] - 3.0 * b * ddr[k] + 3.0 * c * drr[k] - d * rrr[k]) / (d * rrr[k]);
    zeta[k] = isfinite(v) ? v : 0.0;
}

}  // namespace

extern "C" pcf_status pcf_estimate(pcf_ctx *ctx, int npoint, int nb, const double *h0,
                                   const double *h1, const double *h2, const double *h3,
                                   int64_t n_d, int64_t n_r, double *out) {
    if (!ctx || nb < 1 || !h0 || !h1 || !h2 || !out || (npoint != 2 && npoint != 3) ||
        (npoint == 3 && !h3))
        return PCF_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    const int nh = npoint == 2 ? 3 : 4;
    PCF_CU(ctx, ctx->scratch_b.ensure(sizeof(double) * (size_t)nb * (nh + 1)));
    double *d = ctx->scratch_b.as<double>();
    const double *src[4] = {h0, h1, h2, h3};
    for (int i = 0; i < nh; ++i)
        PCF_CU(ctx, cudaMemcpyAsync(d + (size_t)i * nb, src[i], sizeof(double) * nb, cudaMemcpyDefault,
                                    ctx->stream));
    double *o = d + (size_t)nh * nb;
    const bool norm = n_d > 0 && n_r > 0;
    const double D = (double)n_d, R = (double)n_r;
    if (npoint == 2) {
        // DD, DR, RR
        const double a = norm ? 1.0 / (D * (D - 1)) : 1.0, b = norm ? 1.0 / (D * R) : 1.0,
                     c = norm ? 1.0 / (R * (R - 1)) : 1.0;
        k_ls2<<<(nb + 255) / 256, 256, 0, ctx->stream>>>(d, d + nb, d + 2 * nb, a, b, c, nb, o);
    } else {
        // DDD, DDR, DRR, RRR
        const double a = norm ? 1.0 / (D * (D - 1) * (D - 2)) : 1.0,
                     b = norm ? 1.0 / (D * (D - 1) * R) : 1.0, c = norm ? 1.0 / (D * R * (R - 1)) : 1.0,
                     e = norm ? 1.0 / (R * (R - 1) * (R - 2)) : 1.0;
        k_ls3<<<(nb + 255) / 256, 256, 0, ctx->stream>>>(d, d + nb, d + 2 * nb, d + 3 * nb, a, b, c, e,
                                                         nb, o);
    }
    PCF_CU(ctx, cudaGetLastError());
    ++ctx->launches;
    PCF_CU(ctx, cudaMemcpyAsync(out, o, sizeof(double) * nb, cudaMemcpyDefault, ctx->stream));
    PCF_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return PCF_OK;
}
