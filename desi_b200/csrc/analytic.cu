// analytic.cu -- closed-form periodic-box histograms.
//
//  * pcf_analytic_rr: RR (and DR, written as the same histogram) of
//    pcf_2iso_BPCanalytic (cuda/pcf2isoBPC.cuh:166,199-202) and the kernel
//    RR2iso_BPC_analytic (cuda/kernels/2isoBPC_k.cuh:559):
//    RR[k] = alpha (3k^2 + 3k + 1), alpha = 8 dr^3 acos(0) beta / 3 with
//    dr = dmax/bins and beta = N^2 / L^3 evaluated in FP32 as there.
//  * pcf_analytic_3iso: pcf_3isoBPC_analytic (cuda/pcf3isoBPC.cuh:177): fine
//    DD histograms at ptt*bins and ptt*bn_ref*bins bins (DD2iso_forBPC,
//    3isoBPC_k.cuh:1694), their analytic RR, the bin averages make_ff_av /
//    make_ff_av_ref (:1984, :2001), and make_histo_analitic (:2021).
//
// make_histo_analitic refines every coarse bin that the triangle inequality
// cuts into bn_ref^3 sub-cubes, keeping a sub-cube when all 8 corners
// satisfy the triangle inequality.  FP64 addition is monotone, so the
// 8-corner test equals its worst corner:
//   (ru + rv >= rw + h) and (ru + rw >= rv + h) and (rv + rw >= ru + h),
// every sum rounded as the reference's, and for fixed (u, v) the kept w
// form one interval (the first clause is decreasing in w, the others
// increasing).  Each (u, v) then costs two binary searches and two prefix
// sums over w instead of bn_ref corner tests:
//   sum_w c = (ru+h/2)(rv+h/2) S1,  sum_w f = (ru+h/2)(rv+h/2)[(1+A_u+B_v) S1 + S2]
// with S1 = sum (rw+h/2), S2 = sum ff_ref[k*bn_ref+w]/3 over the interval.
// Sums are in FP64 in a different order than the reference's sequential
// loop (relative differences ~1e-13).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "pcf_internal.cuh"

namespace {

// 3k^2+3k+1 as the reference evaluates it in 32-bit int (2isoBPC_k.cuh:564,
// wrapping once k > 26754), or exactly when wrap == 0.
__device__ __forceinline__ double shell_coef(long long k, int wrap) {
    if (wrap) {
        unsigned u = 3u * (unsigned)k * (unsigned)k + 3u * (unsigned)k + 1u;
        return (double)(int)u;
    }
    return (double)(3 * k * k + 3 * k + 1);
}

__global__ void k_rr_analytic(double *rr, double alpha, long long n, int wrap) {
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) rr[k] = __dmul_rn(alpha, shell_coef(k, wrap));
}

// make_ff_av (3isoBPC_k.cuh:1984): ff[i] = sum_j (ri + rj) (DD/RR - 1) / ptt.
__global__ void k_ff_av(const double *dd, const double *rr, float dmax, int bins, int bn_ff, int ptt,
                        double *ff) {
    const int i = blockIdx.x;
    __shared__ double s[256];
    double acc = 0.0;
    for (int j = threadIdx.x; j < ptt; j += blockDim.x) {
        const int i_ = i * ptt;
        const float idm = __fmul_rn((float)i, dmax);
        const double ri = __ddiv_rn((double)idm, (double)bins);
        const double rj = __ddiv_rn(__dmul_rn((double)j + 0.5, (double)dmax), (double)bn_ff);
        const double q = __dsub_rn(__ddiv_rn(dd[i_ + j], rr[i_ + j]), 1.0);
        acc += __ddiv_rn(__dmul_rn(__dadd_rn(ri, rj), q), (double)ptt);
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) ff[i] = s[0];
}

// make_ff_av_ref (3isoBPC_k.cuh:2001): ffr[i*bn_ref+j] = sum_k (ri+rj+rk)(DD/RR-1)/ptt.
__global__ void k_ff_av_ref(const double *dd, const double *rr, float dmax, int bins, int bn_ref,
                            int ptt, double *ffr) {
    const int ij = blockIdx.x;  // i*bn_ref + j
    const int i = ij / bn_ref, j = ij % bn_ref;
    __shared__ double s[128];
    double acc = 0.0;
    const double dr = __ddiv_rn((double)dmax, (double)bins);
    const double dr_ref = __ddiv_rn(dr, (double)bn_ref);
    const double dr_ptt_ref = __ddiv_rn((double)dmax, (double)((long long)ptt * bn_ref * bins));
    const double ri = __dmul_rn((double)i, dr), rj = __dmul_rn((double)j, dr_ref);
    for (int k = threadIdx.x; k < ptt; k += blockDim.x) {
        const double rk = __dmul_rn((double)k + 0.5, dr_ptt_ref);
        const long long sidx = ((long long)i * bn_ref) * ptt + (long long)j * ptt + k;
        const double q = __dsub_rn(__ddiv_rn(dd[sidx], rr[sidx]), 1.0);
        acc += __ddiv_rn(__dmul_rn(__dadd_rn(__dadd_rn(ri, rj), rk), q), (double)ptt);
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) ffr[ij] = s[0];
}

// Corner count of the cube [r1,r1+h]x[r2,r2+h]x[r3,r3+h] that satisfy the
// triangle inequality, with the reference's roundings (3isoBPC_k.cuh:2040).
__device__ int corners(double ri, double rj, double rk, double h) {
    int v = 0;
    for (int a = 0; a < 2; ++a) {
        const double r1 = __dadd_rn(ri, __dmul_rn((double)a, h));
        for (int b = 0; b < 2; ++b) {
            const double r2 = __dadd_rn(rj, __dmul_rn((double)b, h));
            for (int c = 0; c < 2; ++c) {
                const double r3 = __dadd_rn(rk, __dmul_rn((double)c, h));
                if (__dadd_rn(r1, r2) >= r3 && __dadd_rn(r1, r3) >= r2 && __dadd_rn(r2, r3) >= r1) ++v;
            }
        }
    }
    return v;
}

// Full coarse bins (all 8 corners) in closed form; partial bins flagged.
__global__ void k_coarse(int bins, double dr, double alpha, const double *ff, double *ddr,
                         double *rrr, unsigned char *partial) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n3 = bins * bins * bins;
    if (t >= n3) return;
    const int i = t / (bins * bins), j = (t / bins) % bins, k = t % bins;
    const double dr2 = __dmul_rn(dr, 0.5);
    const double ri = __dmul_rn((double)i, dr), rj = __dmul_rn((double)j, dr), rk = __dmul_rn((double)k, dr);
    const int v = corners(ri, rj, rk, dr);
    partial[t] = (v > 0 && v < 8) ? 1 : 0;
    if (v == 8) {
        const double ai = __dadd_rn(ri, dr2), aj = __dadd_rn(rj, dr2), ak = __dadd_rn(rk, dr2);
        const double s = __dmul_rn(__dmul_rn(__dmul_rn(alpha, ai), aj), ak);
        rrr[t] = s;
        double f = 1.0;
        f = __dadd_rn(f, __ddiv_rn(ff[i], __dmul_rn(3.0, ai)));
        f = __dadd_rn(f, __ddiv_rn(ff[j], __dmul_rn(3.0, aj)));
        f = __dadd_rn(f, __ddiv_rn(ff[k], __dmul_rn(3.0, ak)));
        ddr[t] = __dmul_rn(f, s);
    } else {
        rrr[t] = 0.0;
        ddr[t] = 0.0;
    }
}

constexpr int kRefMax = 512;

// One CTA per coarse bin; partial bins refined on the bn_ref^3 sub-grid.
__global__ void __launch_bounds__(256) k_refine(int bins, int bn_ref, double dr, double alpha_ref,
                                                const double *ffr, const unsigned char *partial,
                                                double *ddr, double *rrr) {
    const int t = blockIdx.x;
    if (!partial[t]) return;
    const int i = t / (bins * bins), j = (t / bins) % bins, k = t % bins;
    const double h = __ddiv_rn(dr, (double)bn_ref);
    const double h2 = __dmul_rn(h, 0.5);
    const double ri = __dmul_rn((double)i, dr), rj = __dmul_rn((double)j, dr), rk = __dmul_rn((double)k, dr);
    __shared__ double rw[kRefMax], S1[kRefMax + 1], S2[kRefMax + 1];
    __shared__ double red[2][256];
    for (int w = threadIdx.x; w < bn_ref; w += blockDim.x) rw[w] = __dadd_rn(rk, __dmul_rn((double)w, h));
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        S1[0] = 0.0;
        S2[0] = 0.0;
        for (int w = 0; w < bn_ref; ++w) {
            a += __dadd_rn(rw[w], h2);
            b += __ddiv_rn(ffr[(long long)k * bn_ref + w], 3.0);
            S1[w + 1] = a;
            S2[w + 1] = b;
        }
    }
    __syncthreads();
    double accS = 0.0, accF = 0.0;
    const int nuv = bn_ref * bn_ref;
    for (int uv = threadIdx.x; uv < nuv; uv += blockDim.x) {
        const int u = uv / bn_ref, v = uv % bn_ref;
        const double ru = __dadd_rn(ri, __dmul_rn((double)u, h));
        const double rv = __dadd_rn(rj, __dmul_rn((double)v, h));
        const double ruh = __dadd_rn(ru, h), rvh = __dadd_rn(rv, h);
        const double suv = __dadd_rn(ru, rv);
        // D(w): ru + rv >= rw + h (decreasing in w); U(w): ru + rw >= rv + h and
        // rv + rw >= ru + h (increasing in w)
        auto D = [&](int w) { return suv >= __dadd_rn(rw[w], h); };
        auto U = [&](int w) { return __dadd_rn(ru, rw[w]) >= rvh && __dadd_rn(rv, rw[w]) >= ruh; };
        // largest w with D(w)
        int lo = 0, hi = bn_ref;  // D true on [0, lo), false on [hi, n)
        while (lo < hi) {
            const int m = (lo + hi) >> 1;
            if (D(m)) lo = m + 1; else hi = m;
        }
        const int wend = lo;  // exclusive
        // smallest w with U(w)
        lo = 0;
        hi = bn_ref;
        while (lo < hi) {
            const int m = (lo + hi) >> 1;
            if (U(m)) hi = m; else lo = m + 1;
        }
        const int wbeg = lo;
        if (wbeg >= wend) continue;
        const double au = __dadd_rn(ru, h2), av = __dadd_rn(rv, h2);
        const double cuv = __dmul_rn(au, av);
        const double s1 = S1[wend] - S1[wbeg], s2 = S2[wend] - S2[wbeg];
        const double A = __ddiv_rn(ffr[(long long)i * bn_ref + u], __dmul_rn(3.0, au));
        const double B = __ddiv_rn(ffr[(long long)j * bn_ref + v], __dmul_rn(3.0, av));
        accS += cuv * s1;
        accF += cuv * ((1.0 + A + B) * s1 + s2);
    }
    red[0][threadIdx.x] = accS;
    red[1][threadIdx.x] = accF;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            red[0][threadIdx.x] += red[0][threadIdx.x + o];
            red[1][threadIdx.x] += red[1][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && red[0][0] != 0.0) {
        rrr[t] += red[0][0] * alpha_ref;
        ddr[t] += red[1][0] * alpha_ref;
    }
}

// alpha of RR2iso_BPC_analytic (pcf2isoBPC.cuh:199-202, pcf3isoBPC.cuh:236-242):
// dr = dmax/bins and beta = (N*N)/L^3 in FP32, then 8 dr^3 acos(0) beta / 3.
double rr_alpha(int64_t np, float L, float dmax, int64_t bins) {
    const float drf = dmax / (float)bins;
    const double dr = (double)drf;
    const float L3 = L * L * L;
    const float betaf = (float)(np * np) / L3;
    const double beta = (double)betaf;
    return 8 * dr * dr * dr * std::acos(0.0) * beta / 3;
}

}  // namespace

extern "C" pcf_status pcf_analytic_rr(pcf_ctx *ctx, int bins, int64_t n, float box, float dmax,
                                      int wrap, double *rr) {
    if (!ctx || bins < 1 || n < 1 || !(box > 0.f) || !(dmax > 0.f) || !rr) return PCF_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    PCF_CU(ctx, ctx->d_hist.ensure(sizeof(double) * (size_t)bins + 64));
    double *d = ctx->d_hist.as<double>();
    k_rr_analytic<<<(bins + 255) / 256, 256, 0, ctx->stream>>>(d, rr_alpha(n, box, dmax, bins), bins,
                                                                wrap);
    PCF_CU(ctx, cudaGetLastError());
    ++ctx->launches;
    PCF_CU(ctx, cudaMemcpyAsync(rr, d, sizeof(double) * bins, cudaMemcpyDeviceToHost, ctx->stream));
    PCF_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return PCF_OK;
}

extern "C" pcf_status pcf_analytic_3iso(pcf_ctx *ctx, const pcf_grid *d_, int bins, float dmax,
                                        int ptt, int bn_ref, int wrap, double *ddd, double *ddr,
                                        double *rrr, pcf_stats *stats) {
    if (!ctx || !d_ || bins < 1 || !(dmax > 0.f) || !ddr || !rrr) return PCF_ERR_INVALID_ARG;
    if (ptt <= 0) ptt = 100;       // pcf3isoBPC.cuh:205
    if (bn_ref <= 0) bn_ref = 200;
    if (bn_ref > kRefMax) return PCF_ERR_UNSUPPORTED;
    cudaSetDevice(ctx->device);
    {
        pcf_status s0 = grid_finish(ctx, d_);
        if (s0 != PCF_OK) return s0;
    }
    pcf_grid *D = const_cast<pcf_grid *>(d_);
    const float L = D->box;
    if (!(2.0 * (double)dmax < (double)L)) return PCF_ERR_UNSUPPORTED;
    const int64_t np = D->n;
    const int64_t bn_ff = (int64_t)ptt * bins;
    const int64_t bn_ffr = (int64_t)ptt * bn_ref * bins;
    if (bn_ffr > (1 << 26)) return PCF_ERR_UNSUPPORTED;
    pcf_status s;
    float kernel_ms = 0.f;
    // DDD, counted (XXX3iso_BPC)
    if (ddd) {
        pcf_stats st{};
        s = pcf_count_triplets(ctx, PCF_ISO, D, nullptr, bins, dmax, PCF_BPC, ddd, &st);
        if (s != PCF_OK) return s;
        kernel_ms += st.kernel_ms;
    }
    // fine DD at bn_ff and bn_ffr bins: ordered pairs, periodic, 0 < d < dmax,
    // ds = (float)bins_fine / dmax as DD2iso_forBPC computes it
    DevBuf fine;
    fine.pool = ctx->pool;
    const size_t n3 = (size_t)bins * bins * bins;
    PCF_CU(ctx, fine.ensure(sizeof(double) * (size_t)(2 * bn_ff + 2 * bn_ffr + bins + bins * bn_ref +
                                                      2 * n3) + n3 + 1024));
    double *dd_ff = fine.as<double>();
    double *dd_ffr = dd_ff + bn_ff;
    double *rr_ff = dd_ffr + bn_ffr;
    double *rr_ffr = rr_ff + bn_ff;
    double *ff = rr_ffr + bn_ffr;
    double *ffr = ff + bins;
    double *d_ddr = ffr + (size_t)bins * bn_ref;
    double *d_rrr = d_ddr + n3;
    unsigned char *partial = reinterpret_cast<unsigned char *>(d_rrr + n3);
    for (int pass = 0; pass < 2; ++pass) {
        const int64_t nbf = pass ? bn_ffr : bn_ff;
        const float dsf = (float)nbf / dmax;
        pcf_stats st{};
        s = pcf_count_pairs_ds(ctx, D, (int)nbf, dmax, (double)dsf, PCF_BPC | PCF_DEVICE_OUT,
                               pass ? dd_ffr : dd_ff, &st);
        if (s != PCF_OK) return s;
        kernel_ms += st.kernel_ms;
    }
    // analytic RR at the fine binnings (RR2iso_BPC_analytic with alpha_ff*)
    const double alpha_ff = rr_alpha(np, L, dmax, bn_ff);
    const double alpha_ffr = rr_alpha(np, L, dmax, bn_ffr);
    cudaStream_t st = ctx->stream;
    k_rr_analytic<<<(unsigned)((bn_ff + 255) / 256), 256, 0, st>>>(rr_ff, alpha_ff, bn_ff, wrap);
    k_rr_analytic<<<(unsigned)((bn_ffr + 255) / 256), 256, 0, st>>>(rr_ffr, alpha_ffr, bn_ffr, wrap);
    k_ff_av<<<bins, 128, 0, st>>>(dd_ff, rr_ff, dmax, bins, (int)bn_ff, ptt, ff);
    k_ff_av_ref<<<bins * bn_ref, 128, 0, st>>>(dd_ffr, rr_ffr, dmax, bins, bn_ref, ptt, ffr);
    // constants of pcf3isoBPC.cuh:244-247
    const double dr = dmax / (double)bins;
    const double dr_ref = dr / bn_ref;
    const float Vf = L * L;
    const double V = (double)Vf;
    const double beta_3D = np / V;
    double gama = 8 * (4 * std::acos(0.0) * std::acos(0.0)) * (np * beta_3D * beta_3D);
    gama /= V;
    const double alpha_ref = gama * dr_ref * dr_ref * dr_ref, alpha = gama * dr * dr * dr;
    k_coarse<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(bins, dr, alpha, ff, d_ddr, d_rrr, partial);
    k_refine<<<(unsigned)n3, 256, 0, st>>>(bins, bn_ref, dr, alpha_ref, ffr, partial, d_ddr, d_rrr);
    PCF_CU(ctx, cudaGetLastError());
    ctx->launches += 6;
    PCF_CU(ctx, cudaMemcpyAsync(ddr, d_ddr, sizeof(double) * n3, cudaMemcpyDeviceToHost, st));
    PCF_CU(ctx, cudaMemcpyAsync(rrr, d_rrr, sizeof(double) * n3, cudaMemcpyDeviceToHost, st));
    PCF_CU(ctx, cudaStreamSynchronize(st));
    if (stats) {
        stats->kernel_ms = kernel_ms;
        stats->partitions = D->cells ? D->cells->P : 0;
    }
    return PCF_OK;
}
