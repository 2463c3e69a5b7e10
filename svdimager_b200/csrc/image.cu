// Moment recombination, ES grid correction and reprojection with bilinear splat.
//
// One thread per rotated-frame pixel (SVDIntegratedImager.cu:1295-1463 fused_interpolation;
// archive/FIPkernels.cu:463-677 accumulation, scaling, coordschange, p2p, finalinterp):
//   t3 = -v33 + sgn(v33) sqrt(1 - (t1 + v13)^2 - (t2 + v23)^2)        (pixel skipped if < 0)
//   R  = | Re sum_slab sum_n J_n(alpha) c_n i^n e^{i beta_slab} M_{slab,n}(x, y) | * (-1)^(x+y)
//        / (Phi(|x|) Phi(|y|)) / N_s,  alpha = 2 pi t3 h, beta_slab = 2 pi t3 centre_slab
// then a SIN deprojection of the pixel to the output grid and a bilinear splat.
// Bessel coefficients and geometry in FP64 (the reference evaluates a FP32 power series,
// SVDIntegratedImager.cu:901-920, whose cancellation grows with alpha).
#include "svdi_internal.cuh"
#include "math.cuh"

namespace svdi {

namespace {

struct SplatTarget {
    double LL, MM;
    bool ok;
};

// Per-launch constants of the deprojection, computed once per block from Vin.
struct ReprojConst {
    double inv_v8;      // 1 / |V[8]|
    double dc_r0_sq;    // (cell in degrees / r0)^2, r0 = 180 / pi
    float xi_f, eta_f;  // V[6] / V[8], V[7] / V[8]
    float r0_dc;        // r0 / cell in degrees
};

__device__ inline ReprojConst reproj_const(const double* V, double dc_rad) {
    ReprojConst c;
    const double r0 = 180.0 / kPi, dc = dc_rad / kPi * 180.0;
    c.inv_v8 = 1.0 / fabs(V[8]);
    c.dc_r0_sq = (dc / r0) * (dc / r0);
    c.xi_f = (float)(V[6] / V[8]);
    c.eta_f = (float)(V[7] / V[8]);
    c.r0_dc = (float)(r0 / dc);
    return c;
}

// SVDIntegratedImager.cu:1325-1379 (simplified SIN deprojection; keeps p1, p2 when h > r0). With
// (x, y) the pixel's offset in degrees and h = |(x, y)|, the reference normalises (x, y) by h,
// scales it back by r = h and adds z r0 (xi, eta), z = 1 - sqrt(1 - (h / r0)^2): the target is
// (p1, p2) moved by z r0 (-xi, eta) / dc pixels. That is evaluated here directly: (p1, p2) in FP64,
// the displacement (at most some tens of pixels) in FP32 with z in the cancellation-free form
// s / (1 + sqrt(1 - s)), s = (h / r0)^2 -- no square root or division in FP64 per pixel.
__device__ inline SplatTarget reproject_sii(long long idx, long long idy, long long N, const ReprojConst& k,
                                            const double* V) {
    const double di2 = (double)N * 0.5;
    const long long half = N / 2;
    const double idxf = (double)idx - di2, idyf = (double)idy - di2;
    const double p1 = (-V[0] * idxf + V[3] * idyf) * k.inv_v8 + di2;
    const double p2 = (-V[1] * idxf + V[4] * idyf) * k.inv_v8 + di2;
    const double xo = p1 - (di2 + 1.0), yo = p2 - (di2 + 1.0);  // offset in pixels
    const double s = fma(xo, xo, yo * yo) * k.dc_r0_sq;          // (h / r0)^2
    double oi0 = p1, oi1 = p2;
    if (s <= 1.0) {  // h <= r0
        const float sf = (float)s;
        const float z = sf / (1.0f + sqrtf(1.0f - sf));
        const float m = z * k.r0_dc;
        oi0 = p1 - (double)(m * k.xi_f);
        oi1 = p2 + (double)(m * k.eta_f);
    }
    return {oi0 - (double)half, oi1 - (double)half, true};
}

// archive/FIPkernels.cu:552-624 (coordschange with the integer half size, then the
// trigonometric SIN p2p of Calabretta & Greisen that drops r^2 > 1)
__device__ inline SplatTarget reproject_fipk(long long idx, long long idy, long long N, double dc_rad,
                                             const double* V) {
    const long long half = N / 2;
    const double dc = dc_rad / kPi * 180.0;
    const double r0 = 180.0 / kPi;
    const double xi = V[6] / V[8], eta = V[7] / V[8];
    const double p1 = (-V[0] * (double)(idx - half) + V[3] * (double)(idy - half)) / fabs(V[8]) + (double)half;
    const double p2 = (-V[1] * (double)(idx - half) + V[4] * (double)(idy - half)) / fabs(V[8]) + (double)half;
    double x = -dc * (p1 - ((double)N / 2.0 + 1.0));
    double y = dc * (p2 - ((double)N / 2.0 + 1.0));
    const double x0 = x / r0, y0 = y / r0, r2 = x0 * x0 + y0 * y0;
    const double phi = (r2 != 0.0) ? atan2(x0, -y0) : 0.0;
    double theta;
    if (r2 < 0.5) theta = acos(sqrt(r2));
    else if (r2 <= 1.0) theta = asin(sqrt(1.0 - r2));
    else return {0.0, 0.0, false};
    double sx, cy;
    sincos(phi, &sx, &cy);
    const double t = kPi / 2.0 - fabs(theta);
    double z, costhe;
    if (t < 1.0e-5) {
        z = theta > 0.0 ? t * t / 2.0 : 2.0 - t * t / 2.0;
        costhe = t;
    } else {
        z = 1.0 - sin(theta);
        costhe = cos(theta);
    }
    const double r = r0 * costhe;
    const double w = xi * xi + eta * eta;
    if (w == 0.0) {
        x = r * sx;
        y = -r * cy;
    } else {
        z *= r0;
        x = r * sx + xi * z;
        y = -r * cy + eta * z;
    }
    const double oi0 = -1.0 / dc * x + (double)N / 2.0 + 1.0;
    const double oi1 = 1.0 / dc * y + (double)N / 2.0 + 1.0;
    return {oi0 - (double)half, oi1 - (double)half, true};
}

// One pixel (x, y) of the rotated frame: moments -> |Re sum| -> grid correction -> reprojection.
template <int KMAX>
__device__ __forceinline__ void recombine_pixel(long long x, long long y, const float2* __restrict__ moments,
                                                const GridGeom& g, long long N, double cell,
                                                const double* __restrict__ vin, const SlabParams& sp,
                                                const float* __restrict__ corr, double inv_n, int reprojection,
                                                int presplat, float* __restrict__ out, double* __restrict__ acc,
                                                int final_batch, bool bad, const ReprojConst& kc) {
    double V[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) V[k] = vin[k];
    const long long half = N / 2;
    const long long xr = x - half, yr = y - half;
    const double t1 = cell * (double)yr, t2 = cell * (double)xr;
    const double ra = 1.0 - (t1 + V[2]) * (t1 + V[2]) - (t2 + V[5]) * (t2 + V[5]);
    if (ra < 0.0) {
        if (presplat && final_batch) out[y * N + x] = __int_as_float(0x7fc00000);  // NaN
        return;
    }
    const double t3 = -V[8] + (V[8] >= 0.0 ? 1.0 : -1.0) * sqrt(ra);

    const int K = sp.K;
    double jv[KMAX];
    bessel_jn_fast(2.0 * kPi * t3 * sp.slab_half, K - 1, jv);
    const long long G = g.G, GG = G * G;
    const long long gidx = GG / 2 + G / 2 + yr * G + xr;  // SVDIntegratedImager.cu:1397
    double sum = 0.0;
    for (int j = 0; j < sp.nslab; ++j) {
        const double centre = sp.r3_min + ((double)j + 0.5) * sp.slab_width;
        const double ph = 2.0 * t3 * centre;     // e^{i pi ph}
        double sb, cb;
        if (fabs(ph) < 0x1p-8) {  // small phase: FP32 is exact to ~1e-7 of ph, far below 1e-9 rad
            float sf, cf;
            sincospif((float)ph, &sf, &cf);
            sb = (double)sf;
            cb = (double)cf;
        } else {
            sincospi(ph, &sb, &cb);
        }
        // the terms n = 4 i + q into four independent FP64 sums (the chain of dependent adds, not
        // the loads, set the pace: wide-field recombination 27.7 -> 22.7 ms)
        const float2* mp = moments + (long long)j * K * GG + gidx;
        double s4[4] = {0.0, 0.0, 0.0, 0.0};
        int n = 0;
        for (; n + 4 <= K; n += 4) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float2 m = mp[(long long)(n + q) * GG];
                const double amp = (n + q == 0) ? jv[0] : 2.0 * jv[n + q];
                double cr, ci;  // amp * i^(n + q) * e^{i beta}, n a multiple of 4
                switch (q) {
                    case 0: cr = amp * cb; ci = amp * sb; break;
                    case 1: cr = -amp * sb; ci = amp * cb; break;
                    case 2: cr = -amp * cb; ci = -amp * sb; break;
                    default: cr = amp * sb; ci = -amp * cb; break;
                }
                s4[q] += cr * (double)m.x - ci * (double)m.y;
            }
        }
        for (; n < K; ++n) {
            const float2 m = mp[(long long)n * GG];
            const double amp = (n == 0) ? jv[0] : 2.0 * jv[n];
            double cr, ci;  // amp * i^n * e^{i beta}
            switch (n & 3) {
                case 0: cr = amp * cb; ci = amp * sb; break;
                case 1: cr = -amp * sb; ci = amp * cb; break;
                case 2: cr = -amp * cb; ci = -amp * sb; break;
                default: cr = amp * sb; ci = -amp * cb; break;
            }
            s4[0] += cr * (double)m.x - ci * (double)m.y;
        }
        sum += (s4[0] + s4[1]) + (s4[2] + s4[3]);
    }
    if ((xr + yr) & 1) sum = -sum;
    const long long ax = xr < 0 ? -xr : xr, ay = yr < 0 ? -yr : yr;
    double signed_sum = sum * (double)corr[ax] * (double)corr[ay];
    if (acc) {  // slab batches: the signed sums add up, |.| is taken once, in the last batch
        signed_sum += acc[y * N + x];
        if (!final_batch) {
            acc[y * N + x] = signed_sum;
            return;
        }
    }
    double value = fabs(signed_sum) * inv_n;
    // a NaN or Inf among the gridded values: every moment cell would be NaN after the FFT, so every
    // valid pixel is NaN (the reference's float atomics, SVDIntegratedImager.cu:1276-1290, carry it)
    if (bad) value = __longlong_as_double(0x7ff8000000000000LL);
    if (presplat) {
        out[y * N + x] = (float)value;
        return;
    }

    const SplatTarget tg = reprojection == SVDI_REPROJ_FIPK ? reproject_fipk(x, y, N, cell, V)
                                                            : reproject_sii(x, y, N, kc, V);
    if (!tg.ok) return;
    const double LL = tg.LL, MM = tg.MM;
    if (!(fabs(LL) < (double)(half - 1) && fabs(MM) < (double)(half - 1))) return;
    const double Lf = floor(LL), Mf = floor(MM), Lc = ceil(LL), Mc = ceil(MM);
    float* d = out + half * N + half;
    atomicAdd(&d[(long long)Mf * N + (long long)Lf], (float)((1 - LL + Lf) * (1 - MM + Mf) * value));
    atomicAdd(&d[(long long)Mc * N + (long long)Lf], (float)((1 - LL + Lf) * (0 + MM - Mf) * value));
    atomicAdd(&d[(long long)Mf * N + (long long)Lc], (float)((0 + LL - Lf) * (1 - MM + Mf) * value));
    atomicAdd(&d[(long long)Mc * N + (long long)Lc], (float)((0 + LL - Lf) * (0 + MM - Mf) * value));
}

// Persistent over 32 x 8 pixel tiles: the per-launch constants (slab geometry, reprojection
// constants, the non-finite flag) are set up once per block.
template <int KMAX>
__global__ void __launch_bounds__(256, 4) k_recombine(const float2* __restrict__ moments, GridGeom g, long long N,
                                                  double cell, const double* __restrict__ vin,
                                                  SlabParams sp, const float* __restrict__ corr,
                                                  double inv_n, int reprojection, int presplat,
                                                  float* __restrict__ out, double* __restrict__ acc,
                                                  int final_batch, const DevPlan* __restrict__ plan,
                                                  const unsigned long long* __restrict__ nonfinite) {
    if (plan) {  // one batch of all slabs: the device plan's slab geometry
        sp.r3_min = plan->sp.r3_min;
        sp.slab_width = plan->sp.slab_width;
        sp.slab_half = plan->sp.slab_half;
        sp.inv_half = plan->sp.inv_half;
    }
    __shared__ ReprojConst kc;
    if (threadIdx.x == 0 && threadIdx.y == 0) kc = reproj_const(vin, cell);
    __syncthreads();
    const bool bad = nonfinite && *nonfinite;
    const long long ntx = (N + 31) / 32, nty = (N + 7) / 8;
    for (long long t = blockIdx.x; t < ntx * nty; t += gridDim.x) {
        const long long ty = t / ntx, tx = t - ty * ntx;
        const long long x = tx * 32 + threadIdx.x, y = ty * 8 + threadIdx.y;
        if (x < N && y < N)
            recombine_pixel<KMAX>(x, y, moments, g, N, cell, vin, sp, corr, inv_n, reprojection, presplat, out, acc,
                                  final_batch, bad, kc);
    }
}

}  // namespace

int launch_recombine(const float2* d_moments, const GridGeom& g, long long N, double cell,
                     const double* d_vin64, const SlabParams& sp, const float* d_corr,
                     double inv_n_total, int reprojection, int presplat, float* d_out,
                     cudaStream_t st, double* d_acc, bool final_batch, const DevPlan* d_plan,
                     const unsigned long long* d_nonfinite) {
    const dim3 block(32, 8);
    const long long tiles = ((N + 31) / 32) * ((N + 7) / 8);
    const dim3 grid((unsigned)std::min<long long>(tiles, 8LL * current_sm_count()));
    if (sp.K <= 1) k_recombine<1><<<grid, block, 0, st>>>(d_moments, g, N, cell, d_vin64, sp, d_corr, inv_n_total, reprojection, presplat, d_out, d_acc, final_batch ? 1 : 0, d_plan, d_nonfinite);
    else if (sp.K <= 8) k_recombine<8><<<grid, block, 0, st>>>(d_moments, g, N, cell, d_vin64, sp, d_corr, inv_n_total, reprojection, presplat, d_out, d_acc, final_batch ? 1 : 0, d_plan, d_nonfinite);
    else if (sp.K <= 16) k_recombine<16><<<grid, block, 0, st>>>(d_moments, g, N, cell, d_vin64, sp, d_corr, inv_n_total, reprojection, presplat, d_out, d_acc, final_batch ? 1 : 0, d_plan, d_nonfinite);
    else if (sp.K <= 32) k_recombine<32><<<grid, block, 0, st>>>(d_moments, g, N, cell, d_vin64, sp, d_corr, inv_n_total, reprojection, presplat, d_out, d_acc, final_batch ? 1 : 0, d_plan, d_nonfinite);
    else if (sp.K <= kMaxTerms) k_recombine<kMaxTerms><<<grid, block, 0, st>>>(d_moments, g, N, cell, d_vin64, sp, d_corr, inv_n_total, reprojection, presplat, d_out, d_acc, final_batch ? 1 : 0, d_plan, d_nonfinite);
    else {
        set_error("recombine: too many Chebyshev terms");
        return SVDI_ERR_UNSUPPORTED;
    }
    SVDI_LAUNCHED();
    return SVDI_OK;
}

}  // namespace svdi
