// Pre-processing kernels: FP64 SVD rotation of the baselines, flag/weight polarisation collapse,
// Chebyshev statistics.
//
// The reference (SVDIntegratedImager.cu:409-865) expands every sample's baseline in FP32
// (3 x N_s floats), reduces it with float atomics, runs a cuBLAS SGEMM for the covariance and
// cuSOLVER SYEVD. Here the baselines b_k = uvw_row * f_chan / c are separable, so the mean and
// covariance come from per-row sums times per-channel sums (one pass over the rows only):
//   sum_k b = (sum_row uvw) (sum_chan s),  sum_k b b^T = (sum_row uvw uvw^T) (sum_chan s^2),
// with s = f / c, all in FP64 with a fixed reduction order (deterministic). The 3x3
// eigenproblem is solved by Jacobi rotations in one thread, and the projection keeps the
// separable form: r[row + chan*R] = s[chan] * (Vin . uvw_row).
#include "svdi_internal.cuh"
#include "math.cuh"

namespace svdi {

namespace {

constexpr int kThreads = 256;

template <typename T, int N>
__device__ inline void block_sum(T (&v)[N], T* smem /* [N][kThreads] */) {
    const int t = threadIdx.x;
    for (int k = 0; k < N; ++k) smem[k * kThreads + t] = v[k];
    __syncthreads();
    for (int stride = kThreads / 2; stride > 0; stride >>= 1) {
        if (t < stride)
            for (int k = 0; k < N; ++k) smem[k * kThreads + t] += smem[k * kThreads + t + stride];
        __syncthreads();
    }
    for (int k = 0; k < N; ++k) v[k] = smem[k * kThreads];
    __syncthreads();
}

// Per-block partial sums of uvw (3) and uvw uvw^T (6) over rows.
__global__ void __launch_bounds__(kThreads) k_row_moments(const float* __restrict__ uvw, long long R,
                                                         double* __restrict__ partial) {
    __shared__ double sm[9 * kThreads];
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (long long r = blockIdx.x * (long long)kThreads + threadIdx.x; r < R;
         r += (long long)gridDim.x * kThreads) {
        const double u = uvw[r * 3 + 0], w1 = uvw[r * 3 + 1], w2 = uvw[r * 3 + 2];
        v[0] += u; v[1] += w1; v[2] += w2;
        v[3] += u * u; v[4] += u * w1; v[5] += u * w2;
        v[6] += w1 * w1; v[7] += w1 * w2; v[8] += w2 * w2;
    }
    block_sum<double, 9>(v, sm);
    if (threadIdx.x == 0)
        for (int k = 0; k < 9; ++k) partial[blockIdx.x * 9 + k] = v[k];
}

// One block: final reduction, channel sums, covariance, Jacobi, orientation.
__global__ void __launch_bounds__(kThreads) k_basis(const double* __restrict__ partial, int nblocks,
                                                   const float* __restrict__ freq, long long C,
                                                   long long R, float array_center_x,
                                                   double* __restrict__ vin64, float* __restrict__ vin32,
                                                   double* __restrict__ s_out, double* __restrict__ stats) {
    __shared__ double sm[9 * kThreads];
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < nblocks; b += kThreads)
        for (int k = 0; k < 9; ++k) v[k] += partial[b * 9 + k];
    block_sum<double, 9>(v, sm);
    double cs[2] = {0, 0};
    double smin = 1e300, smax = -1e300;
    for (long long c = threadIdx.x; c < C; c += kThreads) {
        const double s = (double)freq[c] / kCLight;
        s_out[c] = s;
        cs[0] += s;
        cs[1] += s * s;
        smin = fmin(smin, s);
        smax = fmax(smax, s);
    }
    block_sum<double, 2>(cs, sm);
    // min / max of s
    sm[threadIdx.x] = smin;
    sm[kThreads + threadIdx.x] = smax;
    __syncthreads();
    for (int stride = kThreads / 2; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride) {
            sm[threadIdx.x] = fmin(sm[threadIdx.x], sm[threadIdx.x + stride]);
            sm[kThreads + threadIdx.x] = fmax(sm[kThreads + threadIdx.x], sm[kThreads + threadIdx.x + stride]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double ns = (double)R * (double)C;
        double m[3], cov[9];
        for (int a = 0; a < 3; ++a) m[a] = v[a] * cs[0] / ns;
        const int sym[9] = {3, 4, 5, 4, 6, 7, 5, 7, 8};
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) cov[a * 3 + b] = v[sym[a * 3 + b]] * cs[1] - ns * m[a] * m[b];
        double ev[3], evec[9], vin[9];
        jacobi3(cov, ev, evec);
        orient_basis(evec, array_center_x, vin);
        for (int k = 0; k < 9; ++k) {
            vin64[k] = vin[k];
            vin32[k] = (float)vin[k];
        }
        stats[ST_S_MIN] = sm[0];
        stats[ST_S_MAX] = sm[kThreads];
        stats[ST_EIG0] = ev[0];
        stats[ST_EIG1] = ev[1];
        stats[ST_EIG2] = ev[2];
    }
}

// q[row] = Vin . uvw_row (FP64) and per-block min/max of r3 = s * q3 over the row's channels.
__global__ void __launch_bounds__(kThreads) k_project_rows(const float* __restrict__ uvw, long long R,
                                                          const double* __restrict__ vin,
                                                          const double* __restrict__ stats,
                                                          double* __restrict__ q,
                                                          double* __restrict__ partial) {
    __shared__ double sm[2 * kThreads];
    double v[9];
    for (int k = 0; k < 9; ++k) v[k] = vin[k];
    const double smin = stats[ST_S_MIN], smax = stats[ST_S_MAX];
    double lo = 1e300, hi = -1e300;
    for (long long r = blockIdx.x * (long long)kThreads + threadIdx.x; r < R;
         r += (long long)gridDim.x * kThreads) {
        const double u = uvw[r * 3 + 0], w1 = uvw[r * 3 + 1], w2 = uvw[r * 3 + 2];
        double qq[3];
        for (int a = 0; a < 3; ++a) {
            qq[a] = v[a * 3 + 0] * u + v[a * 3 + 1] * w1 + v[a * 3 + 2] * w2;
            q[r * 3 + a] = qq[a];
        }
        // s > 0: the extremes of s * q3 over channels sit at s_min / s_max
        const double e0 = smin * qq[2], e1 = smax * qq[2];
        lo = fmin(lo, fmin(e0, e1));
        hi = fmax(hi, fmax(e0, e1));
    }
    sm[threadIdx.x] = lo;
    sm[kThreads + threadIdx.x] = hi;
    __syncthreads();
    for (int stride = kThreads / 2; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride) {
            sm[threadIdx.x] = fmin(sm[threadIdx.x], sm[threadIdx.x + stride]);
            sm[kThreads + threadIdx.x] = fmax(sm[kThreads + threadIdx.x], sm[kThreads + threadIdx.x + stride]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[blockIdx.x * 2 + 0] = sm[0];
        partial[blockIdx.x * 2 + 1] = sm[kThreads];
    }
}

// Final min/max of r3 partials -> stats.
__global__ void __launch_bounds__(kThreads) k_minmax_final(const double* __restrict__ partial, int nblocks,
                                                          double* __restrict__ stats) {
    __shared__ double sm[2 * kThreads];
    double lo = 1e300, hi = -1e300;
    for (int b = threadIdx.x; b < nblocks; b += kThreads) {
        lo = fmin(lo, partial[b * 2 + 0]);
        hi = fmax(hi, partial[b * 2 + 1]);
    }
    sm[threadIdx.x] = lo;
    sm[kThreads + threadIdx.x] = hi;
    __syncthreads();
    for (int stride = kThreads / 2; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride) {
            sm[threadIdx.x] = fmin(sm[threadIdx.x], sm[threadIdx.x + stride]);
            sm[kThreads + threadIdx.x] = fmax(sm[kThreads + threadIdx.x], sm[kThreads + threadIdx.x + stride]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        stats[ST_R3_MIN] = sm[0];
        stats[ST_R3_MAX] = sm[kThreads];
    }
}

// Flag / WEIGHT_SPECTRUM collapse (SVDIntegratedImager.cu:588-617), one rounding per operation.
__global__ void __launch_bounds__(kThreads) k_collapse(const float* __restrict__ v0r, const float* __restrict__ v0i,
                                                      const float* __restrict__ v3r, const float* __restrict__ v3i,
                                                      const uint8_t* __restrict__ f0, const uint8_t* __restrict__ f3,
                                                      const float* __restrict__ w0in, const float* __restrict__ w3in,
                                                      float* __restrict__ outr, float* __restrict__ outi,
                                                      long long n) {
    for (long long k = blockIdx.x * (long long)kThreads + threadIdx.x; k < n;
         k += (long long)gridDim.x * kThreads) {
        const float w0 = f0[k] ? 0.0f : w0in[k];
        const float w3 = f3[k] ? 0.0f : w3in[k];
        const float ws = __fadd_rn(w0, w3);
        float re = 0.0f, im = 0.0f;
        if (ws > 0.0f) {
            re = __fdiv_rn(__fadd_rn(__fmul_rn(v0r[k], w0), __fmul_rn(v3r[k], w3)), ws);
            im = __fdiv_rn(__fadd_rn(__fmul_rn(v0i[k], w0), __fmul_rn(v3i[k], w3)), ws);
        }
        outr[k] = re;
        outi[k] = im;
    }
}

__device__ __forceinline__ void collapse_one(float a0r, float a0i, float a3r, float a3i, uint8_t g0, uint8_t g3,
                                             float w0in, float w3in, float& re, float& im) {
    const float w0 = g0 ? 0.0f : w0in;
    const float w3 = g3 ? 0.0f : w3in;
    const float ws = __fadd_rn(w0, w3);
    re = 0.0f;
    im = 0.0f;
    if (ws > 0.0f) {
        re = __fdiv_rn(__fadd_rn(__fmul_rn(a0r, w0), __fmul_rn(a3r, w3)), ws);
        im = __fdiv_rn(__fadd_rn(__fmul_rn(a0i, w0), __fmul_rn(a3i, w3)), ws);
    }
}

// The same collapse on four consecutive samples per thread with 16-byte loads and stores (all
// float arrays 16-byte and both flag arrays 4-byte aligned; n4 = n / 4 groups, the tail of
// n % 4 samples by the first threads). Its grid fills half of each SM, so that kernels of the
// main stream (rotation, statistics, histogram) run beside it.
__global__ void __launch_bounds__(kThreads) k_collapse4(const float4* __restrict__ v0r, const float4* __restrict__ v0i,
                                                       const float4* __restrict__ v3r, const float4* __restrict__ v3i,
                                                       const uchar4* __restrict__ f0, const uchar4* __restrict__ f3,
                                                       const float4* __restrict__ w0in, const float4* __restrict__ w3in,
                                                       float4* __restrict__ outr, float4* __restrict__ outi,
                                                       long long n) {
    const long long n4 = n >> 2;
    for (long long k = blockIdx.x * (long long)kThreads + threadIdx.x; k < n4;
         k += (long long)gridDim.x * kThreads) {
        const float4 a0r = v0r[k], a0i = v0i[k], a3r = v3r[k], a3i = v3i[k], b0 = w0in[k], b3 = w3in[k];
        const uchar4 g0 = f0[k], g3 = f3[k];
        float4 re, im;
        collapse_one(a0r.x, a0i.x, a3r.x, a3i.x, g0.x, g3.x, b0.x, b3.x, re.x, im.x);
        collapse_one(a0r.y, a0i.y, a3r.y, a3i.y, g0.y, g3.y, b0.y, b3.y, re.y, im.y);
        collapse_one(a0r.z, a0i.z, a3r.z, a3i.z, g0.z, g3.z, b0.z, b3.z, re.z, im.z);
        collapse_one(a0r.w, a0i.w, a3r.w, a3i.w, g0.w, g3.w, b0.w, b3.w, re.w, im.w);
        outr[k] = re;
        outi[k] = im;
    }
    const long long t = blockIdx.x * (long long)kThreads + threadIdx.x;
    const long long k = (n4 << 2) + t;
    if (t < (n & 3)) {
        const float* s0r = reinterpret_cast<const float*>(v0r);
        const float* s0i = reinterpret_cast<const float*>(v0i);
        const float* s3r = reinterpret_cast<const float*>(v3r);
        const float* s3i = reinterpret_cast<const float*>(v3i);
        const uint8_t* h0 = reinterpret_cast<const uint8_t*>(f0);
        const uint8_t* h3 = reinterpret_cast<const uint8_t*>(f3);
        const float* c0 = reinterpret_cast<const float*>(w0in);
        const float* c3 = reinterpret_cast<const float*>(w3in);
        float re, im;
        collapse_one(s0r[k], s0i[k], s3r[k], s3i[k], h0[k], h3[k], c0[k], c3[k], re, im);
        reinterpret_cast<float*>(outr)[k] = re;
        reinterpret_cast<float*>(outi)[k] = im;
    }
}

// Optional float Bin [N_s][3] of the reference layout: bin[k] = float(s[chan] * q[row]).
__global__ void __launch_bounds__(kThreads) k_expand_bin(const double* __restrict__ q, const double* __restrict__ s,
                                                        long long R, long long C, float* __restrict__ bin) {
    const long long n = R * C;
    for (long long k = blockIdx.x * (long long)kThreads + threadIdx.x; k < n;
         k += (long long)gridDim.x * kThreads) {
        const long long row = k % R, c = k / R;
        const double sc = s[c];
        for (int a = 0; a < 3; ++a) bin[k * 3 + a] = (float)(sc * q[row * 3 + a]);
    }
}

// Archive path: min/max of the third Bin coordinate (FIPkernels.cu:327-334).
__global__ void __launch_bounds__(kThreads) k_bin_r3(const float* __restrict__ bin, long long n,
                                                    double* __restrict__ partial) {
    __shared__ double sm[2 * kThreads];
    double lo = 1e300, hi = -1e300;
    for (long long k = blockIdx.x * (long long)kThreads + threadIdx.x; k < n;
         k += (long long)gridDim.x * kThreads) {
        const double r3 = bin[k * 3 + 2];
        lo = fmin(lo, r3);
        hi = fmax(hi, r3);
    }
    sm[threadIdx.x] = lo;
    sm[kThreads + threadIdx.x] = hi;
    __syncthreads();
    for (int stride = kThreads / 2; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride) {
            sm[threadIdx.x] = fmin(sm[threadIdx.x], sm[threadIdx.x + stride]);
            sm[kThreads + threadIdx.x] = fmax(sm[kThreads + threadIdx.x], sm[kThreads + threadIdx.x + stride]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[blockIdx.x * 2 + 0] = sm[0];
        partial[blockIdx.x * 2 + 1] = sm[kThreads];
    }
}

__global__ void k_vin_from_float(const float* __restrict__ v32, double* __restrict__ v64) {
    if (threadIdx.x < 9) v64[threadIdx.x] = (double)v32[threadIdx.x];
}

// max |t3| and the valid-pixel count over the N x N rotated-frame pixels
// (SVDIntegratedImager.cu:1029-1077), FP64, pixel offsets from the integer image centre.
// max |t3| and the valid-pixel count over the image. t3 = -v33 + sgn(v33) sqrt(ra) is monotone in
// the radicand ra (FP64 square root and subtraction of a constant preserve order), so the largest
// |t3| sits at the smallest or the largest valid radicand: the pixel loop keeps only those two and
// the final reduction takes the square roots (the same values the per-pixel form would produce).
// Rows are spread over blocks and columns over threads (no 64-bit division per pixel).
__global__ void __launch_bounds__(kThreads) k_t3_stats(const double* __restrict__ vin, long long N, double cell,
                                                      double* __restrict__ partial) {
    __shared__ double sm[3 * kThreads];
    const double v13 = vin[2], v23 = vin[5];
    const long long half = N / 2;
    double lo = 2.0, hi = -1.0, cnt = 0.0;  // radicands lie in [0, 1]
    for (long long y = blockIdx.x; y < N; y += gridDim.x) {
        const double t1 = cell * (double)(y - half) + v13;
        const double r1 = 1.0 - t1 * t1;
        for (long long x = threadIdx.x; x < N; x += kThreads) {
            const double t2 = cell * (double)(x - half) + v23;
            const double ra = r1 - t2 * t2;
            if (ra >= 0.0) {
                lo = fmin(lo, ra);
                hi = fmax(hi, ra);
                cnt += 1.0;
            }
        }
    }
    sm[threadIdx.x] = lo;
    sm[kThreads + threadIdx.x] = hi;
    sm[2 * kThreads + threadIdx.x] = cnt;
    __syncthreads();
    for (int stride = kThreads / 2; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride) {
            sm[threadIdx.x] = fmin(sm[threadIdx.x], sm[threadIdx.x + stride]);
            sm[kThreads + threadIdx.x] = fmax(sm[kThreads + threadIdx.x], sm[kThreads + threadIdx.x + stride]);
            sm[2 * kThreads + threadIdx.x] += sm[2 * kThreads + threadIdx.x + stride];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[blockIdx.x * 3 + 0] = sm[0];
        partial[blockIdx.x * 3 + 1] = sm[kThreads];
        partial[blockIdx.x * 3 + 2] = sm[2 * kThreads];
    }
}

__global__ void __launch_bounds__(kThreads) k_t3_final(const double* __restrict__ partial, int nblocks,
                                                      const double* __restrict__ vin, double* __restrict__ stats) {
    __shared__ double sm[3 * kThreads];
    double lo = 2.0, hi = -1.0, cnt = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += kThreads) {
        lo = fmin(lo, partial[b * 3 + 0]);
        hi = fmax(hi, partial[b * 3 + 1]);
        cnt += partial[b * 3 + 2];
    }
    sm[threadIdx.x] = lo;
    sm[kThreads + threadIdx.x] = hi;
    sm[2 * kThreads + threadIdx.x] = cnt;
    __syncthreads();
    for (int stride = kThreads / 2; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride) {
            sm[threadIdx.x] = fmin(sm[threadIdx.x], sm[threadIdx.x + stride]);
            sm[kThreads + threadIdx.x] = fmax(sm[kThreads + threadIdx.x], sm[kThreads + threadIdx.x + stride]);
            sm[2 * kThreads + threadIdx.x] += sm[2 * kThreads + threadIdx.x + stride];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double v33 = vin[8], sg = v33 >= 0.0 ? 1.0 : -1.0;
        double mx = 0.0;
        if (sm[2 * kThreads] > 0.0)
            mx = fmax(fabs(-v33 + sg * sqrt(sm[0])), fabs(-v33 + sg * sqrt(sm[kThreads])));
        stats[ST_MAX_T3] = mx;
        stats[ST_VALID_PIX] = sm[2 * kThreads];
    }
}

// Sampled truncation error of exp(i a s) ~ J0 + 2 sum_{1<=n<K} i^n J_n(a) T_n(s) for all K at
// once: err[K-1] = max over a = amax*i/(na-1), s = -1 + 2j/(ns-1). One block per a. FP64. The
// errors are non-negative, so their bit patterns order like unsigned integers (atomicMax).
// Same quantity as cheb_bucket_error_kernel (SVDIntegratedImager.cu:1112-1202) and
// host_chebyshev_error_sample_range (archive/FIPkernels.cu:287-318).
constexpr int kErrMaxK = 32;
__global__ void __launch_bounds__(kThreads) k_cheb_errors(double amax, int na, int ns, int kmax,
                                                         unsigned long long* __restrict__ err) {
    __shared__ double jv[kErrMaxK];
    __shared__ double red[kErrMaxK][kThreads / 32];
    const int ia = blockIdx.x;
    const double a = (na == 1) ? amax : amax * (double)ia / (double)(na - 1);
    if (threadIdx.x == 0) bessel_jn(a, kmax - 1, jv);
    __syncthreads();
    double local[kErrMaxK];
    for (int n = 0; n < kErrMaxK; ++n) local[n] = 0.0;
    for (int is = threadIdx.x; is < ns; is += kThreads) {
        const double s = -1.0 + 2.0 * (double)is / (double)(ns - 1);
        double sn, cs;
        sincos(a * s, &sn, &cs);
        double ar = 0.0, ai = 0.0, tm2 = 1.0, tm1 = s;
#pragma unroll
        for (int n = 0; n < kErrMaxK; ++n) {
            if (n >= kmax) break;
            double tn = (n == 0) ? 1.0 : (n == 1 ? s : 2.0 * s * tm1 - tm2);
            if (n >= 2) {
                tm2 = tm1;
                tm1 = tn;
            }
            if (n == 0) {
                ar += jv[0] * tn;
            } else {
                const double amp = 2.0 * jv[n] * tn;
                switch (n & 3) {
                    case 0: ar += amp; break;
                    case 1: ai += amp; break;
                    case 2: ar -= amp; break;
                    default: ai -= amp; break;
                }
            }
            local[n] = fmax(local[n], hypot(cs - ar, sn - ai));
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int n = 0; n < kErrMaxK; ++n) {
        double v = local[n];
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) red[n][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < kmax) {
        double v = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) v = fmax(v, red[threadIdx.x][w]);
        atomicMax(&err[threadIdx.x], (unsigned long long)__double_as_longlong(v));
    }
}

int grid_for(long long n, int cap) {
    long long b = (n + kThreads - 1) / kThreads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (int)b;
}

}  // namespace

int launch_preprocess(const float* d_uvw, const float* d_freq, long long R, long long C,
                      float array_center_x, double* d_partial, int partial_cap, double* d_vin64,
                      float* d_vin32, double* d_q, double* d_s, double* d_stats, cudaStream_t st) {
    const int nb = grid_for(R, partial_cap);
    k_row_moments<<<nb, kThreads, 0, st>>>(d_uvw, R, d_partial);
    SVDI_LAUNCHED();
    k_basis<<<1, kThreads, 0, st>>>(d_partial, nb, d_freq, C, R, array_center_x, d_vin64, d_vin32, d_s, d_stats);
    SVDI_LAUNCHED();
    k_project_rows<<<nb, kThreads, 0, st>>>(d_uvw, R, d_vin64, d_stats, d_q, d_partial);
    SVDI_LAUNCHED();
    k_minmax_final<<<1, kThreads, 0, st>>>(d_partial, nb, d_stats);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

int launch_collapse(const float* v0r, const float* v0i, const float* v3r, const float* v3i,
                    const uint8_t* f0, const uint8_t* f3, const float* w0, const float* w3,
                    float* outr, float* outi, long long n, cudaStream_t st) {
    auto al = [](const void* p, uintptr_t a) { return ((uintptr_t)p & (a - 1)) == 0; };
    if (al(v0r, 16) && al(v0i, 16) && al(v3r, 16) && al(v3i, 16) && al(w0, 16) && al(w3, 16) && al(outr, 16) &&
        al(outi, 16) && al(f0, 4) && al(f3, 4)) {
        const int sms = current_sm_count();
        long long b = ((n >> 2) + kThreads - 1) / kThreads;
        if (b > (long long)sms * 4) b = (long long)sms * 4;   // 4 of the 8 resident 256-thread blocks per SM
        if (b < 1) b = 1;
        k_collapse4<<<(int)b, kThreads, 0, st>>>(
            reinterpret_cast<const float4*>(v0r), reinterpret_cast<const float4*>(v0i),
            reinterpret_cast<const float4*>(v3r), reinterpret_cast<const float4*>(v3i),
            reinterpret_cast<const uchar4*>(f0), reinterpret_cast<const uchar4*>(f3),
            reinterpret_cast<const float4*>(w0), reinterpret_cast<const float4*>(w3),
            reinterpret_cast<float4*>(outr), reinterpret_cast<float4*>(outi), n);
    } else {
        k_collapse<<<grid_for(n, 16 * current_sm_count()), kThreads, 0, st>>>(v0r, v0i, v3r, v3i, f0, f3, w0, w3, outr, outi, n);
    }
    SVDI_LAUNCHED();
    return SVDI_OK;
}

int launch_expand_bin(const double* d_q, const double* d_s, long long R, long long C, float* d_bin,
                      cudaStream_t st) {
    k_expand_bin<<<grid_for(R * C, 16 * current_sm_count()), kThreads, 0, st>>>(d_q, d_s, R, C, d_bin);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

int launch_bin_stats(const float* d_bin, long long n, double* d_partial, int partial_cap,
                     double* d_stats, cudaStream_t st) {
    const int nb = grid_for(n, partial_cap);
    k_bin_r3<<<nb, kThreads, 0, st>>>(d_bin, n, d_partial);
    SVDI_LAUNCHED();
    k_minmax_final<<<1, kThreads, 0, st>>>(d_partial, nb, d_stats);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

int launch_vin_from_float(const float* d_vin32, double* d_vin64, cudaStream_t st) {
    k_vin_from_float<<<1, 32, 0, st>>>(d_vin32, d_vin64);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

int launch_t3_stats(const double* d_vin64, long long N, double cell, double* d_partial,
                    int partial_cap, double* d_stats, cudaStream_t st) {
    const int nb = (int)std::max<long long>(1, std::min<long long>(N, partial_cap));  // one row per block and step
    k_t3_stats<<<nb, kThreads, 0, st>>>(d_vin64, N, cell, d_partial);
    SVDI_LAUNCHED();
    k_t3_final<<<1, kThreads, 0, st>>>(d_partial, nb, d_vin64, d_stats);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

__global__ void k_plan(const double* __restrict__ stats, const double* __restrict__ vin, int archive,
                       int nslab, int K, DevPlan* __restrict__ plan) {
    if (threadIdx.x != 0) return;
    slab_params_for(archive != 0, nslab, K, stats[ST_R3_MIN], stats[ST_R3_MAX], plan->sp);
    plan->inv_det = (float)(1.0 / basis_det(vin));  // inf or NaN for a degenerate basis, which the host rejects
}

int launch_plan(const double* d_stats, const double* d_vin64, bool archive, int nslab, int K,
                DevPlan* d_plan, cudaStream_t st) {
    k_plan<<<1, 32, 0, st>>>(d_stats, d_vin64, archive ? 1 : 0, nslab, K, d_plan);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

int launch_cheb_errors(double amax, int na, int ns, int kmax, unsigned long long* d_err,
                       cudaStream_t st) {
    if (kmax > kErrMaxK || kmax < 1 || na < 1 || ns < 2) {
        set_error("cheb_errors: unsupported sampling");
        return SVDI_ERR_UNSUPPORTED;
    }
    SVDI_CUDA(cudaMemsetAsync(d_err, 0, sizeof(unsigned long long) * kmax, st));
    k_cheb_errors<<<na, kThreads, 0, st>>>(amax, na, ns, kmax, d_err);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

}  // namespace svdi
