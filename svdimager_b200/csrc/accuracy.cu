// FP64 direct-DFT accuracy probe: the rotated-frame image value at chosen pixels computed straight
// from the samples, for the autotuner's accuracy check and for users who want an error estimate
// of an image without a CPU oracle.
//
// R(x, y) = | sum_k [vr_k cos(2 pi r_k . t) - vi_k sin(2 pi r_k . t)] | / |det V| / N_s
// over the samples that the gridder keeps (the binning rules of binning_rules.cuh, so edge
// clipping and strict inclusion match the image bit for bit), with the pixel direction
// t = (t1, t2, t3) of the imaging kernels (t3 from SVDIntegratedImager.cu:1029-1077) and the
// 1 / N_s normalisation of SVDIntegratedImager.cu:1445.
#include "binning_rules.cuh"
#include "svdi_internal.cuh"

namespace svdi {

namespace {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_dft_probe(SampleSource src, GridGeom g, SlabParams sp,
                                                        const double* __restrict__ vin, long long N, double cell,
                                                        const long long* __restrict__ px,
                                                        const long long* __restrict__ py, double* __restrict__ acc) {
    __shared__ double part[kThreads / 32];
    const int p = blockIdx.x;
    const long long half = N / 2;
    const double t1 = cell * (double)(py[p] - half), t2 = cell * (double)(px[p] - half);
    const double v13 = vin[2], v23 = vin[5], v33 = vin[8];
    const double ra = 1.0 - (t1 + v13) * (t1 + v13) - (t2 + v23) * (t2 + v23);
    if (ra < 0.0) return;  // outside the projection: the host reports NaN
    const double t3 = -v33 + (v33 >= 0.0 ? 1.0 : -1.0) * sqrt(ra);
    double sum = 0.0;
    for (long long idx = (long long)blockIdx.y * kThreads + threadIdx.x; idx < src.n;
         idx += (long long)gridDim.y * kThreads) {
        if (binrules::sample_key(src, idx, g, sp).key < 0) continue;
        double r1, r2, r3;
        binrules::sample_coords(src, idx, r1, r2, r3);
        double sn, cs;
        sincospi(2.0 * (r1 * t1 + r2 * t2 + r3 * t3), &sn, &cs);
        sum += (double)src.vr[idx] * cs - (double)src.vi[idx] * sn;
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) t += part[w];
        atomicAdd(&acc[p], t);
    }
}

}  // namespace

int launch_dft_probe(const SampleSource& src, const GridGeom& g, const SlabParams& sp, const double* d_vin,
                     long long N, double cell, const long long* d_px, const long long* d_py, int npix,
                     double* d_acc, int sm_count, cudaStream_t st) {
    if (npix <= 0) return SVDI_OK;
    const int split = std::max(1, (4 * sm_count + npix - 1) / npix);
    dim3 grid((unsigned)npix, (unsigned)std::min(split, 1024));
    k_dft_probe<<<grid, kThreads, 0, st>>>(src, g, sp, d_vin, N, cell, d_px, d_py, d_acc);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

}  // namespace svdi
