// Tile-local FP32 ES gridder (plain CUDA-core form).
//
// Replaces fused_gridding (SVDIntegratedImager.cu:1218-1293) / gridding (archive/FIPkernels.cu:
// 383-452), which issue 64 * K * 2 float atomics per sample to global memory. Samples arrive
// binned by tile (binning.cu); a persistent CTA walks equal-size chunks of the binned record array,
// accumulates each tile's (T+W)^2 footprint region in shared memory, and flushes the touched
// bounding box to the moment planes with 8-byte vector reductions (red.global.add.v2.f32) --
// one per cell, instead of one per sample-cell.
//
// Inner loop: one warp per sample. Lanes 0..W-1 evaluate the W x-weights and lanes W..2W-1 the
// W y-weights from a piecewise polynomial of the ES kernel (degree kPolyDeg in the fractional
// grid position, FP32 Horner); lane (a, b) then owns footprint cells (a + p * 32/W, b), whose
// shared-memory addresses are bank-conflict free because the row stride is == W (mod 32).
#include "svdi_internal.cuh"

#include <cmath>
#include <vector>

namespace svdi {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ void red_add_v2(float2* addr, float a, float b) {
    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(addr), "f"(a), "f"(b) : "memory");
}

template <int W, int T, int KC>
struct TileCfg {
    static constexpr int R = T + W;       // region side (footprint origins in [0, T))
    static constexpr int RS = R;          // row stride; R == W (mod 32) for T in {32, 64}
    static constexpr int PLANE = R * RS;  // floats per re or im plane
    static constexpr size_t SMEM = (size_t)KC * 2 * PLANE * sizeof(float);
    static_assert((RS % 32) == (W % 32), "row stride must be == W (mod 32)");
};

template <int W, int T, int KC>
__global__ void __launch_bounds__(kThreads) k_grid_fp32(
    const SampleRec* __restrict__ rec, const float* __restrict__ rec_s,
    const unsigned int* __restrict__ offsets, int key_lo, int key_hi, int slab_lo, GridGeom g,
    SlabParams sp, EsPoly poly, float2* __restrict__ planes, int term0, unsigned int chunk) {
    using C = TileCfg<W, T, KC>;
    extern __shared__ float tile[];  // [KC][2][R][RS]
    __shared__ int bbox[4];          // row min, row max, col min, col max
    __shared__ int seg_key;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int HW = W / 2;
    constexpr int RPP = 32 / W;                // footprint rows per pass
    constexpr int PASSES = (W + RPP - 1) / RPP;
    const int la = lane / W, lb = lane % W;
    const bool lane_cell = lane < RPP * W;

    // this lane's polynomial piece (lanes 0..2W-1)
    float coef[kPolyDeg + 1];
    {
        const int piece = lane % W;
#pragma unroll
        for (int d = 0; d <= kPolyDeg; ++d) coef[d] = poly.c[piece][d];
    }
    const float edge_w = poly.edge;

    for (int i = threadIdx.x; i < KC * 2 * C::PLANE; i += kThreads) tile[i] = 0.0f;
    if (threadIdx.x == 0) {
        bbox[0] = C::R; bbox[1] = -1; bbox[2] = C::R; bbox[3] = -1;
    }
    __syncthreads();

    const unsigned int rec_lo = offsets[key_lo], rec_hi = offsets[key_hi];
    const unsigned int n_chunks = (rec_hi - rec_lo + chunk - 1) / chunk;
    const long long GG = g.G * g.G;
    const int tiles2 = g.ntile * g.ntile;

    for (unsigned int ch = blockIdx.x; ch < n_chunks; ch += gridDim.x) {
        const unsigned int c_beg = rec_lo + ch * chunk;
        const unsigned int c_end = min(rec_hi, c_beg + chunk);
        if (threadIdx.x == 0) {  // last key in [key_lo, key_hi) with offsets[key] <= c_beg
            int lo = key_lo, hi = key_hi;  // offsets[key_hi] = rec_hi > c_beg
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (offsets[mid] <= c_beg) lo = mid; else hi = mid;
            }
            seg_key = lo;
        }
        __syncthreads();
        int key = seg_key;
        while (key < key_hi && offsets[key] < c_end) {
            const unsigned int s_beg = max(c_beg, offsets[key]);
            const unsigned int s_end = min(c_end, offsets[key + 1]);
            if (s_beg < s_end) {
                const int slab = key / tiles2;
                const int t1 = (key / g.ntile) % g.ntile, t2 = key % g.ntile;
                int rmin = C::R, rmax = -1, cmin = C::R, cmax = -1;
                for (unsigned int b0 = s_beg + warp * 32; b0 < s_end; b0 += kWarps * 32) {
                    const unsigned int my = b0 + lane;
                    SampleRec r = {0, 0, 0.0f, 0.0f};
                    float sv = 0.0f;
                    if (my < s_end) {
                        r = rec[my];
                        if (rec_s) sv = rec_s[my];
                    }
                    const int nb = min(32u, s_end - b0);
                    for (int j = 0; j < nb; ++j) {
                        const int xq = __shfl_sync(0xffffffffu, r.xq, j);
                        const int yq = __shfl_sync(0xffffffffu, r.yq, j);
                        const float vre = __shfl_sync(0xffffffffu, r.vre, j);
                        const float vim = __shfl_sync(0xffffffffu, r.vim, j);
                        const int cx = xq >> 24, cy = yq >> 24;
                        const int fxq = xq & 0xFFFFFF, fyq = yq & 0xFFFFFF;
                        // weight of this lane's piece
                        const float f = (float)(lane < W ? fxq : fyq) * (1.0f / 16777216.0f);
                        const float u = fmaf(2.0f, f, -1.0f);
                        float w = coef[kPolyDeg];
#pragma unroll
                        for (int d = kPolyDeg - 1; d >= 0; --d) w = fmaf(w, u, coef[d]);
                        const float wy = __shfl_sync(0xffffffffu, w, W + lb);
                        float tv[KC];
                        if (KC == 1 && term0 == 0) {
                            tv[0] = 1.0f;
                        } else {
                            const float s = __shfl_sync(0xffffffffu, sv, j);
                            float tm2 = 1.0f, tm1 = s;
                            for (int t = 0; t < term0 + KC; ++t) {
                                float tn = t == 0 ? 1.0f : (t == 1 ? s : 2.0f * s * tm1 - tm2);
                                if (t >= 2) { tm2 = tm1; tm1 = tn; }
                                if (t >= term0) tv[t - term0] = tn;
                            }
                        }
                        const int r0 = cx - (HW - 1), c0 = cy - (HW - 1);
#pragma unroll
                        for (int p = 0; p < PASSES; ++p) {
                            const int i = la + p * RPP;
                            const float wx = __shfl_sync(0xffffffffu, w, (i < W ? i : 0));
                            const int rr = r0 + i, cc = c0 + lb;
                            if (lane_cell && i < W && rr >= 0 && cc >= 0) {
                                const float kv = wx * wy;
                                const float ar = kv * vre, ai = kv * vim;
#pragma unroll
                                for (int t = 0; t < KC; ++t) {
                                    float* pl = tile + (size_t)t * 2 * C::PLANE + rr * C::RS + cc;
                                    atomicAdd(pl, ar * tv[t]);
                                    atomicAdd(pl + C::PLANE, ai * tv[t]);
                                }
                            }
                        }
                        // frac == 0: the footprint has W+1 cells; the extra one sits at offset -W/2
                        // and carries psi(-1) = exp(-beta).
                        if ((fxq == 0) | (fyq == 0)) {
                            const float wxe = __shfl_sync(0xffffffffu, w, lane < W ? lane : 0);
                            float wy_l = __shfl_sync(0xffffffffu, w, W + (lane < W ? lane : 0));
                            for (int e = 0; e < 3; ++e) {
                                int rr, cc;
                                float kv;
                                bool act;
                                if (e == 0) {        // extra row x normal columns
                                    act = (fxq == 0) && lane < W;
                                    rr = cx - HW; cc = c0 + lane; kv = edge_w * wy_l;
                                } else if (e == 1) { // normal rows x extra column
                                    act = (fyq == 0) && lane < W;
                                    rr = r0 + lane; cc = cy - HW; kv = wxe * edge_w;
                                } else {             // corner
                                    act = (fxq == 0) && (fyq == 0) && lane == 0;
                                    rr = cx - HW; cc = cy - HW; kv = edge_w * edge_w;
                                }
                                if (act && rr >= 0 && cc >= 0) {
                                    const float ar = kv * vre, ai = kv * vim;
                                    for (int t = 0; t < KC; ++t) {
                                        float* pl = tile + (size_t)t * 2 * C::PLANE + rr * C::RS + cc;
                                        atomicAdd(pl, ar * tv[t]);
                                        atomicAdd(pl + C::PLANE, ai * tv[t]);
                                    }
                                }
                            }
                        }
                        // bounding box of touched cells
                        const int rlo = max(0, fxq ? r0 : r0 - 1), rhi = cx + HW;
                        const int clo = max(0, fyq ? c0 : c0 - 1), chi = cy + HW;
                        rmin = min(rmin, rlo); rmax = max(rmax, rhi);
                        cmin = min(cmin, clo); cmax = max(cmax, chi);
                    }
                }
                if (lane == 0 && rmax >= 0) {
                    atomicMin(&bbox[0], rmin); atomicMax(&bbox[1], rmax);
                    atomicMin(&bbox[2], cmin); atomicMax(&bbox[3], cmax);
                }
                __syncthreads();
                // flush the bounding box: checkerboard sign, clip to the grid, zero behind
                const int br0 = bbox[0], br1 = min(bbox[1], C::R - 1);
                const int bc0 = bbox[2], bc1 = min(bbox[3], C::R - 1);
                if (br1 >= br0 && bc1 >= bc0) {
                    const int bw = bc1 - bc0 + 1;
                    const int ncell = (br1 - br0 + 1) * bw;
                    const long long o1 = g.gmin + (long long)t1 * T;
                    const long long o2 = g.gmin + (long long)t2 * T;
                    for (int cidx = threadIdx.x; cidx < ncell; cidx += kThreads) {
                        const int rr = br0 + cidx / bw, cc = bc0 + cidx % bw;
                        const long long g1 = o1 + rr, g2 = o2 + cc;
                        const bool on_grid = g1 <= g.gmax && g2 <= g.gmax;
                        const float sgn = ((g1 + g2) & 1) ? -1.0f : 1.0f;
                        const long long cell = (g1 - g.gmin) * g.G + (g2 - g.gmin);
#pragma unroll
                        for (int t = 0; t < KC; ++t) {
                            float* pl = tile + (size_t)t * 2 * C::PLANE + rr * C::RS + cc;
                            const float re = pl[0], im = pl[C::PLANE];
                            if (on_grid && (re != 0.0f || im != 0.0f)) {
                                const long long plane = (long long)(slab - slab_lo) * sp.K + term0 + t;
                                red_add_v2(planes + plane * GG + cell, sgn * re, sgn * im);
                            }
                            pl[0] = 0.0f;
                            pl[C::PLANE] = 0.0f;
                        }
                    }
                }
                __syncthreads();
                if (threadIdx.x == 0) {
                    bbox[0] = C::R; bbox[1] = -1; bbox[2] = C::R; bbox[3] = -1;
                }
                __syncthreads();
            }
            ++key;
        }
    }
}

template <int W, int T, int KC>
int launch_variant(const SampleRec* d_rec, const float* d_rec_s, const unsigned int* d_offsets,
                   int key_lo, int key_hi, int slab_lo, const GridGeom& g, const SlabParams& sp,
                   const EsPoly& poly, float2* d_planes, int term0, unsigned int chunk, int sm_count,
                   cudaStream_t st) {
    using C = TileCfg<W, T, KC>;
    auto kern = k_grid_fp32<W, T, KC>;
    static bool configured = false;  // per instantiation
    if (!configured) {
        SVDI_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
        configured = true;
    }
    int per_sm = 0;
    SVDI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, C::SMEM));
    if (per_sm < 1) per_sm = 1;
    kern<<<sm_count * per_sm, kThreads, C::SMEM, st>>>(d_rec, d_rec_s, d_offsets, key_lo, key_hi, slab_lo,
                                                        g, sp, poly, d_planes, term0, chunk);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

template <int W>
int launch_w(const SampleRec* d_rec, const float* d_rec_s, const unsigned int* d_offsets, int key_lo,
             int key_hi, int slab_lo, const GridGeom& g, const SlabParams& sp, const EsPoly& poly,
             float2* d_planes, int sm_count, cudaStream_t st) {
    const unsigned int chunk = 4096;
    if (g.T == 64) {
        for (int t0 = 0; t0 < sp.K; ++t0)
            SVDI_TRY((launch_variant<W, 64, 1>(d_rec, d_rec_s, d_offsets, key_lo, key_hi, slab_lo, g, sp,
                                               poly, d_planes, t0, chunk, sm_count, st)));
        return SVDI_OK;
    }
    if (g.T == 32) {
        int t0 = 0;
        for (; t0 + 8 <= sp.K; t0 += 8)
            SVDI_TRY((launch_variant<W, 32, 8>(d_rec, d_rec_s, d_offsets, key_lo, key_hi, slab_lo, g, sp,
                                               poly, d_planes, t0, chunk, sm_count, st)));
        for (; t0 + 4 <= sp.K; t0 += 4)
            SVDI_TRY((launch_variant<W, 32, 4>(d_rec, d_rec_s, d_offsets, key_lo, key_hi, slab_lo, g, sp,
                                               poly, d_planes, t0, chunk, sm_count, st)));
        for (; t0 < sp.K; ++t0)
            SVDI_TRY((launch_variant<W, 32, 1>(d_rec, d_rec_s, d_offsets, key_lo, key_hi, slab_lo, g, sp,
                                               poly, d_planes, t0, chunk, sm_count, st)));
        return SVDI_OK;
    }
    set_error("gridder: tile size must be 32 or 64");
    return SVDI_ERR_UNSUPPORTED;
}

}  // namespace

int launch_grid_fp32(const SampleRec* d_rec, const float* d_rec_s, const unsigned int* d_offsets,
                     int n_keys, int key_lo, int key_hi, int slab_lo, const GridGeom& g,
                     const SlabParams& sp, const EsPoly& poly, float2* d_planes, int sm_count,
                     cudaStream_t st) {
    if (key_lo < 0 || key_hi > n_keys || key_lo >= key_hi) {
        set_error("gridder: bad key range");
        return SVDI_ERR_INTERNAL;
    }
    switch (g.W) {
        case 6: return launch_w<6>(d_rec, d_rec_s, d_offsets, key_lo, key_hi, slab_lo, g, sp, poly, d_planes, sm_count, st);
        case 8: return launch_w<8>(d_rec, d_rec_s, d_offsets, key_lo, key_hi, slab_lo, g, sp, poly, d_planes, sm_count, st);
        case 10: return launch_w<10>(d_rec, d_rec_s, d_offsets, key_lo, key_hi, slab_lo, g, sp, poly, d_planes, sm_count, st);
        case 12: return launch_w<12>(d_rec, d_rec_s, d_offsets, key_lo, key_hi, slab_lo, g, sp, poly, d_planes, sm_count, st);
        default:
            set_error("gridder: ES support must be one of 6, 8, 10, 12");
            return SVDI_ERR_UNSUPPORTED;
    }
}

// Piecewise polynomial of the ES kernel: piece i (0 <= i < W) interpolates
// psi((i - (W/2 - 1) - f) / (W/2)), f in [0, 1], at kPolyDeg + 1 Chebyshev nodes in u = 2f - 1
// (FP64), converted to monomial coefficients in u for Horner evaluation.
// psi(x) = exp(beta (sqrt(1 - x^2) - 1)) = exp(-beta x^2 / (1 + sqrt((1 - x)(1 + x)))).
void build_es_poly(int W, double beta, EsPoly* out) {
    const int D = kPolyDeg, n = D + 1;
    const int hw = W / 2;
    auto psi = [&](double x) {
        if (fabs(x) > 1.0) return 0.0;
        return exp(-beta * x * x / (1.0 + sqrt((1.0 - x) * (1.0 + x))));
    };
    std::vector<double> nodes(n), vals(n), cheb(n), mono(n), tkm2(n), tkm1(n), tk(n);
    for (int k = 0; k < n; ++k) nodes[k] = cos(kPi * (k + 0.5) / n);
    out->W = W;
    out->edge = (float)exp(-beta);
    for (int i = 0; i < kMaxSupport; ++i)
        for (int d = 0; d <= D; ++d) out->c[i][d] = 0.0f;
    for (int i = 0; i < W; ++i) {
        for (int k = 0; k < n; ++k) {
            const double f = 0.5 * (nodes[k] + 1.0);
            vals[k] = psi((i - (hw - 1) - f) / hw);
        }
        for (int j = 0; j < n; ++j) {  // Chebyshev coefficients of the interpolant
            double s = 0.0;
            for (int k = 0; k < n; ++k) s += vals[k] * cos(kPi * j * (k + 0.5) / n);
            cheb[j] = (j == 0 ? 1.0 : 2.0) * s / n;
        }
        for (int d = 0; d < n; ++d) mono[d] = 0.0;
        // accumulate cheb[j] * T_j(u) in the monomial basis
        for (int d = 0; d < n; ++d) { tkm2[d] = 0.0; tkm1[d] = 0.0; }
        tkm2[0] = 1.0;          // T0
        if (n > 1) tkm1[1] = 1.0;  // T1
        for (int d = 0; d < n; ++d) mono[d] += cheb[0] * tkm2[d];
        if (n > 1)
            for (int d = 0; d < n; ++d) mono[d] += cheb[1] * tkm1[d];
        for (int j = 2; j < n; ++j) {
            for (int d = 0; d < n; ++d) tk[d] = -tkm2[d] + (d > 0 ? 2.0 * tkm1[d - 1] : 0.0);
            for (int d = 0; d < n; ++d) mono[d] += cheb[j] * tk[d];
            tkm2 = tkm1;
            tkm1 = tk;
        }
        for (int d = 0; d <= D; ++d) out->c[i][d] = (float)mono[d];
    }
}

}  // namespace svdi
