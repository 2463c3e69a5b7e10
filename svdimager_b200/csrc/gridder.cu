// Tile-local FP32 ES gridder (plain CUDA-core form).
//
// Replaces fused_gridding (SVDIntegratedImager.cu:1218-1293) / gridding (archive/FIPkernels.cu:
// 383-452), which issue 64 * K * 2 float atomics per sample to global memory. Samples arrive
// binned by tile (binning.cu); a persistent CTA walks equal-size chunks of the binned record array,
// accumulates each tile's (T+W)^2 footprint region in shared memory, and flushes the touched
// bounding box to the moment planes with 8-byte vector reductions (red.global.add.v2.f32) --
// one per cell, instead of one per sample-cell.
//
// Accumulation is 32-bit fixed point: on sm_100a a float atomicAdd to shared memory executes as a
// load + compare-and-swap loop (~3 clk per warp instruction, ~6 under inter-warp overlap, measured),
// whereas red.shared.add.u32 is native (~1 clk). A tile segment (the records of one key within one
// chunk of kGridChunk records) gets the scale 0.999 * 2^s with s = min(22 - e, 31 - e_sum) for
// max|v| < 2^e over the key and sum max(|v_re|, |v_im|) < 2^e_sum over the chunk: every contribution
// stays below 2^22 (one FMA against 1.5 * 2^23 rounds it to an integer exactly) and no cell sum can
// reach 2^31, since |psi psi| <= 1. On ordinary data the sum bound leaves s = 22 - e, a quantisation
// step of 2^-22 max|v|. Integer sums are order-independent, so a segment's contribution is
// deterministic.
//
// Inner loop: one warp per sample. Lanes 0..W-1 evaluate the W x-weights and lanes W..2W-1 the
// W y-weights from a piecewise polynomial of the ES kernel (degree kPolyDeg in the fractional
// grid position, FP32 Horner), two samples per polynomial pass when 2W <= 16; lane (a, b) then
// owns footprint cells (a + p * 32/W, b), whose shared-memory addresses are bank-conflict free
// because the row stride is == W (mod 32).
//
// W = 8 (the main form, any number of terms): the loop is bound by the MIO pipe (shared-memory reductions,
// loads and shuffles, about one warp instruction per SM clock), so each warp instruction serves
// the two samples of a polynomial pass: lanes 16h .. 16h + 15 grid sample j + h, lane (a, rho)
// the four cells (a, c0), (a, c1), (a + 4, c0), (a + 4, c1) with c1 = c0 ^ 4 and c0 the footprint
// column whose bank residue (mod 8) is rho for the first half-warp and rho + 4 for the second
// (the row stride is == 8 mod 32, so a row's eight cells cover the eight residues once). Every
// reduction instruction then puts one half-warp on residues 0-3 and the other on 4-7 of distinct
// rows: conflict-free whatever the two footprints' positions. Per sample: four reductions per
// term, two shuffles and one load (the one-sample form: three shuffles and one and a half loads).
#include "svdi_internal.cuh"

#include <cmath>
#include <vector>

namespace svdi {

namespace {


// Exact ES kernel psi(x) = exp(beta (sqrt(1 - x^2) - 1)) written without cancellation (rare path).
__device__ __forceinline__ float es_exact(float beta, float x) {
    if (fabsf(x) > 1.0f) return 0.0f;
    return expf(-beta * x * x / (1.0f + sqrtf((1.0f - x) * (1.0f + x))));
}

// Round-to-nearest integer of x for |x| < 2^22: fmaf(a, b, kMagic) rounds a*b + 1.5 2^23 once into
// [2^23, 2^24), whose ulp is 1, and the low mantissa bits are then the integer.
constexpr float kMagic = 12582912.0f;   // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;  // bit pattern of kMagic
__device__ __forceinline__ int fx_round(float x_plus_magic) {
    return __float_as_int(x_plus_magic) - kMagicBits;
}

// red.shared.add.u32 at shared-window address addr + OFF (OFF an immediate)
template <int OFF>
__device__ __forceinline__ void red_shared(unsigned int addr, int v) {
    asm volatile("red.shared.add.u32 [%0+%2], %1;" ::"r"(addr), "r"(v), "n"(OFF) : "memory");
}

__device__ __forceinline__ void red_add_v4(float2* addr, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

__device__ __forceinline__ void red_add_v2(float2* addr, float a, float b) {
    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(addr), "f"(a), "f"(b) : "memory");
}

// Passes P..PASSES-1 of one sample's footprint for this lane (one cell per pass): x-weight from the
// lane that evaluated it, then one fixed-point reduction per component at an immediate offset.
template <int P, int PASSES, int RPP, int RS, int PLANE, bool ALL>
__device__ __forceinline__ void grid_passes(unsigned int a, float w, float wy, float vr, float vi, int src0,
                                            const int* wx_src, const bool* pass_on) {
    if constexpr (P < PASSES) {
        const float wx = __shfl_sync(0xffffffffu, w, src0 + wx_src[P]);
        if (ALL || pass_on[P]) {
            const float kv = wx * wy;
            red_shared<4 * P * RPP * RS>(a, fx_round(fmaf(kv, vr, kMagic)));
            red_shared<4 * (P * RPP * RS + PLANE)>(a, fx_round(fmaf(kv, vi, kMagic)));
        }
        grid_passes<P + 1, PASSES, RPP, RS, PLANE, ALL>(a, w, wy, vr, vi, src0, wx_src, pass_on);
    }
}

// The KC terms of one cell at shared-window address addr + OFF: term t's real and imaginary planes
// lie 2 t PLANE and (2 t + 1) PLANE words further (t = T0 .. KC - 1).
template <int T0, int KC, int OFF, int PLANE>
__device__ __forceinline__ void red_terms(unsigned int addr, float ar, float ai, const float (&tv)[KC]) {
    if constexpr (T0 < KC) {
        red_shared<OFF + 8 * T0 * PLANE>(addr, fx_round(fmaf(ar, tv[T0], kMagic)));
        red_shared<OFF + 8 * T0 * PLANE + 4 * PLANE>(addr, fx_round(fmaf(ai, tv[T0], kMagic)));
        red_terms<T0 + 1, KC, OFF, PLANE>(addr, ar, ai, tv);
    }
}

template <int W, int T, int KC>
struct TileCfg {
    static constexpr int R = T + W;       // region side (footprint origins in [0, T))
    static constexpr int RS = R;          // row stride; R == W (mod 32) for T in {32, 64}
    static constexpr int PLANE = R * RS;  // floats per re or im plane
    static constexpr size_t SMEM = (size_t)KC * 2 * PLANE * sizeof(float);
    static constexpr int NT = 256;  // threads per CTA
    static constexpr int NW = NT / 32;
    static_assert((RS % 32) == (W % 32), "row stride must be == W (mod 32)");
};

// Reduces the integer region's bounding box, times inv_scale, into the moment plane of key `key`
// (checkerboard sign, clipped to the grid) and zeroes it behind. The region's accumulation must
// be complete (the caller synchronises the CTA before and after).
template <class C, int T, int KC>
__device__ __forceinline__ void flush_region(int* __restrict__ tile, const int* bbox, int key, int slab_lo,
                                             int term0, float inv_scale, const GridGeom& g, const SlabParams& sp,
                                             float2* __restrict__ planes, int warp, int lane) {
    constexpr int kWarps = C::NW;
    const long long GG = g.G * g.G;
    const int tiles2 = g.ntile * g.ntile2;
    const int slab = key / tiles2;
    const int t1 = (key / g.ntile2) % g.ntile, t2 = key % g.ntile2;
    // flush the bounding box: checkerboard sign, clip to the grid, zero behind. Consecutive
    // threads take consecutive cells of a row (coalesced reductions along a plane row).
    const int br0 = bbox[0], br1 = min(bbox[1], C::R - 1);
    const int bc0 = bbox[2], bc1 = min(bbox[3], C::R - 1);
    if (br1 >= br0 && bc1 >= bc0) {
        const long long o1 = g.gmin + (long long)t1 * T;
        const long long o2 = g.gmin + (long long)t2 * T;
        const long long row_lim = g.gmax - o1;  // rows rr <= row_lim lie on the grid
        const int col_lim = (int)min((long long)bc1, g.gmax - o2);
        const long long plane0 = (long long)(slab - slab_lo) * sp.K + term0;
        if constexpr (C::RS % 4 == 0) {
            // four cells per thread: 16-byte shared loads and stores, 16-byte reductions of two
            // interleaved complex cells where the plane row allows. The CTA's threads take the
            // box's (row, quad) pairs in row-major order (a region row holds fewer quads than a
            // warp has lanes), stepping NT pairs at a time with an incremental row/quad split.
            const int q0 = bc0 >> 2, nq = (bc1 >> 2) - q0 + 1, nr = br1 - br0 + 1;
            const int tid = warp * 32 + lane;
            const int dr = C::NT / nq, dq = C::NT - dr * nq;
            int ri = tid / nq, gi = tid - ri * nq;
            const int row_lim_i = (int)max(-1LL, min((long long)C::R, row_lim));
            const long long base0 = plane0 * GG + (o1 - g.gmin) * g.G + (o2 - g.gmin);
            const int par0 = (int)((o1 + o2) & 1);
            for (; ri < nr; ri += dr, gi += dq) {
                if (gi >= nq) {
                    gi -= nq;
                    if (++ri >= nr) break;
                }
                const int rr = br0 + ri;
                const bool row_on = rr <= row_lim_i;
                const long long rbase = base0 + (long long)(rr * (int)g.G);
                float2* prow = planes + rbase;
                // cc is a multiple of 4, so the sign of cell cc + j is s0 for even j
                const float s0 = ((par0 ^ rr) & 1) ? -inv_scale : inv_scale;
                int* trow = tile + rr * C::RS;
                {
                    const int cc = (q0 + gi) * 4;
#pragma unroll
                    for (int t = 0; t < KC; ++t) {
                        int* pl = trow + (size_t)t * 2 * C::PLANE + cc;
                        const int4 a = *reinterpret_cast<int4*>(pl);
                        const int4 b = *reinterpret_cast<int4*>(pl + C::PLANE);
                        *reinterpret_cast<int4*>(pl) = make_int4(0, 0, 0, 0);
                        *reinterpret_cast<int4*>(pl + C::PLANE) = make_int4(0, 0, 0, 0);
                        if (!row_on || !(a.x | a.y | a.z | a.w | b.x | b.y | b.z | b.w)) continue;
                        const float r0 = s0 * (float)a.x, i0 = s0 * (float)b.x;
                        const float r1 = -s0 * (float)a.y, i1 = -s0 * (float)b.y;
                        const float r2 = s0 * (float)a.z, i2 = s0 * (float)b.z;
                        const float r3 = -s0 * (float)a.w, i3 = -s0 * (float)b.w;
                        float2* p = prow + (long long)t * GG + cc;
                        if (cc + 3 <= col_lim && ((rbase + (long long)t * GG) & 1) == 0) {
                            red_add_v4(p, r0, i0, r1, i1);
                            red_add_v4(p + 2, r2, i2, r3, i3);
                        } else {
                            if (cc <= col_lim) red_add_v2(p, r0, i0);
                            if (cc + 1 <= col_lim) red_add_v2(p + 1, r1, i1);
                            if (cc + 2 <= col_lim) red_add_v2(p + 2, r2, i2);
                            if (cc + 3 <= col_lim) red_add_v2(p + 3, r3, i3);
                        }
                    }
                }
            }
        } else {
            for (int rr = br0 + warp; rr <= br1; rr += kWarps) {
                const bool row_on = rr <= row_lim;
                const long long g1 = o1 + rr;
                float2* prow = planes + plane0 * GG + (g1 - g.gmin) * g.G + (o2 - g.gmin);
                const int par = (int)((g1 + o2) & 1);
                int* trow = tile + rr * C::RS;
                for (int cc = bc0 + lane; cc <= bc1; cc += 32) {
                    const bool on = row_on && cc <= col_lim;
                    const float s = ((par ^ cc) & 1) ? -inv_scale : inv_scale;
#pragma unroll
                    for (int t = 0; t < KC; ++t) {
                        int* pl = trow + (size_t)t * 2 * C::PLANE + cc;
                        const int ire = pl[0], iim = pl[C::PLANE];
                        if (on && (ire | iim))
                            red_add_v2(prow + (long long)t * GG + cc, s * (float)ire, s * (float)iim);
                        pl[0] = 0;
                        pl[C::PLANE] = 0;
                    }
                }
            }
        }
    }
}

// KC <= 2: four CTAs per SM (at most 64 registers; the two-term form otherwise takes 80 and three)
template <int W, int T, int KC>
__global__ void __launch_bounds__(TileCfg<W, T, KC>::NT, (KC <= 2 ? 4 : 1)) k_grid_fp32(
    const SampleRec* __restrict__ rec, const float* __restrict__ rec_s,
    const unsigned int* __restrict__ offsets, const unsigned int* __restrict__ chunk_key,
    const unsigned int* __restrict__ keymax, unsigned int* __restrict__ work, int key_lo, int key_hi,
    int slab_lo, GridGeom g, SlabParams sp, EsPoly poly, float2* __restrict__ planes, int term0) {
    using C = TileCfg<W, T, KC>;
    extern __shared__ int tile[];    // [KC][2][R][RS] 32-bit fixed-point accumulators
    __shared__ int bbox[4];          // row min, row max, col min, col max
    __shared__ float chunk_part[2][TileCfg<W, T, KC>::NW];  // per-warp partial sums of the chunk
    // per-warp staging of the decoded batch: {u_x, u_y, vre, vim} and {fast-path base, s}
    constexpr int kThreads = C::NT, kWarps = C::NW;
    // per-warp staging of the decoded batch (32 samples + the zero pad): the polynomial arguments
    // {u_x, u_y}, and {v_re, v_im, shared address of the footprint origin, Chebyshev argument}
    // W = 8: two samples per warp instruction (header comment)
    constexpr bool kSplit = (W == 8) && (C::RS % 32 == 8);
    __shared__ float2 st_u[kWarps][33];
    __shared__ float4 st_v[kWarps][33];
    __shared__ float2 st_t[kWarps][33];  // KC > 1: T_term0(s), T_term0+1(s) of the staged sample

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int HW = W / 2;
    constexpr int RPP = 32 / W;                  // footprint rows per pass
    constexpr int PASSES = (W + RPP - 1) / RPP;
    constexpr bool PAIR = 2 * W <= 16;           // two samples per polynomial pass
    constexpr bool kAllLanes = (32 % W) == 0;    // every lane owns a cell in every pass
    const int la = lane / W, lb = lane % W;
    const bool lane_cell = lane < RPP * W;
    const int lane_off = la * C::RS + lb;
    // polynomial piece of this lane: x-piece (local < W) or y-piece (W <= local < 2W)
    const int local = PAIR ? (lane & 15) : lane;
    const bool is_x = local < W;
    const int piece = is_x ? local : (local < 2 * W ? local - W : 0);
    float coef[kPolyDeg + 1];
#pragma unroll
    for (int d = 0; d <= kPolyDeg; ++d) coef[d] = poly.c[piece][d];
    int wx_src[PASSES];     // lane holding the x-weight of this lane's row in pass p
    bool pass_on[PASSES];   // this lane owns a footprint cell in pass p
#pragma unroll
    for (int p = 0; p < PASSES; ++p) {
        const int i = la + p * RPP;
        wx_src[p] = i < W ? i : 0;
        pass_on[p] = lane_cell && i < W;
    }
    const unsigned int tile_s = (unsigned int)__cvta_generic_to_shared(tile);
    const unsigned int lane_off_bytes = 4u * (unsigned int)lane_off;
    // this lane's polynomial argument in the staged pair {u_x, u_y} of sample j: u_arg[2 j]
    const float* u_arg = reinterpret_cast<const float*>(&st_u[warp][0]) + (PAIR ? 2 * (lane >> 4) : 0) + (is_x ? 0 : 1);
    // kSplit: this lane's sample in the pass (h), its rows (ra, ra + 4) and its first column's
    // bank residue
    const int sp_h = lane >> 4, sp_ra = (lane >> 2) & 3, sp_rho = (lane & 3) + 4 * sp_h;

    for (int i = threadIdx.x; i < KC * 2 * C::PLANE; i += kThreads) tile[i] = 0;
    if (threadIdx.x == 0) {
        bbox[0] = C::R; bbox[1] = -1; bbox[2] = C::R; bbox[3] = -1;
    }
    __syncthreads();

    // chunks of kGridChunk records at absolute record positions (the first and last ones of the
    // key range may be partial); the scan's table gives each chunk's first key
    const unsigned int rec_lo = offsets[key_lo], rec_hi = offsets[key_hi];
    const unsigned int ch_lo = rec_lo / kGridChunk, ch_hi = (rec_hi + kGridChunk - 1) / kGridChunk;
    const bool need_s = !(KC == 1 && term0 == 0);

    // A CTA takes chunks from a global counter (runs of kRun consecutive chunks; measured on the
    // precision snapshot: 1 is fastest, longer runs of one key leave a tail). A segment that
    // continues the key accumulated in the region joins it (one fixed-point scale) while the
    // running sum bound holds; otherwise the region is reduced into the plane first.
    constexpr unsigned int kRun = 1;
    int run_key = -1;  // key accumulated in the region (-1: none); the same in every thread
    float run_scale = 0.0f, run_inv = 0.0f, run_sum = 0.0f;
    const unsigned int n_ch = ch_hi - ch_lo;
    unsigned int it = 0;
    __shared__ unsigned int s_run;
    for (;;) {
    if (threadIdx.x == 0) s_run = atomicAdd(work, 1u);
    __syncthreads();
    const unsigned int run = s_run;
    __syncthreads();
    if ((unsigned long long)run * kRun >= n_ch) break;
    const unsigned int q_end = min(n_ch, (run + 1) * kRun);
    for (unsigned int q = run * kRun; q < q_end; ++q, ++it) {
        const unsigned int ch = ch_lo + q;
        const unsigned int c_beg = max(rec_lo, ch * kGridChunk);
        const unsigned int c_end = min(rec_hi, (ch + 1) * kGridChunk);
        int key = max(key_lo, (int)chunk_key[ch]);
        // sum of max(|v_re|, |v_im|) over the chunk (fixed reduction order: the same in every thread)
        float csum = 0.0f;
        {
            float part = 0.0f;
            for (unsigned int k = c_beg + threadIdx.x; k < c_end; k += kThreads) {
                const SampleRec q = rec[k];
                part += fmaxf(fabsf(q.vre), fabsf(q.vim));
            }
            for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
            if (lane == 0) chunk_part[it & 1][warp] = part;  // two buffers: no race with the next chunk
            __syncthreads();
#pragma unroll
            for (int w = 0; w < kWarps; ++w) csum += chunk_part[it & 1][w];
        }
        while (key < key_hi && offsets[key] < c_end) {
            const unsigned int s_beg = max(c_beg, offsets[key]);
            const unsigned int s_end = min(c_end, offsets[key + 1]);
            if (s_beg < s_end) {
                // join the region's run of this key, or reduce the region and start a new run
                if (!(key == run_key && (run_sum + csum) * run_scale < 0.998f * 2147483648.0f)) {
                    if (run_key >= 0) {
                        __syncthreads();
                        flush_region<C, T, KC>(tile, bbox, run_key, slab_lo, term0, run_inv, g, sp, planes, warp, lane);
                        __syncthreads();
                        if (threadIdx.x == 0) {
                            bbox[0] = C::R; bbox[1] = -1; bbox[2] = C::R; bbox[3] = -1;
                        }
                        __syncthreads();
                    }
                    // Fixed-point scale of the run (header comment): the key's largest record (the
                    // scatter's per-key maximum) bounds each contribution, the sum over the run's
                    // chunks every cell (|psi psi T_n| <= 1 up to the polynomial's 1e-7).
                    run_key = key;
                    run_sum = 0.0f;
                    run_scale = 0.0f;
                    run_inv = 0.0f;
                    const float vmax = __uint_as_float(keymax[key]);
                    if (vmax > 0.0f && vmax < 3.0e38f && csum < 3.0e38f) {
                        int ex, es;
                        frexpf(vmax, &ex);  // vmax = f 2^ex, f in [0.5, 1)
                        frexpf(csum, &es);
                        run_scale = ldexpf(0.999f, min(kGridScaleBits - ex, 31 - es));
                        run_inv = 1.0f / run_scale;
                    }
                }
                run_sum += csum;
                const float scale = run_scale;
                for (unsigned int b0 = s_beg + warp * 32; b0 < s_end; b0 += kWarps * 32) {
                    // ---- decode this lane's record once per batch
                    const unsigned int my = b0 + lane;
                    const bool valid = my < s_end;
                    SampleRec r = {0, 0, 0.0f, 0.0f};
                    float sv = 0.0f;
                    if (valid) {
                        r = rec[my];
                        if (need_s) sv = rec_s[my];
                    }
                    const int cx = r.xq >> 24, cy = r.yq >> 24;
                    const int fxq = r.xq & 0xFFFFFF, fyq = r.yq & 0xFFFFFF;
                    const int r0 = cx - (HW - 1), c0 = cy - (HW - 1);
                    const bool rare = valid && (fxq == 0 || fyq == 0 || r0 < 0 || c0 < 0);
                    // fast samples compacted into slots [0, nfast); slot nfast is a zero pad, so
                    // the pair loop below needs no per-sample test
                    const unsigned int fast_mask = __ballot_sync(0xffffffffu, valid && !rare);
                    const int nfast = __popc(fast_mask);
                    if (valid && !rare) {
                        const int pos = __popc(fast_mask & ((1u << lane) - 1u));
                        st_u[warp][pos] = make_float2(fmaf(2.0f, (float)fxq * (1.0f / 16777216.0f), -1.0f),
                                                      fmaf(2.0f, (float)fyq * (1.0f / 16777216.0f), -1.0f));
                        // Chebyshev terms of the sample, once per sample (lane-parallel): one term per
                        // launch is folded into the sample's values, so the plain inner loop below grids
                        // it (|T_n(s)| <= 1 keeps the scale bound); KC > 1 stages T_term0 and
                        // T_term0+1, from which the inner loop runs the recurrence KC - 2 steps
                        float tn = 1.0f, tn1 = sv;
                        if (need_s) {
                            float tm2 = 1.0f, tm1 = sv;  // T_0, T_1
                            for (int t = 2; t <= term0 + 1; ++t) {
                                const float tt = 2.0f * sv * tm1 - tm2;
                                tm2 = tm1;
                                tm1 = tt;
                            }
                            tn = term0 == 0 ? 1.0f : tm2;  // T_term0
                            tn1 = term0 == 0 ? sv : tm1;    // T_term0+1
                            if (KC > 1) st_t[warp][pos] = make_float2(tn, tn1);
                        }
                        if (KC > 1) tn = 1.0f;
                        st_v[warp][pos] = make_float4(r.vre * scale * tn, r.vim * scale * tn,
                                                      __uint_as_float(tile_s + 4u * (unsigned int)(r0 * C::RS + c0)),
                                                      sv);
                    }
                    if (lane == 0) {
                        st_t[warp][nfast] = make_float2(0.0f, 0.0f);
                        st_u[warp][nfast] = make_float2(0.0f, 0.0f);
                        st_v[warp][nfast] = make_float4(0.0f, 0.0f, __uint_as_float(tile_s), 0.0f);
                    }
                    // bounding box of the batch (one warp reduction per 32 samples)
                    const int rlo = valid ? max(0, fxq ? r0 : r0 - 1) : C::R;
                    const int rhi = valid ? cx + HW : -1;
                    const int clo = valid ? max(0, fyq ? c0 : c0 - 1) : C::R;
                    const int chi = valid ? cy + HW : -1;
                    const int brlo = __reduce_min_sync(0xffffffffu, rlo);
                    const int brhi = __reduce_max_sync(0xffffffffu, rhi);
                    const int bclo = __reduce_min_sync(0xffffffffu, clo);
                    const int bchi = __reduce_max_sync(0xffffffffu, chi);
                    if (lane == 0 && brhi >= 0) {
                        atomicMin(&bbox[0], brlo); atomicMax(&bbox[1], brhi);
                        atomicMin(&bbox[2], bclo); atomicMax(&bbox[3], bchi);
                    }
                    unsigned int rare_mask = __ballot_sync(0xffffffffu, rare);
                    __syncwarp();
                    // ---- fast path: W x W footprint, polynomial weights, no bounds checks
                    constexpr int STEP = PAIR ? 2 : 1;
                    if constexpr (kSplit) {
                        // two samples per warp instruction (header comment); slot nfast is the
                        // zero pad when nfast is odd
                        const int sh = 16 * sp_h;
#pragma unroll 2
                        for (int j = 0; j < nfast; j += 2) {
                            const float u = u_arg[2 * j];
                            float w = coef[kPolyDeg];
#pragma unroll
                            for (int d = kPolyDeg - 1; d >= 0; --d) w = fmaf(w, u, coef[d]);
                            const float4 sf = st_v[warp][j + sp_h];
                            const unsigned int org = __float_as_uint(sf.z);
                            const int c0 = (sp_rho - (int)(org >> 2)) & 7;
                            const int c1 = c0 ^ 4;
                            const float wx0 = __shfl_sync(0xffffffffu, w, sh + sp_ra);
                            const float wx1 = __shfl_sync(0xffffffffu, w, sh + sp_ra + 4);
                            const float wy0 = __shfl_sync(0xffffffffu, w, sh + 8 + c0);
                            const float wy1 = __shfl_sync(0xffffffffu, w, sh + 8 + c1);
                            const unsigned int a0 = org + 4u * (unsigned int)(sp_ra * C::RS + c0);
                            const unsigned int a1 = org + 4u * (unsigned int)(sp_ra * C::RS + c1);
                            if constexpr (KC > 1) {
                                // the lane's sample's terms T_term0 .. T_term0+KC-1 (staged pair, recurrence)
                                float tv[KC];
                                const float2 t01 = st_t[warp][j + sp_h];
                                tv[0] = t01.x;
                                tv[1] = t01.y;
#pragma unroll
                                for (int t = 2; t < KC; ++t) tv[t] = 2.0f * sf.w * tv[t - 1] - tv[t - 2];
                                float kv = wx0 * wy0;
                                red_terms<0, KC, 0, C::PLANE>(a0, kv * sf.x, kv * sf.y, tv);
                                kv = wx0 * wy1;
                                red_terms<0, KC, 0, C::PLANE>(a1, kv * sf.x, kv * sf.y, tv);
                                kv = wx1 * wy0;
                                red_terms<0, KC, 16 * C::RS, C::PLANE>(a0, kv * sf.x, kv * sf.y, tv);
                                kv = wx1 * wy1;
                                red_terms<0, KC, 16 * C::RS, C::PLANE>(a1, kv * sf.x, kv * sf.y, tv);
                                continue;
                            }
                            float kv = wx0 * wy0;
                            red_shared<0>(a0, fx_round(fmaf(kv, sf.x, kMagic)));
                            red_shared<4 * C::PLANE>(a0, fx_round(fmaf(kv, sf.y, kMagic)));
                            kv = wx0 * wy1;
                            red_shared<0>(a1, fx_round(fmaf(kv, sf.x, kMagic)));
                            red_shared<4 * C::PLANE>(a1, fx_round(fmaf(kv, sf.y, kMagic)));
                            kv = wx1 * wy0;
                            red_shared<16 * C::RS>(a0, fx_round(fmaf(kv, sf.x, kMagic)));
                            red_shared<16 * C::RS + 4 * C::PLANE>(a0, fx_round(fmaf(kv, sf.y, kMagic)));
                            kv = wx1 * wy1;
                            red_shared<16 * C::RS>(a1, fx_round(fmaf(kv, sf.x, kMagic)));
                            red_shared<16 * C::RS + 4 * C::PLANE>(a1, fx_round(fmaf(kv, sf.y, kMagic)));
                        }
                    } else if (KC == 1) {
#pragma unroll 2
                        for (int j = 0; j < nfast; j += STEP) {
                            const float u = u_arg[2 * j];
                            float w = coef[kPolyDeg];
#pragma unroll
                            for (int d = kPolyDeg - 1; d >= 0; --d) w = fmaf(w, u, coef[d]);
#pragma unroll
                            for (int h = 0; h < STEP; ++h) {
                                const float4 sf = st_v[warp][j + h];
                                const float wy = __shfl_sync(0xffffffffu, w, 16 * h + W + lb);
                                const unsigned int a = __float_as_uint(sf.z) + lane_off_bytes;
                                grid_passes<0, PASSES, RPP, C::RS, C::PLANE, kAllLanes>(
                                    a, w, wy, sf.x, sf.y, 16 * h, wx_src, pass_on);
                            }
                        }
                    } else {
                        for (int j = 0; j < nfast; j += STEP) {
                            const float u = u_arg[2 * j];
                            float w = coef[kPolyDeg];
#pragma unroll
                            for (int d = kPolyDeg - 1; d >= 0; --d) w = fmaf(w, u, coef[d]);
#pragma unroll
                            for (int h = 0; h < STEP; ++h) {
                                const float4 sf = st_v[warp][j + h];
                                const float wy = __shfl_sync(0xffffffffu, w, 16 * h + W + lb);
                                float tv[KC];
                                {
                                    const float s = sf.w;
                                    const float2 t01 = st_t[warp][j + h];
                                    tv[0] = t01.x;
                                    if (KC > 1) tv[KC > 1 ? 1 : 0] = t01.y;
#pragma unroll
                                    for (int t = 2; t < KC; ++t) tv[t] = 2.0f * s * tv[t - 1] - tv[t - 2];
                                }
                                const int base = (int)((__float_as_uint(sf.z) - tile_s) >> 2) + lane_off;
#pragma unroll
                                for (int p = 0; p < PASSES; ++p) {
                                    const float wx = __shfl_sync(0xffffffffu, w, 16 * h + wx_src[p]);
                                    if (pass_on[p]) {
                                        const float kv = wx * wy;
                                        int* pl = tile + base + p * RPP * C::RS;
                                        const float ar = kv * sf.x, ai = kv * sf.y;
#pragma unroll
                                        for (int t = 0; t < KC; ++t) {
                                            atomicAdd(pl + (size_t)t * 2 * C::PLANE, fx_round(fmaf(ar, tv[t], kMagic)));
                                            atomicAdd(pl + (size_t)t * 2 * C::PLANE + C::PLANE,
                                                      fx_round(fmaf(ai, tv[t], kMagic)));
                                        }
                                    }
                                }
                            }
                        }
                    }
                    // ---- rare path: exactly-integer positions (W+1 cells, psi(-1) at the ends) and
                    // footprints clipped at the low grid edge; exact ES formula, lanes over cells
                    while (rare_mask) {
                        const int js = __ffs(rare_mask) - 1;
                        rare_mask &= rare_mask - 1;
                        const SampleRec rr_ = rec[b0 + js];
                        const float s = need_s ? rec_s[b0 + js] : 0.0f;
                        const int rcx = rr_.xq >> 24, rcy = rr_.yq >> 24;
                        const int rfx = rr_.xq & 0xFFFFFF, rfy = rr_.yq & 0xFFFFFF;
                        const int lo_r = rfx ? rcx - (HW - 1) : rcx - HW, nr = rfx ? W : W + 1;
                        const int lo_c = rfy ? rcy - (HW - 1) : rcy - HW, nc = rfy ? W : W + 1;
                        const float px = (float)rfx * (1.0f / 16777216.0f), py = (float)rfy * (1.0f / 16777216.0f);
                        float tv[KC];
                        {
                            float tm2 = 1.0f, tm1 = s;
                            for (int t = 0; t < term0 + KC; ++t) {
                                const float tn = t == 0 ? 1.0f : (t == 1 ? s : 2.0f * s * tm1 - tm2);
                                if (t >= 2) { tm2 = tm1; tm1 = tn; }
                                if (t >= term0) tv[t - term0] = tn;
                            }
                        }
                        for (int c = lane; c < nr * nc; c += 32) {
                            const int i = c / nc, jj = c % nc;
                            const int rr = lo_r + i, cc = lo_c + jj;
                            if (rr < 0 || cc < 0) continue;
                            const float x = ((float)(lo_r + i - rcx) - px) / (float)HW;
                            const float y = ((float)(lo_c + jj - rcy) - py) / (float)HW;
                            const float kv = es_exact(poly.beta, x) * es_exact(poly.beta, y);
                            const float ar = kv * (rr_.vre * scale), ai = kv * (rr_.vim * scale);
                            for (int t = 0; t < KC; ++t) {
                                int* pl = tile + (size_t)t * 2 * C::PLANE + rr * C::RS + cc;
                                atomicAdd(pl, fx_round(fmaf(ar, tv[t], kMagic)));
                                atomicAdd(pl + C::PLANE, fx_round(fmaf(ai, tv[t], kMagic)));
                            }
                        }
                    }
                    __syncwarp();
                }
                __syncthreads();
            }
            ++key;
        }
    }
    }
    if (run_key >= 0) {
        __syncthreads();
        flush_region<C, T, KC>(tile, bbox, run_key, slab_lo, term0, run_inv, g, sp, planes, warp, lane);
    }
}
template <int W, int T, int KC>
int launch_variant(const SampleRec* d_rec, const float* d_rec_s, const unsigned int* d_offsets,
                   const unsigned int* d_chunk_key, const unsigned int* d_keymax, unsigned int* d_work,
                   int key_lo, int key_hi, int slab_lo, const GridGeom& g, const SlabParams& sp,
                   const EsPoly& poly, float2* d_planes, int term0, int sm_count, cudaStream_t st) {
    using C = TileCfg<W, T, KC>;
    auto kern = k_grid_fp32<W, T, KC>;
    SVDI_TRY(ensure_dynamic_smem((const void*)kern, C::SMEM));
    int per_sm = 0;
    SVDI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::NT, C::SMEM));
    if (per_sm < 1) per_sm = 1;
    SVDI_CUDA(cudaMemsetAsync(d_work, 0, sizeof(unsigned int), st));
    kern<<<sm_count * per_sm, C::NT, C::SMEM, st>>>(d_rec, d_rec_s, d_offsets, d_chunk_key, d_keymax, d_work,
                                                     key_lo, key_hi, slab_lo, g, sp, poly, d_planes, term0);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

template <int W>
int launch_w(const SampleRec* d_rec, const float* d_rec_s, const unsigned int* d_offsets,
             const unsigned int* d_chunk_key, const unsigned int* d_keymax, unsigned int* d_work, int key_lo,
             int key_hi, int slab_lo, const GridGeom& g, const SlabParams& sp, const EsPoly& poly,
             float2* d_planes, int sm_count, cudaStream_t st) {

    if (g.T == 64) {
        for (int t0 = 0; t0 < sp.K; ++t0)
            SVDI_TRY((launch_variant<W, 64, 1>(d_rec, d_rec_s, d_offsets, d_chunk_key, d_keymax, d_work, key_lo, key_hi,
                                               slab_lo, g, sp, poly, d_planes, t0, sm_count, st)));
        return SVDI_OK;
    }
    if (g.T == 32) {
        int t0 = 0;
        for (; t0 + 8 <= sp.K; t0 += 8)
            SVDI_TRY((launch_variant<W, 32, 8>(d_rec, d_rec_s, d_offsets, d_chunk_key, d_keymax, d_work, key_lo, key_hi,
                                               slab_lo, g, sp, poly, d_planes, t0, sm_count, st)));
        for (; t0 + 4 <= sp.K; t0 += 4)
            SVDI_TRY((launch_variant<W, 32, 4>(d_rec, d_rec_s, d_offsets, d_chunk_key, d_keymax, d_work, key_lo, key_hi,
                                               slab_lo, g, sp, poly, d_planes, t0, sm_count, st)));
        for (; t0 + 2 <= sp.K; t0 += 2)
            SVDI_TRY((launch_variant<W, 32, 2>(d_rec, d_rec_s, d_offsets, d_chunk_key, d_keymax, d_work, key_lo, key_hi,
                                               slab_lo, g, sp, poly, d_planes, t0, sm_count, st)));
        for (; t0 < sp.K; ++t0)
            SVDI_TRY((launch_variant<W, 32, 1>(d_rec, d_rec_s, d_offsets, d_chunk_key, d_keymax, d_work, key_lo, key_hi,
                                               slab_lo, g, sp, poly, d_planes, t0, sm_count, st)));
        return SVDI_OK;
    }
    set_error("gridder: tile size must be 32 or 64");
    return SVDI_ERR_UNSUPPORTED;
}

}  // namespace

int launch_grid_fp32(const SampleRec* d_rec, const float* d_rec_s, const unsigned int* d_offsets,
                     const unsigned int* d_chunk_key, const unsigned int* d_keymax, unsigned int* d_work,
                     int n_keys, int key_lo, int key_hi, int slab_lo, const GridGeom& g,
                     const SlabParams& sp, const EsPoly& poly, float2* d_planes, int sm_count,
                     cudaStream_t st) {
    if (key_lo < 0 || key_hi > n_keys || key_lo >= key_hi || !d_chunk_key || !d_keymax || !d_work) {
        set_error("gridder: bad key range or missing chunk table");
        return SVDI_ERR_INTERNAL;
    }
    switch (g.W) {
        case 6: return launch_w<6>(d_rec, d_rec_s, d_offsets, d_chunk_key, d_keymax, d_work, key_lo, key_hi, slab_lo, g, sp, poly, d_planes, sm_count, st);
        case 8: return launch_w<8>(d_rec, d_rec_s, d_offsets, d_chunk_key, d_keymax, d_work, key_lo, key_hi, slab_lo, g, sp, poly, d_planes, sm_count, st);
        case 10: return launch_w<10>(d_rec, d_rec_s, d_offsets, d_chunk_key, d_keymax, d_work, key_lo, key_hi, slab_lo, g, sp, poly, d_planes, sm_count, st);
        case 12: return launch_w<12>(d_rec, d_rec_s, d_offsets, d_chunk_key, d_keymax, d_work, key_lo, key_hi, slab_lo, g, sp, poly, d_planes, sm_count, st);
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
    out->beta = (float)beta;
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
