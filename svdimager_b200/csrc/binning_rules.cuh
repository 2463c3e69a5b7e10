// Per-sample rules of the tile-binning contract (position quantisation, footprint clipping,
// tile and slab keys), shared by the binning kernels and the FP64 accuracy probe so that both
// apply the same inclusion rule bit for bit. The contract itself is stated in binning.cu.
#pragma once

#include "svdi_internal.cuh"

namespace svdi {
namespace binrules {

struct KeyRec {
    int key;     // -1: dropped
    int xq, yq;
    float s;
};

// floor(x / T) for 0 <= x < 2^24 and 1 <= T < 2^24, exact: a float estimate (off by at most one
// for these ranges) and one integer correction.
__device__ inline int tile_div(int x, int T) {
    int t = __float2int_rz(__fmul_rn(__int2float_rn(x), __frcp_rn(__int2float_rn(T))));
    if (t * T > x) --t;
    else if ((t + 1) * T <= x) ++t;
    return t;
}

// Q = floor(p 2^24) split into cell = floor(p) = Q >> 24 and frac = Q & (2^24 - 1): p 2^24 is exact
// (power-of-two scaling) and one round-down conversion to a 64-bit integer gives Q exactly
// (|Q| < 1e9 2^24 < 2^54), so the split is integer arithmetic. |p| >= 1e9 lies beyond every grid
// (G < 2^24) and is dropped under both edge rules, like the contract's 1e15 bound; within it every
// cell fits 32 bits (tiles T <= 64).
__device__ inline bool quantise_axis(double p, const GridGeom& g, int T, int& tile, int& qrel) {
    if (!(fabs(p) < 1e9)) return false;
    const long long Q = __double2ll_rd(p * 16777216.0);
    const int cell = (int)(Q >> 24);
    const int frac = (int)(Q & 0xFFFFFF);
    const int hw = g.W / 2;
    const int gmin = (int)g.gmin, gmax = (int)g.gmax;
    int lo = frac ? cell - (hw - 1) : cell - hw;
    int hi = cell + hw;
    if (g.edge_mode == SVDI_EDGE_STRICT) {
        if (lo < gmin || hi > gmax) return false;
    } else {
        if (lo < gmin) lo = gmin;
        if (hi > gmax) hi = gmax;
        if (lo > hi) return false;
    }
    tile = tile_div(lo - gmin, T);  // 0 <= lo - gmin < G < 2^24
    const int origin = gmin + tile * T;
    qrel = (int)((unsigned)(cell - origin) * 16777216u + (unsigned)frac);  // Q - origin 2^24
    return true;
}

__device__ inline double grid_pos(double r, const GridGeom& g) {
    if (g.coord_mode == SVDI_COORD_REF32) return (double)__fmul_rn((float)r, g.scale32);
    return __dmul_rn(r, g.scale);
}

__device__ inline void sample_coords(const SampleSource& src, long long idx, double& r1, double& r2,
                                     double& r3) {
    if (src.bin) {
        r1 = (double)src.bin[idx * 3 + 0];
        r2 = (double)src.bin[idx * 3 + 1];
        r3 = (double)src.bin[idx * 3 + 2];
    } else {
        const long long row = idx % src.R, c = idx / src.R;
        const double sc = src.s[c];
        r1 = __dmul_rn(sc, src.q[row * 3 + 0]);
        r2 = __dmul_rn(sc, src.q[row * 3 + 1]);
        r3 = __dmul_rn(sc, src.q[row * 3 + 2]);
    }
}

// Key of a sample at rotated coordinate (r1, r2, r3).
__device__ inline KeyRec coord_key(double r1, double r2, double r3, const GridGeom& g, const SlabParams& sp) {
    KeyRec k;
    k.key = -1;
    int t1, t2;
    if (!quantise_axis(grid_pos(r1, g), g, g.T, t1, k.xq) || !quantise_axis(grid_pos(r2, g), g, g.T2, t2, k.yq))
        return k;
    int j = 0;
    double sv = 0.0;
    if (sp.nslab > 1 || sp.K > 1) {
        double jf = floor(__ddiv_rn(__dsub_rn(r3, sp.r3_min), sp.slab_width));
        if (!(jf >= 0.0)) jf = 0.0;  // also NaN
        if (jf > (double)(sp.nslab - 1)) jf = (double)(sp.nslab - 1);
        j = (int)jf;
        const double centre = __dadd_rn(sp.r3_min, __dmul_rn((double)j + 0.5, sp.slab_width));
        sv = __dmul_rn(__dsub_rn(r3, centre), sp.inv_half);
        sv = fmin(1.0, fmax(-1.0, sv));
    }
    k.s = (float)sv;
    k.key = (j * g.ntile + t1) * g.ntile2 + t2;
    return k;
}

__device__ inline KeyRec sample_key(const SampleSource& src, long long idx, const GridGeom& g,
                                    const SlabParams& sp) {
    double r1, r2, r3;
    sample_coords(src, idx, r1, r2, r3);
    return coord_key(r1, r2, r3, g, sp);
}

// Key of channel scale `sc` on the row with rotated coordinates q: the separable form of
// sample_coords (the same three FP64 products) followed by coord_key.
__device__ inline KeyRec row_chan_key(double sc, double q1, double q2, double q3, const GridGeom& g,
                                      const SlabParams& sp) {
    return coord_key(__dmul_rn(sc, q1), __dmul_rn(sc, q2), __dmul_rn(sc, q3), g, sp);
}

}  // namespace binrules
}  // namespace svdi
