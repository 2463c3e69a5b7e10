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

__device__ inline bool quantise_axis(double p, const GridGeom& g, int T, int& tile, int& qrel) {
    if (!(fabs(p) < 1e15)) return false;
    const long long Q = (long long)floor(p * 16777216.0);
    const long long cell = Q >> 24;
    const long long frac = Q & 0xFFFFFFLL;
    const long long hw = g.W / 2;
    long long lo = frac ? cell - (hw - 1) : cell - hw;
    long long hi = cell + hw;
    if (g.edge_mode == SVDI_EDGE_STRICT) {
        if (lo < g.gmin || hi > g.gmax) return false;
    } else {
        if (lo < g.gmin) lo = g.gmin;
        if (hi > g.gmax) hi = g.gmax;
        if (lo > hi) return false;
    }
    tile = (int)((lo - g.gmin) / T);
    const long long origin = g.gmin + (long long)tile * T;
    qrel = (int)(Q - origin * 16777216LL);
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

__device__ inline KeyRec sample_key(const SampleSource& src, long long idx, const GridGeom& g,
                                    const SlabParams& sp) {
    KeyRec k;
    k.key = -1;
    double r1, r2, r3;
    sample_coords(src, idx, r1, r2, r3);
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

}  // namespace binrules
}  // namespace svdi
