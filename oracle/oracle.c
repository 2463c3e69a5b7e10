/*
 * ORACLE — test infrastructure only.
 *
 * CPU restatement of the reference snapshot imager (egbdfX/SVDimager) and an FP64 direct-DFT
 * imager. Only tests/, the smoke check in __graft_entry__.py and bench.py's cpu_baseline /
 * reference legs load this library, and only as the checker or the CPU baseline. The product
 * (svdimager_b200) never links or calls it.
 *
 * Every function cites the reference lines it restates. Reference paths are relative to the
 * reference project root:
 *   SII  = SVDIntegratedImager.cu            (latest release, slab + bucket-K main path)
 *   FIPK = archive/FIPkernels.cu             (archive FIpipe path)
 *   MFS  = archive/SVD_MFS.py                (archive Python pre-processor)
 *
 * Precision conventions of this restatement (they mirror the B200 implementation, which the
 * parity tests compare against it):
 *   - flag/weight collapse in FP32 with one rounding per operation (no contraction), exactly the
 *     operation order of SII:606-616;
 *   - baselines, SVD rotation and grid coordinates in FP64 (the reference uses FP32 there);
 *   - gridding weights and accumulation in FP64;
 *   - Bessel coefficients in FP64.
 * The reference's FP32 Bessel power series (SII:901-920) is restated separately
 * (orc_bessel_series_f32) to quantify the reference's own error.
 *
 * Compile: see oracle/Makefile (-O2 -fopenmp -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_C_LIGHT 299792458.0
#define ORC_PI 3.14159265358979323846

/* ------------------------------------------------------------------------------------------ */
/* Flag / WEIGHT_SPECTRUM polarisation collapse.  SII:588-617 (also MFS.py:74-90).            */
/* w_p = flag_p ? 0 : weight_p ; V = (V0 w0 + V3 w3) / (w0 + w3), or 0 when the sum is 0.      */
/* ------------------------------------------------------------------------------------------ */
void orc_collapse(long n, const float* v0r, const float* v0i, const float* v3r, const float* v3i,
                  const uint8_t* f0, const uint8_t* f3, const float* w0in, const float* w3in,
                  float* outr, float* outi) {
    for (long k = 0; k < n; ++k) {
        const float w0 = f0[k] ? 0.0f : w0in[k];
        const float w3 = f3[k] ? 0.0f : w3in[k];
        const float ws = w0 + w3;
        if (ws > 0.0f) {
            const float a = v0r[k] * w0;
            const float b = v3r[k] * w3;
            const float c = v0i[k] * w0;
            const float d = v3i[k] * w3;
            outr[k] = (a + b) / ws;
            outi[k] = (c + d) / ws;
        } else {
            outr[k] = 0.0f;
            outi[k] = 0.0f;
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* 3x3 symmetric eigen-decomposition by cyclic Jacobi rotations (FP64).                        */
/* Replaces cusolverDnSsyevd (SII:736-760); eigenvalues returned in ascending order like it.   */
/* evec is column-major: column j is the eigenvector of eval[j].                               */
/* ------------------------------------------------------------------------------------------ */
void orc_jacobi3(const double* a_in, double* eval, double* evec) {
    double a[9];
    memcpy(a, a_in, sizeof(a));
    double v[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = a[1] * a[1] + a[2] * a[2] + a[5] * a[5];
        double diag = a[0] * a[0] + a[4] * a[4] + a[8] * a[8];
        if (off <= 1e-300 || off <= diag * 1e-34) break;
        for (int p = 0; p < 2; ++p) {
            for (int q = p + 1; q < 3; ++q) {
                const double apq = a[p * 3 + q];
                if (apq == 0.0) continue;
                const double app = a[p * 3 + p], aqq = a[q * 3 + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) { /* A <- A J */
                    const double akp = a[k * 3 + p], akq = a[k * 3 + q];
                    a[k * 3 + p] = c * akp - s * akq;
                    a[k * 3 + q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) { /* A <- J^T A */
                    const double apk = a[p * 3 + k], aqk = a[q * 3 + k];
                    a[p * 3 + k] = c * apk - s * aqk;
                    a[q * 3 + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) { /* V <- V J */
                    const double vkp = v[k * 3 + p], vkq = v[k * 3 + q];
                    v[k * 3 + p] = c * vkp - s * vkq;
                    v[k * 3 + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    int idx[3] = {0, 1, 2};
    double d[3] = {a[0], a[4], a[8]};
    for (int i = 0; i < 3; ++i)
        for (int j = i + 1; j < 3; ++j)
            if (d[idx[j]] < d[idx[i]]) { int t = idx[i]; idx[i] = idx[j]; idx[j] = t; }
    for (int j = 0; j < 3; ++j) {
        eval[j] = d[idx[j]];
        for (int k = 0; k < 3; ++k) evec[j * 3 + k] = v[k * 3 + idx[j]];
    }
}

/* ------------------------------------------------------------------------------------------ */
/* SVD/PCA rotation of the baselines, FP64.                                                    */
/* b_k = uvw_row * f_chan / c                          SII:409-429 (flattened idx=row+chan*R)  */
/* mean, covariance (b-m)^T (b-m)                      SII:431-488, SII:717-734                */
/* eigenvectors, descending rows                       SII:736-762, SII:490-507                */
/* orientation (row0 u>=0, row1 v ~ ARRAY_CENTER.x, row2 = row0 x row1)   SII:538-586          */
/* projection r = Vin b (un-centred baselines)         SII:509-536, SII:772-777                */
/* Outputs vin (row-major 3x3), q[row] = Vin uvw_row and s[chan] = f/c, so r_k = s_chan q_row. */
/* ------------------------------------------------------------------------------------------ */
void orc_preprocess64(long nrows, long nch, const float* uvw, const float* freq,
                      float array_center_x, double* vin, double* q, double* s, double* evals) {
    const long ns = nrows * nch;
    for (long c = 0; c < nch; ++c) s[c] = (double)freq[c] / ORC_C_LIGHT;
    double sum[3] = {0, 0, 0};
    for (long c = 0; c < nch; ++c)
        for (long r = 0; r < nrows; ++r)
            for (int a = 0; a < 3; ++a) sum[a] += (double)uvw[r * 3 + a] * s[c];
    double m[3];
    for (int a = 0; a < 3; ++a) m[a] = sum[a] / (double)ns;
    double cov[9] = {0};
    for (long c = 0; c < nch; ++c)
        for (long r = 0; r < nrows; ++r) {
            double d[3];
            for (int a = 0; a < 3; ++a) d[a] = (double)uvw[r * 3 + a] * s[c] - m[a];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) cov[a * 3 + b] += d[a] * d[b];
        }
    double ev[3], evec[9];
    orc_jacobi3(cov, ev, evec);
    if (evals) memcpy(evals, ev, sizeof(ev));
    /* rows of the basis in descending eigenvalue order (build_basis_kernel) */
    double v[9];
    for (int a = 0; a < 3; ++a) {
        v[0 * 3 + a] = evec[2 * 3 + a];
        v[1 * 3 + a] = evec[1 * 3 + a];
        v[2 * 3 + a] = evec[0 * 3 + a];
    }
    if (v[0] < 0.0)
        for (int a = 0; a < 3; ++a) v[a] = -v[a];
    if (array_center_x != 0.0f && v[4] * (double)array_center_x < 0.0)
        for (int a = 0; a < 3; ++a) v[3 + a] = -v[3 + a];
    double r20 = v[1] * v[5] - v[2] * v[4];
    double r21 = v[2] * v[3] - v[0] * v[5];
    double r22 = v[0] * v[4] - v[1] * v[3];
    const double nrm = sqrt(r20 * r20 + r21 * r21 + r22 * r22);
    if (nrm > 0.0) { r20 /= nrm; r21 /= nrm; r22 /= nrm; }
    v[6] = r20; v[7] = r21; v[8] = r22;
    memcpy(vin, v, sizeof(v));
    for (long r = 0; r < nrows; ++r)
        for (int a = 0; a < 3; ++a)
            q[r * 3 + a] = v[a * 3 + 0] * (double)uvw[r * 3 + 0] + v[a * 3 + 1] * (double)uvw[r * 3 + 1] +
                           v[a * 3 + 2] * (double)uvw[r * 3 + 2];
}

/* Expand the separable coordinates: r[k] = s[chan] * q[row], k = row + chan * nrows (SII:90-92) */
void orc_expand_coords(long nrows, long nch, const double* q, const double* s, double* r) {
    for (long c = 0; c < nch; ++c)
        for (long row = 0; row < nrows; ++row)
            for (int a = 0; a < 3; ++a) r[(row + c * nrows) * 3 + a] = s[c] * q[row * 3 + a];
}

/* ------------------------------------------------------------------------------------------ */
/* Exponential-of-semicircle kernel psi(x) = exp(beta (sqrt(1 - x^2) - 1)), 0 outside |x|<=1.  */
/* SII:884-888, FIPK:60-64.                                                                    */
/* ------------------------------------------------------------------------------------------ */
double orc_es(double beta, double x) {
    const double xx = x * x;
    return xx > 1.0 ? 0.0 : exp(beta * (sqrt(1.0 - xx) - 1.0));
}

/* Fourier transform of the ES kernel at image pixel i of a G-point grid, support W:           */
/* Phi(i) = W * int_0^1 psi(t) cos(pi W (i/G) t) dt. This equals conv_corr_kernel[i] *        */
/* conv_corr_norm_factor of the reference (SII:1204-1216, FIPK:368-381), which approximates    */
/* the same integral with a 28-point Gauss-Legendre rule. Here: composite Gauss-Legendre on   */
/* 64 panels x 16 nodes, FP64.                                                                 */
void orc_es_correction(long half_n, long G, int W, double beta, double* phi) {
    static const double x16[8] = {0.0950125098376374, 0.2816035507792589, 0.4580167776572274,
                                  0.6178762444026438, 0.7554044083550030, 0.8656312023878318,
                                  0.9445750230732326, 0.9894009349916499};
    static const double w16[8] = {0.1894506104550685, 0.1826034150449236, 0.1691565193950025,
                                  0.1495959888165767, 0.1246289712555339, 0.0951585116824928,
                                  0.0622535239386479, 0.0271524594117541};
    const int panels = 64;
    for (long i = 0; i <= half_n; ++i) {
        const double f = ORC_PI * (double)W * ((double)i / (double)G);
        double acc = 0.0;
        for (int p = 0; p < panels; ++p) {
            const double a = (double)p / panels, b = (double)(p + 1) / panels;
            const double mid = 0.5 * (a + b), hw = 0.5 * (b - a);
            for (int j = 0; j < 8; ++j) {
                const double t1 = mid - hw * x16[j], t2 = mid + hw * x16[j];
                acc += w16[j] * hw * (orc_es(beta, t1) * cos(f * t1) + orc_es(beta, t2) * cos(f * t2));
            }
        }
        phi[i] = (double)W * acc;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Footprint of one sample along one axis. The grid position is quantised to 2^-24 cells,     */
/* Q = floor(p 2^24), pq = Q 2^-24 (the binning contract of the B200 path); the footprint is    */
/* [ceil(pq - W/2), floor(pq + W/2)] (SII:1261-1267, FIPK:404-410) clipped to the grid          */
/* [-G/2, (G-1)/2]. edge_mode 1 ("strict") drops the sample instead when its footprint leaves  */
/* the grid. Returns 0 when the sample is dropped; *pq receives the quantised position.       */
/* ------------------------------------------------------------------------------------------ */
static int orc_footprint(double p, int W, long G, int edge_mode, long* lo, long* hi, double* pq) {
    const long gmin = -(G / 2), gmax = (G - 1) / 2;
    if (!(fabs(p) < 1e15)) return 0;
    const long long Q = (long long)floor(p * 16777216.0);
    const long long cell = Q >> 24, frac = Q & 0xFFFFFFLL;
    const long hw = W / 2;
    long a = (long)(frac ? cell - (hw - 1) : cell - hw), b = (long)(cell + hw);
    if (edge_mode == 1 && (a < gmin || b > gmax)) return 0;
    if (a < gmin) a = gmin;
    if (b > gmax) b = gmax;
    if (a > b) return 0;
    *lo = a;
    *hi = b;
    *pq = (double)Q / 16777216.0;
    return 1;
}

/* Grid position of a coordinate. coord_mode 0: FP64 p = r * scale. coord_mode 1: the
 * reference's FP32 rounding, p = fl32(fl32(r) * fl32(scale)) (SII:1246-1247, FIPK:400-401). */
static double orc_pos(double r, double scale, int coord_mode) {
    if (coord_mode == 1) return (double)((float)r * (float)scale);
    return r * scale;
}

/* Slab index and Chebyshev argument of a sample (SII:1248-1260). FP64. */
static void orc_slab(double r3, int nslab, double r3_min, double slab_width, double inv_half,
                     int* slab, double* s) {
    int j = (int)floor((r3 - r3_min) / slab_width);
    if (j < 0) j = 0;
    if (j > nslab - 1) j = nslab - 1;
    const double centre = r3_min + ((double)j + 0.5) * slab_width;
    double x = (r3 - centre) * inv_half;
    if (x > 1.0) x = 1.0;
    if (x < -1.0) x = -1.0;
    *slab = j;
    *s = x;
}

/* ------------------------------------------------------------------------------------------ */
/* Tile binning keys. For every sample: the grid position p = r * scale (FP64, scale =        */
/* cell_size * G, or the reference's FP32 rounding), its clipped footprint origin (lo1, lo2),  */
/* and the key                                                                                  */
/*   key = (slab * ntile + (lo1 + G/2) / T) * ntile2 + (lo2 + G/2) / T2,  ntile = ceil(G / T)  */
/* (square tiles: T2 = T, ntile2 = ntile; the tensor-core gridder uses tall narrow tiles)      */
/* or -1 when the sample touches no cell. xq/yq (optional) receive the record coordinates of   */
/* the B200 path: Q - (tile origin) * 2^24 with Q = floor(p 2^24). This is the binning         */
/* contract of the B200 path (bit-exact); the reference grids unsorted (SII:1218-1293).         */
/* ------------------------------------------------------------------------------------------ */
void orc_tile_keys(long n, const double* r, double scale, int coord_mode, long G, int W, int T,
                   int T2, long ntile2, int edge_mode, int nslab, double r3_min, double slab_width,
                   double inv_half, int64_t* keys, int32_t* xq, int32_t* yq, float* sarg) {
    const long ntile = (G + T - 1) / T;
    const long gmin = -(G / 2);
    for (long k = 0; k < n; ++k) {
        const double p1 = orc_pos(r[k * 3 + 0], scale, coord_mode);
        const double p2 = orc_pos(r[k * 3 + 1], scale, coord_mode);
        long a1, b1, a2, b2;
        double q1, q2;
        if (!orc_footprint(p1, W, G, edge_mode, &a1, &b1, &q1) ||
            !orc_footprint(p2, W, G, edge_mode, &a2, &b2, &q2)) {
            keys[k] = -1;
            continue;
        }
        int slab;
        double s;
        orc_slab(r[k * 3 + 2], nslab, r3_min, slab_width, inv_half, &slab, &s);
        const long t1 = (a1 - gmin) / T, t2 = (a2 - gmin) / T2;
        keys[k] = ((int64_t)slab * ntile + t1) * ntile2 + t2;
        if (xq) xq[k] = (int32_t)((long long)floor(p1 * 16777216.0) - (gmin + t1 * T) * 16777216LL);
        if (yq) yq[k] = (int32_t)((long long)floor(p2 * 16777216.0) - (gmin + t2 * T2) * 16777216LL);
        if (sarg) sarg[k] = (float)s;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* ES gridding of Chebyshev w-moments. SII:1218-1293 (fused_gridding); FIPK:383-452.          */
/* planes: complex128 [nslab*K][G][G], plane = slab*K + term; cell (g1, g2) -> index           */
/* (g1 + G/2) * G + (g2 + G/2). Weight = V * T_term(s) / det * psi1 * psi2 * (-1)^(g1+g2).     */
/* The reference divides by det in the gridder (SII:1285) or beforehand (FIPK:377-381).        */
/* Accumulation in FP64. Threads own 8-row bands of grid rows in turn (band b -> thread b mod  */
/* threads, which spreads a dense uv core over all threads); each cell's contributions add in  */
/* sample order, whatever the thread count.                                                    */
/* ------------------------------------------------------------------------------------------ */
#define ORC_BAND 8
void orc_grid(long n, const double* r, const float* vr, const float* vi, double scale, int coord_mode,
              long G, int W, double beta, int K, int nslab, double r3_min, double slab_width,
              double inv_half, double inv_det, int edge_mode, double* planes /* interleaved re,im */) {
    const long GG = G * G;
    const double half_w_inv = 2.0 / (double)W;
    const long gmin = -(G / 2);
    /* first footprint row of every sample (or -1 when the sample is not gridded) */
    long* row0 = (long*)malloc((size_t)(n > 0 ? n : 1) * sizeof(long));
#pragma omp parallel for schedule(static)
    for (long k = 0; k < n; ++k) {
        long a1, b1, a2, b2;
        double q1, q2;
        const double p1 = orc_pos(r[k * 3 + 0], scale, coord_mode);
        const double p2 = orc_pos(r[k * 3 + 1], scale, coord_mode);
        row0[k] = (orc_footprint(p1, W, G, edge_mode, &a1, &b1, &q1) &&
                   orc_footprint(p2, W, G, edge_mode, &a2, &b2, &q2)) ? a1 - gmin : -1;
    }
#pragma omp parallel
    {
        long nt = 1, tid = 0;
#ifdef _OPENMP
        nt = omp_get_num_threads();
        tid = omp_get_thread_num();
#endif
        double w1[64], w2[64], cheb[64];
        for (long k = 0; k < n; ++k) {
            const long r0 = row0[k];
            if (r0 < 0) continue;
            /* the footprint's W + 1 rows touch at most three bands */
            const long bfirst = r0 / ORC_BAND, blast = (r0 + W) / ORC_BAND;
            int mine = 0;
            for (long b = bfirst; b <= blast; ++b) mine |= (b % nt) == tid;
            if (!mine) continue;
            const double p1 = orc_pos(r[k * 3 + 0], scale, coord_mode);
            const double p2 = orc_pos(r[k * 3 + 1], scale, coord_mode);
            long a1, b1, a2, b2;
            double q1, q2;
            orc_footprint(p1, W, G, edge_mode, &a1, &b1, &q1);
            orc_footprint(p2, W, G, edge_mode, &a2, &b2, &q2);
            int slab;
            double s;
            orc_slab(r[k * 3 + 2], nslab, r3_min, slab_width, inv_half, &slab, &s);
            cheb[0] = 1.0;
            if (K > 1) cheb[1] = s;
            for (int t = 2; t < K; ++t) cheb[t] = 2.0 * s * cheb[t - 1] - cheb[t - 2];
            for (long g = a1; g <= b1; ++g) w1[g - a1] = orc_es(beta, ((double)g - q1) * half_w_inv);
            for (long g = a2; g <= b2; ++g) w2[g - a2] = orc_es(beta, ((double)g - q2) * half_w_inv);
            const double vre = (double)vr[k] * inv_det, vim = (double)vi[k] * inv_det;
            for (long g1 = a1; g1 <= b1; ++g1) {
                if (((g1 - gmin) / ORC_BAND) % nt != tid) continue;
                for (long g2 = a2; g2 <= b2; ++g2) {
                    double kv = w1[g1 - a1] * w2[g2 - a2];
                    if ((g1 + g2) & 1) kv = -kv;
                    const long cell = (g1 + G / 2) * G + (g2 + G / 2);
                    for (int t = 0; t < K; ++t) {
                        double* c = planes + 2 * (((long)slab * K + t) * GG + cell);
                        const double wgt = cheb[t] * kv;
                        c[0] += vre * wgt;
                        c[1] += vim * wgt;
                    }
                }
            }
        }
    }
    free(row0);
}

/* ------------------------------------------------------------------------------------------ */
/* Bessel J_n(x), n = 0..nmax, FP64, Miller's downward recurrence normalised with             */
/* J0 + 2 sum J_2k = 1.  Replaces bessel_sequence (SII:901-920).                               */
/* ------------------------------------------------------------------------------------------ */
void orc_bessel_j(double x, int nmax, double* j) {
    const double ax = fabs(x);
    if (ax < 1e-300) {
        j[0] = 1.0;
        for (int n = 1; n <= nmax; ++n) j[n] = 0.0;
        return;
    }
    int start = (nmax > (int)ax ? nmax : (int)ax) + 40 + (int)sqrt(40.0 * (ax + nmax));
    start += start & 1;
    double jn1 = 0.0, jn = 1e-30, norm = 0.0;
    for (int n = start; n >= 1; --n) {
        if (n <= nmax) j[n] = jn;
        if ((n & 1) == 0) norm += 2.0 * jn;
        const double jm1 = (2.0 * n / ax) * jn - jn1;
        jn1 = jn;
        jn = jm1;
        if (fabs(jn) > 1e200) {
            jn *= 1e-200; jn1 *= 1e-200; norm *= 1e-200;
            for (int m = n; m <= nmax; ++m) j[m] *= 1e-200;
        }
    }
    j[0] = jn;
    norm += jn;
    for (int n = 0; n <= nmax; ++n) {
        double v = j[n] / norm;
        if (x < 0 && (n & 1)) v = -v;
        j[n] = v;
    }
}

/* The reference's FP32 power series (SII:901-920, FIPK:184-205), restated for error studies. */
void orc_bessel_series_f32(float alpha, int max_order, float* jvals) {
    const float half_alpha = 0.5f * alpha;
    const float quarter_alpha_sq = half_alpha * half_alpha;
    for (int n = 0; n <= max_order; ++n) {
        float term = 1.0f;
        for (int m = 1; m <= n; ++m) term *= half_alpha / (float)m;
        float sum = term;
        for (int k = 1; k < 32; ++k) {
            term *= -quarter_alpha_sq / ((float)k * (float)(n + k));
            sum += term;
            if (fabsf(term) < 1.0e-7f * (1.0f + fabsf(sum))) break;
        }
        jvals[n] = sum;
    }
}

/* t3 of rotated-frame pixel (x, y) (SII:1381-1391, SII:1045-1059). Returns 0 when invalid.   */
static int orc_t3(const double* vin, long N, double cell, long x, long y, double* t1o, double* t2o,
                  double* t3o) {
    const long half = N / 2;
    const double t1 = cell * (double)(y - half), t2 = cell * (double)(x - half);
    const double v13 = vin[2], v23 = vin[5], v33 = vin[8];
    const double ra = 1.0 - (t1 + v13) * (t1 + v13) - (t2 + v23) * (t2 + v23);
    if (ra < 0.0) return 0;
    *t1o = t1;
    *t2o = t2;
    *t3o = -v33 + (v33 >= 0.0 ? 1.0 : -1.0) * sqrt(ra);
    return 1;
}

/* ------------------------------------------------------------------------------------------ */
/* Moment recombination + grid correction, pre-splat image R[y][x] (FP64).                    */
/* SII:1392-1445 (fused_interpolation up to fabs); FIPK:463-549 (accumulation + scaling).      */
/* moments: complex128 [nslab*K][G][G] AFTER the unnormalised inverse FFT.                     */
/* phi: ES transform per |pixel offset| (orc_es_correction). Invalid pixels -> NaN.            */
/* Image rows [y0, y1) only (the whole image: 0, N).                                           */
/* R = |Re sum_j sum_n c_jn M_jn| / (Phi(|x|) Phi(|y|)) / n_total.                             */
/* ------------------------------------------------------------------------------------------ */
void orc_recombine(const double* moments, long G, long N, double cell, const double* vin, int K,
                   int nslab, double r3_min, double slab_width, double slab_half, const double* phi,
                   double n_total, long y0, long y1, double* R) {
    const long GG = G * G;
#pragma omp parallel for schedule(static)
    for (long y = y0; y < y1; ++y) {
        double jv[64];
        for (long x = 0; x < N; ++x) {
            double t1, t2, t3;
            if (!orc_t3(vin, N, cell, x, y, &t1, &t2, &t3)) {
                R[y * N + x] = NAN;
                continue;
            }
            const long xr = x - N / 2, yr = y - N / 2;
            const double alpha = 2.0 * ORC_PI * t3 * slab_half;
            orc_bessel_j(alpha, K - 1, jv);
            const long gidx = GG / 2 + G / 2 + yr * G + xr; /* SII:1397 */
            double sum = 0.0;
            for (int j = 0; j < nslab; ++j) {
                const double centre = r3_min + ((double)j + 0.5) * slab_width;
                const double b = 2.0 * ORC_PI * t3 * centre;
                const double cb = cos(b), sb = sin(b);
                for (int n = 0; n < K; ++n) {
                    const double* m = moments + 2 * (((long)j * K + n) * GG + gidx);
                    const double amp = (n == 0) ? jv[0] : 2.0 * jv[n];
                    double cr, ci; /* amp * i^n * exp(i b) */
                    switch (n & 3) {
                        case 0: cr = amp * cb; ci = amp * sb; break;
                        case 1: cr = -amp * sb; ci = amp * cb; break;
                        case 2: cr = -amp * cb; ci = -amp * sb; break;
                        default: cr = amp * sb; ci = -amp * cb; break;
                    }
                    sum += cr * m[0] - ci * m[1];
                }
            }
            if ((xr + yr) & 1) sum = -sum;
            const long ax = xr < 0 ? -xr : xr, ay = yr < 0 ? -yr : yr;
            R[y * N + x] = fabs(sum / (phi[ax] * phi[ay])) / n_total;
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* FP64 direct DFT of the same pre-splat image at a list of pixels:                            */
/* R(x,y) = |Re sum_k (V_k / det) exp(+2 pi i r_k . t)| / n_total, t from orc_t3.              */
/* include (optional) selects the samples the imager grids (its footprint inclusion mask).    */
/* Direct sincos per sample; OpenMP over pixels.                                               */
/* ------------------------------------------------------------------------------------------ */
void orc_dft_pixels(long n, const double* r, const float* vr, const float* vi, const uint8_t* include,
                    double inv_det, double n_total, const double* vin, long N, double cell, long npix,
                    const int64_t* px, const int64_t* py, double* out) {
#pragma omp parallel for schedule(dynamic, 1)
    for (long p = 0; p < npix; ++p) {
        double t1, t2, t3;
        if (!orc_t3(vin, N, cell, px[p], py[p], &t1, &t2, &t3)) {
            out[p] = NAN;
            continue;
        }
        double acc = 0.0;
        for (long k = 0; k < n; ++k) {
            if (include && !include[k]) continue;
            const double ph = 2.0 * ORC_PI * (r[k * 3 + 0] * t1 + r[k * 3 + 1] * t2 + r[k * 3 + 2] * t3);
            acc += (double)vr[k] * cos(ph) - (double)vi[k] * sin(ph);
        }
        out[p] = fabs(acc * inv_det) / n_total;
    }
}

/* Same DFT for separable coordinates r_k = s_chan q_row (k = row + chan*nrows): per (row,     */
/* pixel) one sincos of the base phase, then a channel recurrence on a uniform frequency grid  */
/* s_lin(c) = s0 + c ds, corrected per channel by exp(i (s_c - s_lin(c)) phi) evaluated with a */
/* 6-term Taylor series (|arg| < 1e-2 is asserted by the caller's frequency table).            */
void orc_dft_pixels_sep(long nrows, long nch, const double* q, const double* s, const float* vr,
                        const float* vi, const uint8_t* include, double inv_det, double n_total,
                        const double* vin, long N, double cell, long npix, const int64_t* px,
                        const int64_t* py, double* out) {
    const double s0 = s[0];
    const double ds = nch > 1 ? (s[nch - 1] - s[0]) / (double)(nch - 1) : 0.0;
#pragma omp parallel for schedule(dynamic, 1)
    for (long p = 0; p < npix; ++p) {
        double t1, t2, t3;
        if (!orc_t3(vin, N, cell, px[p], py[p], &t1, &t2, &t3)) {
            out[p] = NAN;
            continue;
        }
        double acc = 0.0;
        for (long row = 0; row < nrows; ++row) {
            const double phi = 2.0 * ORC_PI * (q[row * 3 + 0] * t1 + q[row * 3 + 1] * t2 + q[row * 3 + 2] * t3);
            double zr = cos(s0 * phi), zi = sin(s0 * phi);
            const double stepr = cos(ds * phi), stepi = sin(ds * phi);
            for (long c = 0; c < nch; ++c) {
                const long k = row + c * nrows;
                if (!include || include[k]) {
                    const double e = (s[c] - (s0 + (double)c * ds)) * phi;
                    const double e2 = e * e;
                    const double cr = 1.0 - e2 * (0.5 - e2 * (1.0 / 24.0 - e2 / 720.0));
                    const double ci = e * (1.0 - e2 * (1.0 / 6.0 - e2 / 120.0));
                    const double pr = zr * cr - zi * ci, pi = zr * ci + zi * cr;
                    acc += (double)vr[k] * pr - (double)vi[k] * pi;
                }
                const double nr = zr * stepr - zi * stepi;
                zi = zr * stepi + zi * stepr;
                zr = nr;
            }
        }
        out[p] = fabs(acc * inv_det) / n_total;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Reprojection of the rotated-frame image to the output sky grid, bilinear splat.             */
/* Main path: SII:1325-1379 (simplified SIN deprojection, keeps p1,p2 when h > r0) and the     */
/* splat SII:1447-1461. Archive: FIPK:552-677 (coordschange, full-trig p2p that drops r2 > 1,  */
/* finalinterp). Geometry in FP64 here; the reference uses FP32.                               */
/* R is the pre-splat image (NaN = skipped pixel). out must be zeroed by the caller.           */
/* ------------------------------------------------------------------------------------------ */
static void orc_splat4(double* out, long N, double LL, double MM, double value) {
    const long half = N / 2;
    if (!(fabs(LL) < (double)(half - 1) && fabs(MM) < (double)(half - 1))) return;
    const double Lf = floor(LL), Mf = floor(MM), Lc = ceil(LL), Mc = ceil(MM);
    double* d = out + half * N + half;
    d[(long)Mf * N + (long)Lf] += (1 - LL + Lf) * (1 - MM + Mf) * value;
    d[(long)Mc * N + (long)Lf] += (1 - LL + Lf) * (0 + MM - Mf) * value;
    d[(long)Mf * N + (long)Lc] += (0 + LL - Lf) * (1 - MM + Mf) * value;
    d[(long)Mc * N + (long)Lc] += (0 + LL - Lf) * (0 + MM - Mf) * value;
}

/* Pixel rows [y0, y1) of R only (the whole image: 0, N).                                      */
void orc_reproject_sii(const double* R, long N, double cell, const double* vin, long y0, long y1,
                       double* out) {
    const double r0 = 180.0 / ORC_PI;
    const double dc = cell / ORC_PI * 180.0;
    const double di2 = (double)N * 0.5;
    const long half = N / 2;
    const double xi = vin[6] / vin[8], eta = vin[7] / vin[8];
    for (long idy = y0; idy < y1; ++idy)
        for (long idx = 0; idx < N; ++idx) {
            const double v = R[idy * N + idx];
            double t1, t2, t3; /* invalid pixels (no t3) are skipped; NaN values are splatted */
            if (!orc_t3(vin, N, cell, idx, idy, &t1, &t2, &t3)) continue;
            const double idxf = (double)idx - di2, idyf = (double)idy - di2;
            const double p1 = (-vin[0] * idxf + vin[3] * idyf) / fabs(vin[8]) + di2;
            const double p2 = (-vin[1] * idxf + vin[4] * idyf) / fabs(vin[8]) + di2;
            double x = -dc * (p1 - (di2 + 1.0));
            double y = dc * (p2 - (di2 + 1.0));
            const double h = hypot(x, y), hr0 = h / r0;
            if (h != 0.0) { x /= h; y /= -h; } else { x = 0.0; y = 1.0; }
            double oi0, oi1;
            if (h <= r0) {
                const double r = h;
                double z;
                if (h < r0 * sqrt(0.5)) z = 1.0 - sqrt(1.0 - hr0 * hr0);
                else z = hr0 * hr0 / (1.0 + sqrt(1.0 - hr0 * hr0));
                const double w = xi * xi + eta * eta;
                if (w == 0.0) { x = r * x; y = -r * y; }
                else { x = r * x + z * r0 * xi; y = -r * y + z * r0 * eta; }
                oi0 = -x / dc + di2 + 1.0;
                oi1 = y / dc + di2 + 1.0;
            } else {
                oi0 = p1;
                oi1 = p2;
            }
            orc_splat4(out, N, oi0 - (double)half, oi1 - (double)half, v);
        }
}

/* Archive path FIPK:552-677: coordschange (integer half size), p2p (Calabretta & Greisen SIN */
/* with trig; pixels with r^2 > 1 are dropped), finalinterp.                                  */
void orc_reproject_fipk(const double* R, long N, double cell, const double* vin, long y0, long y1,
                        double* out) {
    const long half = N / 2;
    const double dc = cell / ORC_PI * 180.0;
    const double r0 = 180.0 / ORC_PI;
    const double xi = vin[6] / vin[8], eta = vin[7] / vin[8];
    for (long idx = 0; idx < N; ++idx)
        for (long idy = y0; idy < y1; ++idy) {
            const double v = R[idy * N + idx];
            double t1, t2, t3; /* invalid pixels (no t3) are skipped; NaN values are splatted */
            if (!orc_t3(vin, N, cell, idx, idy, &t1, &t2, &t3)) continue;
            const double p1 = (-vin[0] * ((double)idx - (double)half) + vin[3] * ((double)idy - (double)half)) / fabs(vin[8]) + (double)half;
            const double p2 = (-vin[1] * ((double)idx - (double)half) + vin[4] * ((double)idy - (double)half)) / fabs(vin[8]) + (double)half;
            double x = -dc * (p1 - ((double)N / 2.0 + 1.0));
            double y = dc * (p2 - ((double)N / 2.0 + 1.0));
            const double x0 = x / r0, y0 = y / r0, r2 = x0 * x0 + y0 * y0;
            const double phi = (r2 != 0.0) ? atan2(x0, -y0) : 0.0; /* radians */
            double theta; /* radians */
            if (r2 < 0.5) theta = acos(sqrt(r2));
            else if (r2 <= 1.0) theta = asin(sqrt(1.0 - r2));
            else continue;
            const double sx = sin(phi), cy = cos(phi);
            const double t = ORC_PI / 2.0 - fabs(theta);
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
            if (w == 0.0) { x = r * sx; y = -r * cy; }
            else { z *= r0; x = r * sx + xi * z; y = -r * cy + eta * z; }
            const double oi0 = -1.0 / dc * x + (double)N / 2.0 + 1.0;
            const double oi1 = 1.0 / dc * y + (double)N / 2.0 + 1.0;
            orc_splat4(out, N, oi0 - (double)half, oi1 - (double)half, v);
        }
}

/* max |t3| and valid-pixel count over the image (SII:1029-1077, FIPK:333-348). FP64.        */
void orc_t3_stats(const double* vin, long N, double cell, double* max_abs_t3, long* valid) {
    double m = 0.0;
    long cnt = 0;
    for (long y = 0; y < N; ++y)
        for (long x = 0; x < N; ++x) {
            double t1, t2, t3;
            if (!orc_t3(vin, N, cell, x, y, &t1, &t2, &t3)) continue;
            if (fabs(t3) > m) m = fabs(t3);
            ++cnt;
        }
    *max_abs_t3 = m;
    *valid = cnt;
}

/* Sampled truncation error of the Jacobi-Anger series exp(i a s) ~ J0 + 2 sum_{n<K} i^n Jn Tn */
/* max over a in {amax*i/(na-1)} and s in {-1 + 2 j/(ns-1)} of |exact - approx|, for every     */
/* K = 1..kmax at once (err[K-1]). FIPK:287-318 (na=513, ns=2048, FP64) and SII:1112-1202     */
/* (na=257, ns=1024) evaluate the same quantity.                                               */
void orc_cheb_errors(double amax, int na, int ns, int kmax, double* err) {
    for (int K = 0; K < kmax; ++K) err[K] = 0.0;
#pragma omp parallel
    {
        double local[64] = {0};
        double jv[64];
#pragma omp for schedule(static)
        for (int ia = 0; ia < na; ++ia) {
            const double a = na == 1 ? amax : amax * (double)ia / (double)(na - 1);
            orc_bessel_j(a, kmax - 1, jv);
            for (int is = 0; is < ns; ++is) {
                const double s = -1.0 + 2.0 * (double)is / (double)(ns - 1);
                const double er = cos(a * s), ei = sin(a * s);
                double ar = 0.0, ai = 0.0, tm2 = 1.0, tm1 = s;
                for (int n = 0; n < kmax; ++n) {
                    double tn = n == 0 ? 1.0 : (n == 1 ? s : 2.0 * s * tm1 - tm2);
                    if (n >= 2) { tm2 = tm1; tm1 = tn; }
                    if (n == 0) ar += jv[0] * tn;
                    else {
                        const double amp = 2.0 * jv[n] * tn;
                        switch (n & 3) {
                            case 0: ar += amp; break;
                            case 1: ai += amp; break;
                            case 2: ar -= amp; break;
                            default: ai -= amp; break;
                        }
                    }
                    const double e = hypot(er - ar, ei - ai);
                    if (e > local[n]) local[n] = e;
                }
            }
        }
#pragma omp critical
        for (int K = 0; K < kmax; ++K) if (local[K] > err[K]) err[K] = local[K];
    }
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
