// Small numerical helpers shared by host and device code.
#pragma once

#include <cmath>

namespace svdi {

// Bessel functions J_0..J_nmax of the first kind, FP64.
// |x| < 1e-3: the ascending series (three terms reach double precision there);
// otherwise Miller's downward recurrence from an even start order well above max(nmax, |x|),
// normalised by J_0 + 2 sum_k J_2k = 1, with rescaling against overflow.
__host__ __device__ inline void bessel_jn(double x, int nmax, double* j) {
    const double ax = fabs(x);
    if (ax < 1e-300) {
        j[0] = 1.0;
        for (int n = 1; n <= nmax; ++n) j[n] = 0.0;
        return;
    }
    if (ax < 1e-3) {
        const double h = 0.5 * x, q = -h * h;
        double lead = 1.0;  // (x/2)^n / n!
        for (int n = 0; n <= nmax; ++n) {
            if (n > 0) lead *= h / n;
            const double t1 = q / (n + 1);
            const double t2 = t1 * q / (2.0 * (n + 2));
            j[n] = lead * (1.0 + t1 + t2);
        }
        return;
    }
    const int top = (nmax > (int)ax ? nmax : (int)ax);
    int start = top + 40 + (int)sqrt(40.0 * (ax + nmax));
    start += start & 1;
    double jn1 = 0.0, jn = 1e-30, norm = 0.0;
    for (int n = start; n >= 1; --n) {
        if (n <= nmax) j[n] = jn;
        if ((n & 1) == 0) norm += 2.0 * jn;
        const double jm1 = (2.0 * n / ax) * jn - jn1;
        jn1 = jn;
        jn = jm1;
        if (fabs(jn) > 1e200) {
            jn *= 1e-200;
            jn1 *= 1e-200;
            norm *= 1e-200;
            for (int m = n; m <= nmax; ++m) j[m] *= 1e-200;
        }
    }
    norm += jn;
    j[0] = jn;
    const double inv = 1.0 / norm;
    for (int n = 0; n <= nmax; ++n) {
        double v = j[n] * inv;
        if (x < 0 && (n & 1)) v = -v;
        j[n] = v;
    }
}

// The same functions for the per-pixel recombination, with the divisions of the series and of the
// recurrence replaced by multiplications with reciprocals (1/n from a table, 1/|x| once): FP64
// division is a long instruction sequence, and the recurrence divides once per step. The results
// differ from bessel_jn by rounding only (relative ~1e-16); host-side decisions keep bessel_jn.
__device__ __constant__ const double kRecipSmall[72] = {
    1.0 / 1,  1.0 / 2,  1.0 / 3,  1.0 / 4,  1.0 / 5,  1.0 / 6,  1.0 / 7,  1.0 / 8,  1.0 / 9,  1.0 / 10,
    1.0 / 11, 1.0 / 12, 1.0 / 13, 1.0 / 14, 1.0 / 15, 1.0 / 16, 1.0 / 17, 1.0 / 18, 1.0 / 19, 1.0 / 20,
    1.0 / 21, 1.0 / 22, 1.0 / 23, 1.0 / 24, 1.0 / 25, 1.0 / 26, 1.0 / 27, 1.0 / 28, 1.0 / 29, 1.0 / 30,
    1.0 / 31, 1.0 / 32, 1.0 / 33, 1.0 / 34, 1.0 / 35, 1.0 / 36, 1.0 / 37, 1.0 / 38, 1.0 / 39, 1.0 / 40,
    1.0 / 41, 1.0 / 42, 1.0 / 43, 1.0 / 44, 1.0 / 45, 1.0 / 46, 1.0 / 47, 1.0 / 48, 1.0 / 49, 1.0 / 50,
    1.0 / 51, 1.0 / 52, 1.0 / 53, 1.0 / 54, 1.0 / 55, 1.0 / 56, 1.0 / 57, 1.0 / 58, 1.0 / 59, 1.0 / 60,
    1.0 / 61, 1.0 / 62, 1.0 / 63, 1.0 / 64, 1.0 / 65, 1.0 / 66, 1.0 / 67, 1.0 / 68, 1.0 / 69, 1.0 / 70,
    1.0 / 71, 1.0 / 72};

// nmax <= 69.
__device__ inline void bessel_jn_fast(double x, int nmax, double* j) {
    const double ax = fabs(x);
    if (ax < 1e-300) {
        j[0] = 1.0;
        for (int n = 1; n <= nmax; ++n) j[n] = 0.0;
        return;
    }
    if (ax < 1e-3) {
        const double h = 0.5 * x, q = -h * h;
        double lead = 1.0;  // (x/2)^n / n!
        for (int n = 0; n <= nmax; ++n) {
            if (n > 0) lead *= h * kRecipSmall[n - 1];
            const double t1 = q * kRecipSmall[n];
            const double t2 = t1 * q * (0.5 * kRecipSmall[n + 1]);
            j[n] = lead * (1.0 + t1 + t2);
        }
        return;
    }
    const double inv_ax = 1.0 / ax;
    const int top = (nmax > (int)ax ? nmax : (int)ax);
    int start = top + 40 + (int)sqrt(40.0 * (ax + nmax));
    start += start & 1;
    double jn1 = 0.0, jn = 1e-30, norm = 0.0;
    for (int n = start; n >= 1; --n) {
        if (n <= nmax) j[n] = jn;
        if ((n & 1) == 0) norm += 2.0 * jn;
        const double jm1 = (2.0 * n * inv_ax) * jn - jn1;
        jn1 = jn;
        jn = jm1;
        if (fabs(jn) > 1e200) {
            jn *= 1e-200;
            jn1 *= 1e-200;
            norm *= 1e-200;
            for (int m = n; m <= nmax; ++m) j[m] *= 1e-200;
        }
    }
    norm += jn;
    j[0] = jn;
    const double inv = 1.0 / norm;
    for (int n = 0; n <= nmax; ++n) {
        double v = j[n] * inv;
        if (x < 0 && (n & 1)) v = -v;
        j[n] = v;
    }
}

// Cyclic Jacobi eigen-decomposition of a symmetric 3x3 matrix (row-major), FP64. Eigenvalues in
// ascending order; evec row j is the eigenvector of eval[j]. Replaces cusolverDnSsyevd
// (SVDIntegratedImager.cu:736-760), whose eigenvalues are ascending as well.
__host__ __device__ inline void jacobi3(const double* a_in, double* eval, double* evec) {
    double a[9];
    for (int i = 0; i < 9; ++i) a[i] = a_in[i];
    double v[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int sweep = 0; sweep < 64; ++sweep) {
        const double off = a[1] * a[1] + a[2] * a[2] + a[5] * a[5];
        const double diag = a[0] * a[0] + a[4] * a[4] + a[8] * a[8];
        if (off <= 1e-300 || off <= diag * 1e-34) break;
        for (int p = 0; p < 2; ++p) {
            for (int q = p + 1; q < 3; ++q) {
                const double apq = a[p * 3 + q];
                if (apq == 0.0) continue;
                const double app = a[p * 3 + p], aqq = a[q * 3 + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    const double akp = a[k * 3 + p], akq = a[k * 3 + q];
                    a[k * 3 + p] = c * akp - s * akq;
                    a[k * 3 + q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double apk = a[p * 3 + k], aqk = a[q * 3 + k];
                    a[p * 3 + k] = c * apk - s * aqk;
                    a[q * 3 + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    const double vkp = v[k * 3 + p], vkq = v[k * 3 + q];
                    v[k * 3 + p] = c * vkp - s * vkq;
                    v[k * 3 + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    int idx[3] = {0, 1, 2};
    const double d[3] = {a[0], a[4], a[8]};
    for (int i = 0; i < 3; ++i)
        for (int k = i + 1; k < 3; ++k)
            if (d[idx[k]] < d[idx[i]]) {
                const int t = idx[i];
                idx[i] = idx[k];
                idx[k] = t;
            }
    for (int jj = 0; jj < 3; ++jj) {
        eval[jj] = d[idx[jj]];
        for (int k = 0; k < 3; ++k) evec[jj * 3 + k] = v[k * 3 + idx[jj]];
    }
}

// Orientation of the PCA basis (SVDIntegratedImager.cu:538-586): rows in descending eigenvalue
// order; row 0 with non-negative u component; row 1 with a v component of the sign of
// ARRAY_CENTER.x (skipped when that is 0); row 2 = row0 x row1, normalised.
__host__ __device__ inline void orient_basis(const double* evec_asc, float array_center_x, double* vin) {
    for (int a = 0; a < 3; ++a) {
        vin[0 * 3 + a] = evec_asc[2 * 3 + a];
        vin[1 * 3 + a] = evec_asc[1 * 3 + a];
        vin[2 * 3 + a] = evec_asc[0 * 3 + a];
    }
    if (vin[0] < 0.0)
        for (int a = 0; a < 3; ++a) vin[a] = -vin[a];
    if (array_center_x != 0.0f && vin[4] * (double)array_center_x < 0.0)
        for (int a = 0; a < 3; ++a) vin[3 + a] = -vin[3 + a];
    double r20 = vin[1] * vin[5] - vin[2] * vin[4];
    double r21 = vin[2] * vin[3] - vin[0] * vin[5];
    double r22 = vin[0] * vin[4] - vin[1] * vin[3];
    const double nrm = sqrt(r20 * r20 + r21 * r21 + r22 * r22);
    if (nrm > 0.0) {
        r20 /= nrm;
        r21 /= nrm;
        r22 /= nrm;
    }
    vin[6] = r20;
    vin[7] = r21;
    vin[8] = r22;
}

}  // namespace svdi
