// Second pass of the pruned inverse 2-D FFT: the column transforms of the N columns the
// recombination reads, in shared memory, for grid sizes G = 2^a 3^b (b <= 1, 16 <= G <= 12288).
//
// cuFFT transforms a strided column batch of a large plane at a fraction of the bandwidth of its
// contiguous row transforms (6144-row columns: ~1.1 TB/s). Here a CTA takes CB adjacent columns
// whole (G x CB complex values, CB * 8-byte row segments, up to 192 KB of shared memory), runs an
// in-place mixed-radix decimation-in-frequency FFT over the rows -- one radix-3 pass first (when
// 3 | G), then radix-16 passes, then one radix-2/4/8 pass -- and writes each output row back from
// its digit-reversed position. Pass p with radix R and stride S (the product of the later radices,
// a power of two) takes the R elements b R S + j + S m (m < R) of a column, forms their inverse DFT
// (e^{+2 pi i m k / R}), multiplies element k by e^{+2 pi i j k / (R S)} and writes it back to
// b R S + j + S k. The twiddles come from a table of e^{+2 pi i t / G} (FP64-rounded), element k of
// pass p reading entry j k G / (R S) (< G); the output permutation is a table too (the output row
// of each block row, so the block is read back in order). The transform is the inverse,
// unnormalised one, as cuFFT's CUFFT_INVERSE.
//
// Shared-memory rows are swizzled: block row r sits at row r ^ (f(r >> 3) & mask), f(x) = x ^
// (x >> 2) ^ (x >> 4), mask = 16 / CB - 1 (the rows that share a 128-byte bank line). The last
// passes take rows R or 2 R apart in a warp, which without it fall on the same banks (a 6144-row
// block lost half its shared-memory wavefronts to conflicts).
#include "svdi_internal.cuh"

#include <cmath>
#include <vector>

namespace svdi {

namespace {


__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 c_i(float2 a) { return make_float2(-a.y, a.x); }    // i a

// inverse DFTs (e^{+2 pi i m k / R}) in place
__device__ __forceinline__ void dft2(float2& a, float2& b) {
    const float2 t = a;
    a = c_add(t, b);
    b = c_sub(t, b);
}

__device__ __forceinline__ void dft3(float2& a, float2& b, float2& c) {
    constexpr float kS = 0.866025403784438647f;  // sqrt(3) / 2
    const float2 t1 = c_add(b, c), t2 = c_sub(b, c);
    const float2 m = make_float2(fmaf(-0.5f, t1.x, a.x), fmaf(-0.5f, t1.y, a.y));
    const float2 r = make_float2(-kS * t2.y, kS * t2.x);  // i sqrt(3)/2 (b - c)
    a = c_add(a, t1);
    b = c_add(m, r);
    c = c_sub(m, r);
}

__device__ __forceinline__ void dft4(float2& a, float2& b, float2& c, float2& d) {
    const float2 s0 = c_add(a, c), d0 = c_sub(a, c), s1 = c_add(b, d), d1 = c_sub(b, d);
    a = c_add(s0, s1);
    c = c_sub(s0, s1);
    b = c_add(d0, c_i(d1));
    d = c_sub(d0, c_i(d1));
}

__device__ __forceinline__ void dft8(float2 (&v)[16]) {
    constexpr float kC = 0.707106781186547524f;
    dft4(v[0], v[2], v[4], v[6]);
    dft4(v[1], v[3], v[5], v[7]);
    // odd half times e^{+2 pi i k / 8}, k = 0..3
    const float2 o1 = make_float2(kC * (v[3].x - v[3].y), kC * (v[3].x + v[3].y));
    const float2 o2 = c_i(v[5]);
    const float2 o3 = make_float2(-kC * (v[7].x + v[7].y), kC * (v[7].x - v[7].y));
    const float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1];
    v[0] = c_add(e0, o0);
    v[4] = c_sub(e0, o0);
    v[1] = c_add(e1, o1);
    v[5] = c_sub(e1, o1);
    v[2] = c_add(e2, o2);
    v[6] = c_sub(e2, o2);
    v[3] = c_add(e3, o3);
    v[7] = c_sub(e3, o3);
}

__device__ __forceinline__ void dft16(float2 (&v)[16]) {
    // x[b + 4 a]: four radix-4 DFTs over a, twiddles e^{+2 pi i b k1 / 16}, four over b;
    // y[k1 + 4 k2] = sum_b e^{2 pi i b k2 / 4} e^{2 pi i b k1 / 16} Z_b[k1]
    constexpr float kC1 = 0.923879532511286756f, kS1 = 0.382683432365089772f, kC = 0.707106781186547524f;
#pragma unroll
    for (int b = 0; b < 4; ++b) dft4(v[b], v[b + 4], v[b + 8], v[b + 12]);
    // Z_b[k1] sits in v[b + 4 k1]
    v[5] = c_mul(v[5], make_float2(kC1, kS1));     // b 1, k1 1: e^{i pi / 8}
    v[9] = c_mul(v[9], make_float2(kC, kC));       // b 1, k1 2: e^{i pi / 4}
    v[13] = c_mul(v[13], make_float2(kS1, kC1));   // b 1, k1 3: e^{3 i pi / 8}
    v[6] = c_mul(v[6], make_float2(kC, kC));       // b 2, k1 1
    v[10] = c_i(v[10]);                            // b 2, k1 2: i
    v[14] = c_mul(v[14], make_float2(-kC, kC));    // b 2, k1 3: e^{3 i pi / 4}
    v[7] = c_mul(v[7], make_float2(kS1, kC1));     // b 3, k1 1: e^{3 i pi / 8}
    v[11] = c_mul(v[11], make_float2(-kC, kC));    // b 3, k1 2: e^{3 i pi / 4}
    v[15] = c_mul(v[15], make_float2(-kC1, -kS1)); // b 3, k1 3: e^{9 i pi / 8}
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    // y[k1 + 4 k2] now sits in v[4 k1 + k2]: transpose the 4 x 4 index
    float2 t;
    t = v[1]; v[1] = v[4]; v[4] = t;
    t = v[2]; v[2] = v[8]; v[8] = t;
    t = v[3]; v[3] = v[12]; v[12] = t;
    t = v[6]; v[6] = v[9]; v[9] = t;
    t = v[7]; v[7] = v[13]; v[13] = t;
    t = v[11]; v[11] = v[14]; v[14] = t;
}

template <int R>
__device__ __forceinline__ void dft_r(float2 (&v)[16]) {
    if constexpr (R == 2) dft2(v[0], v[1]);
    else if constexpr (R == 3) dft3(v[0], v[1], v[2]);
    else if constexpr (R == 4) dft4(v[0], v[1], v[2], v[3]);
    else if constexpr (R == 8) dft8(v);
    else dft16(v);
}

// asynchronous global -> shared copies of 8 or 16 bytes (the block's rows stay in flight together)
__device__ __forceinline__ void cp_async8(float2* dst, const float2* src) {
    const unsigned int d = (unsigned int)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(float2* dst, const float2* src) {
    const unsigned int d = (unsigned int)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

// the shared-memory row of block row r (file comment)
__device__ __forceinline__ int srow(int r, int mask) {
    const int x = r >> 3;
    return r ^ ((x ^ (x >> 2) ^ (x >> 4)) & mask);
}

// one pass of radix R over the CTA's G x CB block (see the file comment)
template <int R, int NT>
__device__ __forceinline__ void col_pass(float2* __restrict__ sh, int G, int lcb, int s_log, int tw_step,
                                         const float2* __restrict__ tw) {
    // a thread takes one butterfly of two adjacent columns: 16-byte shared-memory accesses and
    // the twiddles loaded once for both
    const int S = 1 << s_log, CP = 1 << (lcb - 1);
    const int nbf = (G / R) << (lcb - 1);
    const int mask = (16 >> lcb) - 1;
    for (int t = threadIdx.x; t < nbf; t += NT) {
        const int c = (t & (CP - 1)) * 2, q = t >> (lcb - 1);
        const int b = q >> s_log, j = q & (S - 1);
        const int base = b * R * S + j;
        float2 v[16], u[16];
#pragma unroll
        for (int m = 0; m < R; ++m) {
            const float4 w = *reinterpret_cast<const float4*>(sh + (srow(base + S * m, mask) << lcb) + c);
            v[m] = make_float2(w.x, w.y);
            u[m] = make_float2(w.z, w.w);
        }
        dft_r<R>(v);
        dft_r<R>(u);
        if (j) {
            const int st = j * tw_step;
            int ix = st;
#pragma unroll
            for (int k = 1; k < R; ++k, ix += st) {
                const float2 w = __ldg(&tw[ix]);
                v[k] = c_mul(v[k], w);
                u[k] = c_mul(u[k], w);
            }
        }
#pragma unroll
        for (int m = 0; m < R; ++m)
            *reinterpret_cast<float4*>(sh + (srow(base + S * m, mask) << lcb) + c) =
                make_float4(v[m].x, v[m].y, u[m].x, u[m].y);
    }
}

// NT threads; NT = 256: two CTAs per SM (blocks of up to 96 KB), NT = 512: one (up to 192 KB)
template <int NT>
__global__ void __launch_bounds__(NT, 512 / NT) k_fft_cols(float2* __restrict__ planes, int G, long long c0,
                                                             int ncols, ColFftPlan P,
                                                             const float2* __restrict__ tw,
                                                             const int* __restrict__ out_row) {
    extern __shared__ __align__(16) float2 sh[];
    const int lcb = P.lcb, CB = 1 << lcb;
    const int mask = (16 >> lcb) - 1;
    const int cb0 = blockIdx.x * CB;
    const int ncb = min(CB, ncols - cb0);
    float2* const pl = planes + (long long)blockIdx.y * G * G + c0 + cb0;
    const int n = G << lcb;
    // pairs of columns: 16-byte copies where the pair is whole and 16-byte aligned (c0 + cb0 even;
    // G even keeps every row aligned alike), else 8-byte copies; columns past the block's end are 0
    const bool al16 = ((c0 + cb0) & 1) == 0;
    for (int i = threadIdx.x; i < (n >> 1); i += NT) {
        const int r = i >> (lcb - 1), c = (i & ((CB >> 1) - 1)) * 2;
        const float2* src = pl + (long long)r * G + c;
        float2* dst = sh + (srow(r, mask) << lcb) + c;
        if (al16 && c + 1 < ncb) {
            cp_async16(dst, src);
        } else {
            if (c < ncb) cp_async8(dst, src);
            else dst[0] = make_float2(0.0f, 0.0f);
            if (c + 1 < ncb) cp_async8(dst + 1, src + 1);
            else dst[1] = make_float2(0.0f, 0.0f);
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    for (int p = 0; p < P.npass; ++p) {
        switch (P.rad[p]) {
            case 2: col_pass<2, NT>(sh, G, lcb, P.s_log[p], P.tw_step[p], tw); break;
            case 3: col_pass<3, NT>(sh, G, lcb, P.s_log[p], P.tw_step[p], tw); break;
            case 4: col_pass<4, NT>(sh, G, lcb, P.s_log[p], P.tw_step[p], tw); break;
            case 8: col_pass<8, NT>(sh, G, lcb, P.s_log[p], P.tw_step[p], tw); break;
            default: col_pass<16, NT>(sh, G, lcb, P.s_log[p], P.tw_step[p], tw); break;
        }
        __syncthreads();
    }
    // block row r to its output row (digit reversal), pairs of columns as on the way in
    for (int i = threadIdx.x; i < (n >> 1); i += NT) {
        const int r = i >> (lcb - 1), c = (i & ((CB >> 1) - 1)) * 2;
        const float2* src = sh + (srow(r, mask) << lcb) + c;
        float2* dst = pl + (long long)__ldg(&out_row[r]) * G + c;
        if (al16 && c + 1 < ncb) {
            *reinterpret_cast<float4*>(dst) = *reinterpret_cast<const float4*>(src);
        } else {
            if (c < ncb) dst[0] = src[0];
            if (c + 1 < ncb) dst[1] = src[1];
        }
    }
}

}  // namespace

// Where it is used: grid sizes at which it measured faster than cuFFT's strided column plan on
// B200 -- up to 1536 rows (two CTAs per SM; 1536: configuration B 49.5 -> 46.6 ms per 256
// snapshots) and from 4096 (6144: 0.38 -> 0.17 ms per plane). At 3072 rows cuFFT's column kernel
// stays ahead (0.091 against 0.093 ms for the precision snapshot's whole FFT).
bool col_fft_supported(long long G) {
    if (G < 16 || G > 12288 || (G > 1536 && G < 4096)) return false;
    long long r = G;
    while (r % 2 == 0) r /= 2;
    return r == 1 || r == 3;
}

int make_col_fft(long long G, ColFftPlan& P, float2** d_tw, int** d_perm) {
    if (!col_fft_supported(G)) {
        set_error("column FFT: unsupported grid size");
        return SVDI_ERR_UNSUPPORTED;
    }
    // radices: 3 first (when 3 | G), then 16s, then the remaining power of two
    std::vector<int> rad;
    long long g = G;
    int k2 = 0;
    while (g % 2 == 0) {
        g /= 2;
        ++k2;
    }
    if (g == 3) rad.push_back(3);
    while (k2 >= 4) {
        rad.push_back(16);
        k2 -= 4;
    }
    if (k2) rad.push_back(1 << k2);
    P = ColFftPlan{};
    P.npass = (int)rad.size();
    long long before = 1;  // product of the earlier radices = G / (R S)
    for (int p = 0; p < P.npass; ++p) {
        long long S = 1;
        for (int q = p + 1; q < P.npass; ++q) S *= rad[q];
        int sl = 0;
        while ((1LL << sl) < S) ++sl;
        P.rad[p] = rad[p];
        P.s_log[p] = sl;
        P.tw_step[p] = (int)before;
        before *= rad[p];
    }
    // columns per CTA: the largest power of two up to 16 with G * CB * 8 bytes <= 96 KB up to 1536
    // rows (two CTAs per SM), <= 192 KB beyond (one CTA per SM; 6144 rows x 4 columns: 32-byte row
    // segments, where pairs of columns at 96 KB measured slower)
    const long long cap = G <= 1536 ? 96 * 1024 : 192 * 1024;
    int lcb = 1;
    while (lcb < 4 && G * (2LL << lcb) * 8 <= cap) ++lcb;
    P.lcb = lcb;  // >= 1 for every supported G (the copies take pairs of columns)
    // tables: e^{+2 pi i t / G} and the digit-reversed position of each output row
    std::vector<float2> tw((size_t)G);
    for (long long t = 0; t < G; ++t) {
        const double a = 2.0 * 3.14159265358979323846 * (double)t / (double)G;
        tw[(size_t)t] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    std::vector<int> perm((size_t)G);
    for (long long nrow = 0; nrow < G; ++nrow) {
        long long t = nrow, pos = 0;
        for (int p = 0; p < P.npass; ++p) {
            const long long k = t % rad[p];
            t /= rad[p];
            pos += k << P.s_log[p];
        }
        perm[(size_t)pos] = (int)nrow;  // block row pos holds output row nrow
    }
    SVDI_CUDA(cudaMalloc(d_tw, (size_t)G * sizeof(float2)));
    SVDI_CUDA(cudaMalloc(d_perm, (size_t)G * sizeof(int)));
    SVDI_CUDA(cudaMemcpy(*d_tw, tw.data(), (size_t)G * sizeof(float2), cudaMemcpyHostToDevice));
    SVDI_CUDA(cudaMemcpy(*d_perm, perm.data(), (size_t)G * sizeof(int), cudaMemcpyHostToDevice));
    return SVDI_OK;
}

int launch_col_fft(float2* d_planes, int nplanes, long long G, long long c0, long long ncols, const ColFftPlan& P,
                   const float2* d_tw, const int* d_perm, cudaStream_t st) {
    const size_t smem = (size_t)G * ((size_t)1 << P.lcb) * sizeof(float2);
    const dim3 grid((unsigned)((ncols + (1LL << P.lcb) - 1) >> P.lcb), (unsigned)nplanes);
    if (smem <= 96 * 1024) {
        SVDI_TRY(ensure_dynamic_smem((const void*)k_fft_cols<256>, smem, true));
        k_fft_cols<256><<<grid, 256, smem, st>>>(d_planes, (int)G, c0, (int)ncols, P, d_tw, d_perm);
    } else {
        SVDI_TRY(ensure_dynamic_smem((const void*)k_fft_cols<512>, smem, true));
        k_fft_cols<512><<<grid, 512, smem, st>>>(d_planes, (int)G, c0, (int)ncols, P, d_tw, d_perm);
    }
    SVDI_LAUNCHED();
    return SVDI_OK;
}

}  // namespace svdi
