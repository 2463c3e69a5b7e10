// Internal declarations shared by the svdimager_b200 CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/svdimager_b200.h"

namespace svdi {

constexpr double kCLight = 299792458.0;  // SVDIntegratedImager.cu:382
constexpr double kPi = 3.14159265358979323846;
constexpr int kMaxTerms = 64;            // Chebyshev terms the kernels support
constexpr int kMaxSupport = 16;          // ES support the kernels support
constexpr int kPolyDeg = 8;              // degree of the piecewise ES polynomials (FP32 error
                                         // within 3e-8 of degree 11 for W = 6..12)
constexpr int kQuantBits = 24;           // grid positions are quantised to 2^-24 cells

// Record of one binned sample (16 bytes). xq/yq: quantised position relative to the tile origin,
// (cell offset << 24) | frac24; vre/vim: visibility / |det(Vin[0:2,0:2])| as float bits.
struct __align__(16) SampleRec {
    int xq, yq;
    float vre, vim;
};

// Device-resident scalar statistics (double slots, one D2H copy per snapshot).
enum StatSlot {
    ST_R3_MIN = 0, ST_R3_MAX, ST_MAX_T3, ST_VALID_PIX, ST_S_MIN, ST_S_MAX, ST_NUM_GRIDDED,
    ST_NUM_DROPPED, ST_EIG0, ST_EIG1, ST_EIG2, ST_COUNT = 16
};

// Geometry of one imaging call (passed by value to kernels).
struct GridGeom {
    long long G;          // grid side
    long long gmin, gmax; // first/last cell index relative to the centre: -G/2 .. (G-1)/2
    int W;                // ES support (even)
    int T;                // tile rows (first grid axis)
    int ntile;            // ceil(G / T)
    int T2;               // tile columns (second grid axis)
    int ntile2;           // tiles along the second axis (>= ceil(G / T2))
    int edge_mode;
    int coord_mode;
    double scale;         // cell_size * G  (grid position = r * scale)
    float scale32;        // float(cell_size * G) of the reference (coord_mode 1)
};

struct SlabParams {
    int nslab;
    int K;
    double r3_min;
    double slab_width;
    double inv_half;      // 1 / slab half width
    double slab_half;
};

// Continuous slab parameters of nslab slabs over the w range [r3min, r3max] (SVDIntegratedImager.cu:
// 973-991; the archive path's single centred slab, archive/FIPkernels.cu:327-366). One definition
// for the host decision and the device plan, so that both give the same bits.
__host__ __device__ inline void slab_params_for(bool archive, int nslab, int K, double r3min, double r3max,
                                                SlabParams& sp) {
    const double half_range = fmax(0.5 * (r3max - r3min), 1.0e-6);
    sp.nslab = nslab;
    sp.K = K;
    if (archive) {
        const double centre = 0.5 * (r3max + r3min);
        sp.r3_min = centre - half_range;
        sp.slab_width = 2.0 * half_range;
        sp.slab_half = half_range;
        sp.inv_half = 1.0 / half_range;
    } else {
        const double r3_range = fmax(r3max - r3min, 2.0e-6);
        sp.r3_min = r3min;
        sp.slab_width = r3_range / nslab;
        sp.slab_half = fmax(0.5 * sp.slab_width, 1.0e-6);
        sp.inv_half = 1.0 / sp.slab_half;
    }
}

// |V00 V11 - V01 V10| of the row-major basis, rounded once per operation on host and device.
__host__ __device__ inline double basis_det(const double* V) {
#ifdef __CUDA_ARCH__
    return fabs(__dsub_rn(__dmul_rn(V[0], V[4]), __dmul_rn(V[1], V[3])));
#else
    const volatile double a = V[0] * V[4], b = V[1] * V[3];
    return fabs(a - b);
#endif
}

// The slab parameters and 1 / |det| of one snapshot computed on the device from its statistics,
// for kernels launched before the host has read the statistics back.
struct DevPlan {
    SlabParams sp;
    float inv_det;
};

// ES kernel as W polynomial pieces in the fractional position: piece i evaluates
// psi((i - (W/2 - 1) - f) / (W/2)) for f in [0, 1).
struct EsPoly {
    float c[kMaxSupport][kPolyDeg + 1];
    float edge;           // psi(+-1) = exp(-beta), weight of the extra cell when frac == 0
    float beta;           // ES beta (exact evaluation on the rare path)
    int W;
};

// ---- launch accounting -------------------------------------------------------------------
void note_launch(int n = 1);

// ---- status helpers ------------------------------------------------------------------------
void set_error(const std::string& msg);

// Raises kernel `func`'s dynamic shared-memory limit on the current device to at least `bytes`
// (and, with carveout_max, asks for the largest shared-memory carveout), once per kernel and
// device. Thread-safe: engines image from several host threads, and the limit only ever grows, so
// a launch that needed less stays valid while another thread raises it. Returns an SVDI status.
int ensure_dynamic_smem(const void* func, size_t bytes, bool carveout_max = false);

// Streaming-multiprocessor count of the current device, queried once per device (148 on a
// B200; launch caps are multiples of it). Thread-safe.
int current_sm_count();

#define SVDI_CUDA(call)                                                                       \
    do {                                                                                      \
        cudaError_t e__ = (call);                                                             \
        if (e__ != cudaSuccess) {                                                             \
            ::svdi::set_error(std::string("CUDA error ") + cudaGetErrorString(e__) + " at " + \
                              __FILE__ + ":" + std::to_string(__LINE__));                     \
            return SVDI_ERR_CUDA;                                                             \
        }                                                                                     \
    } while (0)

#define SVDI_LAUNCHED()                                                                       \
    do {                                                                                      \
        ::svdi::note_launch();                                                                \
        cudaError_t e__ = cudaGetLastError();                                                 \
        if (e__ != cudaSuccess) {                                                             \
            ::svdi::set_error(std::string("kernel launch failed: ") + cudaGetErrorString(e__) \
                              + " at " + __FILE__ + ":" + std::to_string(__LINE__));          \
            return SVDI_ERR_CUDA;                                                             \
        }                                                                                     \
    } while (0)

#define SVDI_TRY(call)                  \
    do {                                \
        int s__ = (call);               \
        if (s__ != SVDI_OK) return s__; \
    } while (0)

// ---- kernel launchers (stream-ordered, no synchronisation) ---------------------------------
// preprocess.cu
int launch_preprocess(const float* d_uvw, const float* d_freq, long long R, long long C,
                      float array_center_x, double* d_partial, int partial_cap, double* d_vin64,
                      float* d_vin32, double* d_q, double* d_s, double* d_stats, cudaStream_t st);
int launch_collapse(const float* v0r, const float* v0i, const float* v3r, const float* v3i,
                    const uint8_t* f0, const uint8_t* f3, const float* w0, const float* w3,
                    float* outr, float* outi, long long n, cudaStream_t st);
int launch_expand_bin(const double* d_q, const double* d_s, long long R, long long C, float* d_bin,
                      cudaStream_t st);
int launch_bin_stats(const float* d_bin, long long n, double* d_partial, int partial_cap,
                     double* d_stats, cudaStream_t st);
int launch_vin_from_float(const float* d_vin32, double* d_vin64, cudaStream_t st);
int launch_t3_stats(const double* d_vin64, long long N, double cell, double* d_partial,
                    int partial_cap, double* d_stats, cudaStream_t st);
int launch_cheb_errors(double amax, int na, int ns, int kmax, unsigned long long* d_err,
                       cudaStream_t st);
// The device plan for nslab slabs and K terms from the statistics (ST_R3_MIN, ST_R3_MAX) and Vin.
int launch_plan(const double* d_stats, const double* d_vin64, bool archive, int nslab, int K,
                DevPlan* d_plan, cudaStream_t st);

// binning.cu
struct SampleSource {
    // separable (main path): r = s[chan] * q[row], idx = row + chan * R
    const double* q;
    const double* s;
    long long R;
    // explicit (archive path): r = bin[idx]
    const float* bin;
    // collapsed visibilities
    const float* vr;
    const float* vi;
    long long n;
    float inv_det;
    // optional: the scatter adds the number of records it writes whose value is NaN or +-Inf
    unsigned long long* nonfinite;
};
// d_plan (optional): slab parameters and 1 / |det| read on the device instead of sp and src.inv_det
int launch_histogram(const SampleSource& src, const GridGeom& g, const SlabParams& sp,
                     unsigned int* d_counts, int n_keys, unsigned long long* d_dropped,
                     cudaStream_t st, const DevPlan* d_plan = nullptr);
// d_kb_offsets (optional): exclusive scan of ceil(count / kb_size) per key, n_keys + 1 entries.
// d_chunk_key (optional): for every chunk c of chunk_size records, the last key whose records
// start at or before c * chunk_size (ceil(total / chunk_size) entries, total = offsets[n_keys]).
int launch_scan(const unsigned int* d_counts, int n_keys, unsigned int* d_offsets,
                unsigned int* d_cursor, cudaStream_t st, unsigned int* d_kb_offsets = nullptr,
                int kb_size = 32, unsigned int* d_chunk_key = nullptr, int chunk_size = 512);
// d_vmax (optional, zeroed by the caller): receives max(|vre|, |vim|) over the records as float bits
// d_keymax (optional, n_keys entries zeroed by the caller): the same maximum per key
int launch_scatter(const SampleSource& src, const GridGeom& g, const SlabParams& sp,
                   unsigned int* d_cursor, int n_keys, SampleRec* d_rec, float* d_rec_s,
                   unsigned int* d_vmax, cudaStream_t st, unsigned int* d_keymax = nullptr,
                   const DevPlan* d_plan = nullptr);

// gridder_tc.cu: split-precision tcgen05 gridder (one moment plane, support <= 8)
constexpr int kTcTileRows = 56;    // tile rows: footprint origins; 64-row accumulator with halo
constexpr int kTcTileCols = 8;     // tile columns: footprint origins of one column block
constexpr int kTcBlocks = 4;       // column blocks per super-tile accumulator (4 x 32 TMEM columns)
// accuracy.cu: FP64 direct DFT at pixels (px, py) of the samples the gridder keeps; d_acc (npix,
// zeroed by the caller) receives the signed sums before |.| / |det| / N_s
int launch_dft_probe(const SampleSource& src, const GridGeom& g, const SlabParams& sp, const double* d_vin,
                     long long N, double cell, const long long* d_px, const long long* d_py, int npix,
                     double* d_acc, int sm_count, cudaStream_t st);

// fft_cols.cu: the pruned inverse FFT's column transforms in shared memory (G = 2^a 3^b, b <= 1,
// 16 <= G <= 12288): pass radices, log2 of each pass's stride, twiddle-table steps, log2 of the
// columns per CTA
struct ColFftPlan {
    int npass = 0;
    int lcb = 0;
    int rad[6] = {};
    int s_log[6] = {};
    int tw_step[6] = {};
};
bool col_fft_supported(long long G);
// allocates the twiddle and output-permutation tables (cudaFree both)
int make_col_fft(long long G, ColFftPlan& P, float2** d_tw, int** d_perm);
// columns [c0, c0 + ncols) of each of nplanes G x G planes, in place
int launch_col_fft(float2* d_planes, int nplanes, long long G, long long c0, long long ncols, const ColFftPlan& P,
                   const float2* d_tw, const int* d_perm, cudaStream_t st);

// host_stage.cu: copies between pageable host memory and the device through a pinned staging
// ring that a pool of host threads fills and drains. A pageable cudaMemcpyAsync stages through the
// driver's buffer with one host thread and so runs at about one core's memcpy speed; here several
// threads copy slices of one slot while the copy engine moves the previous slot, so the host side
// keeps up with the PCIe link. Pinned, registered or managed memory and copies below a few MB take
// the plain cudaMemcpyAsync. The ring (three 16 MB slots) and the threads start on the first
// staged copy; if its pinned memory cannot be had, every copy takes the plain path. Not
// thread-safe: one stager serves one engine, whose calls are serialised.
class HostStager {
public:
    HostStager() = default;
    HostStager(const HostStager&) = delete;
    HostStager& operator=(const HostStager&) = delete;
    ~HostStager();
    // true for host memory that CUDA neither allocated nor registered
    static bool pageable(const void* host);
    // Stream-ordered upload. Returns once `host` has been read (the caller may reuse it), like a
    // pageable cudaMemcpyAsync; the device copy completes in stream order on `st`.
    int h2d(void* dev, const void* host, size_t bytes, cudaStream_t st);
    // Download after the work queued on `st`; returns once `host` holds the bytes.
    int d2h(void* host, const void* dev, size_t bytes, cudaStream_t st);
    int threads() const;

private:
    struct Impl;
    Impl* impl_ = nullptr;
    bool unavailable_ = false;  // the ring could not be set up: plain copies from then on
    int init();
    bool staged(const void* host, size_t bytes);
};

constexpr int kTcKBlock = 32;      // records per K-block (one MMA pair of K steps)
// gridder_i8.cu: exact integer tcgen05 gridder (support <= 8; one launch per Chebyshev term)
constexpr int kI8TileRows = 24;    // tile rows: footprint origins; 32-row accumulator window with halo
constexpr int kI8TileCols = 8;     // tile columns: footprint origins; 16-column window with halo
// d_keymax: the scatter's per-key max |value| (float bits); d_rec_s: the records' Chebyshev
// arguments (K > 1); moment plane (slab - slab_lo) * K + n receives term n
int launch_grid_i8(const SampleRec* d_rec, const float* d_rec_s, const unsigned int* d_offsets,
                   const unsigned int* d_kb_offsets, int n_keys, int key_lo, int key_hi, int slab_lo, int K,
                   const GridGeom& g, const EsPoly& poly, float2* d_planes, const unsigned int* d_keymax,
                   unsigned int* d_status, int sm_count, cudaStream_t st);
int launch_grid_tc(const SampleRec* d_rec, const unsigned int* d_offsets, const unsigned int* d_kb_offsets,
                   int n_keys, int key_lo, int key_hi, int slab_lo, const GridGeom& g, const EsPoly& poly,
                   float2* d_planes, const unsigned int* d_vmax, unsigned int* d_status, int sm_count,
                   cudaStream_t st, bool bf16 = false);

// gridder.cu
// d_chunk_key, d_keymax: the scan's chunk table (chunks of kGridChunk records) and the scatter's
// per-key max |value|
constexpr int kGridChunk = 1024;
// Fixed-point contributions of the FP32 gridder stay below 2^kGridScaleBits (exact rounding with
// one FMA needs < 2^22)
constexpr int kGridScaleBits = 22;
// d_work: one counter the launch resets and its CTAs take runs of chunks from
int launch_grid_fp32(const SampleRec* d_rec, const float* d_rec_s, const unsigned int* d_offsets,
                     const unsigned int* d_chunk_key, const unsigned int* d_keymax, unsigned int* d_work,
                     int n_keys, int key_lo, int key_hi, int slab_lo, const GridGeom& g,
                     const SlabParams& sp, const EsPoly& poly, float2* d_planes, int sm_count,
                     cudaStream_t st);
void build_es_poly(int W, double beta, EsPoly* out);

// image.cu
// d_acc (N x N doubles, zeroed before the first batch) when the slabs are split over several
// batches: every batch adds its signed sum, the final batch takes |.| and writes the image.
int launch_recombine(const float2* d_moments, const GridGeom& g, long long N, double cell,
                     const double* d_vin64, const SlabParams& sp, const float* d_corr,
                     double inv_n_total, int reprojection, int presplat, float* d_out,
                     cudaStream_t st, double* d_acc = nullptr, bool final_batch = true,
                     const DevPlan* d_plan = nullptr, const unsigned long long* d_nonfinite = nullptr);

}  // namespace svdi
