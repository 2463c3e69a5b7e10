// Imaging engine and the C ABI.
//
// Orchestration replaces FIpipeDevice (SVDIntegratedImager.cu:1498-1761) and FIpipe
// (archive/FIPkernels.cu:679-911). Differences by design:
//   - device buffers, cuFFT plans, grid-correction tables and ES polynomials are kept resident in
//     an engine and grown on demand (the reference allocates, plans and frees on every call);
//   - the Chebyshev/slab statistics need one small device-to-host read per snapshot (the
//     reference needs two, plus a serial single-thread reduction kernel);
//   - samples are binned by tile before gridding (binning.cu, gridder.cu).
#include "svdi_internal.cuh"
#include "math.cuh"

#include <cufft.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

namespace svdi {

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void set_error(const std::string& msg) { g_last_error = msg; }

int ensure_dynamic_smem(const void* func, size_t bytes, bool carveout_max) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> limit;  // (kernel, device) -> bytes set
    int dev = 0;
    SVDI_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    auto it = limit.find({func, dev});
    const bool first = it == limit.end();
    if (!first && it->second >= bytes) return SVDI_OK;
    // set explicitly even below 48 KiB: without it the default limit is 48 KiB minus the kernel's
    // static shared memory
    if (bytes > 0)
        SVDI_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    if (carveout_max && first)
        SVDI_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
    limit[{func, dev}] = bytes;
    return SVDI_OK;
}
int current_sm_count() {
    static std::mutex mu;
    static std::map<int, int> count;  // device -> SM count
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    std::lock_guard<std::mutex> lock(mu);
    auto it = count.find(dev);
    if (it != count.end()) return it->second;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    count[dev] = sms;
    return sms;
}
void note_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

namespace {

constexpr double kRefBeta = 15.3704324328;   // SVDIntegratedImager.cu:1235
constexpr int kRefSupport = 8;               // SVDIntegratedImager.cu:1234
constexpr int kChebMaxMoments = 32;          // SVDIntegratedImager.cu:35
constexpr double kChebTargetError = 1.0e-2;  // SVDIntegratedImager.cu:36
constexpr double kChebTargetAlpha = 10.0;    // SVDIntegratedImager.cu:37
constexpr int kPartialCap = 4096;

#define SVDI_CUFFT(call)                                                                  \
    do {                                                                                  \
        cufftResult r__ = (call);                                                         \
        if (r__ != CUFFT_SUCCESS) {                                                       \
            ::svdi::set_error(std::string("cuFFT error ") + std::to_string((int)r__) +    \
                              " at " + __FILE__ + ":" + std::to_string(__LINE__));        \
            return SVDI_ERR_CUFFT;                                                        \
        }                                                                                 \
    } while (0)

// Grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    int ensure(size_t bytes) {
        if (bytes <= cap) return SVDI_OK;
        if (p) {
            cudaFree(p);
            p = nullptr;
            cap = 0;
        }
        const size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error(std::string("device allocation of ") + std::to_string(want) + " bytes failed: " +
                      cudaGetErrorString(e));
            return SVDI_ERR_OUT_OF_MEMORY;
        }
        cap = want;
        return SVDI_OK;
    }
    template <typename T>
    T* as() const { return reinterpret_cast<T*>(p); }
};

long long next_nice_even(long long n) {
    for (long long m = std::max<long long>(2, n + (n & 1));; m += 2) {
        long long r = m;
        for (long long f : {2, 3, 5, 7})
            while (r % f == 0) r /= f;
        if (r == 1) return m;
    }
}

// The plans of a pruned inverse 2-D FFT (make_fft_plan).
struct FftPlan {
    enum Mode { kFull2D = 0, kRowsCufftCols = 1, kRowsSharedCols = 2 };
    Mode mode = kFull2D;
    cufftHandle rows = 0, cols = 0;  // kFull2D: `rows` is one 2-D plan of the whole grid
    ColFftPlan cp{};                 // kRowsSharedCols: the shared-memory column transforms
    float2* d_tw = nullptr;
    int* d_perm = nullptr;
    cudaStream_t stream = nullptr;
    long long G = 0, N = 0;
    int batch = 0;
};

void destroy_fft_plan(FftPlan& plan) {
    if (plan.rows) cufftDestroy(plan.rows);
    if (plan.cols) cufftDestroy(plan.cols);
    if (plan.d_tw) cudaFree(plan.d_tw);
    if (plan.d_perm) cudaFree(plan.d_perm);
    plan.rows = plan.cols = 0;
    plan.d_tw = nullptr;
    plan.d_perm = nullptr;
}

}  // namespace

}  // namespace svdi

struct svdi_engine {
    svdi_options opt;
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    // the flag/weight collapse runs on `side`, beside the rotation, statistics and histogram
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_vis = nullptr;
    std::mutex mu;
    // staging for host inputs
    svdi::DevBuf in_uvw, in_freq, in_v0r, in_v0i, in_v3r, in_v3i, in_f0, in_f3, in_w0, in_w3;
    svdi::DevBuf in_bin, in_vin;
    // intermediates
    svdi::DevBuf vr, vi, q, s, vin64, vin32, stats, partial, counts, offsets, cursor, dropped, rec,
        rec_s, planes, corr, image, cheb_err, bin_out, grid_keep, tc_status, kb_offsets, acc, chunk_key, keymax,
        plan_buf;
    size_t sz_vr = 0, sz_q = 0, sz_s = 0, sz_off = 0, sz_rec = 0, sz_rec_s = 0, sz_grid = 0, sz_mom = 0;
    const float* cur_vr = nullptr;
    const float* cur_vi = nullptr;
    const double* cur_q = nullptr;
    const double* cur_s = nullptr;
    double* h_stats = nullptr;  // pinned: ST_COUNT statistics, then the 9 entries of Vin
    // Speculative plan: a call with the same shape as the last one launches its gridding with the
    // last call's slab and Chebyshev counts (the slab geometry itself computed on the device from
    // this call's statistics) and checks the counts against its own host decision afterwards,
    // imaging again in the rare case they differ. The device never waits for the host decision.
    bool spec_valid = false, spec_archive = false, spec_bin = false;
    long long spec_N = 0, spec_n = 0, spec_R = 0;
    float spec_cell = 0.0f;
    svdi::SlabParams spec_sp{};
    cudaEvent_t ev_stats = nullptr;
    // slabs per batch of every (slab count, terms, grid size) asked for (a server slot alternates
    // between request shapes)
    std::map<std::tuple<int, int, long long>, size_t> bslab_cache;
    // Completion of the last call, read lazily (finish_pending): the device-API call returns once
    // its work is enqueued, so that the host can enqueue the next snapshot meanwhile.
    unsigned long long* h_ndrop = nullptr;  // pinned: dropped-sample count of the last call
    bool pending = false;                   // last call's device-side statistics not yet read
    bool pending_times = false;             // its stage events are valid (single slab batch)
    bool pending_total = false;             // ev[0] -> ev[7] spans the whole call
    bool pending_need_s = false;
    long long pending_n = 0;
    std::map<std::tuple<long long, long long, int>, svdi::FftPlan> plans;
    std::map<std::tuple<long long, long long, int, double>, std::vector<float>> corr_cache;
    std::tuple<long long, long long, int, double> corr_key{-1, -1, -1, 0.0};
    std::map<std::tuple<double, int, int>, std::vector<double>> cheb_cache;
    svdi::EsPoly poly{};
    int poly_W = -1;
    double poly_beta = 0.0;
    svdi_stats last{};
    cudaEvent_t ev[8] = {};
    // the last imaging call's sample source and geometry (for the accuracy probe)
    svdi::SampleSource last_src{};
    svdi::GridGeom last_g{};
    svdi::SlabParams last_sp{};
    long long last_N = 0;
    double last_cell = 0.0;
    bool have_last = false;
    svdi::DevBuf probe;
    // pageable host uploads and image downloads of the archive entry and the host-input call
    svdi::HostStager stager;
    bool batch_bound = false;  // a batch's captured graph refers to this engine's buffers

    ~svdi_engine() {
        if (device >= 0) cudaSetDevice(device);
        for (auto& kv : plans) svdi::destroy_fft_plan(kv.second);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (h_stats) cudaFreeHost(h_stats);
        if (h_ndrop) cudaFreeHost(h_ndrop);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_stats) cudaEventDestroy(ev_stats);
        if (ev_vis) cudaEventDestroy(ev_vis);
        if (side) cudaStreamDestroy(side);
        if (stream && own_stream) cudaStreamDestroy(stream);
    }
};

namespace svdi {
namespace {

int engine_init(svdi_engine* e, const svdi_options* opt) {
    e->opt = *opt;
    e->device = opt->device;
    SVDI_CUDA(cudaSetDevice(e->device));
    SVDI_CUDA(cudaDeviceGetAttribute(&e->sm_count, cudaDevAttrMultiProcessorCount, e->device));
    // the main stream at the highest priority: when blocks of the side stream's collapse retire,
    // the block scheduler starts the main stream's kernels first
    int prio_low = 0, prio_high = 0;
    SVDI_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    SVDI_CUDA(cudaStreamCreateWithPriority(&e->stream, cudaStreamNonBlocking, prio_high));
    SVDI_CUDA(cudaStreamCreateWithPriority(&e->side, cudaStreamNonBlocking, prio_low));
    SVDI_CUDA(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
    SVDI_CUDA(cudaEventCreateWithFlags(&e->ev_vis, cudaEventDisableTiming));
    SVDI_CUDA(cudaEventCreateWithFlags(&e->ev_stats, cudaEventDisableTiming));
    SVDI_CUDA(cudaMallocHost(&e->h_stats, (ST_COUNT + 9) * sizeof(double)));
    SVDI_CUDA(cudaMallocHost(&e->h_ndrop, 2 * sizeof(unsigned long long)));
    for (auto& ev : e->ev) SVDI_CUDA(cudaEventCreate(&ev));
    return SVDI_OK;
}

template <typename T>
int upload(DevBuf& b, const T* host, size_t n, cudaStream_t st) {
    SVDI_TRY(b.ensure(n * sizeof(T)));
    if (n) SVDI_CUDA(cudaMemcpyAsync(b.p, host, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return SVDI_OK;
}

// upload through the engine's staging ring (pageable sources of several MB; others copy directly)
template <typename T>
int upload_staged(svdi_engine* e, DevBuf& b, const T* host, size_t n, cudaStream_t st) {
    SVDI_TRY(b.ensure(n * sizeof(T)));
    return e->stager.h2d(b.p, host, n * sizeof(T), st);
}

double read_target_alpha(const svdi_options& o) {
    if (o.target_alpha > 0) return o.target_alpha;
    if (const char* env = std::getenv("SVD_CHEB_TARGET_ALPHA")) {  // SVDIntegratedImager.cu:963-971
        const double v = std::atof(env);
        if (v > 0) return v;
    }
    return kChebTargetAlpha;
}

// Sampled Jacobi-Anger truncation errors for K = 1..32 at alpha_max (device FP64, cached).
int cheb_errors(svdi_engine* e, double amax, int na, int ns, std::vector<double>& out) {
    auto key = std::make_tuple(amax, na, ns);
    auto it = e->cheb_cache.find(key);
    if (it != e->cheb_cache.end()) {
        out = it->second;
        return SVDI_OK;
    }
    SVDI_TRY(e->cheb_err.ensure(kChebMaxMoments * sizeof(unsigned long long)));
    SVDI_TRY(launch_cheb_errors(amax, na, ns, kChebMaxMoments, e->cheb_err.as<unsigned long long>(),
                                e->stream));
    unsigned long long h[kChebMaxMoments];
    SVDI_CUDA(cudaMemcpyAsync(h, e->cheb_err.p, sizeof(h), cudaMemcpyDeviceToHost, e->stream));
    SVDI_CUDA(cudaStreamSynchronize(e->stream));
    out.resize(kChebMaxMoments);
    for (int k = 0; k < kChebMaxMoments; ++k) {
        double d;
        memcpy(&d, &h[k], sizeof(d));
        out[k] = d;
    }
    if (e->cheb_cache.size() > 4096) e->cheb_cache.clear();
    e->cheb_cache[key] = out;
    return SVDI_OK;
}

// Upper bound of the Jacobi-Anger truncation error on |s| <= 1 when K terms are kept:
// 2 sum_{n >= K} |J_n(a)| (|T_n| <= 1).
double truncation_bound(double a, int K) {
    double j[200];
    const int nmax = std::min(199, K + 60 + (int)std::fabs(a));
    bessel_jn(a, nmax, j);
    double s = 0.0;
    for (int n = K; n <= nmax; ++n) s += std::fabs(j[n]);
    return 2.0 * s;
}

int k_for_target(double a, double target) {
    for (int K = 1; K <= kMaxTerms; ++K)
        if (truncation_bound(a, K) <= target) return K;
    return -1;
}

// Slab / Chebyshev configuration from the device statistics.
int choose_slabs(svdi_engine* e, bool archive, double r3min, double r3max, double mt3, SlabParams& sp,
                 double& alpha_max, double& slab_alpha) {
    const svdi_options& o = e->opt;
    const double half_range = std::max(0.5 * (r3max - r3min), 1.0e-6);
    alpha_max = 2.0 * kPi * mt3 * half_range;
    int nslab = 1;  // archive/FIPkernels.cu:327-366: one slab centred on the range
    if (!archive) {  // SVDIntegratedImager.cu:973-991
        const double r3_range = std::max(r3max - r3min, 2.0e-6);
        if (o.k_rule == SVDI_KRULE_TARGET && o.target_alpha <= 0) {
            // minimise the number of moment planes nslab * K(alpha_slab) at the error target; among
            // equal plane counts take the smallest K (a sample is gridded into K planes of its slab,
            // so fewer terms and more slabs grid the same planes with less work)
            int best_n = 1, best_p = 1 << 30;
            for (int n = 1; n <= 64; ++n) {
                const double h = std::max(0.5 * r3_range / n, 1.0e-6);
                const int K = k_for_target(2.0 * kPi * mt3 * h, o.target_error);
                if (K < 0) continue;
                if (n * K <= best_p) {
                    best_p = n * K;
                    best_n = n;
                }
                if (K == 1) break;
            }
            nslab = best_n;
        } else {
            nslab = (int)std::ceil(std::max(alpha_max, 0.0) / read_target_alpha(o));
            if (nslab < 1) nslab = 1;
        }
    }
    slab_params_for(archive, nslab, 0, r3min, r3max, sp);
    slab_alpha = 2.0 * kPi * mt3 * sp.slab_half;
    int K = kChebMaxMoments;
    std::vector<double> err;
    switch (o.k_rule) {
        case SVDI_KRULE_BUCKET: {  // SVDIntegratedImager.cu:1577-1603
            SVDI_TRY(cheb_errors(e, slab_alpha, 257, 1024, err));
            for (int kb : {8, 16, 24, 32})
                if (err[kb - 1] <= kChebTargetError) {
                    K = kb;
                    break;
                }
            break;
        }
        case SVDI_KRULE_MIN: {  // archive/FIPkernels.cu:287-366
            SVDI_TRY(cheb_errors(e, slab_alpha, 513, 2048, err));
            for (int k = 1; k <= kChebMaxMoments; ++k)
                if (err[k - 1] <= kChebTargetError) {
                    K = k;
                    break;
                }
            break;
        }
        case SVDI_KRULE_TARGET: {
            const int k = k_for_target(slab_alpha, o.target_error);
            if (k < 0) {
                set_error("no Chebyshev order <= 64 reaches the error target; increase the slab count");
                return SVDI_ERR_UNSUPPORTED;
            }
            K = k;
            break;
        }
        case SVDI_KRULE_FIXED:
            K = o.fixed_k;
            break;
        default:
            set_error("unknown k_rule");
            return SVDI_ERR_INVALID_ARGUMENT;
    }
    if (K < 1 || K > kMaxTerms) {
        set_error("Chebyshev order out of range");
        return SVDI_ERR_UNSUPPORTED;
    }
    sp.K = K;
    return SVDI_OK;
}

// The inverse 2-D FFT of `batch` moment planes of G x G, pruned to what the recombination reads:
// every row (length G, contiguous) is transformed, then only the N columns it reads (the checkerboard
// sign centres the transform, so pixel x reads column G / 2 + x - N / 2: one contiguous run) are
// transformed along the rows' stride. The second pass does N / G of the full 2-D transform's work
// there; the other columns keep their first-pass values and are never read. For G = 2^a 3^b
// (b <= 1, up to 12288) the column pass is this library's shared-memory transform (fft_cols.cu: a
// CTA per block of adjacent columns, one launch over all planes); other 2,3,5,7-smooth sizes use a
// strided cuFFT column plan per plane. Grid sizes with a prime factor above 7 (cuFFT's Bluestein
// path, which gave wrong in-place results for the interleaved column batches on B200) keep one 2-D
// plan.
int make_fft_plan(long long G, long long N, int batch, cudaStream_t st, FftPlan& plan) {
    long long r = G;
    for (long long f : {2, 3, 5, 7})
        while (r % f == 0) r /= f;
    int n = (int)G;
    if (r == 1) {
        SVDI_CUFFT(cufftPlanMany(&plan.rows, 1, &n, &n, 1, n, &n, 1, n, CUFFT_C2C, (int)(G * batch)));
        if (col_fft_supported(G)) {
            SVDI_TRY(make_col_fft(G, plan.cp, &plan.d_tw, &plan.d_perm));
            plan.mode = FftPlan::kRowsSharedCols;
        } else {
            SVDI_CUFFT(cufftPlanMany(&plan.cols, 1, &n, &n, n, 1, &n, n, 1, CUFFT_C2C, (int)N));
            plan.mode = FftPlan::kRowsCufftCols;
        }
    } else {
        int dims[2] = {n, n};
        SVDI_CUFFT(cufftPlanMany(&plan.rows, 2, dims, nullptr, 1, n * n, nullptr, 1, n * n, CUFFT_C2C, batch));
        plan.cols = 0;
        plan.mode = FftPlan::kFull2D;
    }
    SVDI_CUFFT(cufftSetStream(plan.rows, st));
    if (plan.cols) SVDI_CUFFT(cufftSetStream(plan.cols, st));
    plan.stream = st;
    plan.G = G;
    plan.N = N;
    plan.batch = batch;
    return SVDI_OK;
}

int get_plan(svdi_engine* e, long long G, long long N, int batch, FftPlan& plan) {
    auto key = std::make_tuple(G, N, batch);
    auto it = e->plans.find(key);
    if (it != e->plans.end()) {
        plan = it->second;
        return SVDI_OK;
    }
    SVDI_TRY(make_fft_plan(G, N, batch, e->stream, plan));
    e->plans[key] = plan;
    return SVDI_OK;
}

int exec_fft(const FftPlan& plan, cufftComplex* planes, int nplanes) {
    SVDI_CUFFT(cufftExecC2C(plan.rows, planes, planes, CUFFT_INVERSE));
    if (plan.mode == FftPlan::kFull2D) return SVDI_OK;
    const long long c0 = plan.G / 2 - plan.N / 2;
    if (plan.mode == FftPlan::kRowsSharedCols)
        return launch_col_fft(reinterpret_cast<float2*>(planes), nplanes, plan.G, c0, plan.N, plan.cp, plan.d_tw,
                              plan.d_perm, plan.stream);
    for (int p = 0; p < nplanes; ++p) {
        cufftComplex* col0 = planes + (long long)p * plan.G * plan.G + c0;
        SVDI_CUFFT(cufftExecC2C(plan.cols, col0, col0, CUFFT_INVERSE));
    }
    return SVDI_OK;
}

// 1 / Phi(i), i = 0..N/2: inverse of the ES kernel's Fourier transform at image offset i, computed
// in FP64 by composite Gauss-Legendre quadrature (the reference tabulates the same integral with a
// 28-point rule in FP32, SVDIntegratedImager.cu:867-882, 1204-1216).
int ensure_corr(svdi_engine* e, long long N, long long G, int W, double beta) {
    auto key = std::make_tuple(N, G, W, beta);
    if (e->corr_key == key) return SVDI_OK;
    auto it = e->corr_cache.find(key);
    if (it == e->corr_cache.end()) {
        static const double x16[8] = {0.0950125098376374, 0.2816035507792589, 0.4580167776572274,
                                      0.6178762444026438, 0.7554044083550030, 0.8656312023878318,
                                      0.9445750230732326, 0.9894009349916499};
        static const double w16[8] = {0.1894506104550685, 0.1826034150449236, 0.1691565193950025,
                                      0.1495959888165767, 0.1246289712555339, 0.0951585116824928,
                                      0.0622535239386479, 0.0271524594117541};
        auto psi = [&](double x) {
            if (std::fabs(x) > 1.0) return 0.0;
            return std::exp(-beta * x * x / (1.0 + std::sqrt((1.0 - x) * (1.0 + x))));
        };
        std::vector<float> c(N / 2 + 1);
        const int panels = 64;
        for (long long i = 0; i <= N / 2; ++i) {
            const double f = kPi * (double)W * ((double)i / (double)G);
            double acc = 0.0;
            for (int p = 0; p < panels; ++p) {
                const double a = (double)p / panels, b = (double)(p + 1) / panels;
                const double mid = 0.5 * (a + b), hw = 0.5 * (b - a);
                for (int j = 0; j < 8; ++j) {
                    const double t1 = mid - hw * x16[j], t2 = mid + hw * x16[j];
                    acc += w16[j] * hw * (psi(t1) * std::cos(f * t1) + psi(t2) * std::cos(f * t2));
                }
            }
            c[i] = (float)(1.0 / ((double)W * acc));
        }
        if (e->corr_cache.size() > 64) e->corr_cache.clear();
        it = e->corr_cache.emplace(key, std::move(c)).first;
    }
    SVDI_TRY(e->corr.ensure(it->second.size() * sizeof(float)));
    SVDI_CUDA(cudaMemcpyAsync(e->corr.p, it->second.data(), it->second.size() * sizeof(float),
                              cudaMemcpyHostToDevice, e->stream));
    e->corr_key = key;
    return SVDI_OK;
}

bool is_tc_gridder(int gridder) {
    return gridder == SVDI_GRIDDER_TC || gridder == SVDI_GRIDDER_TC_BF16 || gridder == SVDI_GRIDDER_TC_I8;
}

// Tile geometry of the tensor-core gridders (the grid size g.G set): 56 x 8 tiles for the FP16 /
// BF16 form, 24 x 8 for the integer form.
void tc_tiles(int gridder, GridGeom& g) {
    if (gridder == SVDI_GRIDDER_TC_I8) {
        g.T = kI8TileRows;
        g.T2 = kI8TileCols;
        g.ntile = (int)((g.G + g.T - 1) / g.T);
        g.ntile2 = (int)((g.G + g.T2 - 1) / g.T2);
    } else {
        g.T = kTcTileRows;
        g.T2 = kTcTileCols;
        g.ntile = (int)((g.G + g.T - 1) / g.T);
        g.ntile2 = (int)((g.G + g.T2 - 1) / g.T2);
        g.ntile2 = (g.ntile2 + kTcBlocks - 1) / kTcBlocks * kTcBlocks;
    }
}

long long grid_size(long long N, double sigma) {
    if (sigma == 1.5) return (3 * N + 1) / 2;  // ceil(1.5 N), SVDIntegratedImager.cu:1510
    return next_nice_even((long long)std::ceil(sigma * (double)N - 1e-9));
}

size_t batch_slabs_for(svdi_engine* e, int nslab, int K, long long G) {
    // SVDIntegratedImager.cu:1470-1496 (env SVDIMAGER_MAX_BATCH_SLABS or 25 % of free HBM)
    if (e->opt.max_batch_slabs > 0) return std::min<size_t>(nslab, e->opt.max_batch_slabs);
    if (const char* env = std::getenv("SVDIMAGER_MAX_BATCH_SLABS")) {
        const long long v = std::atoll(env);
        if (v > 0) return std::min<size_t>(nslab, (size_t)v);
    }
    // The free-memory query takes a driver lock that other processes on the GPU contend for (it
    // stalled calls by up to tens of milliseconds), so it is asked once per configuration.
    const auto key = std::make_tuple(nslab, K, G);
    const auto hit = e->bslab_cache.find(key);
    if (hit != e->bslab_cache.end()) return hit->second;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    const size_t per_slab = (size_t)K * (size_t)G * (size_t)G * sizeof(float2);
    const size_t budget = (free_b + e->planes.cap) / 4;
    const size_t b = std::min<size_t>(nslab, std::max<size_t>(1, budget / per_slab));
    if (e->bslab_cache.size() > 64) e->bslab_cache.clear();
    e->bslab_cache.emplace(key, b);
    return b;
}

// The host decisions of one snapshot: everything image_core reads back from the device before
// it can launch the gridding (basis determinant, w range, slab and Chebyshev configuration,
// slabs per batch). With a fixed plan image_core issues device work only (no synchronisation,
// no allocation when the buffers are already large enough), so it can be captured in a graph.
struct ExecPlan {
    float inv_det = 0.0f;
    SlabParams sp{};
    double alpha_max = 0, slab_alpha = 0, r3min = 0, r3max = 0, mt3 = 0;
    size_t bslabs = 1;
};

// Imaging core: given vin64 and sample source on the device, produce the image in d_out.
// fixed: replay a recorded plan (device work only; *d_status_out receives the tensor-core
// gridder's status word); record: store this call's plan.
// Reads the last call's device-side results once its work has completed: the dropped-sample
// count and, when its stage events are valid, the stage and total device times.
int finish_pending(svdi_engine* e) {
    if (!e->pending) return SVDI_OK;
    SVDI_CUDA(cudaEventSynchronize(e->pending_total ? e->ev[7] : e->ev[6]));
    svdi_stats& L = e->last;
    const unsigned long long ndrop = *e->h_ndrop;
    L.num_gridded = (size_t)(e->pending_n - (long long)ndrop);
    e->sz_rec = (size_t)(e->pending_n - (long long)ndrop) * sizeof(SampleRec);
    e->sz_rec_s = e->pending_need_s ? (size_t)(e->pending_n - (long long)ndrop) * 4 : 0;
    if (e->pending_times) {
        float a = 0, b = 0, c = 0, d = 0;
        cudaEventElapsedTime(&d, e->ev[1], e->ev[2]);
        cudaEventElapsedTime(&a, e->ev[3], e->ev[4]);
        cudaEventElapsedTime(&b, e->ev[4], e->ev[5]);
        cudaEventElapsedTime(&c, e->ev[5], e->ev[6]);
        L.ms_bin = d;
        L.ms_grid = a;
        L.ms_fft = b;
        L.ms_image = c;
    }
    if (e->pending_total) {
        float mp = 0, mt = 0;
        cudaEventElapsedTime(&mp, e->ev[0], e->ev[1]);
        cudaEventElapsedTime(&mt, e->ev[0], e->ev[7]);
        L.ms_preprocess = mp;
        L.ms_total = mt;
    }
    e->pending = false;
    return SVDI_OK;
}

// The host decision from the statistics and Vin read back into h_stats: 1 / |det|, w range, slab
// and Chebyshev configuration.
int host_decision(svdi_engine* e, bool archive, SampleSource& src, SlabParams& sp, double& alpha_max,
                  double& slab_alpha, double& r3min, double& r3max, double& mt3) {
    r3min = e->h_stats[ST_R3_MIN];
    r3max = e->h_stats[ST_R3_MAX];
    mt3 = e->h_stats[ST_MAX_T3];
    std::memcpy(e->last.vin, e->h_stats + ST_COUNT, 9 * sizeof(double));
    const double det = basis_det(e->last.vin);
    if (!(det > 0.0) || !std::isfinite(det)) {
        set_error("degenerate basis: |V00 V11 - V01 V10| is zero");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    src.inv_det = (float)(1.0 / det);
    return choose_slabs(e, archive, r3min, r3max, mt3, sp, alpha_max, slab_alpha);
}

// vis_ready (optional): event after which src.vr / src.vi hold the collapsed visibilities; only
// the scatter reads them.
int image_core(svdi_engine* e, bool archive, SampleSource src, long long N, float cell_f,
               float* d_out, const ExecPlan* fixed = nullptr, ExecPlan* record = nullptr,
               unsigned int* d_status_out = nullptr, cudaEvent_t vis_ready = nullptr, bool allow_spec = true) {
    cudaStream_t st = e->stream;
    const svdi_options& o = e->opt;
    const double cell = (double)cell_f;
    const long long n = src.n;
    const bool timed = fixed == nullptr;  // events, statistics and status read-back
    if (timed) e->pending = false;         // the previous call's statistics are superseded
    SlabParams sp{};
    double alpha_max = 0, slab_alpha = 0, r3min = 0, r3max = 0, mt3 = 0;
    const DevPlan* dplan = nullptr;  // speculative: slab geometry and 1 / |det| from the device
    size_t spec_bslabs = 0;
    if (fixed) {
        src.inv_det = fixed->inv_det;
        sp = fixed->sp;
        alpha_max = fixed->alpha_max;
        slab_alpha = fixed->slab_alpha;
        r3min = fixed->r3min;
        r3max = fixed->r3max;
        mt3 = fixed->mt3;
    } else {
        // statistics: max |t3|, then one small read
        SVDI_TRY(launch_t3_stats(e->vin64.as<double>(), N, cell, e->partial.as<double>(), kPartialCap,
                                 e->stats.as<double>(), st));
        SVDI_CUDA(cudaMemcpyAsync(e->h_stats, e->stats.p, ST_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st));
        SVDI_CUDA(cudaMemcpyAsync(e->h_stats + ST_COUNT, e->vin64.p, 9 * sizeof(double), cudaMemcpyDeviceToHost, st));
        bool spec = allow_spec && !record && e->spec_valid && e->spec_archive == archive && e->spec_N == N &&
                    e->spec_cell == cell_f && e->spec_n == n && e->spec_R == src.R &&
                    e->spec_bin == (src.bin != nullptr);
        if (spec) {  // one batch of all slabs only
            spec_bslabs = batch_slabs_for(e, e->spec_sp.nslab, e->spec_sp.K, grid_size(N, o.sigma));
            spec = (int)spec_bslabs >= e->spec_sp.nslab;
        }
        if (spec) {
            SVDI_CUDA(cudaEventRecord(e->ev_stats, st));
            sp = e->spec_sp;
            SVDI_TRY(e->plan_buf.ensure(sizeof(DevPlan)));
            SVDI_TRY(launch_plan(e->stats.as<double>(), e->vin64.as<double>(), archive, sp.nslab, sp.K,
                                 e->plan_buf.as<DevPlan>(), st));
            dplan = e->plan_buf.as<DevPlan>();
        } else {
            SVDI_CUDA(cudaStreamSynchronize(st));
            SVDI_TRY(host_decision(e, archive, src, sp, alpha_max, slab_alpha, r3min, r3max, mt3));
        }
    }

    GridGeom g{};
    g.G = grid_size(N, o.sigma);
    g.gmin = -(g.G / 2);
    g.gmax = (g.G - 1) / 2;
    g.W = o.support;
    // the tensor-core gridders accumulate one moment plane at a time in TMEM: the FP16 / BF16 form
    // (K == 1) bins into 56 x 8 tiles (64 x 16 accumulator window, gridder_tc.cu), the integer form
    // (any K, one launch per Chebyshev term) into 24 x 8 tiles (32 x 16 window, gridder_i8.cu);
    // the integer form scales each key by its own max |value| from the scatter
    const bool use_tc = is_tc_gridder(o.gridder) && (sp.K == 1 || o.gridder == SVDI_GRIDDER_TC_I8) && g.W <= 8;
    const bool use_i8 = use_tc && o.gridder == SVDI_GRIDDER_TC_I8;
    if (use_tc) {
        tc_tiles(o.gridder, g);
    } else {
        g.T = o.tile ? o.tile : (sp.K == 1 ? 64 : 32);
        g.ntile = (int)((g.G + g.T - 1) / g.T);
        g.T2 = g.T;
        g.ntile2 = g.ntile;
    }
    g.edge_mode = o.edge_mode;
    g.coord_mode = o.coord_mode;
    g.scale = cell * (double)g.G;
    g.scale32 = cell_f * (float)g.G;
    const long long n_keys_ll = (long long)sp.nslab * g.ntile * g.ntile2;
    if (n_keys_ll > (1LL << 26)) {
        set_error("too many tile keys");
        return SVDI_ERR_UNSUPPORTED;
    }
    const int n_keys = (int)n_keys_ll;

    if (e->poly_W != g.W || e->poly_beta != o.beta) {
        build_es_poly(g.W, o.beta, &e->poly);
        e->poly_W = g.W;
        e->poly_beta = o.beta;
    }

    // binning
    if (timed) SVDI_CUDA(cudaEventRecord(e->ev[1], st));
    SVDI_TRY(e->counts.ensure((size_t)n_keys * 4));
    SVDI_TRY(e->offsets.ensure((size_t)(n_keys + 1) * 4));
    SVDI_TRY(e->cursor.ensure((size_t)n_keys * 4));
    SVDI_TRY(e->dropped.ensure(16));  // [0] dropped samples, [1] non-finite gridded values
    SVDI_TRY(e->rec.ensure((size_t)std::max<long long>(n, 1) * sizeof(SampleRec)));
    const bool need_s = sp.K > 1;
    if (need_s) SVDI_TRY(e->rec_s.ensure((size_t)std::max<long long>(n, 1) * sizeof(float)));
    SVDI_CUDA(cudaMemsetAsync(e->counts.p, 0, (size_t)n_keys * 4, st));
    SVDI_CUDA(cudaMemsetAsync(e->dropped.p, 0, 16, st));
    // a NaN or Inf among the gridded values makes the image NaN, as the reference's float atomics
    // and FFT do (SVDIntegratedImager.cu:606-612 keeps NaN under a zero weight)
    src.nonfinite = e->dropped.as<unsigned long long>() + 1;
    SVDI_TRY(launch_histogram(src, g, sp, e->counts.as<unsigned int>(), n_keys,
                              e->dropped.as<unsigned long long>(), st, dplan));
    if (use_tc) {
        SVDI_TRY(e->kb_offsets.ensure((size_t)(n_keys + 1) * 4));
    } else {  // the FP32 gridder's chunk table
        SVDI_TRY(e->chunk_key.ensure(((size_t)std::max<long long>(n, 1) / kGridChunk + 2) * 4));
    }
    const bool need_keymax = !use_tc || use_i8;  // per-key max |value| (FP32 and integer gridders)
    if (need_keymax) {
        SVDI_TRY(e->keymax.ensure((size_t)n_keys * 4));
        SVDI_CUDA(cudaMemsetAsync(e->keymax.p, 0, (size_t)n_keys * 4, st));
    }
    SVDI_TRY(launch_scan(e->counts.as<unsigned int>(), n_keys, e->offsets.as<unsigned int>(),
                         e->cursor.as<unsigned int>(), st,
                         use_tc ? e->kb_offsets.as<unsigned int>() : nullptr, kTcKBlock,
                         use_tc ? nullptr : e->chunk_key.as<unsigned int>(), kGridChunk));
    // tensor-core gridder: [0] give-up status, [1] max |record value| (float bits) from the scatter
    if (use_tc) {
        SVDI_TRY(e->tc_status.ensure(4 * sizeof(unsigned int)));
        SVDI_CUDA(cudaMemsetAsync(e->tc_status.p, 0, 4 * sizeof(unsigned int), st));
    }
    if (vis_ready) SVDI_CUDA(cudaStreamWaitEvent(st, vis_ready, 0));
    SVDI_TRY(launch_scatter(src, g, sp, e->cursor.as<unsigned int>(), n_keys, e->rec.as<SampleRec>(),
                            need_s ? e->rec_s.as<float>() : nullptr,
                            use_tc ? e->tc_status.as<unsigned int>() + 1 : nullptr, st,
                            need_keymax ? e->keymax.as<unsigned int>() : nullptr, dplan));
    if (timed) SVDI_CUDA(cudaEventRecord(e->ev[2], st));

    // slab batches: grid -> FFT -> recombine
    const size_t bslabs = fixed ? fixed->bslabs : (dplan ? spec_bslabs : batch_slabs_for(e, sp.nslab, sp.K, g.G));
    if (record) {
        record->inv_det = src.inv_det;
        record->sp = sp;
        record->alpha_max = alpha_max;
        record->slab_alpha = slab_alpha;
        record->r3min = r3min;
        record->r3max = r3max;
        record->mt3 = mt3;
        record->bslabs = bslabs;
    }
    const int planes_per_batch = (int)bslabs * sp.K;
    const size_t plane_bytes = (size_t)g.G * g.G * sizeof(float2);
    SVDI_TRY(e->planes.ensure(plane_bytes * planes_per_batch));
    FftPlan plan;
    SVDI_TRY(get_plan(e, g.G, N, planes_per_batch, plan));
    SVDI_TRY(ensure_corr(e, N, g.G, g.W, o.beta));
    SVDI_CUDA(cudaMemsetAsync(d_out, 0, (size_t)N * N * sizeof(float), st));
    // slabs split over several batches: the signed sums of all batches before |.| (the reference
    // takes |.| per batch, SVDIntegratedImager.cu:1445, inside its batch loop at :1681)
    const bool multi_batch = (int)bslabs < sp.nslab;
    if (multi_batch) {
        SVDI_TRY(e->acc.ensure((size_t)N * N * sizeof(double)));
        SVDI_CUDA(cudaMemsetAsync(e->acc.p, 0, (size_t)N * N * sizeof(double), st));
    }
    float ms_grid = 0, ms_fft = 0, ms_img = 0;
    for (int s0 = 0; s0 < sp.nslab; s0 += (int)bslabs) {
        const int s1 = std::min(sp.nslab, s0 + (int)bslabs);
        SlabParams bp = sp;
        if (timed) SVDI_CUDA(cudaEventRecord(e->ev[3], st));
        SVDI_CUDA(cudaMemsetAsync(e->planes.p, 0, plane_bytes * planes_per_batch, st));
        const int tiles2 = g.ntile * g.ntile2;
        if (use_i8) {
            SVDI_TRY(launch_grid_i8(e->rec.as<SampleRec>(), need_s ? e->rec_s.as<float>() : nullptr,
                                    e->offsets.as<unsigned int>(), e->kb_offsets.as<unsigned int>(), n_keys,
                                    s0 * tiles2, s1 * tiles2, s0, sp.K, g, e->poly, e->planes.as<float2>(),
                                    e->keymax.as<unsigned int>(), e->tc_status.as<unsigned int>(), e->sm_count,
                                    st));
        } else if (use_tc) {
            SVDI_TRY(launch_grid_tc(e->rec.as<SampleRec>(), e->offsets.as<unsigned int>(),
                                    e->kb_offsets.as<unsigned int>(), n_keys, s0 * tiles2,
                                    s1 * tiles2, s0, g, e->poly, e->planes.as<float2>(),
                                    e->tc_status.as<unsigned int>() + 1, e->tc_status.as<unsigned int>(),
                                    e->sm_count, st, o.gridder == SVDI_GRIDDER_TC_BF16));
        } else {
            SVDI_TRY(launch_grid_fp32(e->rec.as<SampleRec>(), need_s ? e->rec_s.as<float>() : nullptr,
                                      e->offsets.as<unsigned int>(), e->chunk_key.as<unsigned int>(),
                                      e->keymax.as<unsigned int>(),
                                      e->chunk_key.as<unsigned int>() + (size_t)std::max<long long>(n, 1) / kGridChunk + 1,
                                      n_keys, s0 * tiles2, s1 * tiles2, s0, g,
                                      sp, e->poly, e->planes.as<float2>(), e->sm_count, st));
        }
        if (o.keep_grid && s0 == 0) {
            SVDI_TRY(e->grid_keep.ensure(plane_bytes * planes_per_batch));
            SVDI_CUDA(cudaMemcpyAsync(e->grid_keep.p, e->planes.p, plane_bytes * planes_per_batch,
                                      cudaMemcpyDeviceToDevice, st));
            e->sz_grid = plane_bytes * (size_t)(std::min(sp.nslab, (int)bslabs) * sp.K);
        }
        if (timed) SVDI_CUDA(cudaEventRecord(e->ev[4], st));
        SVDI_TRY(exec_fft(plan, e->planes.as<cufftComplex>(), planes_per_batch));
        if (timed) SVDI_CUDA(cudaEventRecord(e->ev[5], st));
        // recombine the slabs of this batch (moment plane index relative to the batch)
        bp.nslab = s1 - s0;
        bp.r3_min = sp.r3_min + (double)s0 * sp.slab_width;
        SVDI_TRY(launch_recombine(e->planes.as<float2>(), g, N, cell, e->vin64.as<double>(), bp,
                                  e->corr.as<float>(), 1.0 / (double)n, o.reprojection, o.presplat, d_out,
                                  st, multi_batch ? e->acc.as<double>() : nullptr, s1 == sp.nslab, dplan,
                                  src.nonfinite));
        if (!timed) continue;
        SVDI_CUDA(cudaEventRecord(e->ev[6], st));
        if (!multi_batch) continue;  // one batch: its stage times are read when the call completes
        SVDI_CUDA(cudaEventSynchronize(e->ev[6]));
        float a = 0, b = 0, c = 0;
        cudaEventElapsedTime(&a, e->ev[3], e->ev[4]);
        cudaEventElapsedTime(&b, e->ev[4], e->ev[5]);
        cudaEventElapsedTime(&c, e->ev[5], e->ev[6]);
        ms_grid += a;
        ms_fft += b;
        ms_img += c;
    }
    if (dplan) {  // the host decision of this call, taken while the device images
        SVDI_CUDA(cudaEventSynchronize(e->ev_stats));
        SlabParams real{};
        const int rc = host_decision(e, archive, src, real, alpha_max, slab_alpha, r3min, r3max, mt3);
        if (rc != SVDI_OK) {
            e->spec_valid = false;
            return rc;
        }
        if (real.nslab != sp.nslab || real.K != sp.K) {  // other counts: image again with them
            e->spec_valid = false;
            return image_core(e, archive, src, N, cell_f, d_out, nullptr, nullptr, d_status_out, vis_ready, false);
        }
        sp = real;  // the same bits as the device plan (slab_params_for, basis_det)
    }
    if (!fixed && !record) {
        e->spec_valid = true;
        e->spec_archive = archive;
        e->spec_bin = src.bin != nullptr;
        e->spec_N = N;
        e->spec_cell = cell_f;
        e->spec_n = n;
        e->spec_R = src.R;
        e->spec_sp = sp;
    }
    e->last_src = src;
    e->last_g = g;
    e->last_sp = sp;
    e->last_N = N;
    e->last_cell = cell;
    e->have_last = true;
    if (!timed) {
        if (d_status_out) {
            if (use_tc)
                SVDI_CUDA(cudaMemcpyAsync(d_status_out, e->tc_status.p, sizeof(unsigned int),
                                          cudaMemcpyDeviceToDevice, st));
            else
                SVDI_CUDA(cudaMemsetAsync(d_status_out, 0, sizeof(unsigned int), st));
        }
        return SVDI_OK;
    }
    SVDI_CUDA(cudaMemcpyAsync(e->h_ndrop, e->dropped.p, 8, cudaMemcpyDeviceToHost, st));
    if (use_tc) {  // the tensor-core gridder's give-up status is checked before the call returns
        unsigned int tc_status = 0;
        SVDI_CUDA(cudaMemcpyAsync(&tc_status, e->tc_status.p, 4, cudaMemcpyDeviceToHost, st));
        SVDI_CUDA(cudaStreamSynchronize(st));
        if (tc_status != 0) {
            set_error("tensor-core gridder gave up waiting for an MMA completion (status " +
                      std::to_string(tc_status) + "); the grid is incomplete");
            return SVDI_ERR_INTERNAL;
        }
    }
    e->pending = true;
    e->pending_times = !multi_batch;
    e->pending_total = false;
    e->pending_need_s = need_s;
    e->pending_n = n;
    if (multi_batch) {
        float mb = 0;
        cudaEventElapsedTime(&mb, e->ev[1], e->ev[2]);
        e->last.ms_bin = mb;
        e->last.ms_grid = ms_grid;
        e->last.ms_fft = ms_fft;
        e->last.ms_image = ms_img;
    }

    e->sz_off = (size_t)(n_keys + 1) * 4;
    e->sz_mom = plane_bytes * (size_t)planes_per_batch;
    e->cur_vr = src.vr;
    e->cur_vi = src.vi;
    e->sz_vr = (size_t)n * 4;
    e->cur_q = src.q;
    e->cur_s = src.s;
    svdi_stats& L = e->last;
    L.tile = g.T;
    L.tile_cols = g.T2;
    L.used_tc = use_tc ? 1 : 0;
    L.num_keys = n_keys;
    L.slab_r3_min = sp.r3_min;
    L.slab_width = sp.slab_width;
    L.slab_half = sp.slab_half;
    L.num_samples = (size_t)n;
    L.grid_size = (size_t)g.G;
    L.num_slabs = sp.nslab;
    L.num_terms = sp.K;
    L.num_planes = sp.nslab * sp.K;
    L.r3_min = r3min;
    L.r3_max = r3max;
    L.max_abs_t3 = mt3;
    L.valid_pixels = (size_t)e->h_stats[ST_VALID_PIX];
    L.alpha_max = alpha_max;
    L.slab_alpha_max = slab_alpha;
    return SVDI_OK;
}

int check_ms(const svdi_host_ms* h) {
    if (!h) {
        set_error("null measurement-set descriptor");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    if (h->num_samples == 0 || h->num_rows == 0 || h->num_channels == 0) {
        set_error("Measurement set is empty");  // SVDIntegratedImager.cu:640-642
        return SVDI_ERR_EMPTY_INPUT;
    }
    if (h->num_samples != h->num_rows * h->num_channels) {
        set_error("num_samples must equal num_rows * num_channels");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    if (h->num_samples >= (1ULL << 32) - 1) {
        set_error("more than 2^32 - 2 samples per snapshot");
        return SVDI_ERR_UNSUPPORTED;
    }
    if (!h->uvw || !h->frequencies_hz || !h->vis0_real || !h->vis0_imag || !h->vis3_real ||
        !h->vis3_imag || !h->flag0 || !h->flag3 || !h->weight0 || !h->weight3) {
        set_error("null array in measurement-set descriptor");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    return SVDI_OK;
}

int check_image_args(size_t N, float cell) {
    if (N == 0 || N > 65536) {
        set_error("Image_Size must be in 1..65536");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    if (!(cell > 0.0f) || !std::isfinite(cell)) {
        set_error("Cell_Size must be greater than zero");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    return SVDI_OK;
}

int check_options(const svdi_options& o) {
    if (o.support != 6 && o.support != 8 && o.support != 10 && o.support != 12) {
        set_error("support must be 6, 8, 10 or 12");
        return SVDI_ERR_UNSUPPORTED;
    }
    if (!(o.beta > 0) || !(o.sigma >= 1.0) || o.sigma > 4.0) {
        set_error("beta must be > 0 and sigma in [1, 4]");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    if (o.tile != 0 && o.tile != 32 && o.tile != 64) {
        set_error("tile must be 0, 32 or 64");
        return SVDI_ERR_UNSUPPORTED;
    }
    if (o.gridder != SVDI_GRIDDER_FP32 && !is_tc_gridder(o.gridder)) {
        set_error("unknown gridder");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    return SVDI_OK;
}

// Main path on device-resident raw snapshot arrays.
int main_path_device(svdi_engine* e, const svdi_host_ms* d, size_t N, float cell, float* d_out,
                     const ExecPlan* fixed = nullptr, ExecPlan* record = nullptr,
                     unsigned int* d_status_out = nullptr) {
    cudaStream_t st = e->stream;
    const long long R = (long long)d->num_rows, C = (long long)d->num_channels;
    const long long n = (long long)d->num_samples;
    if (!fixed) SVDI_CUDA(cudaEventRecord(e->ev[0], st));
    SVDI_TRY(e->vr.ensure(n * 4));
    SVDI_TRY(e->vi.ensure(n * 4));
    SVDI_TRY(e->q.ensure(R * 24));
    SVDI_TRY(e->s.ensure(C * 8));
    SVDI_TRY(e->vin64.ensure(9 * 8));
    SVDI_TRY(e->vin32.ensure(9 * 4));
    SVDI_TRY(e->stats.ensure(ST_COUNT * 8));
    SVDI_TRY(e->partial.ensure((size_t)kPartialCap * 9 * 8));
    // the collapse (HBM-bound) overlaps the rotation, the statistics read-back and the histogram
    // (compute-bound), which need only uvw and frequencies; the scatter waits for it
    SVDI_CUDA(cudaEventRecord(e->ev_fork, st));
    SVDI_CUDA(cudaStreamWaitEvent(e->side, e->ev_fork, 0));
    SVDI_TRY(launch_collapse(d->vis0_real, d->vis0_imag, d->vis3_real, d->vis3_imag, d->flag0, d->flag3,
                             d->weight0, d->weight3, e->vr.as<float>(), e->vi.as<float>(), n, e->side));
    SVDI_CUDA(cudaEventRecord(e->ev_vis, e->side));
    SVDI_TRY(launch_preprocess(d->uvw, d->frequencies_hz, R, C, d->array_center_x, e->partial.as<double>(),
                               kPartialCap, e->vin64.as<double>(), e->vin32.as<float>(), e->q.as<double>(),
                               e->s.as<double>(), e->stats.as<double>(), st));
    SampleSource src{};
    src.q = e->q.as<double>();
    src.s = e->s.as<double>();
    src.R = R;
    src.vr = e->vr.as<float>();
    src.vi = e->vi.as<float>();
    src.n = n;
    e->sz_q = (size_t)R * 24;
    e->sz_s = (size_t)C * 8;
    SVDI_TRY(image_core(e, false, src, (long long)N, cell, d_out, fixed, record, d_status_out, e->ev_vis));
    if (fixed) return SVDI_OK;
    SVDI_CUDA(cudaEventRecord(e->ev[7], st));
    e->pending_total = true;  // preprocessing and total times are read with the other statistics
    return SVDI_OK;
}

int check_archive_args(const float* Visreal, const float* Visimag, const float* Bin, const float* Vin,
                       const float* dirty_image, size_t n, size_t N, float cell) {
    if (!Visreal || !Visimag || !Bin || !Vin || !dirty_image) {
        set_error("null pointer argument");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    if (n == 0) {
        set_error("num_baselines must be greater than zero");
        return SVDI_ERR_EMPTY_INPUT;
    }
    if (n >= (1ULL << 32) - 1) {
        set_error("more than 2^32 - 2 samples per call");
        return SVDI_ERR_UNSUPPORTED;
    }
    return check_image_args(N, cell);
}

int archive_path(svdi_engine* e, const float* Visreal, const float* Visimag, const float* Bin,
                 const float* Vin, float* dirty_image, size_t n, size_t N, float cell) {
    SVDI_TRY(check_archive_args(Visreal, Visimag, Bin, Vin, dirty_image, n, N, cell));
    cudaStream_t st = e->stream;
    SVDI_CUDA(cudaSetDevice(e->device));
    SVDI_CUDA(cudaEventRecord(e->ev[0], st));
    SVDI_TRY(upload_staged(e, e->vr, Visreal, n, st));
    SVDI_TRY(upload_staged(e, e->vi, Visimag, n, st));
    SVDI_TRY(upload_staged(e, e->in_bin, Bin, n * 3, st));
    SVDI_TRY(upload(e->vin32, Vin, 9, st));
    SVDI_TRY(e->vin64.ensure(9 * 8));
    SVDI_TRY(e->stats.ensure(ST_COUNT * 8));
    SVDI_TRY(e->partial.ensure((size_t)kPartialCap * 9 * 8));
    SVDI_TRY(e->image.ensure(N * N * 4));
    SVDI_TRY(launch_vin_from_float(e->vin32.as<float>(), e->vin64.as<double>(), st));
    SVDI_TRY(launch_bin_stats(e->in_bin.as<float>(), (long long)n, e->partial.as<double>(), kPartialCap,
                              e->stats.as<double>(), st));
    SampleSource src{};
    src.bin = e->in_bin.as<float>();
    src.vr = e->vr.as<float>();
    src.vi = e->vi.as<float>();
    src.n = (long long)n;
    e->sz_q = 0;
    e->sz_s = 0;
    SVDI_TRY(image_core(e, true, src, (long long)N, cell, e->image.as<float>()));
    SVDI_TRY(e->stager.d2h(dirty_image, e->image.p, N * N * 4, st));
    SVDI_CUDA(cudaEventRecord(e->ev[7], st));
    SVDI_CUDA(cudaStreamSynchronize(st));
    SVDI_TRY(finish_pending(e));
    float mt = 0;
    cudaEventElapsedTime(&mt, e->ev[0], e->ev[7]);
    e->last.ms_total = mt;
    return SVDI_OK;
}

svdi_options archive_defaults() {
    svdi_options o;
    svdi_default_options(&o);
    o.k_rule = SVDI_KRULE_MIN;
    o.reprojection = SVDI_REPROJ_FIPK;
    return o;
}

std::mutex g_default_mu;
std::map<int, std::unique_ptr<svdi_engine>> g_default_engines;

int default_engine(svdi_engine** out) {
    int dev = 0;
    SVDI_CUDA(cudaGetDevice(&dev));
    auto it = g_default_engines.find(dev);
    if (it == g_default_engines.end()) {
        std::unique_ptr<svdi_engine> e(new svdi_engine());
        svdi_options o = archive_defaults();
        o.device = dev;
        SVDI_TRY(engine_init(e.get(), &o));
        it = g_default_engines.emplace(dev, std::move(e)).first;
    }
    *out = it->second.get();
    return SVDI_OK;
}

}  // namespace
}  // namespace svdi

using namespace svdi;

extern "C" {

const char* svdi_last_error(void) { return g_last_error.c_str(); }

uint64_t svdi_kernel_launch_count(void) { return g_launches.load(); }

void svdi_default_options(svdi_options* opt) {
    if (!opt) return;
    memset(opt, 0, sizeof(*opt));
    opt->device = 0;
    opt->k_rule = SVDI_KRULE_BUCKET;
    opt->fixed_k = 1;
    opt->target_error = 1e-6;
    opt->target_alpha = 0.0;
    opt->edge_mode = SVDI_EDGE_CLIP;
    opt->coord_mode = SVDI_COORD_FP64;
    opt->reprojection = SVDI_REPROJ_SII;
    opt->support = kRefSupport;
    opt->beta = kRefBeta;
    opt->sigma = 1.5;
    opt->tile = 0;
    opt->gridder = SVDI_GRIDDER_FP32;
    opt->max_batch_slabs = 0;
}

int svdi_engine_create(const svdi_options* opt, svdi_engine** out) {
    g_last_error.clear();
    if (!out) {
        set_error("null output handle");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    svdi_options o;
    if (opt) o = *opt;
    else svdi_default_options(&o);
    SVDI_TRY(check_options(o));
    std::unique_ptr<svdi_engine> e(new svdi_engine());
    SVDI_TRY(engine_init(e.get(), &o));
    *out = e.release();
    return SVDI_OK;
}

void svdi_engine_destroy(svdi_engine* e) { delete e; }

int svdi_engine_image_host(svdi_engine* e, const svdi_host_ms* h, size_t N, float cell, float* dirty_image) {
    g_last_error.clear();
    if (!e || !dirty_image) {
        set_error("null argument");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    SVDI_TRY(check_ms(h));
    SVDI_TRY(check_image_args(N, cell));
    std::lock_guard<std::mutex> lk(e->mu);
    SVDI_CUDA(cudaSetDevice(e->device));
    cudaStream_t st = e->stream;
    const size_t n = h->num_samples, R = h->num_rows, C = h->num_channels;
    // uvw and frequencies first on the main stream: the rotation, statistics, histogram and scan
    // need only these and run while the visibilities, flags and weights upload on the side
    // stream, which then collapses them (main_path_device)
    SVDI_TRY(upload(e->in_uvw, h->uvw, R * 3, st));
    SVDI_TRY(upload(e->in_freq, h->frequencies_hz, C, st));
    SVDI_CUDA(cudaEventRecord(e->ev_fork, st));
    SVDI_CUDA(cudaStreamWaitEvent(e->side, e->ev_fork, 0));
    cudaStream_t sd = e->side;
    SVDI_TRY(upload_staged(e, e->in_v0r, h->vis0_real, n, sd));
    SVDI_TRY(upload_staged(e, e->in_v0i, h->vis0_imag, n, sd));
    SVDI_TRY(upload_staged(e, e->in_v3r, h->vis3_real, n, sd));
    SVDI_TRY(upload_staged(e, e->in_v3i, h->vis3_imag, n, sd));
    SVDI_TRY(upload_staged(e, e->in_f0, h->flag0, n, sd));
    SVDI_TRY(upload_staged(e, e->in_f3, h->flag3, n, sd));
    SVDI_TRY(upload_staged(e, e->in_w0, h->weight0, n, sd));
    SVDI_TRY(upload_staged(e, e->in_w3, h->weight3, n, sd));
    svdi_host_ms d = *h;
    d.uvw = e->in_uvw.as<float>();
    d.frequencies_hz = e->in_freq.as<float>();
    d.vis0_real = e->in_v0r.as<float>();
    d.vis0_imag = e->in_v0i.as<float>();
    d.vis3_real = e->in_v3r.as<float>();
    d.vis3_imag = e->in_v3i.as<float>();
    d.flag0 = e->in_f0.as<uint8_t>();
    d.flag3 = e->in_f3.as<uint8_t>();
    d.weight0 = e->in_w0.as<float>();
    d.weight3 = e->in_w3.as<float>();
    SVDI_TRY(e->image.ensure(N * N * 4));
    SVDI_TRY(main_path_device(e, &d, N, cell, e->image.as<float>()));
    SVDI_TRY(e->stager.d2h(dirty_image, e->image.p, N * N * 4, st));
    SVDI_TRY(finish_pending(e));
    return SVDI_OK;
}

int svdi_engine_image_device(svdi_engine* e, const svdi_host_ms* d, size_t N, float cell, float* d_out,
                             void* cuda_stream) {
    g_last_error.clear();
    if (!e || !d_out) {
        set_error("null argument");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    SVDI_TRY(check_ms(d));
    SVDI_TRY(check_image_args(N, cell));
    std::lock_guard<std::mutex> lk(e->mu);
    SVDI_CUDA(cudaSetDevice(e->device));
    // the call is ordered on the caller's stream (0: the legacy default stream): it starts after
    // the caller's earlier work there and the caller's later work there sees the image
    cudaStream_t user = (cudaStream_t)cuda_stream;
    SVDI_CUDA(cudaEventRecord(e->ev[0], user));
    SVDI_CUDA(cudaStreamWaitEvent(e->stream, e->ev[0], 0));
    SVDI_TRY(main_path_device(e, d, N, cell, d_out));
    SVDI_CUDA(cudaEventRecord(e->ev[7], e->stream));
    SVDI_CUDA(cudaStreamWaitEvent(user, e->ev[7], 0));
    return SVDI_OK;
}

int svdi_engine_fipipe_host(svdi_engine* e, const float* Visreal, const float* Visimag, const float* Bin,
                            const float* Vin, float* dirty_image, size_t n, size_t N, float cell) {
    g_last_error.clear();
    if (!e) {
        set_error("null engine");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lk(e->mu);
    return archive_path(e, Visreal, Visimag, Bin, Vin, dirty_image, n, N, cell);
}

int svdi_engine_last_stats(const svdi_engine* e, svdi_stats* out) {
    if (!e || !out) {
        set_error("null argument");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    svdi_engine* m = const_cast<svdi_engine*>(e);
    std::lock_guard<std::mutex> lk(m->mu);
    SVDI_CUDA(cudaSetDevice(m->device));
    SVDI_TRY(finish_pending(m));
    *out = e->last;
    return SVDI_OK;
}

static int buffer_of(const svdi_engine* e, int which, const void** p, size_t* bytes) {
    switch (which) {
        case SVDI_BUF_VIS_REAL: *p = e->cur_vr; *bytes = e->cur_vr ? e->sz_vr : 0; return SVDI_OK;
        case SVDI_BUF_VIS_IMAG: *p = e->cur_vi; *bytes = e->cur_vi ? e->sz_vr : 0; return SVDI_OK;
        case SVDI_BUF_Q: *p = e->cur_q; *bytes = e->cur_q ? e->sz_q : 0; return SVDI_OK;
        case SVDI_BUF_S: *p = e->cur_s; *bytes = e->cur_s ? e->sz_s : 0; return SVDI_OK;
        case SVDI_BUF_VIN: *p = e->vin64.p; *bytes = e->vin64.p ? 72 : 0; return SVDI_OK;
        case SVDI_BUF_OFFSETS: *p = e->offsets.p; *bytes = e->sz_off; return SVDI_OK;
        case SVDI_BUF_RECORDS: *p = e->rec.p; *bytes = e->sz_rec; return SVDI_OK;
        case SVDI_BUF_RECORDS_S: *p = e->rec_s.p; *bytes = e->sz_rec_s; return SVDI_OK;
        case SVDI_BUF_GRID: *p = e->grid_keep.p; *bytes = e->sz_grid; return SVDI_OK;
        case SVDI_BUF_MOMENTS: *p = e->planes.p; *bytes = e->sz_mom; return SVDI_OK;
        default:
            set_error("unknown buffer id");
            return SVDI_ERR_INVALID_ARGUMENT;
    }
}

int svdi_engine_buffer_size(const svdi_engine* e, int which, size_t* bytes) {
    if (!e || !bytes) {
        set_error("null argument");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    svdi_engine* m = const_cast<svdi_engine*>(e);
    std::lock_guard<std::mutex> lk(m->mu);
    SVDI_CUDA(cudaSetDevice(m->device));
    SVDI_TRY(finish_pending(m));
    const void* p = nullptr;
    return buffer_of(e, which, &p, bytes);
}

int svdi_engine_copy_buffer(svdi_engine* e, int which, void* host_dst, size_t bytes) {
    if (!e || !host_dst) {
        set_error("null argument");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lk(e->mu);
    SVDI_CUDA(cudaSetDevice(e->device));
    SVDI_TRY(finish_pending(e));
    const void* p = nullptr;
    size_t have = 0;
    SVDI_TRY(buffer_of(e, which, &p, &have));
    if (!p || bytes > have) {
        set_error("buffer not available or request larger than the buffer");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    SVDI_CUDA(cudaSetDevice(e->device));
    SVDI_CUDA(cudaMemcpyAsync(host_dst, p, bytes, cudaMemcpyDeviceToHost, e->stream));
    SVDI_CUDA(cudaStreamSynchronize(e->stream));
    return SVDI_OK;
}

int svdi_fipipe(const float* Visreal, const float* Visimag, const float* Bin, const float* Vin,
                float* dirty_image, size_t num_baselines, size_t image_size, float cell_size) {
    g_last_error.clear();
    SVDI_TRY(check_archive_args(Visreal, Visimag, Bin, Vin, dirty_image, num_baselines, image_size, cell_size));
    std::lock_guard<std::mutex> lk(g_default_mu);
    svdi_engine* e = nullptr;
    SVDI_TRY(default_engine(&e));
    std::lock_guard<std::mutex> lk2(e->mu);
    return archive_path(e, Visreal, Visimag, Bin, Vin, dirty_image, num_baselines, image_size, cell_size);
}

// ---- main-path mirror ----------------------------------------------------------------------
struct svdi_pre_internal {
    svdi_engine* engine;
};

int svdi_preprocess_measurement_set(const svdi_host_ms* h, svdi_device_buffers* dev, int want_bin) {
    g_last_error.clear();
    if (!dev) {
        set_error("null device buffers");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    memset(dev, 0, sizeof(*dev));
    SVDI_TRY(check_ms(h));
    svdi_options o;
    svdi_default_options(&o);
    SVDI_CUDA(cudaGetDevice(&o.device));
    svdi_engine* e = nullptr;
    SVDI_TRY(svdi_engine_create(&o, &e));
    std::unique_ptr<svdi_engine> guard(e);
    cudaStream_t st = e->stream;
    const size_t n = h->num_samples, R = h->num_rows, C = h->num_channels;
    SVDI_TRY(upload(e->in_uvw, h->uvw, R * 3, st));
    SVDI_TRY(upload(e->in_freq, h->frequencies_hz, C, st));
    SVDI_TRY(upload(e->in_v0r, h->vis0_real, n, st));
    SVDI_TRY(upload(e->in_v0i, h->vis0_imag, n, st));
    SVDI_TRY(upload(e->in_v3r, h->vis3_real, n, st));
    SVDI_TRY(upload(e->in_v3i, h->vis3_imag, n, st));
    SVDI_TRY(upload(e->in_f0, h->flag0, n, st));
    SVDI_TRY(upload(e->in_f3, h->flag3, n, st));
    SVDI_TRY(upload(e->in_w0, h->weight0, n, st));
    SVDI_TRY(upload(e->in_w3, h->weight3, n, st));
    SVDI_TRY(e->vr.ensure(n * 4));
    SVDI_TRY(e->vi.ensure(n * 4));
    SVDI_TRY(e->q.ensure(R * 24));
    SVDI_TRY(e->s.ensure(C * 8));
    SVDI_TRY(e->vin64.ensure(9 * 8));
    SVDI_TRY(e->vin32.ensure(9 * 4));
    SVDI_TRY(e->stats.ensure(ST_COUNT * 8));
    SVDI_TRY(e->partial.ensure((size_t)kPartialCap * 9 * 8));
    SVDI_TRY(launch_collapse(e->in_v0r.as<float>(), e->in_v0i.as<float>(), e->in_v3r.as<float>(),
                             e->in_v3i.as<float>(), e->in_f0.as<uint8_t>(), e->in_f3.as<uint8_t>(),
                             e->in_w0.as<float>(), e->in_w3.as<float>(), e->vr.as<float>(), e->vi.as<float>(),
                             (long long)n, st));
    SVDI_TRY(launch_preprocess(e->in_uvw.as<float>(), e->in_freq.as<float>(), (long long)R, (long long)C,
                               h->array_center_x, e->partial.as<double>(), kPartialCap, e->vin64.as<double>(),
                               e->vin32.as<float>(), e->q.as<double>(), e->s.as<double>(), e->stats.as<double>(),
                               st));
    if (want_bin) {
        SVDI_TRY(e->bin_out.ensure(n * 12));
        SVDI_TRY(launch_expand_bin(e->q.as<double>(), e->s.as<double>(), (long long)R, (long long)C,
                                   e->bin_out.as<float>(), st));
    }
    SVDI_CUDA(cudaStreamSynchronize(st));
    // hand the buffers over to the descriptor; the engine keeps ownership of the rest
    dev->d_vis_real = e->vr.as<float>();
    dev->d_vis_imag = e->vi.as<float>();
    dev->d_vin = e->vin32.as<float>();
    dev->d_bin = want_bin ? e->bin_out.as<float>() : nullptr;
    dev->num_samples = n;
    dev->num_rows = R;
    dev->num_channels = C;
    dev->d_vin64 = e->vin64.as<double>();
    dev->d_q = e->q.as<double>();
    dev->d_s = e->s.as<double>();
    dev->d_stats = e->stats.as<double>();
    auto* in = new svdi_pre_internal{guard.release()};
    dev->internal = in;
    return SVDI_OK;
}

int svdi_fipipe_device(const svdi_device_buffers* dev, float* dirty_image, size_t N, float cell) {
    g_last_error.clear();
    if (!dev || !dev->internal || !dirty_image) {
        set_error("device buffers not initialised by svdi_preprocess_measurement_set");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    SVDI_TRY(check_image_args(N, cell));
    svdi_engine* e = static_cast<svdi_pre_internal*>(dev->internal)->engine;
    std::lock_guard<std::mutex> lk(e->mu);
    SVDI_CUDA(cudaSetDevice(e->device));
    SVDI_TRY(e->image.ensure(N * N * 4));
    SampleSource src{};
    src.q = dev->d_q;
    src.s = dev->d_s;
    src.R = (long long)dev->num_rows;
    src.vr = dev->d_vis_real;
    src.vi = dev->d_vis_imag;
    src.n = (long long)dev->num_samples;
    SVDI_TRY(image_core(e, false, src, (long long)N, cell, e->image.as<float>()));
    SVDI_CUDA(cudaMemcpyAsync(dirty_image, e->image.p, N * N * 4, cudaMemcpyDeviceToHost, e->stream));
    SVDI_CUDA(cudaStreamSynchronize(e->stream));
    SVDI_TRY(finish_pending(e));
    return SVDI_OK;
}

int svdi_copy_to_host(void* host_dst, const void* device_src, size_t bytes) {
    g_last_error.clear();
    if (!host_dst || !device_src) {
        set_error("null pointer argument");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    SVDI_CUDA(cudaMemcpy(host_dst, device_src, bytes, cudaMemcpyDeviceToHost));
    return SVDI_OK;
}

void svdi_free_device_buffers(svdi_device_buffers* dev) {
    if (!dev) return;
    if (dev->internal) {
        auto* in = static_cast<svdi_pre_internal*>(dev->internal);
        delete in->engine;
        delete in;
    }
    memset(dev, 0, sizeof(*dev));
}

}  // extern "C"

// C++-linkage archive entry, exactly archive/pipe_interface.cpp:8.
int FIpipe(float* Visreal, float* Visimag, float* Bin, float* Vin, float* dirty_image, size_t num_baselines,
           size_t image_size, float cell_size) {
    return svdi_fipipe(Visreal, Visimag, Bin, Vin, dirty_image, num_baselines, image_size, cell_size);
}

// ---------------------------------------------------------------------------------------------
// Batches: many snapshots imaged by one CUDA-graph launch (no counterpart in the reference,
// whose driver images one snapshot per process, SVDIntegratedImager.cu:1773-1854).
// ---------------------------------------------------------------------------------------------
struct svdi_batch {
    svdi_engine* e = nullptr;
    std::vector<svdi_host_ms> snaps;
    std::vector<svdi::ExecPlan> plans;
    size_t N = 0;
    float cell = 0.0f;
    float* d_images = nullptr;
    svdi::DevBuf status;  // per snapshot (chained graph) or per gridder launch (wide): give-up status
    int num_status = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t last_stream = nullptr;
    // Wide batch: every stage over all snapshots at once (batch-owned buffers, one gridder launch
    // per Chebyshev order over the keys of all snapshots, one FFT over all moment planes).
    bool wide = false;
    svdi::DevBuf vr, vi, q, s, vin64, vin32, stats, partial, counts, offsets, cursor, keymax, chunk_key,
        kb_offsets, rec, rec_s, planes, dropped, work, corr;
    svdi::FftPlan fft;
    std::vector<cudaStream_t> lanes;
    std::vector<cudaEvent_t> lane_ev;
    cudaEvent_t ev_fork = nullptr;
    // Split batch (svdi_batch_create with many snapshots): the second half of the snapshots is a
    // batch of its own on an engine this batch owns, launched on `split_stream` beside this half,
    // so that one half's FFT and recombinations overlap the other half's gridding.
    svdi_batch* second = nullptr;
    svdi_engine* own_engine = nullptr;
    size_t first_count = 0;
    cudaStream_t split_stream = nullptr;
    cudaEvent_t ev_split_fork = nullptr, ev_split_join = nullptr;
    ~svdi_batch() {
        if (second) delete second;  // releases own_engine's binding
        if (own_engine) svdi_engine_destroy(own_engine);
        if (e) cudaSetDevice(e->device);
        if (ev_split_fork) cudaEventDestroy(ev_split_fork);
        if (ev_split_join) cudaEventDestroy(ev_split_join);
        if (split_stream) cudaStreamDestroy(split_stream);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        svdi::destroy_fft_plan(fft);
        for (auto ev : lane_ev) cudaEventDestroy(ev);
        for (auto st : lanes) cudaStreamDestroy(st);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (e) e->batch_bound = false;
    }
};

namespace svdi {
namespace {

// Grid geometry of an imaging call (the same rules as image_core).
GridGeom geom_for(const svdi_options& o, long long N, float cell_f, int K, bool use_tc) {
    GridGeom g{};
    g.G = grid_size(N, o.sigma);
    g.gmin = -(g.G / 2);
    g.gmax = (g.G - 1) / 2;
    g.W = o.support;
    if (use_tc) {
        tc_tiles(o.gridder, g);
    } else {
        g.T = o.tile ? o.tile : (K == 1 ? 64 : 32);
        g.ntile = (int)((g.G + g.T - 1) / g.T);
        g.T2 = g.T;
        g.ntile2 = g.ntile;
    }
    g.edge_mode = o.edge_mode;
    g.coord_mode = o.coord_mode;
    g.scale = (double)cell_f * (double)g.G;
    g.scale32 = cell_f * (float)g.G;
    return g;
}

// The wide batch's device work, captured into b->graph from the engine's stream. Snapshots are
// grouped by Chebyshev order; group g owns a contiguous range of tile keys (its snapshots' keys in
// turn, slabs first), of global slabs and of moment planes. Per snapshot: collapse, rotation and
// histogram (into its key range of one counts array), on kLanes side streams so that the small
// per-snapshot kernels overlap; then one scan over all keys; the scatters (side streams); one
// gridder launch per group walking the chunks of all its snapshots' records from a device counter;
// one cuFFT execution over all planes; the recombination of every snapshot into its image.
// Returns SVDI_ERR_UNSUPPORTED (nothing captured) when a snapshot's plan splits its slabs over
// several FFT batches or all planes do not fit in half of the free device memory.
int wide_capture(svdi_batch* b) {
    svdi_engine* e = b->e;
    const svdi_options& o = e->opt;
    const size_t B = b->snaps.size();
    const long long N = (long long)b->N;
    const float cell_f = b->cell;
    for (const auto& p : b->plans)
        if ((int)p.bslabs < p.sp.nslab) return SVDI_ERR_UNSUPPORTED;
    const bool tc_opt = is_tc_gridder(o.gridder);
    // groups of equal Chebyshev order, in order of first appearance
    std::vector<int> group_k;
    std::vector<int> group_of(B);
    for (size_t s = 0; s < B; ++s) {
        const int K = b->plans[s].sp.K;
        auto it = std::find(group_k.begin(), group_k.end(), K);
        group_of[s] = (int)(it - group_k.begin());
        if (it == group_k.end()) group_k.push_back(K);
    }
    const int NG = (int)group_k.size();
    struct Group {
        int K = 1;
        bool tc = false;
        GridGeom g{};
        long long key_lo = 0, key_hi = 0, slab_lo = 0, plane_lo = 0;
    };
    std::vector<Group> groups(NG);
    std::vector<long long> key_base(B), plane_base(B), samp_off(B), row_off(B), chan_off(B);
    long long nkeys = 0, nplanes = 0, ntot = 0, rtot = 0, ctot = 0;
    bool need_s = false, any_tc = false;
    for (int gi = 0; gi < NG; ++gi) {
        Group& G = groups[gi];
        G.K = group_k[gi];
        G.tc = tc_opt && (G.K == 1 || o.gridder == SVDI_GRIDDER_TC_I8) && o.support <= 8;
        G.g = geom_for(o, N, cell_f, G.K, G.tc);
        // the gridders take a key's slab as key / (tiles per slab): start the group on a multiple of
        // its tiles per slab (the keys skipped stay empty)
        const long long tiles2 = (long long)G.g.ntile * G.g.ntile2;
        nkeys = (nkeys + tiles2 - 1) / tiles2 * tiles2;
        G.key_lo = nkeys;
        G.slab_lo = nkeys / tiles2;
        G.plane_lo = nplanes;
        for (size_t s = 0; s < B; ++s) {
            if (group_of[s] != gi) continue;
            const SlabParams& sp = b->plans[s].sp;
            key_base[s] = nkeys;
            plane_base[s] = nplanes;
            nkeys += (long long)sp.nslab * G.g.ntile * G.g.ntile2;
            nplanes += (long long)sp.nslab * sp.K;
        }
        G.key_hi = nkeys;
        need_s = need_s || G.K > 1;
        any_tc = any_tc || G.tc;
    }
    for (size_t s = 0; s < B; ++s) {
        samp_off[s] = ntot;
        row_off[s] = rtot;
        chan_off[s] = ctot;
        ntot += (long long)b->snaps[s].num_samples;
        rtot += (long long)b->snaps[s].num_rows;
        ctot += (long long)b->snaps[s].num_channels;
    }
    if (nkeys > (1LL << 28) || ntot >= (1LL << 32) - 1) return SVDI_ERR_UNSUPPORTED;
    const long long Gs = groups[0].g.G, GG = Gs * Gs;
    size_t free_b = 0, total_b = 0;
    SVDI_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t plane_bytes = (size_t)nplanes * (size_t)GG * sizeof(float2);
    if (plane_bytes > free_b / 2) return SVDI_ERR_UNSUPPORTED;

    const size_t NN = (size_t)N * (size_t)N;
    SVDI_TRY(b->vr.ensure((size_t)ntot * 4));
    SVDI_TRY(b->vi.ensure((size_t)ntot * 4));
    SVDI_TRY(b->q.ensure((size_t)rtot * 24));
    SVDI_TRY(b->s.ensure((size_t)ctot * 8));
    SVDI_TRY(b->vin64.ensure(B * 9 * 8));
    SVDI_TRY(b->vin32.ensure(B * 9 * 4));
    SVDI_TRY(b->stats.ensure(B * ST_COUNT * 8));
    const int L = (int)std::min<size_t>(8, B);
    SVDI_TRY(b->partial.ensure((size_t)L * kPartialCap * 9 * 8));
    SVDI_TRY(b->counts.ensure((size_t)nkeys * 4));
    SVDI_TRY(b->offsets.ensure((size_t)(nkeys + 1) * 4));
    SVDI_TRY(b->cursor.ensure((size_t)nkeys * 4));
    SVDI_TRY(b->keymax.ensure((size_t)nkeys * 4));
    SVDI_TRY(b->chunk_key.ensure(((size_t)std::max<long long>(ntot, 1) / kGridChunk + 2) * 4));
    if (any_tc) SVDI_TRY(b->kb_offsets.ensure((size_t)(nkeys + 1) * 4));
    SVDI_TRY(b->rec.ensure((size_t)std::max<long long>(ntot, 1) * sizeof(SampleRec)));
    if (need_s) SVDI_TRY(b->rec_s.ensure((size_t)std::max<long long>(ntot, 1) * 4));
    SVDI_TRY(b->planes.ensure(plane_bytes));
    SVDI_TRY(b->dropped.ensure(B * 2 * 8));
    SVDI_TRY(b->work.ensure(4 * sizeof(unsigned int) * (size_t)(NG + 1)));
    SVDI_TRY(b->status.ensure((size_t)NG * 4 * sizeof(unsigned int)));
    b->num_status = NG;
    // correction table and ES polynomial of this geometry (the table copied: the batch owns it)
    SVDI_TRY(ensure_corr(e, N, Gs, o.support, o.beta));
    SVDI_TRY(b->corr.ensure((size_t)(N / 2 + 1) * 4));
    SVDI_CUDA(cudaMemcpyAsync(b->corr.p, e->corr.p, (size_t)(N / 2 + 1) * 4, cudaMemcpyDeviceToDevice, e->stream));
    if (e->poly_W != o.support || e->poly_beta != o.beta) {
        build_es_poly(o.support, o.beta, &e->poly);
        e->poly_W = o.support;
        e->poly_beta = o.beta;
    }
    SVDI_TRY(make_fft_plan(Gs, N, (int)nplanes, e->stream, b->fft));
    int prio_low = 0, prio_high = 0;
    SVDI_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    for (int l = 0; l < L; ++l) {
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        SVDI_CUDA(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio_low));
        b->lanes.push_back(st);
        SVDI_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        b->lane_ev.push_back(ev);
    }
    SVDI_CUDA(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
    SVDI_CUDA(cudaStreamSynchronize(e->stream));

    cudaStream_t st = e->stream;
    auto fork = [&]() -> int {
        SVDI_CUDA(cudaEventRecord(b->ev_fork, st));
        for (int l = 0; l < L; ++l) SVDI_CUDA(cudaStreamWaitEvent(b->lanes[l], b->ev_fork, 0));
        return SVDI_OK;
    };
    auto join = [&]() -> int {
        for (int l = 0; l < L; ++l) {
            SVDI_CUDA(cudaEventRecord(b->lane_ev[l], b->lanes[l]));
            SVDI_CUDA(cudaStreamWaitEvent(st, b->lane_ev[l], 0));
        }
        return SVDI_OK;
    };
    auto source = [&](size_t s) {
        SampleSource src{};
        src.q = b->q.as<double>() + 3 * row_off[s];
        src.s = b->s.as<double>() + chan_off[s];
        src.R = (long long)b->snaps[s].num_rows;
        src.vr = b->vr.as<float>() + samp_off[s];
        src.vi = b->vi.as<float>() + samp_off[s];
        src.n = (long long)b->snaps[s].num_samples;
        src.inv_det = b->plans[s].inv_det;
        src.nonfinite = b->dropped.as<unsigned long long>() + 2 * s + 1;
        return src;
    };
    unsigned int* vmax = b->work.as<unsigned int>() + 4 * NG + 1;  // max |record value| for the TC gridder

    SVDI_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = [&]() -> int {
        SVDI_CUDA(cudaMemsetAsync(b->counts.p, 0, (size_t)nkeys * 4, st));
        SVDI_CUDA(cudaMemsetAsync(b->keymax.p, 0, (size_t)nkeys * 4, st));
        SVDI_CUDA(cudaMemsetAsync(b->dropped.p, 0, B * 2 * 8, st));
        SVDI_CUDA(cudaMemsetAsync(b->status.p, 0, (size_t)NG * 4 * sizeof(unsigned int), st));
        SVDI_CUDA(cudaMemsetAsync(vmax, 0, sizeof(unsigned int), st));
        SVDI_CUDA(cudaMemsetAsync(b->d_images, 0, B * NN * 4, st));
        // per snapshot: collapse, rotation, histogram
        SVDI_TRY(fork());
        for (size_t s = 0; s < B; ++s) {
            cudaStream_t ls = b->lanes[s % L];
            const svdi_host_ms& d = b->snaps[s];
            const Group& G = groups[group_of[s]];
            SVDI_TRY(launch_collapse(d.vis0_real, d.vis0_imag, d.vis3_real, d.vis3_imag, d.flag0, d.flag3, d.weight0,
                                     d.weight3, b->vr.as<float>() + samp_off[s], b->vi.as<float>() + samp_off[s],
                                     (long long)d.num_samples, ls));
            SVDI_TRY(launch_preprocess(d.uvw, d.frequencies_hz, (long long)d.num_rows, (long long)d.num_channels,
                                       d.array_center_x, b->partial.as<double>() + (size_t)(s % L) * kPartialCap * 9,
                                       kPartialCap, b->vin64.as<double>() + 9 * s, b->vin32.as<float>() + 9 * s,
                                       b->q.as<double>() + 3 * row_off[s], b->s.as<double>() + chan_off[s],
                                       b->stats.as<double>() + ST_COUNT * s, ls));
            const SlabParams& sp = b->plans[s].sp;
            const int nk = (int)((long long)sp.nslab * G.g.ntile * G.g.ntile2);
            SVDI_TRY(launch_histogram(source(s), G.g, sp, b->counts.as<unsigned int>() + key_base[s], nk,
                                      b->dropped.as<unsigned long long>() + 2 * s, ls));
        }
        SVDI_TRY(join());
        SVDI_TRY(launch_scan(b->counts.as<unsigned int>(), (int)nkeys, b->offsets.as<unsigned int>(),
                             b->cursor.as<unsigned int>(), st, any_tc ? b->kb_offsets.as<unsigned int>() : nullptr,
                             kTcKBlock, b->chunk_key.as<unsigned int>(), kGridChunk));
        // per snapshot: scatter into the global record order
        SVDI_TRY(fork());
        for (size_t s = 0; s < B; ++s) {
            cudaStream_t ls = b->lanes[s % L];
            const Group& G = groups[group_of[s]];
            const SlabParams& sp = b->plans[s].sp;
            const int nk = (int)((long long)sp.nslab * G.g.ntile * G.g.ntile2);
            SVDI_TRY(launch_scatter(source(s), G.g, sp, b->cursor.as<unsigned int>() + key_base[s], nk,
                                    b->rec.as<SampleRec>(), need_s ? b->rec_s.as<float>() : nullptr,
                                    G.tc ? vmax : nullptr, ls, b->keymax.as<unsigned int>() + key_base[s]));
        }
        SVDI_TRY(join());
        // one gridder launch per Chebyshev order over the records of all its snapshots
        SVDI_CUDA(cudaMemsetAsync(b->planes.p, 0, plane_bytes, st));
        for (int gi = 0; gi < NG; ++gi) {
            const Group& G = groups[gi];
            if (G.key_hi == G.key_lo) continue;
            SlabParams sg{};
            sg.K = G.K;
            sg.nslab = (int)((G.key_hi - G.key_lo) / ((long long)G.g.ntile * G.g.ntile2));
            float2* pl = b->planes.as<float2>() + G.plane_lo * GG;
            unsigned int* stw = b->status.as<unsigned int>() + 4 * gi;
            if (G.tc && o.gridder == SVDI_GRIDDER_TC_I8) {
                // status in [0], work counter in [2]; per-key scales from the scatter's maxima
                SVDI_TRY(launch_grid_i8(b->rec.as<SampleRec>(), need_s ? b->rec_s.as<float>() : nullptr,
                                        b->offsets.as<unsigned int>(), b->kb_offsets.as<unsigned int>(), (int)nkeys,
                                        (int)G.key_lo, (int)G.key_hi, (int)G.slab_lo, G.K, G.g, e->poly, pl,
                                        b->keymax.as<unsigned int>(), stw, e->sm_count, st));
            } else if (G.tc) {
                // the TC gridder keeps its status in [0], reads max |v| from the pointer and counts work in [2]
                SVDI_TRY(launch_grid_tc(b->rec.as<SampleRec>(), b->offsets.as<unsigned int>(),
                                        b->kb_offsets.as<unsigned int>(), (int)nkeys, (int)G.key_lo, (int)G.key_hi,
                                        (int)G.slab_lo, G.g, e->poly, pl, vmax, stw, e->sm_count, st,
                                        o.gridder == SVDI_GRIDDER_TC_BF16));
            } else {
                SVDI_TRY(launch_grid_fp32(b->rec.as<SampleRec>(), need_s ? b->rec_s.as<float>() : nullptr,
                                          b->offsets.as<unsigned int>(), b->chunk_key.as<unsigned int>(),
                                          b->keymax.as<unsigned int>(), b->work.as<unsigned int>() + gi, (int)nkeys,
                                          (int)G.key_lo, (int)G.key_hi, (int)G.slab_lo, G.g, sg, e->poly, pl,
                                          e->sm_count, st));
            }
        }
        SVDI_TRY(exec_fft(b->fft, b->planes.as<cufftComplex>(), (int)nplanes));
        for (size_t s = 0; s < B; ++s) {
            const Group& G = groups[group_of[s]];
            SVDI_TRY(launch_recombine(b->planes.as<float2>() + plane_base[s] * GG, G.g, N, (double)cell_f,
                                      b->vin64.as<double>() + 9 * s, b->plans[s].sp, b->corr.as<float>(),
                                      1.0 / (double)b->snaps[s].num_samples, o.reprojection, o.presplat,
                                      b->d_images + s * NN, st, nullptr, true, nullptr,
                                      b->dropped.as<unsigned long long>() + 2 * s + 1));
        }
        return SVDI_OK;
    }();
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (rc != SVDI_OK) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return rc == SVDI_ERR_UNSUPPORTED ? SVDI_ERR_INTERNAL : rc;
    }
    if (ce != cudaSuccess || !graph) {
        set_error(std::string("graph capture failed: ") + cudaGetErrorString(ce));
        cudaGetLastError();
        return SVDI_ERR_CUDA;
    }
    b->graph = graph;
    SVDI_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->wide = true;
    return SVDI_OK;
}

}  // namespace
}  // namespace svdi

extern "C" {

namespace {

int batch_create_one(svdi_engine* e, const svdi_host_ms* snapshots, size_t num_snapshots, size_t image_size,
                     float cell_size, float* d_images, svdi_batch** out) {
    using namespace svdi;
    g_last_error.clear();
    if (!e || !snapshots || !d_images || !out) {
        set_error("null argument");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (num_snapshots == 0) {
        set_error("a batch needs at least one snapshot");
        return SVDI_ERR_EMPTY_INPUT;
    }
    SVDI_TRY(check_image_args(image_size, cell_size));
    for (size_t s = 0; s < num_snapshots; ++s) SVDI_TRY(check_ms(&snapshots[s]));
    if (e->opt.keep_grid) {
        set_error("batches do not keep grids: create the engine with keep_grid = 0");
        return SVDI_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lk(e->mu);
    if (e->batch_bound) {
        set_error("this engine already holds a batch; destroy it first");
        return SVDI_ERR_UNSUPPORTED;
    }
    SVDI_CUDA(cudaSetDevice(e->device));
    std::unique_ptr<svdi_batch> b(new svdi_batch());
    b->snaps.assign(snapshots, snapshots + num_snapshots);
    b->plans.resize(num_snapshots);
    b->N = image_size;
    b->cell = cell_size;
    b->d_images = d_images;
    SVDI_TRY(b->status.ensure(num_snapshots * sizeof(unsigned int)));
    const size_t NN = image_size * image_size;
    // plan: one ordinary pass per snapshot records its host decisions and sizes every buffer
    for (size_t s = 0; s < num_snapshots; ++s)
        SVDI_TRY(main_path_device(e, &b->snaps[s], image_size, cell_size, d_images + s * NN, nullptr, &b->plans[s]));
    SVDI_CUDA(cudaStreamSynchronize(e->stream));
    SVDI_TRY(finish_pending(e));
    b->e = e;
    // every stage over all snapshots at once; when that is not possible (a snapshot's slabs span
    // several FFT batches, or the planes of all snapshots do not fit), the chained graph below
    const int wrc = wide_capture(b.get());
    if (wrc == SVDI_OK) {
        e->batch_bound = true;
        *out = b.release();
        return SVDI_OK;
    }
    if (wrc != SVDI_ERR_UNSUPPORTED) {
        b->e = nullptr;
        return wrc;
    }
    b->e = nullptr;
    b->num_status = (int)num_snapshots;
    // capture the device work of every snapshot with its plan
    SVDI_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    int rc = SVDI_OK;
    for (size_t s = 0; s < num_snapshots && rc == SVDI_OK; ++s)
        rc = main_path_device(e, &b->snaps[s], image_size, cell_size, d_images + s * NN, &b->plans[s], nullptr,
                              b->status.as<unsigned int>() + s);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(e->stream, &graph);
    if (rc != SVDI_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (ce != cudaSuccess || !graph) {
        set_error(std::string("graph capture failed: ") + cudaGetErrorString(ce));
        cudaGetLastError();
        return SVDI_ERR_CUDA;
    }
    b->graph = graph;
    SVDI_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->e = e;
    e->batch_bound = true;
    *out = b.release();
    return SVDI_OK;
}

// Batches of at least this many snapshots are split in two halves (the measured configuration B:
// 5,480 snapshots/s as one graph, 5,732/s as two graphs side by side).
constexpr size_t kSplitBatchMin = 16;

}  // namespace

int svdi_batch_create(svdi_engine* e, const svdi_host_ms* snapshots, size_t num_snapshots, size_t image_size,
                      float cell_size, float* d_images, svdi_batch** out) {
    using namespace svdi;
    if (e && snapshots && d_images && out && num_snapshots >= kSplitBatchMin && !e->opt.keep_grid &&
        !e->batch_bound && check_image_args(image_size, cell_size) == SVDI_OK) {
        // two halves on two engines (the second owned by the batch), each captured as a wide batch;
        // when either half cannot be a wide batch, one batch of all the snapshots below
        svdi_engine* e2 = nullptr;
        if (svdi_engine_create(&e->opt, &e2) == SVDI_OK) {
            const size_t h = num_snapshots / 2;
            svdi_batch* b1 = nullptr;
            svdi_batch* b2 = nullptr;
            int rc = batch_create_one(e, snapshots, h, image_size, cell_size, d_images, &b1);
            if (rc == SVDI_OK)
                rc = batch_create_one(e2, snapshots + h, num_snapshots - h, image_size, cell_size,
                                      d_images + h * image_size * image_size, &b2);
            if (rc == SVDI_OK && b1->wide && b2->wide &&
                cudaStreamCreateWithFlags(&b1->split_stream, cudaStreamNonBlocking) == cudaSuccess &&
                cudaEventCreateWithFlags(&b1->ev_split_fork, cudaEventDisableTiming) == cudaSuccess &&
                cudaEventCreateWithFlags(&b1->ev_split_join, cudaEventDisableTiming) == cudaSuccess) {
                b1->second = b2;
                b1->own_engine = e2;
                b1->first_count = h;
                *out = b1;
                g_last_error.clear();
                return SVDI_OK;
            }
            cudaGetLastError();
            if (b2) svdi_batch_destroy(b2);
            if (b1) svdi_batch_destroy(b1);
            svdi_engine_destroy(e2);
        }
    }
    return batch_create_one(e, snapshots, num_snapshots, image_size, cell_size, d_images, out);
}

int svdi_batch_launch(svdi_batch* b, void* cuda_stream) {
    using namespace svdi;
    g_last_error.clear();
    if (!b || !b->exec) {
        set_error("null batch");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    SVDI_CUDA(cudaSetDevice(b->e->device));
    cudaStream_t st = cuda_stream ? (cudaStream_t)cuda_stream : b->e->stream;
    if (b->second) {  // the second half on its own stream, both ordered after `st`'s earlier work
        SVDI_CUDA(cudaEventRecord(b->ev_split_fork, st));
        SVDI_CUDA(cudaStreamWaitEvent(b->split_stream, b->ev_split_fork, 0));
        SVDI_CUDA(cudaGraphLaunch(b->second->exec, b->split_stream));
        SVDI_CUDA(cudaGraphLaunch(b->exec, st));
        SVDI_CUDA(cudaEventRecord(b->ev_split_join, b->split_stream));
        SVDI_CUDA(cudaStreamWaitEvent(st, b->ev_split_join, 0));
        b->second->last_stream = b->split_stream;
    } else {
        SVDI_CUDA(cudaGraphLaunch(b->exec, st));
    }
    b->last_stream = st;
    return SVDI_OK;
}

int svdi_batch_check(svdi_batch* b) {
    using namespace svdi;
    g_last_error.clear();
    if (!b) {
        set_error("null batch");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    SVDI_CUDA(cudaSetDevice(b->e->device));
    if (b->last_stream) SVDI_CUDA(cudaStreamSynchronize(b->last_stream));
    if (b->second) SVDI_TRY(svdi_batch_check(b->second));
    if (b->wide) {  // one status block of 4 words per gridder launch
        std::vector<unsigned int> st((size_t)b->num_status * 4);
        SVDI_CUDA(cudaMemcpy(st.data(), b->status.p, st.size() * sizeof(unsigned int), cudaMemcpyDeviceToHost));
        for (int gi = 0; gi < b->num_status; ++gi)
            if (st[4 * gi]) {
                set_error("gridder launch " + std::to_string(gi) + ": the tensor-core gridder gave up waiting (status " +
                          std::to_string(st[4 * gi]) + "); the batch's images are incomplete");
                return SVDI_ERR_INTERNAL;
            }
        return SVDI_OK;
    }
    std::vector<unsigned int> st(b->snaps.size());
    SVDI_CUDA(cudaMemcpy(st.data(), b->status.p, st.size() * sizeof(unsigned int), cudaMemcpyDeviceToHost));
    for (size_t s = 0; s < st.size(); ++s)
        if (st[s]) {
            set_error("snapshot " + std::to_string(s) + ": the tensor-core gridder gave up waiting (status " +
                      std::to_string(st[s]) + "); its image is incomplete");
            return SVDI_ERR_INTERNAL;
        }
    return SVDI_OK;
}

int svdi_batch_plan(const svdi_batch* b, size_t index, int* num_slabs, int* num_terms) {
    using namespace svdi;
    if (b && b->second && index >= b->first_count) return svdi_batch_plan(b->second, index - b->first_count, num_slabs, num_terms);
    if (!b || index >= b->plans.size()) {
        set_error("bad batch or snapshot index");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    if (num_slabs) *num_slabs = b->plans[index].sp.nslab;
    if (num_terms) *num_terms = b->plans[index].sp.K;
    return SVDI_OK;
}

int svdi_batch_mode(const svdi_batch* b) {
    if (!b) {
        svdi::set_error("null batch");
        return -SVDI_ERR_INVALID_ARGUMENT;
    }
    return (b->wide && (!b->second || b->second->wide)) ? 1 : 0;
}

void svdi_batch_destroy(svdi_batch* b) { delete b; }

int svdi_engine_dft_pixels(svdi_engine* e, const int64_t* px, const int64_t* py, size_t npix, double* out) {
    using namespace svdi;
    g_last_error.clear();
    if (!e || !px || !py || !out) {
        set_error("null argument");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    if (npix == 0) return SVDI_OK;
    if (npix > 65536) {
        set_error("at most 65536 pixels per call");
        return SVDI_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lk(e->mu);
    if (!e->have_last) {
        set_error("no image has been made with this engine yet");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    const long long N = e->last_N;
    for (size_t p = 0; p < npix; ++p)
        if (px[p] < 0 || py[p] < 0 || px[p] >= N || py[p] >= N) {
            set_error("pixel index outside the image");
            return SVDI_ERR_INVALID_ARGUMENT;
        }
    SVDI_CUDA(cudaSetDevice(e->device));
    cudaStream_t st = e->stream;
    SVDI_TRY(e->probe.ensure(npix * 3 * sizeof(long long)));
    long long* d_px = e->probe.as<long long>();
    long long* d_py = d_px + npix;
    double* d_acc = reinterpret_cast<double*>(d_py + npix);
    SVDI_CUDA(cudaMemcpyAsync(d_px, px, npix * 8, cudaMemcpyHostToDevice, st));
    SVDI_CUDA(cudaMemcpyAsync(d_py, py, npix * 8, cudaMemcpyHostToDevice, st));
    SVDI_CUDA(cudaMemsetAsync(d_acc, 0, npix * 8, st));
    SVDI_TRY(launch_dft_probe(e->last_src, e->last_g, e->last_sp, e->vin64.as<double>(), N, e->last_cell, d_px,
                              d_py, (int)npix, d_acc, e->sm_count, st));
    std::vector<double> acc(npix);
    SVDI_CUDA(cudaMemcpyAsync(acc.data(), d_acc, npix * 8, cudaMemcpyDeviceToHost, st));
    SVDI_CUDA(cudaStreamSynchronize(st));
    const double* V = e->last.vin;
    const double inv_det = 1.0 / std::fabs(V[0] * V[4] - V[1] * V[3]);
    const double cell = e->last_cell;
    for (size_t p = 0; p < npix; ++p) {
        const double t1 = cell * (double)(py[p] - N / 2), t2 = cell * (double)(px[p] - N / 2);
        const double ra = 1.0 - (t1 + V[2]) * (t1 + V[2]) - (t2 + V[5]) * (t2 + V[5]);
        out[p] = ra < 0.0 ? std::nan("") : std::fabs(acc[p] * inv_det) / (double)e->last_src.n;
    }
    return SVDI_OK;
}

}  // extern "C"
