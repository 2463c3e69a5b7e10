// Allocation-free tile binning.
//
// Some callers cannot call cudaMalloc once they are running: a correlator's real-time loop that
// reserves all of its device memory at start-up and must never stall on the allocator, or a host
// framework that owns the device's memory pool and forbids outside allocations. For them,
// svdi_bin_samples_noalloc bins samples into the caller's output buffers and keeps its own
// scratch (per-key counters, per-key write cursors, the dropped-sample counter) in the
// file-scope device array below, which every GPU that loads this library holds until the process
// exits. It runs the same histogram / scan / scatter kernels as the engine's binning.
#include "svdi_internal.cuh"

#include <mutex>

namespace svdi {
namespace {

constexpr int kNoallocMaxKeys = SVDI_NOALLOC_MAX_KEYS;
constexpr int kMaxDevices = 64;

// [0, K): key counts; [K, 2K): write cursors; [2K, 2K + 2): 64-bit dropped-sample counter.
static __device__ __align__(256) unsigned int g_noalloc_scratch[2 * kNoallocMaxKeys + 4];

std::mutex g_scratch_mu;
unsigned int* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array for the current device; resolved once per device and kept
// for the life of the process (a cudaDeviceReset of that device would leave it stale).
int scratch_for_current_device(unsigned int** out) {
    int dev = 0;
    SVDI_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device ordinal out of range for the allocation-free entry point");
        return SVDI_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        SVDI_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch_ptr[dev] = static_cast<unsigned int*>(p);
    }
    *out = g_scratch_ptr[dev];
    return SVDI_OK;
}

}  // namespace
}  // namespace svdi

extern "C" int svdi_bin_samples_noalloc(const float* d_bin, const float* d_vis_real, const float* d_vis_imag,
                                        size_t num_samples, size_t image_size, float cell_size, int tile,
                                        float inv_det, void* d_records, uint32_t* d_offsets,
                                        size_t offsets_capacity, void* cuda_stream) {
    using namespace svdi;
    set_error("");  // a successful call leaves no message from an earlier failed one
    if (!d_bin || !d_vis_real || !d_vis_imag || !d_records || !d_offsets) {
        set_error("null pointer argument");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    if (num_samples == 0) {
        set_error("num_samples must be greater than zero");
        return SVDI_ERR_EMPTY_INPUT;
    }
    if (num_samples >= (1ULL << 32) - 1) {
        set_error("more than 2^32 - 2 samples per call");
        return SVDI_ERR_UNSUPPORTED;
    }
    if (image_size == 0 || image_size > 65536 || !(cell_size > 0.0f)) {
        set_error("Image_Size must be in 1..65536 and Cell_Size greater than zero");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    if (tile != 32 && tile != 64) {
        set_error("tile must be 32 or 64");
        return SVDI_ERR_UNSUPPORTED;
    }
    GridGeom g{};
    g.G = (3 * (long long)image_size + 1) / 2;  // ceil(1.5 N), SVDIntegratedImager.cu:1510
    g.gmin = -(g.G / 2);
    g.gmax = (g.G - 1) / 2;
    g.W = 8;
    g.T = tile;
    g.ntile = (int)((g.G + g.T - 1) / g.T);
    g.T2 = tile;
    g.ntile2 = g.ntile;
    g.edge_mode = SVDI_EDGE_CLIP;
    g.coord_mode = SVDI_COORD_FP64;
    g.scale = (double)cell_size * (double)g.G;
    g.scale32 = cell_size * (float)g.G;
    const long long n_keys = (long long)g.ntile * g.ntile;
    if (n_keys > SVDI_NOALLOC_MAX_KEYS) {
        set_error("ceil(1.5 * image_size / tile)^2 = " + std::to_string(n_keys) +
                  " tile keys exceed the allocation-free limit of " + std::to_string(SVDI_NOALLOC_MAX_KEYS) +
                  "; use a larger tile or the engine API");
        return SVDI_ERR_UNSUPPORTED;
    }
    if (offsets_capacity < (size_t)n_keys + 1) {
        set_error("offsets buffer needs ceil(1.5 * image_size / tile)^2 + 1 entries");
        return SVDI_ERR_INVALID_ARGUMENT;
    }
    unsigned int* scratch = nullptr;
    SVDI_TRY(scratch_for_current_device(&scratch));
    unsigned int* counts = scratch;
    unsigned int* cursor = scratch + kNoallocMaxKeys;
    unsigned long long* dropped = reinterpret_cast<unsigned long long*>(scratch + 2 * kNoallocMaxKeys);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    SlabParams sp{};
    sp.nslab = 1;
    sp.K = 1;
    sp.slab_width = 1.0;
    sp.slab_half = 0.5;
    sp.inv_half = 2.0;
    SampleSource src{};
    src.bin = d_bin;
    src.vr = d_vis_real;
    src.vi = d_vis_imag;
    src.n = (long long)num_samples;
    src.inv_det = inv_det;
    // the array keeps the previous call's contents: counters and the dropped count start at zero
    SVDI_CUDA(cudaMemsetAsync(counts, 0, sizeof(unsigned int) * (size_t)n_keys, st));
    SVDI_CUDA(cudaMemsetAsync(dropped, 0, sizeof(unsigned long long), st));
    SVDI_TRY(launch_histogram(src, g, sp, counts, (int)n_keys, dropped, st));
    SVDI_TRY(launch_scan(counts, (int)n_keys, d_offsets, cursor, st));
    SVDI_TRY(launch_scatter(src, g, sp, cursor, (int)n_keys, static_cast<SampleRec*>(d_records), nullptr, nullptr, st));
    return SVDI_OK;
}
