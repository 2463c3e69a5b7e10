/*
 * svdimager_b200 — B200-native snapshot imager (drop-in for the imaging path of the
 * Transient-Oriented Imager, egbdfX/SVDimager).
 *
 * C ABI: plain pointers and sizes, status codes, no exceptions across the boundary.
 * Reference files cited by path relative to the reference project root:
 *   SVDIntegratedImager.cu (main path), archive/FIPkernels.cu and archive/pipe_interface.cpp
 *   (archive path).
 *
 * Thread safety: every function may be called from any host thread. An engine handle is owned by
 * one caller at a time (calls on one handle serialise on an internal mutex). The process-wide
 * default engine used by FIpipe / svdi_fipipe is guarded the same way.
 */
#ifndef SVDIMAGER_B200_H
#define SVDIMAGER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------ */
#define SVDI_OK 0
#define SVDI_ERR_INVALID_ARGUMENT 1   /* null pointer, zero size, non-positive cell size, ... */
#define SVDI_ERR_EMPTY_INPUT 2        /* zero samples (SVDIntegratedImager.cu:640-642)          */
#define SVDI_ERR_CUDA 3               /* a CUDA runtime call failed                             */
#define SVDI_ERR_CUFFT 4              /* a cuFFT call failed                                    */
#define SVDI_ERR_OUT_OF_MEMORY 5      /* admission refused / device allocation failed          */
#define SVDI_ERR_UNSUPPORTED 6        /* option outside the implemented range                  */
#define SVDI_ERR_INTERNAL 7

/* Message of the last failing call on this host thread ("" when none). */
const char* svdi_last_error(void);

/* ---- archive entry point ----------------------------------------------------------------- */
/*
 * Replaces int FIpipe(float* Visreal, float* Visimag, float* Bin, float* Vin, float* dirty_image,
 *                     size_t num_baselines, size_t image_size, float cell_size)
 * declared at archive/pipe_interface.cpp:8 and defined at archive/FIPkernels.cu:679.
 * All pointers are HOST pointers owned by the caller. Visreal/Visimag: [num_baselines] collapsed
 * visibilities; Bin: [num_baselines][3] rotated baselines in wavelengths (row-major); Vin: 3x3
 * row-major basis; dirty_image: [image_size][image_size] output. num_baselines counts samples
 * (rows x channels). Semantics of the archive path: one w-slab, the smallest Chebyshev order in
 * 1..32 whose sampled Jacobi-Anger error is <= 1e-2 (archive/FIPkernels.cu:287-366), the
 * trigonometric SIN reprojection (archive/FIPkernels.cu:577-677). Returns SVDI_OK (0) or an error
 * status (the reference always returns 0 and reports nothing).
 * The library also exports the C++-linkage symbol `int FIpipe(float*, float*, float*, float*,
 * float*, size_t, size_t, float)` so that archive/pipe_interface.cpp links against it unchanged.
 */
int svdi_fipipe(const float* Visreal, const float* Visimag, const float* Bin, const float* Vin,
                float* dirty_image, size_t num_baselines, size_t image_size, float cell_size);

/* ---- main-path mirror ---------------------------------------------------------------------- */
/* Field for field HostMeasurementSetData (SVDIntegratedImager.cu:39-54). Samples are flattened
 * channel-major: idx = row + chan * num_rows (SVDIntegratedImager.cu:90-92). Host pointers. */
typedef struct svdi_host_ms {
    size_t num_rows;
    size_t num_channels;
    size_t num_samples;            /* must equal num_rows * num_channels */
    const float* uvw;              /* [num_rows][3] metres */
    const float* frequencies_hz;   /* [num_channels] */
    const float* vis0_real;        /* [num_samples] polarisation 0 */
    const float* vis0_imag;
    const float* vis3_real;        /* [num_samples] polarisation 3 */
    const float* vis3_imag;
    const uint8_t* flag0;          /* [num_samples] 1 = flagged */
    const uint8_t* flag3;
    const float* weight0;          /* [num_samples] WEIGHT_SPECTRUM */
    const float* weight3;
    float array_center_x;          /* ARRAY_CENTER.x of the OBSERVATION table (0 = unknown) */
} svdi_host_ms;

/* Mirror of DevicePreprocessBuffers (SVDIntegratedImager.cu:63-69) with the FP64 extensions the
 * B200 path keeps: rotated baselines are separable, r[row + chan*R] = s[chan] * q[row]. */
typedef struct svdi_device_buffers {
    float* d_bin;                  /* [num_samples][3] float rotated baselines (only if requested) */
    float* d_vin;                  /* [9] float basis, row-major                               */
    float* d_vis_real;             /* [num_samples] collapsed visibilities                     */
    float* d_vis_imag;
    size_t num_samples;
    /* extensions */
    size_t num_rows;
    size_t num_channels;
    double* d_vin64;               /* [9] FP64 basis                                            */
    double* d_q;                   /* [num_rows][3] FP64 Vin . uvw_row (metres)                 */
    double* d_s;                   /* [num_channels] FP64 f / c                                 */
    double* d_stats;               /* device scalars: r3 min/max etc. (internal layout)         */
    void* internal;
} svdi_device_buffers;

/* Replaces preprocess_measurement_set_gpu (SVDIntegratedImager.cu:635-853): uploads the host data
 * and computes the FP64 SVD rotation and the flag/weight collapse on the device. want_bin != 0
 * also materialises the float d_bin array of the reference layout. */
int svdi_preprocess_measurement_set(const svdi_host_ms* host, svdi_device_buffers* dev, int want_bin);

/* Replaces FIpipeDevice (SVDIntegratedImager.cu:1498-1761): images preprocessed device buffers into
 * the HOST array dirty_image [image_size][image_size]. Slab + bucket-K semantics
 * (SVDIntegratedImager.cu:926-991, 1577-1603), simplified SIN reprojection
 * (SVDIntegratedImager.cu:1325-1379). */
int svdi_fipipe_device(const svdi_device_buffers* dev, float* dirty_image, size_t image_size,
                       float cell_size);

/* Replaces free_device_preprocess_buffers (SVDIntegratedImager.cu:855-865). */
void svdi_free_device_buffers(svdi_device_buffers* dev);

/* Copies `bytes` from a device array of svdi_device_buffers (or any device pointer of this process)
 * into host memory and waits for the copy; for callers without their own CUDA runtime. No
 * counterpart in the reference (its callers read DevicePreprocessBuffers with cudaMemcpy). */
int svdi_copy_to_host(void* host_dst, const void* device_src, size_t bytes);

/* ---- engine (device-resident, reusable) -------------------------------------------------- */
/* New export: the reference allocates, plans and frees on every call (SVDIntegratedImager.cu:1630-
 * 1676); an engine keeps grids, cuFFT plans, bins and staging buffers resident between calls. */
typedef struct svdi_engine svdi_engine;

#define SVDI_KRULE_BUCKET 0      /* K in {8,16,24,32}, sampled error <= 1e-2 (main path)        */
#define SVDI_KRULE_MIN 1         /* smallest K in 1..32, sampled error <= 1e-2 (archive path)   */
#define SVDI_KRULE_TARGET 2      /* smallest K whose truncation error <= target_error           */
#define SVDI_KRULE_FIXED 3       /* K = fixed_k                                                 */

#define SVDI_EDGE_CLIP 0         /* reference rule: truncate footprints at the grid edge        */
#define SVDI_EDGE_STRICT 1       /* drop samples whose footprint leaves the grid                */

#define SVDI_COORD_FP64 0        /* grid coordinates in FP64                                    */
#define SVDI_COORD_REF32 1       /* the reference's FP32 rounding of Bin * (cell * G)          */

#define SVDI_REPROJ_SII 0        /* simplified SIN deprojection (SVDIntegratedImager.cu)        */
#define SVDI_REPROJ_FIPK 1       /* trigonometric SIN deprojection (archive/FIPkernels.cu)      */

#define SVDI_GRIDDER_FP32 0      /* tile-local FP32 gridder (CUDA cores, shared memory)         */
#define SVDI_GRIDDER_TC 1        /* split-precision tcgen05 tensor-core gridder, FP16 hi + lo   */
#define SVDI_GRIDDER_TC_BF16 2   /* the same with BF16 hi + lo operands (16-bit significand)    */
#define SVDI_GRIDDER_TC_I8 3     /* exact integer tcgen05 gridder: 3-byte digits, int32 sums    */

typedef struct svdi_options {
    int device;                  /* CUDA device ordinal                                        */
    int k_rule;                  /* SVDI_KRULE_*                                               */
    int fixed_k;                 /* for SVDI_KRULE_FIXED                                       */
    double target_error;         /* for SVDI_KRULE_TARGET                                      */
    double target_alpha;         /* slab alpha target; <= 0: SVD_CHEB_TARGET_ALPHA env or 10   */
    int edge_mode;               /* SVDI_EDGE_*                                                */
    int coord_mode;              /* SVDI_COORD_*                                               */
    int reprojection;            /* SVDI_REPROJ_*                                              */
    int support;                 /* ES support W (8 in the reference)                          */
    double beta;                 /* ES beta (15.3704324328 in the reference)                   */
    double sigma;                /* oversampling, G = ceil(sigma N) (1.5 in the reference)     */
    int tile;                    /* gridder tile size (32 or 64); 0 = automatic                 */
    int gridder;                 /* SVDI_GRIDDER_*                                             */
    size_t max_batch_slabs;      /* 0 = SVDIMAGER_MAX_BATCH_SLABS env or the HBM budget        */
    int keep_grid;               /* != 0: keep a copy of the first slab batch's grid before the
                                    FFT for svdi_engine_copy_buffer (testing aid)              */
    int presplat;                /* != 0: output the rotated-frame image R(x, y) before the
                                    reprojection (NaN where the pixel is invalid)              */
} svdi_options;

/* Defaults of the reference main path (bucket K, clip, FP64 coordinates, SIN-simplified). */
void svdi_default_options(svdi_options* opt);

int svdi_engine_create(const svdi_options* opt, svdi_engine** out);
void svdi_engine_destroy(svdi_engine* e);

/* Full main path from HOST snapshot data to a HOST image (uploads, preprocesses, images). */
int svdi_engine_image_host(svdi_engine* e, const svdi_host_ms* host, size_t image_size,
                           float cell_size, float* dirty_image);

/* Device-resident snapshot: the same fields as svdi_host_ms but DEVICE pointers (no upload).
 * The work is ordered on cuda_stream (0: the legacy default stream): it starts after the caller's
 * earlier work on that stream, and later work there sees the image. The call waits once, for the
 * w statistics that size the plan, and returns while the gridding, FFT and recombination still
 * run; svdi_engine_last_stats and the buffer accessors wait for them. */
int svdi_engine_image_device(svdi_engine* e, const svdi_host_ms* dev_ms, size_t image_size,
                             float cell_size, float* d_dirty_image, void* cuda_stream);

/* Archive path on an engine: host pointers, same contract as svdi_fipipe. */
int svdi_engine_fipipe_host(svdi_engine* e, const float* Visreal, const float* Visimag,
                            const float* Bin, const float* Vin, float* dirty_image,
                            size_t num_baselines, size_t image_size, float cell_size);

/* Statistics of the last imaging call on an engine. */
typedef struct svdi_stats {
    size_t num_samples;          /* N_s (the image normalisation)                              */
    size_t num_gridded;          /* samples with at least one footprint cell on the grid       */
    size_t grid_size;            /* G                                                          */
    int num_slabs;               /* w-slabs                                                    */
    int num_terms;               /* Chebyshev terms K                                          */
    int num_planes;              /* num_slabs * K moment planes                                */
    double r3_min, r3_max;       /* range of the third rotated coordinate (wavelengths)        */
    double max_abs_t3;           /* max |t3| over valid pixels                                 */
    size_t valid_pixels;
    double alpha_max;            /* 2 pi max|t3| (r3 range / 2)                                */
    double slab_alpha_max;
    double vin[9];               /* FP64 basis used                                            */
    int tile;                    /* gridder tile rows                                          */
    int tile_cols;               /* gridder tile columns                                       */
    int used_tc;                 /* 1 when the tensor-core gridder ran                         */
    int num_keys;                /* tile keys: num_slabs * ceil(G/T)^2                         */
    double slab_r3_min, slab_width, slab_half;  /* slab geometry used by the gridder           */
    float ms_total;              /* device time of the call (CUDA events)                      */
    float ms_preprocess, ms_bin, ms_grid, ms_fft, ms_image;
} svdi_stats;

int svdi_engine_last_stats(const svdi_engine* e, svdi_stats* out);

/* FP64 direct DFT of the engine's last snapshot at pixels (px[i], py[i]) of its N x N image:
 * |sum_k Re(V_k e^{2 pi i r_k . t})| / |det V| / N_s over the samples the gridder kept (the same
 * inclusion rule, bit for bit), i.e. the rotated-frame image before reprojection (presplat = 1).
 * NaN where the pixel has no valid direction. An accuracy probe for any image, used by the
 * autotuner; no counterpart in the reference (its only check is the image itself). */
int svdi_engine_dft_pixels(svdi_engine* e, const int64_t* px, const int64_t* py, size_t npix, double* out);

/* ---- batches: many snapshots imaged by one CUDA-graph launch ------------------------------
 * No counterpart in the reference, whose driver images one snapshot per process
 * (SVDIntegratedImager.cu:1773-1854). svdi_batch_create images every snapshot once with the
 * engine (recording each snapshot's host decisions: rotation, w range, slab and Chebyshev
 * configuration, and sizing the engine's buffers for the largest), then captures the device work
 * of all snapshots into one CUDA graph. svdi_batch_launch replays it with one cudaGraphLaunch.
 * The graph runs every stage over all snapshots at once where it can ("wide" batch, the batch's
 * own buffers): the small per-snapshot kernels (collapse, rotation, histogram, scatter) side by
 * side on several streams, one scan over the tile keys of all snapshots, one persistent gridder
 * launch per Chebyshev order that walks the records of all its snapshots from a device work
 * counter, one batched cuFFT over all moment planes, and the recombinations. A batch whose
 * snapshots split their w-slabs over several FFT batches, or whose moment planes do not fit in
 * half of the free device memory, is captured snapshot after snapshot instead.
 *   snapshots: device-resident descriptors as for svdi_engine_image_device; their arrays must
 *              stay allocated at the same addresses (refill them in place to image new data of
 *              the same layout, sizes and w range: the recorded plans are reused as they are);
 *   d_images:  num_snapshots x N x N floats on the device, image s at d_images + s N^2.
 * The engine holds one batch at a time and must not image anything else while a launch is in
 * flight (the graph uses its buffers). With 16 or more snapshots the batch runs as two halves: the
 * second half on an engine the batch creates with the same options and owns until
 * svdi_batch_destroy, launched on a stream of its own beside the first half (svdi_batch_launch
 * orders both after the caller's stream and the caller's stream after both). */
typedef struct svdi_batch svdi_batch;
int svdi_batch_create(svdi_engine* e, const svdi_host_ms* snapshots, size_t num_snapshots, size_t image_size,
                      float cell_size, float* d_images, svdi_batch** out);
int svdi_batch_launch(svdi_batch* b, void* cuda_stream);  /* asynchronous; NULL: the engine's stream */
int svdi_batch_check(svdi_batch* b);   /* waits for the last launch; SVDI_ERR_INTERNAL if a tensor-core
                                          gridder wait gave up in any snapshot                        */
int svdi_batch_plan(const svdi_batch* b, size_t index, int* num_slabs, int* num_terms);
int svdi_batch_mode(const svdi_batch* b);  /* 1: wide batch, 0: snapshot after snapshot         */
void svdi_batch_destroy(svdi_batch* b);

/* Intermediate buffers of the last call, for inspection and tests (device-to-host copy). */
#define SVDI_BUF_VIS_REAL 0      /* float [N_s] collapsed visibilities                         */
#define SVDI_BUF_VIS_IMAG 1
#define SVDI_BUF_Q 2             /* double [rows][3] Vin . uvw_row                             */
#define SVDI_BUF_S 3             /* double [channels] f / c                                    */
#define SVDI_BUF_VIN 4           /* double [9]                                                 */
#define SVDI_BUF_OFFSETS 5       /* uint32 [n_keys + 1] record offsets per tile key            */
#define SVDI_BUF_RECORDS 6       /* 16-byte records {int xq, int yq, float vre, float vim}     */
#define SVDI_BUF_RECORDS_S 7     /* float Chebyshev argument per record (K > 1)                */
#define SVDI_BUF_GRID 8          /* complex64 [planes][G][G] grid before the FFT (keep_grid)   */
#define SVDI_BUF_MOMENTS 9       /* complex64 [planes][G][G] after the FFT (last slab batch)   */
int svdi_engine_buffer_size(const svdi_engine* e, int which, size_t* bytes);
int svdi_engine_copy_buffer(svdi_engine* e, int which, void* host_dst, size_t bytes);

/* ---- serving: continuous batching ---------------------------------------------------------- */
/* New export (the reference images one snapshot per process, SVDIntegratedImager.cu:1773-1854).
 * A server keeps num_slots engines resident (own stream, grids, cuFFT plans, tile bins) and one
 * worker thread per slot. Requests queue in arrival order; a request is admitted when a slot is
 * free and its device-memory estimate fits in the HBM budget beside the running ones (a smaller
 * request may overtake a larger one that waits for memory); admitted requests overlap on the GPU.
 * Requests that can never fit the budget are refused at submit (SVDI_ERR_OUT_OF_MEMORY). The host
 * arrays of a request and its output image must stay valid until svdi_server_wait returns. */
typedef struct svdi_server svdi_server;

typedef struct svdi_request_info {
    int status;                  /* SVDI_OK or the request's error status                      */
    int slot;                    /* slot that ran it                                           */
    size_t num_samples;
    double queue_ms;             /* submit -> start (host wall clock)                          */
    double run_ms;               /* start -> completion                                        */
    double latency_ms;           /* submit -> completion                                       */
} svdi_request_info;

/* hbm_budget_bytes = 0: 80 % of the free device memory. fault_every > 0 makes every
 * fault_every-th request fail on the host before any device work (failure-path testing). */
int svdi_server_create(const svdi_options* opt, int num_slots, size_t hbm_budget_bytes,
                       int fault_every, svdi_server** out);
/* Queue a main-path request (host snapshot, host output [N][N]); returns its ticket. */
int svdi_server_submit(svdi_server* s, const svdi_host_ms* ms, size_t image_size, float cell_size,
                       float* dirty_image, uint64_t* ticket);
/* Block until the request finishes (timeout_s <= 0: no limit); returns the request's status. */
int svdi_server_wait(svdi_server* s, uint64_t ticket, double timeout_s, svdi_request_info* info);
int svdi_server_poll(svdi_server* s, uint64_t ticket, int* done);
int svdi_server_stats(svdi_server* s, size_t* queued, size_t* hbm_in_use, size_t* hbm_budget,
                      uint64_t* admitted);
/* Drains the queue, joins the workers, frees the engines. */
void svdi_server_destroy(svdi_server* s);

/* The serving handle under its short names: svdi_create makes a server with
 * SVDI_DEFAULT_SLOTS resident engines, an automatic HBM budget (80 % of the free device memory)
 * and no fault injection; svdi_submit / svdi_poll / svdi_wait / svdi_destroy are
 * svdi_server_submit / _poll / _wait / _destroy. Status codes, no exceptions across the ABI;
 * submit, poll and wait may be called from any thread. */
#define SVDI_DEFAULT_SLOTS 3
int svdi_create(const svdi_options* opt, svdi_server** out);
int svdi_submit(svdi_server* s, const svdi_host_ms* ms, size_t image_size, float cell_size,
                float* dirty_image, uint64_t* ticket);
int svdi_poll(svdi_server* s, uint64_t ticket, int* done);
int svdi_wait(svdi_server* s, uint64_t ticket, double timeout_s, svdi_request_info* info);
void svdi_destroy(svdi_server* s);

/* ---- allocation-free binning --------------------------------------------------------------- */
/* No counterpart in the reference. For callers that must not allocate device memory once they
 * run: a correlator's real-time loop that reserves all of its device memory at start-up and
 * cannot stall on the allocator, or a host framework that owns the device's memory pool.
 * Bins num_samples samples (archive layout: d_bin [num_samples][3] in wavelengths, collapsed
 * d_vis_real / d_vis_imag) into tile records exactly like the engine's binning with one w-slab,
 * one Chebyshev term, ES support 8, clipping at the grid edge and FP64 grid coordinates, on a
 * grid of side ceil(1.5 image_size); vre/vim of each record are the visibility times inv_det.
 * All pointers are DEVICE pointers owned by the caller: d_records receives up to num_samples
 * 16-byte records {int xq, int yq, float vre, float vim}; d_offsets receives
 * ceil(1.5 image_size / tile)^2 + 1 record offsets per tile key (offsets_capacity entries).
 * The scratch (per-key counters and cursors, the dropped count) is a static device array of
 * 2 * SVDI_NOALLOC_MAX_KEYS + 4 words (128 KiB) that every GPU loading this library holds until
 * the process exits; more tile keys than SVDI_NOALLOC_MAX_KEYS are rejected with
 * SVDI_ERR_UNSUPPORTED. The first call on a device looks the array's address up
 * (cudaGetSymbolAddress): make it before any stream capture. With CUDA's default lazy module
 * loading that first call is also what loads this library's kernels and the array onto the
 * device, which takes device memory once: make the first call at start-up, outside the
 * real-time loop, or set CUDA_MODULE_LOADING=EAGER. The address is kept for the life of the
 * process, so do not cudaDeviceReset a device after calling this on it. Every call shares the
 * array, so calls whose work overlaps on the GPU (other streams or threads on the same device)
 * race; serialise them. Asynchronous on cuda_stream (NULL = legacy default stream); after the
 * first call on a device it allocates no device memory. */
#define SVDI_NOALLOC_MAX_KEYS 16384
int svdi_bin_samples_noalloc(const float* d_bin, const float* d_vis_real, const float* d_vis_imag,
                             size_t num_samples, size_t image_size, float cell_size, int tile,
                             float inv_det, void* d_records, uint32_t* d_offsets,
                             size_t offsets_capacity, void* cuda_stream);

/* Number of kernel launches this library has issued in the calling process. */
uint64_t svdi_kernel_launch_count(void);

#ifdef __cplusplus
}  /* extern "C" */

/* C++ linkage, the exact declaration of archive/pipe_interface.cpp:8. */
int FIpipe(float* Visreal, float* Visimag, float* Bin, float* Vin, float* dirty_image,
           size_t num_baselines, size_t image_size, float cell_size);
#endif

#endif /* SVDIMAGER_B200_H */
