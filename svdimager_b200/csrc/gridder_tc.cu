// Split-precision tensor-core ES gridder (tcgen05 + TMEM), one moment plane, support W <= 8.
//
// Replaces the same reference kernels as the FP32 gridder (fused_gridding,
// SVDIntegratedImager.cu:1218-1293; gridding, archive/FIPkernels.cu:383-452) for the K = 1 case.
//
// Gridding with a separable kernel is a sum of outer products. For the samples k of one tile,
//   G[m][n] = sum_k  wx_k[m] * (wy_k[n] v_k)   =   (A B^T)[m][n],
// where column k of A holds the ES weights of sample k on its W footprint rows and column k of B
// its ES weights on its W footprint columns times the visibility (re and im as separate B rows).
// Each K-block of 32 samples of one tile is written to shared memory as FP16 hi + lo pairs
// (x = hi + lo + O(2^-22 x)) and accumulated in FP32 in tensor memory by
//   D += A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T
// (six tcgen05.mma kind::f16, M = 128, N = 32, K = 16; the lo*lo term is below 2^-22 relative).
//
// Tiles. Binning uses 120-row x 8-column tiles (footprint origins). Four consecutive tile keys
// (the same tile row, 32 consecutive columns) form a super-tile. Its running sum lives in TMEM
// columns [0, 128): block c = key % 4 owns columns [32c, 32c + 32), lanes = the 128 grid rows
// origin1 .. origin1 + 127, columns 0..15 the real and 16..31 the imaginary part of grid columns
// origin2 + 8c .. origin2 + 8c + 15. Neighbouring blocks overlap by 8 grid columns; the epilogue
// adds the overlap while it reads TMEM, and flushes every non-zero cell once with a vector
// reduction to the moment plane, checkerboard sign and 1 / scale applied.
//
// Two-level accumulation. The tensor core's FP32 accumulation is not round-to-nearest: summing
// thousands of MMAs into one accumulator shrank dense grid cells by a relative 3.5e-5 on the 8.4M
// sample snapshot (measured against the oracle). So the MMAs of at most 8 K-blocks of one key
// (48 MMAs) go to one of three "fresh" 32-column accumulators (columns 128..223), which are then
// added into the running block with FP32 round-to-nearest adds (tcgen05.ld / tcgen05.st, two
// K-blocks later, when those MMAs are done).
//
// Work split. Every CTA takes an equal share of the binned records (a contiguous range, which can
// start and end inside a tile) and walks it in K-blocks; a super-tile change flushes the
// accumulator. Warp 0 prefetches the records of the K-block four steps ahead into a shared-memory
// ring with cp.async; all 256 threads build the operands of the current K-block (thread = one
// footprint row/column of one sample) into one of four stages, whose reuse waits on the mbarrier
// that tcgen05.commit signals when the stage's MMAs are done; thread 0 issues the MMAs.
//
// Scaling. The B values are wy * v * 2^(14 - e) with max|v| < 2^e over all records (the scatter
// kernel's max reduction) and the A values 256 * wx, so every FP16 operand is below 65504 and the
// low halves of all but negligible contributions stay normal.
//
// Rare samples (exact-integer positions, whose footprint is W + 1 cells wide, and footprints
// clipped at the low grid edge) skip the matrices: the eight threads of the sample add their
// exact ES weights to the moment plane directly.
//
// Every wait is bounded (about one second of global time); a wait that runs out sets *status,
// the CTA stops, waits (bounded) for its MMAs, frees its tensor memory and returns, and the host
// reports the grid as incomplete.
#include "svdi_internal.cuh"

#include <cuda_fp16.h>

namespace svdi {

namespace {

constexpr int kThreads = 256;
constexpr int kKB = 32;          // samples per K-block
constexpr int kStages = 4;       // operand stages in shared memory
constexpr int kRing = 8;         // record ring slots (K-blocks)
constexpr int kAhead = 4;        // K-blocks of records in flight
constexpr int kAccRows = 128;    // M
constexpr int kBlockCols = 32;   // N per column block (16 re + 16 im)
constexpr int kFreshBufs = 3;    // fresh accumulators: one open interval + two awaiting their merge
constexpr int kFreshKB = 8;      // K-blocks (48 MMAs) per fresh interval at most
constexpr int kFreshCol0 = kTcBlocks * kBlockCols;  // running blocks first, then the fresh buffers
constexpr int kTmemCols = 256;
static_assert(kFreshCol0 + kFreshBufs * kBlockCols <= kTmemCols, "TMEM plan exceeds the allocation");

constexpr int kABytes = kAccRows * kKB * 2;     // 8 KB per FP16 A operand
constexpr int kBBytes = kBlockCols * kKB * 2;   // 2 KB per FP16 B operand
constexpr int kStageBytes = 2 * kABytes + 2 * kBBytes;
constexpr int kRingBytes = kRing * kKB * (int)sizeof(SampleRec);
constexpr int kOldBytes = kStages * kThreads * 4;
constexpr int kSmemUsed = kStages * kStageBytes + kRingBytes + kOldBytes;
// Requested dynamic shared memory: above a third of the SM's 228 KB, so that at most two CTAs of
// this kernel are resident on an SM and their 2 x 256 TMEM columns always fit in its 512.
constexpr int kSmemBytes = 96 * 1024;
static_assert(kSmemUsed <= kSmemBytes, "shared-memory plan exceeds the request");
static_assert(kRing >= kAhead + 1, "record ring too small for the prefetch distance");
static_assert(kTcTileRows + 8 <= kAccRows && kTcTileCols + 8 <= 16, "tile + footprint must fit the accumulator");

// K-major, no-swizzle canonical layout of an FP16 operand with kKB columns: core matrices of
// 8 rows x 16 bytes; the next 8 K-elements at +128 bytes (LBO), the next 8 rows at +512 (SBO).
__device__ __forceinline__ int op_off(int row, int k) {
    return (row & 7) * 16 + (row >> 3) * 512 + (k >> 3) * 128 + (k & 7) * 2;
}
constexpr unsigned long long kDescHi = (512ull >> 4) << 32 | (1ull << 46);  // SBO, version 1
constexpr unsigned long long kDescLbo = (128ull >> 4) << 16;                // LBO

__device__ __forceinline__ unsigned long long smem_desc(uint32_t addr) {
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | kDescLbo | kDescHi;
}

// Instruction descriptor: FP32 accumulator, FP16 A and B, both K-major, N = 32, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | ((uint32_t)(kBlockCols >> 3) << 17) | ((uint32_t)(kAccRows >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the completion of the phase with the given parity: about one second.
__device__ bool mbar_wait(uint32_t addr, uint32_t parity) {
    if (mbar_try(addr, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (unsigned int it = 1; it < (1u << 28); ++it) {
        if (mbar_try(addr, parity)) return true;
        if ((it & 63u) == 0 && global_ns() - t0 > 1000000000ull) return false;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, unsigned long long a, unsigned long long b, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(kIdesc), "r"(accum)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

// 32 consecutive TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};" ::"r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
        "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
        "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
        "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
        "r"(__float_as_uint(v[15]))
        : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void red_add_v2(float2* addr, float a, float b) {
    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(addr), "f"(a), "f"(b) : "memory");
}

// Exact ES kernel psi(x) = exp(beta (sqrt(1 - x^2) - 1)) written without cancellation.
__device__ __forceinline__ float es_exact(float beta, float x) {
    if (fabsf(x) > 1.0f) return 0.0f;
    return expf(-beta * x * x / (1.0f + sqrtf((1.0f - x) * (1.0f + x))));
}

__device__ __forceinline__ void split_store(unsigned char* hi, unsigned char* lo, int off, float x) {
    const __half h = __float2half_rn(x);
    *reinterpret_cast<__half*>(hi + off) = h;
    *reinterpret_cast<__half*>(lo + off) = __float2half_rn(x - __half2float(h));
}

struct KBMeta {
    int key;   // tile key of the K-block
    int cnt;   // samples in it (0 = no more K-blocks)
};

// Walks the CTA's record range [rbeg, rend) in K-blocks of one key each.
struct KIter {
    int key;
    unsigned int pos, end;
    bool ok;
    __device__ void next_key(const unsigned int* off, int key_hi, unsigned int rend) {
        for (;;) {
            ++key;
            if (key >= key_hi) { ok = false; return; }
            const unsigned int b = off[key];
            if (b >= rend) { ok = false; return; }
            const unsigned int e = min(rend, off[key + 1]);
            if (b < e) { pos = b; end = e; return; }
        }
    }
    __device__ void advance(const unsigned int* off, int key_hi, unsigned int rend) {
        pos += kKB;
        if (pos >= end) next_key(off, key_hi, rend);
    }
};

struct TcParams {
    const SampleRec* rec;
    const unsigned int* offsets;
    const unsigned int* vmax;
    float2* planes;
    unsigned int* status;
    int key_lo, key_hi, slab_lo;
};

__global__ void __launch_bounds__(kThreads, 2) k_grid_tc(TcParams P, GridGeom g, EsPoly poly) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) unsigned long long mbar[kStages];
    __shared__ KBMeta meta[kRing];
    __shared__ uint32_t tmem_base_sh;
    __shared__ int start_key_sh;

    unsigned char* stage_base = smem;
    SampleRec* ring = reinterpret_cast<SampleRec*>(smem + kStages * kStageBytes);
    int* oldpos = reinterpret_cast<int*>(smem + kStages * kStageBytes + kRingBytes);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int slot = tid >> 3, fi = tid & 7;  // sample slot of the K-block, footprint row/col index
    const int W = g.W, HW = W / 2;
    const int tiles2 = g.ntile * g.ntile2;
    const long long GG = g.G * g.G;

    // ---- set-up: tensor memory, barriers, the CTA's record range
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[s])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < kStages * kStageBytes / 16; i += kThreads)
        reinterpret_cast<uint4*>(stage_base)[i] = make_uint4(0, 0, 0, 0);
    for (int i = tid; i < kStages * kThreads; i += kThreads) oldpos[i] = -1;

    const unsigned int rec_lo = P.offsets[P.key_lo], rec_hi = P.offsets[P.key_hi];
    const unsigned long long total = rec_hi - rec_lo;
    const unsigned int rbeg = rec_lo + (unsigned int)(total * blockIdx.x / gridDim.x);
    const unsigned int rend = rec_lo + (unsigned int)(total * (blockIdx.x + 1) / gridDim.x);
    if (tid == 0) {  // last key with offsets[key] <= rbeg
        int lo = P.key_lo, hi = P.key_hi;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (P.offsets[mid] <= rbeg) lo = mid; else hi = mid;
        }
        start_key_sh = lo;
    }
    // FP16 operand scale from max |v| over all records
    float vscale = 0.0f;
    {
        const float vmax = __uint_as_float(*P.vmax);
        if (vmax > 0.0f && vmax < 3.0e38f) {
            int ex;
            frexpf(vmax, &ex);
            vscale = ldexpf(1.0f, max(-100, min(100, 14 - ex)));
        }
    }
    const float inv_scale = vscale > 0.0f ? 1.0f / (256.0f * vscale) : 0.0f;
    float coef[kPolyDeg + 1];
#pragma unroll
    for (int d = 0; d <= kPolyDeg; ++d) coef[d] = poly.c[fi][d];

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;

    // ---- record prefetch (warp 0): K-block j goes to ring slot j % kRing, one cp.async group each
    KIter pf;
    if (warp == 0) {
        pf.key = start_key_sh;
        pf.pos = rbeg;
        pf.end = min(rend, P.offsets[pf.key + 1]);
        pf.ok = rbeg < rend;
        if (pf.ok && pf.pos >= pf.end) pf.next_key(P.offsets, P.key_hi, rend);
    }
    auto prefetch = [&](int j) {  // warp 0 only
        const int cnt = pf.ok ? (int)min((unsigned int)kKB, pf.end - pf.pos) : 0;
        if (lane < cnt) cp_async16(smem_u32(ring + (j % kRing) * kKB + lane), P.rec + pf.pos + lane);
        cp_async_commit();
        if (lane == 0) meta[j % kRing] = KBMeta{pf.ok ? pf.key : -1, cnt};
        if (pf.ok) pf.advance(P.offsets, P.key_hi, rend);
    };
    if (warp == 0) {
        for (int j = 0; j < kAhead; ++j) prefetch(j);
        cp_async_wait<kAhead - 1>();
    }
    __syncthreads();

    int cur_st = -1, cur_key = 0;
    int kb = 0;
    bool aborted = false;  // block-uniform (set from __syncthreads_or)
    // Accumulation state, block-uniform. run_valid bit c: running block c holds data. Open interval:
    // fresh buffer ob, block oc, on K-blocks so far (on == 0: none open). Closed intervals waiting
    // for their merge, oldest first: pend[0..np), packed (last K-block << 8) | (block << 4) | buffer.
    unsigned int run_valid = 0;
    int ob = 0, oc = 0, on = 0;
    int pend[3] = {0, 0, 0};
    int np = 0;

    const int q = warp & 3, h = warp >> 2;  // TMEM lane quarter, column half of this warp
    const uint32_t lane_addr = (uint32_t)(32 * q) << 16;

    auto wait_kb = [&](int j) -> bool {  // the MMAs of K-block j are complete (bounded wait)
        return mbar_wait(smem_u32(&mbar[j % kStages]), (uint32_t)((j / kStages) & 1));
    };
    // running[blk] (+)= fresh[buf] with FP32 round-to-nearest adds: this thread's lane, columns
    // [16h, 16h + 16) of the block (h = 0: real, h = 1: imaginary part).
    auto merge = [&](int packed) {
        const int buf = packed & 15, blk = (packed >> 4) & 15;
        float f[16], r[16];
        const uint32_t ra = tmem + lane_addr + (uint32_t)(kBlockCols * blk + 16 * h);
        tmem_ld16(tmem + lane_addr + (uint32_t)(kFreshCol0 + kBlockCols * buf + 16 * h), f);
        if ((run_valid >> blk) & 1u) {
            tmem_ld16(ra, r);
#pragma unroll
            for (int j = 0; j < 16; ++j) f[j] += r[j];
        }
        tmem_st16(ra, f);
        run_valid |= 1u << blk;
    };
    auto close_interval = [&]() {
        if (on > 0) {
            pend[np] = ((kb - 1) << 8) | (oc << 4) | ob;
            ++np;
            on = 0;
        }
    };

    // Flush the super-tile of cur_key: merge every fresh interval, read the running blocks (warp w:
    // rows 32 (w % 4) + lane, blocks 2 (w / 4) and 2 (w / 4) + 1), add the column overlaps and reduce
    // the non-zero on-grid cells into the moment plane.
    auto flush = [&]() {
        bool fail = false;
        close_interval();
        if (np > 0 && !wait_kb(pend[np - 1] >> 8)) {  // the newest commit covers the older MMAs
            fail = true;
            atomicOr(P.status, 2u);
        }
        tc_fence_after();
        for (int k = 0; k < np; ++k) merge(pend[k]);
        np = 0;
        // the merges stored the real halves from warps 0-3 and the imaginary halves from warps 4-7;
        // the epilogue below reads whole blocks across that split
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        const int slab = cur_key / tiles2;
        const int t1 = (cur_key / g.ntile2) % g.ntile;
        const int t2b = (cur_key % g.ntile2) / kTcBlocks * kTcBlocks;
        const int row = 32 * q + lane;
        const long long g1 = g.gmin + (long long)t1 * g.T + row;
        const bool row_ok = g1 <= g.gmax;
        const long long o2 = g.gmin + (long long)t2b * g.T2;  // grid column of block 0, column 0
        float2* plane = P.planes + (long long)(slab - P.slab_lo) * GG + (g1 - g.gmin) * g.G;
        float cre[8], cim[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) { cre[j] = 0.0f; cim[j] = 0.0f; }
        auto emit = [&](long long g2, float re, float im) {
            if (row_ok && g2 <= g.gmax && (re != 0.0f || im != 0.0f)) {
                const float sg = ((g1 + g2) & 1) ? -inv_scale : inv_scale;
                red_add_v2(plane + (g2 - g.gmin), sg * re, sg * im);
            }
        };
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int c = 2 * h + cc;
            float v[32];
            if ((run_valid >> c) & 1u) {
                tmem_ld32(tmem + lane_addr + (uint32_t)(kBlockCols * c), v);
            } else {
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = 0.0f;
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                emit(o2 + 8 * c + j, cre[j] + v[j], cim[j] + v[16 + j]);
                cre[j] = v[8 + j];
                cim[j] = v[24 + j];
            }
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) emit(o2 + 8 * (2 * h + 2) + j, cre[j], cim[j]);
        run_valid = 0;
        tc_fence_before();
        if (__syncthreads_or(fail)) aborted = true;
    };

    for (;;) {
        const KBMeta m = meta[kb % kRing];
        if (m.cnt == 0) break;
        const int st = m.key / kTcBlocks;  // ntile2 is a multiple of kTcBlocks
        if (st != cur_st) {
            if (cur_st >= 0) {
                flush();
                if (aborted) break;
            }
            cur_st = st;
        }
        cur_key = m.key;
        const int c = m.key % kTcBlocks;
        if (on > 0 && (c != oc || on == kFreshKB)) close_interval();
        if (on == 0) {  // a fresh buffer that no closed interval still occupies
            unsigned int used = 0;
            for (int k = 0; k < np; ++k) used |= 1u << (pend[k] & 15);
            ob = (used & 1u) == 0 ? 0 : ((used & 2u) == 0 ? 1 : 2);
            oc = c;
        }
        if (warp == 0) prefetch(kb + kAhead);

        // ---- this thread's sample slot and footprint index
        const int s = kb % kStages;
        unsigned char* A_hi = stage_base + s * kStageBytes;
        unsigned char* A_lo = A_hi + kABytes;
        unsigned char* B_hi = A_lo + kABytes;
        unsigned char* B_lo = B_hi + kBBytes;
        const bool valid = slot < m.cnt;
        SampleRec r = {0, 0, 0.0f, 0.0f};
        if (valid) r = ring[(kb % kRing) * kKB + slot];
        const int cx = r.xq >> 24, cy = r.yq >> 24;
        const int fxq = r.xq & 0xFFFFFF, fyq = r.yq & 0xFFFFFF;
        const int r0 = cx - (HW - 1), c0 = cy - (HW - 1);
        const bool rare = valid && (fxq == 0 || fyq == 0 || r0 < 0 || c0 < 0 || r0 >= g.T || c0 >= g.T2);
        const bool fast = valid && !rare && fi < W;
        float wx = 0.0f, wy = 0.0f;
        if (fast) {
            const float ux = fmaf(2.0f, (float)fxq * (1.0f / 16777216.0f), -1.0f);
            const float uy = fmaf(2.0f, (float)fyq * (1.0f / 16777216.0f), -1.0f);
            wx = coef[kPolyDeg];
            wy = coef[kPolyDeg];
#pragma unroll
            for (int d = kPolyDeg - 1; d >= 0; --d) {
                wx = fmaf(wx, ux, coef[d]);
                wy = fmaf(wy, uy, coef[d]);
            }
        }
        // ---- stage reuse: the MMAs of K-block kb - kStages must be done with it
        bool fail = false;
        if (kb >= kStages && !wait_kb(kb - kStages)) {
            fail = true;
            atomicOr(P.status, 1u);
        }
        {  // clear the entries this thread wrote into the stage last time
            const int old = oldpos[s * kThreads + tid];
            if (old >= 0) {
                const int orow = old >> 8, ocol = old & 0xFF;
                const int oa = op_off(orow, slot);
                *reinterpret_cast<__half*>(A_hi + oa) = __float2half_rn(0.0f);
                *reinterpret_cast<__half*>(A_lo + oa) = __float2half_rn(0.0f);
                const int ob_ = op_off(ocol, slot), obi = op_off(16 + ocol, slot);
                *reinterpret_cast<__half*>(B_hi + ob_) = __float2half_rn(0.0f);
                *reinterpret_cast<__half*>(B_lo + ob_) = __float2half_rn(0.0f);
                *reinterpret_cast<__half*>(B_hi + obi) = __float2half_rn(0.0f);
                *reinterpret_cast<__half*>(B_lo + obi) = __float2half_rn(0.0f);
            }
        }
        __syncwarp();
        if (fast) {
            const int arow = r0 + fi, bcol = c0 + fi;
            split_store(A_hi, A_lo, op_off(arow, slot), 256.0f * wx);
            const float wv = wy * vscale;
            split_store(B_hi, B_lo, op_off(bcol, slot), wv * r.vre);
            split_store(B_hi, B_lo, op_off(16 + bcol, slot), wv * r.vim);
            oldpos[s * kThreads + tid] = (arow << 8) | bcol;
        } else {
            oldpos[s * kThreads + tid] = -1;
        }
        if (rare) {  // exact ES weights straight to the moment plane; the slot's 8 threads over cells
            const int slab = m.key / tiles2;
            const int t1 = (m.key / g.ntile2) % g.ntile, t2 = m.key % g.ntile2;
            const long long o1 = g.gmin + (long long)t1 * g.T, o2 = g.gmin + (long long)t2 * g.T2;
            const int lo_r = fxq ? r0 : cx - HW, nr = fxq ? W : W + 1;
            const int lo_c = fyq ? c0 : cy - HW, nc = fyq ? W : W + 1;
            const float px = (float)fxq * (1.0f / 16777216.0f), py = (float)fyq * (1.0f / 16777216.0f);
            float2* plane = P.planes + (long long)(slab - P.slab_lo) * GG;
            for (int cidx = fi; cidx < nr * nc; cidx += 8) {
                const int rr = lo_r + cidx / nc, cc = lo_c + cidx % nc;
                const long long g1 = o1 + rr, g2 = o2 + cc;
                if (g1 < g.gmin || g2 < g.gmin || g1 > g.gmax || g2 > g.gmax) continue;
                const float x = ((float)(rr - cx) - px) / (float)HW;
                const float y = ((float)(cc - cy) - py) / (float)HW;
                const float kv = es_exact(poly.beta, x) * es_exact(poly.beta, y);
                const float sg = ((g1 + g2) & 1) ? -kv : kv;
                red_add_v2(plane + (g1 - g.gmin) * g.G + (g2 - g.gmin), sg * r.vre, sg * r.vim);
            }
        }
        // ---- merge the intervals closed two or more K-blocks ago (their MMAs are done by now)
        {
            int k = 0;
            while (k < np && (pend[k] >> 8) <= kb - 2) {
                if (!wait_kb(pend[k] >> 8)) {
                    fail = true;
                    atomicOr(P.status, 8u);
                }
                tc_fence_after();
                merge(pend[k]);
                ++k;
            }
            if (k > 0) {
                for (int i = k; i < np; ++i) pend[i - k] = pend[i];
                np -= k;
                tc_fence_before();
            }
        }
        if (warp == 0) cp_async_wait<kAhead - 1>();  // records of K-block kb + 1 have landed
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (__syncthreads_or(fail)) {
            aborted = true;
            break;
        }
        if (tid == 0) {
            tc_fence_after();
            const uint32_t d = tmem + (uint32_t)(kFreshCol0 + kBlockCols * ob);
            const uint32_t ah = smem_u32(A_hi), al = smem_u32(A_lo), bh = smem_u32(B_hi), bl = smem_u32(B_lo);
            uint32_t acc = on > 0 ? 1u : 0u;
#pragma unroll
            for (int k = 0; k < kKB / 16; ++k) {  // 16-element K steps: +256 bytes
                const uint32_t ko = (uint32_t)k * 256u;
                mma_f16(d, smem_desc(ah + ko), smem_desc(bh + ko), acc);
                acc = 1u;
                mma_f16(d, smem_desc(ah + ko), smem_desc(bl + ko), 1u);
                mma_f16(d, smem_desc(al + ko), smem_desc(bh + ko), 1u);
            }
            mma_commit(smem_u32(&mbar[s]));
        }
        ++on;
        ++kb;
    }
    if (cur_st >= 0 && !aborted) flush();

    // ---- teardown: no copies or MMAs in flight, then free the tensor memory
    if (warp == 0) cp_async_wait<0>();
    if (kb > 0) {
        const int s = (kb - 1) % kStages;
        if (!mbar_wait(smem_u32(&mbar[s]), (uint32_t)(((kb - 1) / kStages) & 1))) atomicOr(P.status, 4u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

}  // namespace

int launch_grid_tc(const SampleRec* d_rec, const unsigned int* d_offsets, int n_keys, int key_lo, int key_hi,
                   int slab_lo, const GridGeom& g, const EsPoly& poly, float2* d_planes,
                   const unsigned int* d_vmax, unsigned int* d_status, int sm_count, cudaStream_t st) {
    if (key_lo < 0 || key_hi > n_keys || key_lo >= key_hi) {
        set_error("tensor-core gridder: bad key range");
        return SVDI_ERR_INTERNAL;
    }
    if (g.W > 8 || (g.W & 1) || g.T != kTcTileRows || g.T2 != kTcTileCols || (g.ntile2 % kTcBlocks) != 0 ||
        (key_lo % kTcBlocks) != 0) {
        set_error("tensor-core gridder: needs even support <= 8 and 120 x 8 tiles in groups of 8");
        return SVDI_ERR_UNSUPPORTED;
    }
    static bool configured = false;
    if (!configured) {
        SVDI_CUDA(cudaFuncSetAttribute(k_grid_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
        // without a carveout preference the occupancy query assumes one CTA per SM
        SVDI_CUDA(cudaFuncSetAttribute(k_grid_tc, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
        configured = true;
    }
    // two CTAs per SM by design (2 x 256 of the SM's 512 TMEM columns; shared memory admits no third)
    int per_sm = 0;
    SVDI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_grid_tc, kThreads, kSmemBytes));
    if (per_sm < 1) {
        set_error("tensor-core gridder: kernel does not fit on an SM");
        return SVDI_ERR_UNSUPPORTED;
    }
    per_sm = 2;
    TcParams P{d_rec, d_offsets, d_vmax, d_planes, d_status, key_lo, key_hi, slab_lo};
    k_grid_tc<<<sm_count * per_sm, kThreads, kSmemBytes, st>>>(P, g, poly);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

}  // namespace svdi
