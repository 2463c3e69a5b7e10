// Split-precision tensor-core ES gridder (tcgen05 + TMEM), one moment plane, support W <= 8.
//
// Replaces the same reference kernels as the FP32 gridder (fused_gridding,
// SVDIntegratedImager.cu:1218-1293; gridding, archive/FIPkernels.cu:383-452) for the K = 1 case.
//
// Gridding with a separable kernel is a sum of outer products. For the samples k of one tile,
//   G[m][n] = sum_k  wx_k[m] * (wy_k[n] v_k)   =   (A B^T)[m][n],
// where column k of A holds the ES weights of sample k on its footprint rows and column k of B its
// ES weights on its footprint columns times the visibility (re and im as separate B columns).
// Each K-block of 32 samples of one tile is written to shared memory with both factors split into
// FP16 (or BF16) hi + lo parts (x = hi + lo + O(2^-22 x) in FP16), stacked as
//   A' = [A_hi; A_lo] (128 rows),  B' = [B_hi | B_lo] (64 columns),
// so that ONE tcgen05.mma kind::f16 (M = 128, N = 64, K = 16) per 16 samples computes all four
// products A_hi B_hi, A_hi B_lo, A_lo B_hi, A_lo B_lo into the quarters of a 128 x 64 FP32
// accumulator in tensor memory; the epilogue adds the quarters. Two MMAs per K-block.
//
// Cost model (measured on B200): a skinny tcgen05.mma costs about its operand bytes read from
// shared memory at ~117 B/clk per SM, and in this kernel one issuing thread spent ~110 clk per
// MMA; an mbarrier try_wait costs the issuing thread ~200 clk. Hence few, wide MMAs (6 KB of
// operands each, 2 per K-block instead of 6 skinny ones), two CTAs per SM (two issuing threads)
// and one wait per pipeline stage of four K-blocks.
//
// Operands. Both are MN-major without swizzle: a core matrix is 8 K (samples) x 16 bytes (8
// consecutive rows of A or columns of B). One thread builds one sample's column of A' and of B': its
// eight row taps land at rows r0 .. r0 + 7 of the 64-row accumulator, that is in the 8-row chunks
// r0 / 8 and r0 / 8 + 1 at an offset of r0 % 8. The thread evaluates the taps in order (FP32
// piecewise polynomials whose coefficients are kernel-parameter constants), packs them into hi and
// lo half pairs and shifts the 16-half window into place with byte permutes and word selects, so
// each chunk is one 16-byte store (a warp's stores of one chunk fill four whole shared-memory
// wavefronts, whatever the samples' rows). The A' rows are ordered so that TMEM lane quarter q
// holds grid rows 16q .. 16q + 15 of the hi part and then of the lo part (a_chunk). B's 16 columns
// (8 real + 8 imaginary taps of the 8-column tile plus halo) are written in full; of A only the
// chunks the thread's previous sample in this stage slot covered and the new sample does not are
// cleared.
//
// Accumulation. Consecutive K-blocks of one tile key (at most kIntervalKB of them, 32 MMAs) form
// an interval that accumulates in one of four 64-column TMEM accumulators. The tensor core's FP32
// accumulation is not round-to-nearest: summing thousands of MMAs into one accumulator shrank
// dense grid cells by a relative 3.5e-5 on the 8.4M-sample snapshot (measured against the oracle),
// so intervals stay short and each one is drained by the epilogue into the moment plane with FP32
// round-to-nearest reductions (red.global.add.v2.f32, checkerboard sign and 1 / scale applied).
//
// Tiles. Binning uses 56-row x 8-column tiles (footprint origins); an accumulator covers the tile's
// 64 rows (56 + halo) and 16 columns (8 + halo).
//
// Roles (two CTAs per SM, 14 warps, 256 TMEM columns each):
//   warps 0-7   producers: warps w and w + 4 fill sub-stage w of the two pipeline stages in turn
//               with K-blocks j = w, w + 4, w + 8, ... (one thread per sample), warp w the A'
//               column and warp w + 4 the B' column of each sample; the eight warps arrive on
//               full[stage]; a stage is reused once the MMAs of its previous round commit to
//               empty[stage].
//   warp 8      scheduler: walks the CTA's share of the K-blocks (runs of up to 32 records of one
//               key), publishes their descriptors to a ring and stages each K-block's records
//               (one contiguous run of 16-byte records) into shared memory with a bulk copy
//               (cp.async.bulk, this GPU's own memory, no multicast) that completes on the record
//               slot's mbarrier.
//   warp 9      MMA issuer: issues the MMAs, opens and closes intervals and posts a drain event
//               per interval.
//   warps 10-13 epilogue: TMEM lane quarter (warp % 4); drain the intervals in event order.
// The scheduler warps take chunks of 32 K-blocks from a global counter (a chunk can start and end
// inside a tile).
//
// Scaling. The B values are wy * v * 2^(14 - e) with max|v| < 2^e over all records (the scatter
// kernel's max reduction) and the A values 256 * wx, so every FP16 operand is below 65504 and the
// low halves of all but negligible contributions stay normal.
//
// Rare samples (exact-integer positions, whose footprint is W + 1 cells wide, and footprints
// clipped at the low grid edge) skip the matrices: their thread adds the exact ES weights to the
// moment plane directly.
//
// Every wait is bounded (about one second of global time); a wait that runs out sets *status and
// a CTA-wide abort flag that every other wait also watches, so all roles leave their loops, the
// MMA warp waits (bounded) for its last commit, the scheduler for its last record copies, the
// tensor memory is freed and the host reports the grid as incomplete.
#include "svdi_internal.cuh"
#include "tc_sync.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace svdi {

namespace {

constexpr int kKB = kTcKBlock;          // samples per K-block
constexpr int kRows = 64;               // grid rows of an accumulator: tile rows + footprint halo
constexpr int kCols = 32;               // columns of a split: 16 real + 16 imaginary
constexpr int kM = 2 * kRows;           // MMA rows: A_hi rows, then A_lo rows
constexpr int kN = 2 * kCols;           // MMA columns: B_hi columns, then B_lo columns
constexpr int kSubStages = 4;           // K-blocks per pipeline stage (one per producer warp)
constexpr int kPipe = 2;                // pipeline stages
// producers: warp w < kSubStages writes A' of sub-stage w, warp kSubStages + w its B'
constexpr int kProdWarps = 2 * kSubStages;                 // 8
constexpr int kSchedWarp = kProdWarps;                     // 8
constexpr int kMmaWarp = kProdWarps + 1;                   // 9
constexpr int kEpiWarp0 = kProdWarps + 2;                  // 10..13
constexpr int kWarps = kProdWarps + 2 + 4;
constexpr int kThreads = kWarps * 32;                      // 448
constexpr int kAccBufs = 4;             // TMEM accumulators of kN columns
constexpr int kIntervalKB = 16;         // K-blocks (32 MMAs) per accumulator interval at most
constexpr int kTmemCols = 256;
constexpr int kMetaRing = 64;           // published K-block descriptors
constexpr int kRecSlots = 16;           // record slots: K-blocks staged ahead of the producers
constexpr int kChunkKB = 32;            // K-blocks per chunk of dynamically distributed work
constexpr int kEventRing = 64;

constexpr int kABytes = kRows * kKB * 2;                 // 4 KB per FP16 A half (hi or lo)
constexpr int kBBytes = kCols * kKB * 2;                 // 2 KB per FP16 B half
constexpr int kSubBytes = 2 * kABytes + 2 * kBBytes;     // 12 KB: one K-block
constexpr int kStageBytes = kSubStages * kSubBytes;      // 48 KB
constexpr int kRecOff = kPipe * kStageBytes;             // record slots after the stages
constexpr int kRecBytes = kRecSlots * kKB * 16;          // 8 KB
constexpr int kSmemUsed = kRecOff + kRecBytes;
// Requested dynamic shared memory: more than a third of the SM's 228 KB, so at most two CTAs share
// an SM and their 2 x 256 TMEM columns always fit in its 512.
constexpr int kSmemBytes = kSmemUsed;
static_assert(kSmemBytes > 228 * 1024 / 3 && 2 * (kSmemBytes + 4096) <= 228 * 1024, "two CTAs per SM");
static_assert(kAccBufs * kN <= kTmemCols, "TMEM plan exceeds the allocation");
static_assert(kTcTileRows + 8 <= kRows && kTcTileCols + 8 <= 16, "tile + footprint must fit the accumulator");
static_assert(kEpiWarp0 + 4 == kWarps, "four epilogue warps (one per TMEM lane quarter) come last");
static_assert(kRecSlots <= kMetaRing && kKB == 32, "one record slot per published K-block, one lane per record");

// MN-major, no-swizzle canonical layout of an FP16 operand with kKB K-columns: a core matrix is
// 8 K-rows x 16 bytes (8 consecutive M or N elements); the next 8 K at +128 bytes (LBO), the next
// 8 M / N elements at +512 bytes (SBO). Element (mn, k) sits at byte
// (mn % 8) * 2 + (k % 8) * 16 + (k / 8) * 128 + (mn / 8) * 512.
constexpr unsigned long long kDescFixed = ((128ull >> 4) << 16) | ((512ull >> 4) << 32) | (1ull << 46);
__device__ __forceinline__ unsigned long long smem_desc(uint32_t addr) {
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | kDescFixed;
}
// Instruction descriptor: FP32 accumulator, FP16 A and B, both MN-major, N = 64, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 15) | (1u << 16) | ((uint32_t)(kN >> 3) << 17) |
                            ((uint32_t)(kM >> 4) << 24);
// The same with BF16 A and B (both operands always have the same type).
constexpr uint32_t kIdescBf16 = kIdesc | (1u << 7) | (1u << 10);

using namespace tc;


// Eight values (taps 0..7) as FP16 (or BF16) hi or lo pairs (x = hi + lo + O(2^-22 x) in FP16,
// O(2^-17 x) in BF16): word w holds taps 2w (low half) and 2w + 1.
template <bool kBf16>
__device__ __forceinline__ uint32_t pack_rn(float a, float b) {
    if constexpr (kBf16) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<const uint32_t*>(&h);
    } else {
        const __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<const uint32_t*>(&h);
    }
}
template <bool kBf16>
__device__ __forceinline__ float2 unpack(uint32_t w) {
    if constexpr (kBf16) {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w));
    } else {
        return __half22float2(*reinterpret_cast<const __half2*>(&w));
    }
}
template <bool kBf16>
__device__ __forceinline__ void hi8(const float (&x)[8], uint32_t (&hi)[4]) {
#pragma unroll
    for (int w = 0; w < 4; ++w) hi[w] = pack_rn<kBf16>(x[2 * w], x[2 * w + 1]);
}
template <bool kBf16>
__device__ __forceinline__ void lo8(const float (&x)[8], uint32_t (&lo)[4]) {
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        const float2 f = unpack<kBf16>(pack_rn<kBf16>(x[2 * w], x[2 * w + 1]));
        lo[w] = pack_rn<kBf16>(x[2 * w] - f.x, x[2 * w + 1] - f.y);
    }
}

// The 16-half window of two 8-element chunks with taps 0..7 at positions sh .. sh + 7 (0 <= sh < 8)
// and zeros elsewhere: o[0..3] is the first chunk, o[4..7] the second. A half shift by the low bit
// of sh (byte permutes), then word shifts by 1 and 2 (selects).
__device__ __forceinline__ void window16(const uint32_t (&h)[4], int sh, uint32_t (&o)[8]) {
    const uint32_t sel = (sh & 1) ? 0x5432u : 0x7654u;
    uint32_t g[5];
    g[0] = __byte_perm(0u, h[0], sel);
    g[1] = __byte_perm(h[0], h[1], sel);
    g[2] = __byte_perm(h[1], h[2], sel);
    g[3] = __byte_perm(h[2], h[3], sel);
    g[4] = __byte_perm(h[3], 0u, sel);
    const bool s1 = (sh & 2) != 0, s2 = (sh & 4) != 0;
    uint32_t u[6];
    u[0] = s1 ? 0u : g[0];
#pragma unroll
    for (int w = 1; w < 5; ++w) u[w] = s1 ? g[w - 1] : g[w];
    u[5] = s1 ? g[4] : 0u;
    o[0] = s2 ? 0u : u[0];
    o[1] = s2 ? 0u : u[1];
#pragma unroll
    for (int w = 2; w < 6; ++w) o[w] = s2 ? u[w - 2] : u[w];
    o[6] = s2 ? u[4] : 0u;
    o[7] = s2 ? u[5] : 0u;
}

// A operand row order: the TMEM lane quarter q (accumulator lanes 32q .. 32q + 31) holds grid rows
// 16q .. 16q + 15 of the hi part in its first 16 lanes and the same rows of the lo part in the
// last 16, so one warp adds hi and lo with a shuffle. In 8-row chunks: grid-row chunk j of the hi
// part is A chunk a_chunk(j), of the lo part a_chunk(j) + 2.
__device__ __forceinline__ int a_chunk(int j) { return ((j >> 1) << 2) | (j & 1); }

__device__ __forceinline__ void st_chunk(unsigned char* p, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    *reinterpret_cast<uint4*>(p) = make_uint4(a, b, c, d);
}


enum EventType : int { kEvDrain = 0, kEvExit = 1 };
struct Event {
    int type;
    int buf;     // accumulator to drain
    int key;     // its tile key
    int parity;  // phase parity of the accumulator's MMAs-done barrier
};

struct TcParams {
    const SampleRec* rec;
    const unsigned int* offsets;
    const unsigned int* kb_offsets;  // exclusive scan of ceil(count / kKB) per key
    const unsigned int* vmax;
    float2* planes;
    unsigned int* status;
    unsigned int* work;              // next chunk of K-blocks to hand out (zeroed by the host)
    int key_lo, key_hi, slab_lo;
};

struct __align__(8) TcShared {
    unsigned long long full[kPipe];       // producers -> MMA: the stage's K-blocks written (4 warp arrivals)
    unsigned long long empty[kPipe];      // MMA -> producers: stage read (tcgen05.commit)
    unsigned long long rec_full[kRecSlots];  // scheduler's bulk copy -> producers: records staged
    unsigned long long fdone[kAccBufs];   // MMA -> epilogue: the interval's MMAs done (commit)
    unsigned long long ffree[kAccBufs];   // epilogue -> MMA: accumulator read (4 warp arrivals)
    KBMeta meta[kMetaRing];
    Event events[kEventRing];
    unsigned int published;               // K-block descriptors published
    unsigned int consumed;                // K-blocks whose descriptor and records everyone is done with
    unsigned int sched_done;              // 1 + total K-blocks once the schedule is complete
    unsigned int ev_published;
    unsigned int ev_consumed[4];
    int abort;
    uint32_t tmem_base;
};


template <bool kBf16>
__global__ void __launch_bounds__(kThreads, 2) k_grid_tc(TcParams P, GridGeom g, EsPoly poly) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ TcShared S;
    const SampleRec* recs = reinterpret_cast<const SampleRec*>(smem + kRecOff);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int W = g.W, HW = W / 2;
    const int tiles2 = g.ntile * g.ntile2;
    const long long GG = g.G * g.G;
    volatile int* abort_flag = &S.abort;
    const uint32_t idesc = kBf16 ? kIdescBf16 : kIdesc;

    // ---- set-up: tensor memory, barriers, the CTA's record range
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // the K-blocks of keys [key_lo, key_hi), handed out in chunks by the scheduler warps
    const unsigned int kb_lo = P.kb_offsets[P.key_lo], kb_hi = P.kb_offsets[P.key_hi];
    if (tid == 0) {
        for (int s = 0; s < kPipe; ++s) {
            mbar_init(smem_u32(&S.full[s]), kProdWarps);
            mbar_init(smem_u32(&S.empty[s]), 1);
        }
        for (int s = 0; s < kRecSlots; ++s) mbar_init(smem_u32(&S.rec_full[s]), 1);
        for (int b = 0; b < kAccBufs; ++b) {
            mbar_init(smem_u32(&S.fdone[b]), 1);
            mbar_init(smem_u32(&S.ffree[b]), 4);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        S.published = 0;
        S.consumed = 0;
        S.sched_done = 0;
        S.ev_published = 0;
        for (int q = 0; q < 4; ++q) S.ev_consumed[q] = 0;
        S.abort = 0;
    }
    for (int i = tid; i < kPipe * kStageBytes / 16; i += kThreads)
        reinterpret_cast<uint4*>(smem)[i] = make_uint4(0, 0, 0, 0);
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
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem_base;

    if (warp < kProdWarps) {
        // =========================== producers ===========================
        // warp -> sub-stage (warp % 4) and operand (A' for warps 0-3, B' for warps 4-7); lane ->
        // sample (K-slot) of the K-block; round `it` uses stage it % 2. The A' warp also adds the
        // rare samples to the plane.
        const int sw = warp % kSubStages;
        const bool a_role = warp < kSubStages;
        const int kofs = (lane & 7) * 16 + (lane >> 3) * 128;  // byte offset of this K-slot's 16-byte row
        int oldj0 = -1, oldj1 = -1;  // first A chunk of this lane's previous sample per stage (-1: none)
        int pub_seen = 0;  // lane 0: published count last read (acquire)
        bool failed = false;
        for (int it = 0;; ++it) {
            const int j = it * kSubStages + sw;
            const int stg = it & 1;
            const int use = it >> 1;  // earlier rounds of this stage
            unsigned char* const A = smem + stg * kStageBytes + sw * kSubBytes;  // A_hi and A_lo rows
            unsigned char* const B_hi = A + 2 * kABytes;
            unsigned char* const B_lo = B_hi + kBBytes;
            // wait until K-block j is published or the schedule ends before it (warp-uniform)
            int state = 0;  // 1: produce, 0: done, -1: give up
            unsigned int sdv = 0;
            if (lane == 0) {
                PollClock pc;
                for (unsigned int n = 0;; ++n) {
                    if (pub_seen <= j) pub_seen = (int)ld_acquire(&S.published);
                    if (pub_seen > j) { state = 1; break; }
                    sdv = ld_acquire(&S.sched_done);
                    if (sdv && (unsigned int)j >= sdv - 1) { state = 0; break; }
                    if ((n & 63u) == 63u && (*abort_flag || pc.expired())) {
                        state = -1;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            state = __shfl_sync(0xffffffffu, state, 0);
            if (state == 0) {
                // the schedule holds T = sdv - 1 K-blocks: when a stage-mate has one in this round, this
                // warp still arrives (after the stage is free, so the arrival counts for this use)
                const unsigned int T = __shfl_sync(0xffffffffu, sdv, 0) - 1;
                if ((unsigned int)(it * kSubStages) < T) {
                    bool ok = true;
                    if (use > 0) ok = mbar_wait(smem_u32(&S.empty[stg]), (uint32_t)((use - 1) & 1), abort_flag);
                    if (__all_sync(0xffffffffu, ok)) {
                        if (lane == 0) mbar_arrive(smem_u32(&S.full[stg]));
                    } else {
                        failed = true;
                    }
                }
                break;
            }
            if (state < 0) {
                failed = true;
                break;
            }
            const KBMeta m = S.meta[j % kMetaRing];
            // this K-block's records, staged by the scheduler's bulk copy
            const int slot = j % kRecSlots;
            bool ok = mbar_wait(smem_u32(&S.rec_full[slot]), (uint32_t)((j / kRecSlots) & 1), abort_flag);
            // the stage slot: the MMAs of its previous round must be done with it
            if (ok && use > 0) ok = mbar_wait(smem_u32(&S.empty[stg]), (uint32_t)((use - 1) & 1), abort_flag);
            if (!__all_sync(0xffffffffu, ok)) {
                failed = true;
                break;
            }
            const bool valid = lane < m.cnt;
            SampleRec r = {0, 0, 0.0f, 0.0f};
            if (valid) r = recs[slot * kKB + lane];
            const int cx = r.xq >> 24, cy = r.yq >> 24;
            const int fxq = r.xq & 0xFFFFFF, fyq = r.yq & 0xFFFFFF;
            const int r0 = cx - (HW - 1), c0 = cy - (HW - 1);
            const bool rare = valid && (fxq == 0 || fyq == 0 || r0 < 0 || c0 < 0 || r0 >= g.T || c0 >= g.T2);
            const bool fast = valid && !rare;
            if (rare && a_role) {  // exact ES weights straight to the moment plane
                const int slab = m.key / tiles2;
                const int t1 = (m.key / g.ntile2) % g.ntile, t2 = m.key % g.ntile2;
                const long long o1 = g.gmin + (long long)t1 * g.T, o2 = g.gmin + (long long)t2 * g.T2;
                const int lo_r = fxq ? r0 : cx - HW, nr = fxq ? W : W + 1;
                const int lo_c = fyq ? c0 : cy - HW, nc = fyq ? W : W + 1;
                const float px = (float)fxq * (1.0f / 16777216.0f), py = (float)fyq * (1.0f / 16777216.0f);
                float2* plane = P.planes + (long long)(slab - P.slab_lo) * GG;
                for (int cidx = 0; cidx < nr * nc; ++cidx) {
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
            // ---- A: row taps (256 wx), chunks j0 and j0 + 1 at offset r0 % 8
            if (a_role) {
                const float ux = fmaf(2.0f, (float)fxq * (1.0f / 16777216.0f), -1.0f);
                float a[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    float w = poly.c[t][kPolyDeg];
#pragma unroll
                    for (int d = kPolyDeg - 1; d >= 0; --d) w = fmaf(w, ux, poly.c[t][d]);
                    a[t] = 256.0f * w;
                }
                const int j0 = fast ? (r0 >> 3) : -8;
                const int oldj = stg ? oldj1 : oldj0;
                if (oldj >= 0) {  // clear the previous sample's chunks the new one does not cover
#pragma unroll
                    for (int d = 0; d < 2; ++d) {
                        const int cj = oldj + d;
                        if (cj != j0 && cj != j0 + 1) {
                            st_chunk(A + kofs + a_chunk(cj) * 512, 0u, 0u, 0u, 0u);
                            st_chunk(A + kofs + (a_chunk(cj) + 2) * 512, 0u, 0u, 0u, 0u);
                        }
                    }
                }
                if (fast) {
                    uint32_t h[4], o[8];
                    const int c0h = a_chunk(j0), c1h = a_chunk(j0 + 1);
                    hi8<kBf16>(a, h);
                    window16(h, r0 & 7, o);
                    st_chunk(A + kofs + c0h * 512, o[0], o[1], o[2], o[3]);
                    st_chunk(A + kofs + c1h * 512, o[4], o[5], o[6], o[7]);
                    lo8<kBf16>(a, h);
                    window16(h, r0 & 7, o);
                    st_chunk(A + kofs + (c0h + 2) * 512, o[0], o[1], o[2], o[3]);
                    st_chunk(A + kofs + (c1h + 2) * 512, o[4], o[5], o[6], o[7]);
                }
                if (stg) oldj1 = fast ? j0 : -1;
                else oldj0 = fast ? j0 : -1;
            }
            // ---- B: column taps times the visibility (real: chunks 0-1, imaginary: chunks 2-3)
            else {
                const float uy = fmaf(2.0f, (float)fyq * (1.0f / 16777216.0f), -1.0f);
                float wy[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    float w = poly.c[t][kPolyDeg];
#pragma unroll
                    for (int d = kPolyDeg - 1; d >= 0; --d) w = fmaf(w, uy, poly.c[t][d]);
                    wy[t] = fast ? w * vscale : 0.0f;
                }
                const int sc = fast ? c0 : 0;
#pragma unroll
                for (int part = 0; part < 2; ++part) {
                    const float v = part ? r.vim : r.vre;
                    float b[8];
#pragma unroll
                    for (int t = 0; t < 8; ++t) b[t] = wy[t] * v;
                    uint32_t h[4], o[8];
                    unsigned char* bh = B_hi + kofs + part * 1024;
                    unsigned char* bl = B_lo + kofs + part * 1024;
                    hi8<kBf16>(b, h);
                    window16(h, sc, o);
                    st_chunk(bh, o[0], o[1], o[2], o[3]);
                    st_chunk(bh + 512, o[4], o[5], o[6], o[7]);
                    lo8<kBf16>(b, h);
                    window16(h, sc, o);
                    st_chunk(bl, o[0], o[1], o[2], o[3]);
                    st_chunk(bl + 512, o[4], o[5], o[6], o[7]);
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&S.full[stg]));
        }
        if (failed && lane == 0 && !*abort_flag) {
            atomicOr(P.status, 1u);
            *abort_flag = 1;
        }
    } else if (warp == kSchedWarp) {
        // ============================ scheduler ============================
        schedule_kblocks<kKB, kMetaRing, kRecSlots, kChunkKB>(S, P, smem + kRecOff, kb_lo, kb_hi, nullptr, nullptr,
                                                              abort_flag, lane);
    } else if (warp == kMmaWarp) {
        // ============================ MMA issuer ============================
        // Consecutive K-blocks of one key form an interval (at most kIntervalKB K-blocks) that
        // accumulates in one of the kAccBufs TMEM accumulators; closing it commits the
        // accumulator's MMAs to fdone[b] and hands the accumulator to the epilogue.
        int cur_key = -1;
        int ob = 0, on = 0, next_buf = 0;
        unsigned int fuse[kAccBufs];
#pragma unroll
        for (int b = 0; b < kAccBufs; ++b) fuse[b] = 0;
        unsigned int ev_n = 0;
        int last_commit_stage = -1;
        unsigned int last_commit_parity = 0;
        int open_stage = -1;  // stage whose last K-blocks never came (end of the schedule)
        unsigned int open_stage_parity = 0;
        bool failed = false;
        unsigned int ev_free_seen = 0;  // events consumed by every epilogue warp, last read
        auto push_event = [&](Event ev) {  // lane 0
            if (failed) return;
            PollClock pc;
            for (unsigned int n = 0;; ++n) {
                if (ev_n - ev_free_seen < (unsigned int)kEventRing) break;
                unsigned int mn = 0xFFFFFFFFu;
                for (int q = 0; q < 4; ++q) mn = min(mn, ld_acquire(&S.ev_consumed[q]));
                ev_free_seen = mn;
                if (ev_n - mn < (unsigned int)kEventRing) break;
                if ((n & 63u) == 63u && (*abort_flag || pc.expired())) {
                    failed = true;
                    return;
                }
                __nanosleep(32);
            }
            S.events[ev_n % kEventRing] = ev;
            ++ev_n;
            st_release(&S.ev_published, ev_n);
        };
        auto close_interval = [&]() {  // lane 0
            if (on > 0) {
                mma_commit(smem_u32(&S.fdone[ob]));
                push_event(Event{kEvDrain, ob, cur_key, (int)(fuse[ob] & 1u)});
                ++fuse[ob];
                on = 0;
            }
        };

        unsigned int pub_seen = 0;  // published count last read (acquire): meta[< pub_seen] are visible
        for (unsigned int i = 0;; ++i) {
            // wait until K-block i is published or the schedule ends before it
            int state = 0;
            if (lane == 0) {
                PollClock pc;
                for (unsigned int n = 0;; ++n) {
                    if (pub_seen > i) { state = 1; break; }
                    pub_seen = ld_acquire(&S.published);
                    if (pub_seen > i) { state = 1; break; }
                    const unsigned int sd = ld_acquire(&S.sched_done);
                    if (sd && i >= sd - 1) { state = 0; break; }
                    if ((n & 63u) == 63u && (*abort_flag || pc.expired())) {
                        state = -1;
                        break;
                    }
                    __nanosleep(32);
                }
                if (state < 0) failed = true;
            }
            state = __shfl_sync(0xffffffffu, state, 0);
            if (state <= 0) break;
            if (lane == 0 && !failed) {
                const int key = S.meta[i % kMetaRing].key;
                if (on > 0 && (key != cur_key || on == kIntervalKB)) close_interval();
                cur_key = key;
                if (on == 0) {  // open an interval on the next accumulator, once the epilogue has read it
                    const int b = next_buf;
                    next_buf = (next_buf + 1) % kAccBufs;
                    if (fuse[b] > 0 && !mbar_wait(smem_u32(&S.ffree[b]), (fuse[b] - 1) & 1u, abort_flag))
                        failed = true;
                    ob = b;
                }
                const int stg = (int)((i / kSubStages) % kPipe);
                const unsigned int u = i / (kSubStages * kPipe);
                const int sub = (int)(i % kSubStages);  // sub-stage of K-block i
                // one wait per stage (four K-blocks): a try_wait costs the issuing thread ~200 clk
                if (!failed && sub == 0 && !mbar_wait(smem_u32(&S.full[stg]), u & 1u, abort_flag)) failed = true;
                // producers and this warp are done with the descriptors and records of K-blocks <= i
                if (!failed && sub == kSubStages - 1) st_release(&S.consumed, i + 1);
                if (!failed) {
                    tc_fence_after();
                    const uint32_t d = tmem + (uint32_t)(kN * ob);
                    const uint32_t a = smem_u32(smem + stg * kStageBytes + sub * kSubBytes);
                    const uint32_t b = a + 2 * kABytes;
                    // one MMA per 16-sample K step: [A_hi; A_lo] x [B_hi | B_lo] gives all four
                    // hi/lo products in the accumulator's quarters
                    mma_f16(d, smem_desc(a), smem_desc(b), on > 0 ? 1u : 0u, idesc);
                    mma_f16(d, smem_desc(a + 256u), smem_desc(b + 256u), 1u, idesc);
                    if (sub == kSubStages - 1) {  // all K-blocks of the stage issued
                        mma_commit(smem_u32(&S.empty[stg]));
                        last_commit_stage = stg;
                        last_commit_parity = u & 1u;
                        open_stage = -1;
                    } else {
                        open_stage = stg;
                        open_stage_parity = u & 1u;
                    }
                    ++on;
                }
                if (failed && !*abort_flag) {
                    atomicOr(P.status, 2u);
                    *abort_flag = 1;
                }
            }
            if (__shfl_sync(0xffffffffu, (int)failed, 0) || *abort_flag) break;
        }
        if (lane == 0) {
            if (open_stage >= 0) {
                mma_commit(smem_u32(&S.empty[open_stage]));
                last_commit_stage = open_stage;
                last_commit_parity = open_stage_parity;
            }
            if (!failed && !*abort_flag) close_interval();
            push_event(Event{kEvExit, 0, 0, 0});
            if (failed && !*abort_flag) {
                atomicOr(P.status, 2u);
                *abort_flag = 1;
            }
            // no MMA of this CTA may still run when the tensor memory is freed
            if (last_commit_stage >= 0) {
                const volatile int never = 0;
                if (!mbar_wait(smem_u32(&S.empty[last_commit_stage]), last_commit_parity, &never))
                    atomicOr(P.status, 4u);
            }
        }
        __syncwarp();
    } else {
        // ============================ epilogue ============================
        // Warp q reads TMEM lane quarter q: lanes 0-15 hold accumulator rows 16q .. 16q + 15 of the
        // A_hi products, lanes 16-31 the same rows of the A_lo products; columns 0-31 come from
        // B_hi, 32-63 from B_lo (0-15 real, 16-31 imaginary within each). A lane adds its two column
        // halves, the partner lane (lane ^ 16) supplies the other A half, and the pair emits the
        // row's 16 complex cells to the moment plane (lanes 0-15 cells 0-7, lanes 16-31 cells 8-15),
        // checkerboard sign and 1 / scale applied, zero cells skipped.
        const int q = warp & 3;
        const uint32_t lane_addr = (uint32_t)(32 * q) << 16;
        const int row = 16 * q + (lane & 15);
        const int cell0 = (lane >> 4) * 8;
        for (unsigned int e = 0;; ++e) {
            bool ok = true;
            if (lane == 0) ok = wait_at_least(&S.ev_published, e + 1, abort_flag);
            if (!__shfl_sync(0xffffffffu, (int)ok, 0)) {
                if (lane == 0 && !*abort_flag) {
                    atomicOr(P.status, 8u);
                    *abort_flag = 1;
                }
                break;
            }
            const Event ev = S.events[e % kEventRing];
            if (ev.type == kEvExit) break;
            bool dn = mbar_wait(smem_u32(&S.fdone[ev.buf]), (uint32_t)ev.parity, abort_flag);
            dn = __all_sync(0xffffffffu, dn);
            if (!dn) {
                if (lane == 0 && !*abort_flag) {
                    atomicOr(P.status, 8u);
                    *abort_flag = 1;
                }
                break;
            }
            tc_fence_after();
            const uint32_t base = tmem + lane_addr + (uint32_t)(kN * ev.buf);
            float re[8], im[8];  // this lane's 8 cells of its row: real, imaginary
#pragma unroll
            for (int half = 0; half < 2; ++half) {  // cells 0-7, then 8-15
                uint32_t rh[8], rl[8], ih[8], il[8];
                tmem_ld8(base + (uint32_t)(8 * half), rh);        // real, B_hi
                tmem_ld8(base + (uint32_t)(32 + 8 * half), rl);   // real, B_lo
                tmem_ld8(base + (uint32_t)(16 + 8 * half), ih);   // imaginary, B_hi
                tmem_ld8(base + (uint32_t)(48 + 8 * half), il);   // imaginary, B_lo
                tmem_ld_wait();
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) {
                    float xr = __uint_as_float(rh[jj]) + __uint_as_float(rl[jj]);
                    float xi = __uint_as_float(ih[jj]) + __uint_as_float(il[jj]);
                    xr += __shfl_xor_sync(0xffffffffu, xr, 16);
                    xi += __shfl_xor_sync(0xffffffffu, xi, 16);
                    if ((lane >> 4) == half) {
                        re[jj] = xr;
                        im[jj] = xi;
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&S.ffree[ev.buf]));  // the accumulator is read
            const int slab = ev.key / tiles2;
            const int t1 = (ev.key / g.ntile2) % g.ntile, t2 = ev.key % g.ntile2;
            const long long g1 = g.gmin + (long long)t1 * g.T + row;
            const long long o2 = g.gmin + (long long)t2 * g.T2 + cell0;
            if (g1 <= g.gmax) {
                float2* prow = P.planes + (long long)(slab - P.slab_lo) * GG + (g1 - g.gmin) * g.G - g.gmin;
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) {
                    const long long g2 = o2 + jj;
                    if (g2 <= g.gmax && (re[jj] != 0.0f || im[jj] != 0.0f)) {
                        const float sg = ((g1 + g2) & 1) ? -inv_scale : inv_scale;
                        red_add_v2(prow + g2, sg * re[jj], sg * im[jj]);
                    }
                }
            }
            __syncwarp();
            if (lane == 0) st_release(&S.ev_consumed[q], e + 1);
        }
        if (lane == 0) st_release(&S.ev_consumed[q], 0xFFFFFFF0u);  // never block the event ring again
    }

    // ---- teardown: all roles done, no MMA in flight; free the tensor memory
    tc_fence_before();
    __syncthreads();
    if (warp == kMmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

}  // namespace

int launch_grid_tc(const SampleRec* d_rec, const unsigned int* d_offsets, const unsigned int* d_kb_offsets,
                   int n_keys, int key_lo, int key_hi, int slab_lo, const GridGeom& g, const EsPoly& poly,
                   float2* d_planes, const unsigned int* d_vmax, unsigned int* d_status, int sm_count,
                   cudaStream_t st, bool bf16) {
    if (key_lo < 0 || key_hi > n_keys || key_lo >= key_hi) {
        set_error("tensor-core gridder: bad key range");
        return SVDI_ERR_INTERNAL;
    }
    if (g.W > 8 || (g.W & 1) || g.T != kTcTileRows || g.T2 != kTcTileCols) {
        set_error("tensor-core gridder: needs even support <= 8 and 56 x 8 tiles");
        return SVDI_ERR_UNSUPPORTED;
    }
    if (reinterpret_cast<uintptr_t>(d_rec) % 16 != 0) {
        set_error("tensor-core gridder: records must be 16-byte aligned");
        return SVDI_ERR_INTERNAL;
    }
    auto kern = bf16 ? k_grid_tc<true> : k_grid_tc<false>;
    SVDI_TRY(ensure_dynamic_smem((const void*)kern, kSmemBytes, true));
    int per_sm = 0;
    SVDI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, kSmemBytes));
    if (per_sm < 1) {
        set_error("tensor-core gridder: kernel does not fit on an SM");
        return SVDI_ERR_UNSUPPORTED;
    }
    // d_status: [0] give-up flags, [1] max |value| (read through d_vmax), [2] the work counter
    SVDI_CUDA(cudaMemsetAsync(d_status + 2, 0, sizeof(unsigned int), st));
    TcParams P{d_rec, d_offsets, d_kb_offsets, d_vmax, d_planes, d_status, d_status + 2, key_lo, key_hi, slab_lo};
    // two CTAs per SM (two MMA-issuing threads: one thread issues a skinny MMA every ~46 clk, the
    // tensor pipe takes one every ~26), each with 256 of the SM's 512 TMEM columns; the records must
    // start 16-byte aligned for the bulk copies
    kern<<<2 * sm_count, kThreads, kSmemBytes, st>>>(P, g, poly);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

}  // namespace svdi
