// Exact integer tensor-core ES gridder (tcgen05.mma kind::i8, int32 accumulation in tensor
// memory), one Chebyshev term of the w-slabs' moment planes per launch, support W <= 8.
//
// Replaces the same reference kernels as the other gridders (fused_gridding,
// SVDIntegratedImager.cu:1218-1293, whose inner loop over the K Chebyshev terms is :1276-1290;
// gridding, archive/FIPkernels.cu:383-452). A launch grids term n of every slab in its key range:
// the sample's value is multiplied by T_n(s) (s the record's Chebyshev argument, T_n by the
// three-term recurrence in FP32) before B is quantised, and |T_n| <= 1 keeps the key's scale bound.
// K terms take K launches over the same records.
//
// Gridding with a separable kernel is a sum of outer products: for the samples k of one tile,
//   G[r][c] = sum_k  wx_k[r] * (wy_k[c] v_k)   =   (A B^T)[r][c].
// Here both factors are 22-bit fixed-point integers written as three byte digits,
//   A_q = round(0.999 2^22 wx)           = a_0 + 2^8 a_1 + 2^16 a_2   (unsigned bytes),
//   B_q = round(0.999 2^(22 - e) wy v)   = b_0 + 2^8 b_1 + 2^16 b_2   (signed bytes),
// with max |v| < 2^e over the tile key (the scatter's per-key maximum). The signed digits come from
// one add and one xor: the low three bytes of (B_q + 0x8080) ^ 0x8080 are b_0, b_1, b_2 in
// [-128, 127]. The digits are stacked along the MMA's M and N:
//   A' (M = 128): TMEM lane quarter q holds window rows 8q .. 8q + 7; lane 8d + j of the quarter is
//                 digit d of row 8q + j (lanes 24-31 of each quarter stay zero);
//   B' (N = 96):  column 32 e + 16 comp + c is digit e of window column c, real (comp 0) or
//                 imaginary (comp 1) part;
// so ONE tcgen05.mma kind::i8 (M = 128, N = 96, K = 32, A unsigned, B signed) per 32 samples forms
// all nine digit products D_de in int32, and the epilogue adds sum_de 2^(8 (d + e)) D_de, which is
// sum_k A_q B_q exactly. Integer accumulation does not round, so consecutive K-blocks of a tile key
// share one accumulator for as long as they last within a chunk of the schedule (at most
// kChunkKB = 64 K-blocks; int32 would hold kIntervalKB = 2048 of them: |a_d b_e| <= 255 * 128 for
// 65,536 samples), and the result does not depend on the order of the samples.
//
// Cost model (measured on B200): a tcgen05.mma costs its issuing thread ~140 clk (8-bit) whatever
// its N, and the tensor core reads shared-memory operands at ~100-117 B/clk per SM. The 8-bit form
// moves 7 KB of operands per 32 samples (4 KB A', 3 KB B') where the FP16 hi + lo form moves 12 KB
// in two MMAs. Two CTAs per SM issue in parallel.
//
// Tiles: binning uses 24-row x 8-column tiles of footprint origins; the accumulator covers the
// 32 x 16 window (tile plus the W - 1 halo).
//
// Operands (MN-major, no swizzle, 8-bit): a core matrix is 8 K (samples) x 16 bytes (16
// consecutive rows of A' or columns of B'); the next 8 K at +128 bytes, the next 16 M / N at +512
// bytes. One thread builds one sample's column of A' (warps 0-3) or of B' (warps 4-7) in 16-byte
// stores: A' quarter q is two 16-byte rows {digits 0 and 1 of its 8 rows} and {digit 2, zero}; a
// sample's 8 row taps at window rows r0 .. r0 + 7 fill quarter r0 / 8 shifted up by r0 % 8 bytes and,
// when r0 % 8 > 0, the start of the next quarter. B' group 2 e + comp is the 16 window columns of one
// digit and part, the sample's 8 column taps shifted up by c0 bytes. Of A' only the quarters the
// lane's previous sample in this stage slot wrote and the new one does not are cleared; B' is
// written in full.
//
// Roles, synchronisation, record staging (cp.async.bulk from this GPU's own memory, no multicast),
// rare samples (straight to the plane with exact weights) and the bounded waits with a CTA-wide
// abort flag follow the FP16 tensor-core gridder (gridder_tc.cu).
#include "svdi_internal.cuh"
#include "tc_sync.cuh"

namespace svdi {

namespace {

using namespace tc;

constexpr int kKB = kTcKBlock;          // samples per K-block (the MMA's K)
constexpr int kWinRows = 32;            // window rows: tile rows + halo (4 lane quarters x 8)
constexpr int kWinCols = 16;            // window columns: tile columns + halo
constexpr int kM = 128;                 // MMA rows: 4 quarters x 32 lanes
constexpr int kN = 96;                  // MMA columns: 3 digits x 2 parts x 16 columns
constexpr int kSubStages = 4;           // K-blocks per pipeline stage (one per producer warp pair)
constexpr int kPipe = 3;                // pipeline stages
constexpr int kProdWarps = 2 * kSubStages;                 // 8: A' warps 0-3, B' warps 4-7
constexpr int kSchedWarp = kProdWarps;                     // 8
constexpr int kMmaWarp = kProdWarps + 1;                   // 9
constexpr int kEpiWarp0 = kProdWarps + 2;                  // 10..13
constexpr int kWarps = kProdWarps + 2 + 4;
constexpr int kThreads = kWarps * 32;                      // 448
constexpr int kAccBufs = 2;             // TMEM accumulators of kN columns
constexpr int kAccStride = 128;         // TMEM columns between accumulators
constexpr int kIntervalKB = 2048;       // K-blocks per accumulator interval at most (int32 range)
constexpr int kTmemCols = 256;
constexpr int kMetaRing = 64;           // published K-block descriptors
constexpr int kRecSlots = 16;           // record slots: K-blocks staged ahead of the producers
constexpr int kChunkKB = 64;            // K-blocks per chunk of dynamically distributed work
constexpr int kEventRing = 64;

constexpr int kABytes = kM * kKB;                        // 4 KB
constexpr int kBBytes = kN * kKB;                        // 3 KB
constexpr int kSubBytes = kABytes + kBBytes;             // 7 KB: one K-block
constexpr int kStageBytes = kSubStages * kSubBytes;      // 28 KB
constexpr int kRecOff = kPipe * kStageBytes;             // record slots after the stages
constexpr int kRecBytes = kRecSlots * kKB * 16;          // 8 KB
constexpr int kEpiOff = kRecOff + kRecBytes;             // epilogue staging after the records
constexpr int kEpiStride = 36;                           // floats per staged lane row (32 + 4: no bank conflicts)
constexpr int kEpiBytes = 4 * 24 * kEpiStride * 4;       // 13.5 KB: 24 lanes per epilogue warp
constexpr int kSmemBytes = kEpiOff + kEpiBytes;          // 105.5 KB
static_assert(kSmemBytes > 228 * 1024 / 3 && 2 * (kSmemBytes + 4096) <= 228 * 1024, "two CTAs per SM");
static_assert((kAccBufs - 1) * kAccStride + kN <= kTmemCols, "TMEM plan exceeds the allocation");
static_assert(kI8TileRows + 8 <= kWinRows && kI8TileCols + 8 <= kWinCols, "tile + footprint must fit the window");
static_assert(kSubBytes % 1024 == 0, "K-block operands stay 1 KB aligned");
static_assert(kEpiWarp0 + 4 == kWarps, "four epilogue warps (one per TMEM lane quarter) come last");
static_assert(kRecSlots <= kMetaRing && kKB == 32, "one record slot per published K-block, one lane per record");
static_assert(kChunkKB <= kIntervalKB && kMetaRing % kSubStages == 0,
              "intervals end with their chunk; a stage's interval flags are one aligned word");

// MN-major, no-swizzle 8-bit operand with kKB K-columns: element (mn, k) at byte
// (mn % 16) + (k % 8) * 16 + (k / 8) * 128 + (mn / 16) * 512.
constexpr unsigned long long kDescFixed = ((128ull >> 4) << 16) | ((512ull >> 4) << 32) | (1ull << 46);
__device__ __forceinline__ unsigned long long smem_desc(uint32_t addr) {
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | kDescFixed;
}
// Instruction descriptor: S32 accumulator, A unsigned 8-bit, B signed 8-bit, both MN-major,
// N = 96, M = 128.
constexpr uint32_t kIdescI8 = (2u << 4) | (0u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                              ((uint32_t)(kN >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);

// Round-to-nearest integer of x for |x| < 2^22 through the float bit pattern of x + 1.5 2^23.
constexpr float kMagic = 12582912.0f;
constexpr int kMagicBits = 0x4B400000;
constexpr float kAScale = 0.999f * 4194304.0f;   // 0.999 * 2^22

// Byte d of each of w[0..3] (d = 0, 1, 2), gathered into one word: byte t of the result is byte d
// of w[t]. Used to turn four per-tap digit words into one word per digit.
__device__ __forceinline__ void digit_words(const uint32_t (&w)[4], uint32_t& d0, uint32_t& d1, uint32_t& d2) {
    const uint32_t t01 = __byte_perm(w[0], w[1], 0x5140);  // w0.b0 w1.b0 w0.b1 w1.b1
    const uint32_t t23 = __byte_perm(w[2], w[3], 0x5140);
    const uint32_t u01 = __byte_perm(w[0], w[1], 0x7362);  // w0.b2 w1.b2 w0.b3 w1.b3
    const uint32_t u23 = __byte_perm(w[2], w[3], 0x7362);
    d0 = __byte_perm(t01, t23, 0x5410);
    d1 = __byte_perm(t01, t23, 0x7632);
    d2 = __byte_perm(u01, u23, 0x5410);
}

__device__ __forceinline__ unsigned long long join64(uint32_t lo, uint32_t hi) {
    return ((unsigned long long)hi << 32) | lo;
}

__device__ __forceinline__ void st16(unsigned char* p, unsigned long long a, unsigned long long b) {
    *reinterpret_cast<uint4*>(p) = make_uint4((uint32_t)a, (uint32_t)(a >> 32), (uint32_t)b, (uint32_t)(b >> 32));
}

__device__ __forceinline__ void red_add_v4(float2* addr, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

struct I8Params {
    const SampleRec* rec;
    const unsigned int* offsets;
    const unsigned int* kb_offsets;  // exclusive scan of ceil(count / kKB) per key
    const unsigned int* keymax;      // per key max(|vre|, |vim|), float bits
    float2* planes;
    unsigned int* status;
    unsigned int* work;              // next chunk of K-blocks to hand out (zeroed by the host)
    const float* rec_s;              // per record Chebyshev argument (term > 0 only)
    int key_lo, key_hi, slab_lo;
    int K, term;                     // moment planes per slab; the term this launch grids
};

// T_n(s) by the three-term recurrence T_{k+1} = 2 s T_k - T_{k-1} (FP32, as the FP32 gridder)
__device__ __forceinline__ float cheb_term(int n, float s) {
    if (n == 0) return 1.0f;
    float tm2 = 1.0f, tm1 = s;
    for (int t = 2; t <= n; ++t) {
        const float tt = 2.0f * s * tm1 - tm2;
        tm2 = tm1;
        tm1 = tt;
    }
    return tm1;
}

enum EventType : int { kEvDrain = 0, kEvExit = 1 };
struct Event {
    int type;
    int buf;      // accumulator to drain
    int key;      // its tile key
    int parity;   // phase parity of the accumulator's MMAs-done barrier
    float inv;    // 1 / the key's fixed-point scale of B (0: no finite non-zero value)
};

struct __align__(8) I8Shared {
    unsigned long long full[kPipe];       // producers -> MMA: the stage's K-blocks written (8 warp arrivals)
    unsigned long long empty[kPipe];      // MMA -> producers: stage read (tcgen05.commit)
    unsigned long long rec_full[kRecSlots];  // scheduler's bulk copy -> producers: records staged
    unsigned long long fdone[kAccBufs];   // MMA -> epilogue: the interval's MMAs done (commit)
    unsigned long long ffree[kAccBufs];   // epilogue -> MMA: accumulator read (4 warp arrivals)
    KBMeta meta[kMetaRing];
    unsigned char open[kMetaRing];        // scheduler -> MMA: 1 where a K-block starts an interval
    Event events[kEventRing];
    unsigned int published;               // K-block descriptors published
    unsigned int consumed;                // K-blocks whose descriptor and records everyone is done with
    unsigned int sched_done;              // 1 + total K-blocks once the schedule is complete
    unsigned int ev_published;
    unsigned int ev_consumed[4];
    int abort;
    uint32_t tmem_base;
};

// kTerm: the launch grids a Chebyshev term n > 0 (reads the records' arguments, T_n(s) by the
// recurrence); term 0 is its own instantiation without that code, whose absence the one-term
// snapshots' instruction cache feels (0.656 -> 0.605 ms on the precision snapshot)
template <bool kTerm>
__global__ void __launch_bounds__(kThreads, 2) k_grid_i8(I8Params P, GridGeom g, EsPoly poly) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ I8Shared S;
    const SampleRec* recs = reinterpret_cast<const SampleRec*>(smem + kRecOff);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int W = g.W, HW = W / 2;
    const int tiles2 = g.ntile * g.ntile2;
    const long long GG = g.G * g.G;
    volatile int* abort_flag = &S.abort;

    // ---- set-up: tensor memory, barriers
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
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
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem_base;

    if (warp < kProdWarps) {
        // =========================== producers ===========================
        // warp -> sub-stage (warp % 4) and operand (A' for warps 0-3, B' for warps 4-7); lane ->
        // sample (K-slot) of the K-block; round `it` uses stage it % kPipe. The A' warp also adds
        // the rare samples to the plane.
        const int sw = warp % kSubStages;
        const bool a_role = warp < kSubStages;
        const int kofs = (lane & 7) * 16 + (lane >> 3) * 128;  // byte offset of this K-slot's 16-byte row
        unsigned int oldmask[kPipe];  // A' quarters this lane's previous sample wrote, per stage
#pragma unroll
        for (int s = 0; s < kPipe; ++s) oldmask[s] = 0;
        int pub_seen = 0;  // lane 0: published count last read (acquire)
        bool failed = false;
        for (int it = 0;; ++it) {
            const int j = it * kSubStages + sw;
            const int stg = it % kPipe;
            const int use = it / kPipe;  // earlier rounds of this stage
            unsigned char* const A = smem + stg * kStageBytes + sw * kSubBytes;
            unsigned char* const B = A + kABytes;
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
            // Chebyshev argument of the sample (launches of term n > 0)
            const float sarg = (kTerm && valid) ? P.rec_s[m.pos + lane] : 0.0f;
            const int cx = r.xq >> 24, cy = r.yq >> 24;
            const int fxq = r.xq & 0xFFFFFF, fyq = r.yq & 0xFFFFFF;
            const int r0 = cx - (HW - 1), c0 = cy - (HW - 1);
            const bool rare = valid && (fxq == 0 || fyq == 0 || r0 < 0 || c0 < 0 || r0 >= g.T || c0 >= g.T2);
            const bool fast = valid && !rare;
            if (a_role) {
                if (rare) {  // exact ES weights straight to the moment plane
                    const int slab = m.key / tiles2;
                    const int t1 = (m.key / g.ntile2) % g.ntile, t2 = m.key % g.ntile2;
                    const long long o1 = g.gmin + (long long)t1 * g.T, o2 = g.gmin + (long long)t2 * g.T2;
                    const int lo_r = fxq ? r0 : cx - HW, nr = fxq ? W : W + 1;
                    const int lo_c = fyq ? c0 : cy - HW, nc = fyq ? W : W + 1;
                    const float px = (float)fxq * (1.0f / 16777216.0f), py = (float)fyq * (1.0f / 16777216.0f);
                    const float tn = kTerm ? cheb_term(P.term, sarg) : 1.0f;
                    const float vre = r.vre * tn, vim = r.vim * tn;
                    float2* plane = P.planes + ((long long)(slab - P.slab_lo) * P.K + P.term) * GG;
                    for (int cidx = 0; cidx < nr * nc; ++cidx) {
                        const int rr = lo_r + cidx / nc, cc = lo_c + cidx % nc;
                        const long long g1 = o1 + rr, g2 = o2 + cc;
                        if (g1 < g.gmin || g2 < g.gmin || g1 > g.gmax || g2 > g.gmax) continue;
                        const float x = ((float)(rr - cx) - px) / (float)HW;
                        const float y = ((float)(cc - cy) - py) / (float)HW;
                        const float kv = es_exact(poly.beta, x) * es_exact(poly.beta, y);
                        const float sg = ((g1 + g2) & 1) ? -kv : kv;
                        red_add_v2(plane + (g1 - g.gmin) * g.G + (g2 - g.gmin), sg * vre, sg * vim);
                    }
                }
                // ---- A': row taps as 22-bit unsigned integers, three byte digits per row
                const float ux = fmaf(2.0f, (float)fxq * (1.0f / 16777216.0f), -1.0f);
                uint32_t qa[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    float w = poly.c[t][kPolyDeg];
#pragma unroll
                    for (int d = kPolyDeg - 1; d >= 0; --d) w = fmaf(w, ux, poly.c[t][d]);
                    qa[t] = (uint32_t)max(0, __float_as_int(fmaf(w, kAScale, kMagic)) - kMagicBits);
                }
                uint32_t dl[3], dh[3];  // digit d of taps 0-3 (dl) and 4-7 (dh), one byte per tap
                {
                    const uint32_t w0[4] = {qa[0], qa[1], qa[2], qa[3]};
                    const uint32_t w1[4] = {qa[4], qa[5], qa[6], qa[7]};
                    digit_words(w0, dl[0], dl[1], dl[2]);
                    digit_words(w1, dh[0], dh[1], dh[2]);
                }
                const int q0 = r0 >> 3, s8 = (r0 & 7) * 8;
                const unsigned int newmask = fast ? ((1u << q0) | (s8 ? (2u << q0) : 0u)) : 0u;
                const unsigned int om = stg == 0 ? oldmask[0] : (stg == 1 ? oldmask[1] : oldmask[2]);
                const unsigned int clr = om & ~newmask;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (clr & (1u << q)) {
                        st16(A + kofs + (2 * q) * 512, 0ull, 0ull);
                        st16(A + kofs + (2 * q + 1) * 512, 0ull, 0ull);
                    }
                }
                if (fast) {
                    unsigned long long lo[3], hi[3];  // quarter q0 (taps shifted up by r0 % 8) and q0 + 1
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const unsigned long long x = join64(dl[d], dh[d]);
                        lo[d] = x << s8;
                        hi[d] = s8 ? (x >> (64 - s8)) : 0ull;
                    }
                    st16(A + kofs + (2 * q0) * 512, lo[0], lo[1]);
                    st16(A + kofs + (2 * q0 + 1) * 512, lo[2], 0ull);
                    if (s8) {
                        st16(A + kofs + (2 * q0 + 2) * 512, hi[0], hi[1]);
                        st16(A + kofs + (2 * q0 + 3) * 512, hi[2], 0ull);
                    }
                }
                if (stg == 0) oldmask[0] = newmask;
                else if (stg == 1) oldmask[1] = newmask;
                else oldmask[2] = newmask;
            } else {
                // ---- B': column taps times the visibility as 22-bit signed integers, three signed
                // byte digits, shifted up by c0 bytes in each 16-column group
                const float ks = kTerm ? m.scale * cheb_term(P.term, sarg) : m.scale;
                const float uy = fmaf(2.0f, (float)fyq * (1.0f / 16777216.0f), -1.0f);
                float wy[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    float w = poly.c[t][kPolyDeg];
#pragma unroll
                    for (int d = kPolyDeg - 1; d >= 0; --d) w = fmaf(w, uy, poly.c[t][d]);
                    wy[t] = w;
                }
                const int sc = fast ? c0 * 8 : 0;
#pragma unroll
                for (int comp = 0; comp < 2; ++comp) {
                    const float vs = fast ? (comp ? r.vim : r.vre) * ks : 0.0f;
                    uint32_t qb[8];
#pragma unroll
                    for (int t = 0; t < 8; ++t)
                        qb[t] = (uint32_t)(__float_as_int(fmaf(wy[t], vs, kMagic)) - (kMagicBits - 0x8080)) ^ 0x8080u;
                    uint32_t el[3], eh[3];
                    {
                        const uint32_t w0[4] = {qb[0], qb[1], qb[2], qb[3]};
                        const uint32_t w1[4] = {qb[4], qb[5], qb[6], qb[7]};
                        digit_words(w0, el[0], el[1], el[2]);
                        digit_words(w1, eh[0], eh[1], eh[2]);
                    }
#pragma unroll
                    for (int e = 0; e < 3; ++e) {
                        const unsigned long long x = join64(el[e], eh[e]);
                        st16(B + kofs + (2 * e + comp) * 512, x << sc, sc ? (x >> (64 - sc)) : 0ull);
                    }
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
        schedule_kblocks<kKB, kMetaRing, kRecSlots, kChunkKB>(S, P, smem + kRecOff, kb_lo, kb_hi, P.keymax, S.open,
                                                              abort_flag, lane);
    } else if (warp == kMmaWarp) {
        // ============================ MMA issuer ============================
        // An interval -- K-blocks of one key, opened where the scheduler flagged a key change or a
        // chunk start -- accumulates in one of the kAccBufs
        // TMEM accumulators; closing the interval commits its MMAs to fdone[b] and hands the
        // accumulator to the epilogue.
        int cur_key = -1;
        float cur_inv = 0.0f;
        int ob = 0, on = 0, next_buf = 0;
        unsigned int fuse[kAccBufs];
#pragma unroll
        for (int b = 0; b < kAccBufs; ++b) fuse[b] = 0;
        unsigned int ev_n = 0;
        int last_commit_stage = -1;
        unsigned int last_commit_parity = 0;
        bool failed = false;
        unsigned int ev_free_seen = 0;  // events consumed by every epilogue warp, last read
        const unsigned long long desc0 = smem_desc(smem_u32(smem));
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
                push_event(Event{kEvDrain, ob, cur_key, (int)(fuse[ob] & 1u), cur_inv});
                ++fuse[ob];
                on = 0;
            }
        };

        unsigned int pub_seen = 0;  // published count last read (acquire): meta[< pub_seen] are visible
        // One round per pipeline stage: K-blocks 4s .. 4s + 3 (fewer at the end of the schedule),
        // their descriptors read by four lanes, one full-barrier wait, then the MMAs.
        for (unsigned int s = 0;; ++s) {
            const unsigned int i0 = s * kSubStages;
            const int stg = (int)(s % kPipe);
            const unsigned int u = s / kPipe;
            // how many of the stage's K-blocks exist, once they are all published (warp-uniform;
            // -1: give up)
            int nin = 0;
            if (lane == 0) {
                PollClock pc;
                for (unsigned int n = 0;; ++n) {
                    if (pub_seen >= i0 + kSubStages) { nin = kSubStages; break; }
                    pub_seen = ld_acquire(&S.published);
                    if (pub_seen >= i0 + kSubStages) { nin = kSubStages; break; }
                    const unsigned int sd = ld_acquire(&S.sched_done);
                    if (sd) {  // the schedule is complete: sd - 1 K-blocks, all published
                        pub_seen = sd - 1;
                        nin = pub_seen > i0 ? (int)min((unsigned int)kSubStages, pub_seen - i0) : 0;
                        break;
                    }
                    if ((n & 63u) == 63u && (*abort_flag || pc.expired())) {
                        nin = -1;
                        break;
                    }
                    __nanosleep(32);
                }
                if (nin < 0) failed = true;
            }
            nin = __shfl_sync(0xffffffffu, nin, 0);
            if (nin <= 0) break;
            // the stage's interval starts, one byte per K-block (the scheduler's; published with the
            // descriptors); a K-block's key and scale are read only where an interval opens
            if (lane == 0 && !failed) {
                const uint32_t opens = *reinterpret_cast<const uint32_t*>(&S.open[i0 % kMetaRing]);
                if (!mbar_wait(smem_u32(&S.full[stg]), u & 1u, abort_flag)) failed = true;
                tc_fence_after();  // the producers' operand writes are ordered before the MMAs
                // producers and this warp are done with the descriptors and records of the stage
                if (!failed) st_release(&S.consumed, i0 + (unsigned int)nin);
                const unsigned long long da0 = desc0 + (unsigned long long)((stg * kStageBytes) >> 4);
#pragma unroll
                for (int k = 0; k < kSubStages; ++k) {
                    if (k < nin && !failed) {
                        if ((opens >> (8 * k)) & 1u) {  // a new interval on the next accumulator
                            close_interval();
                            const KBMeta& mt = S.meta[(i0 + k) % kMetaRing];
                            cur_key = mt.key;
                            cur_inv = mt.inv_scale;
                            const int b = next_buf;
                            next_buf = (next_buf + 1) % kAccBufs;
                            if (fuse[b] > 0 && !mbar_wait(smem_u32(&S.ffree[b]), (fuse[b] - 1) & 1u, abort_flag))
                                failed = true;
                            ob = b;
                        }
                        if (!failed) {
                            const unsigned long long da = da0 + (unsigned long long)((k * kSubBytes) >> 4);
                            mma_i8(tmem + (uint32_t)(kAccStride * ob), da, da + (kABytes >> 4), on > 0 ? 1u : 0u,
                                   kIdescI8);
                            ++on;
                        }
                    }
                }
                // the stage is free again once its MMAs are done (the producers wait on empty)
                mma_commit(smem_u32(&S.empty[stg]));
                last_commit_stage = stg;
                last_commit_parity = u & 1u;
                if (failed && !*abort_flag) {
                    atomicOr(P.status, 2u);
                    *abort_flag = 1;
                }
            }
            if (__shfl_sync(0xffffffffu, (int)failed, 0) || *abort_flag) break;
        }
        if (lane == 0) {
            if (!failed && !*abort_flag) close_interval();
            push_event(Event{kEvExit, 0, 0, 0, 0.0f});
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
        // Warp q reads TMEM lane quarter q: lane 8d + j (d < 3) holds the digit-d products of window
        // row 8q + j against the 96 B' columns. The lane adds its three B digits per (part, column),
        // F = D_0 + 2^8 D_1 + 2^16 D_2 in FP32, and stages 2^(8d) F in shared memory as (re, im)
        // pairs of its row's 16 columns. The warp then emits the 8 rows x 16 cells: lane L takes
        // cells 2k, 2k + 1 (k = L % 8) of row 4 it + L / 8 (it = 0, 1), adds the three digit rows and
        // issues one 16-byte reduction of the two complex cells (checkerboard sign and 1 / scale
        // applied); eight lanes cover a row's 128 bytes.
        const int q = warp & 3;
        const uint32_t lane_addr = (uint32_t)(32 * q) << 16;
        const int d = lane >> 3, jr = lane & 7;
        const float w_own = d == 0 ? 1.0f : (d == 1 ? 256.0f : 65536.0f);
        float* const stage = reinterpret_cast<float*>(smem + kEpiOff) + q * 24 * kEpiStride;
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
            const uint32_t base = tmem + lane_addr + (uint32_t)(kAccStride * ev.buf);
#pragma unroll
            for (int half = 0; half < 2; ++half) {  // columns 0-7, then 8-15
                uint32_t x0[8], x1[8], x2[8], y0[8], y1[8], y2[8];
                const uint32_t col = (uint32_t)(8 * half);
                tmem_ld8(base + col, x0);        // real, B digit 0
                tmem_ld8(base + 32 + col, x1);   // real, B digit 1
                tmem_ld8(base + 64 + col, x2);   // real, B digit 2
                tmem_ld8(base + 16 + col, y0);   // imaginary, B digit 0
                tmem_ld8(base + 48 + col, y1);
                tmem_ld8(base + 80 + col, y2);
                tmem_ld_wait();
                if (d < 3) {
                    float4* dst = reinterpret_cast<float4*>(stage + (8 * d + jr) * kEpiStride + 16 * half);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        float f[4];
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int c = 2 * k + h;
                            f[2 * h] = w_own * fmaf(65536.0f, (float)(int)x2[c], fmaf(256.0f, (float)(int)x1[c], (float)(int)x0[c]));
                            f[2 * h + 1] = w_own * fmaf(65536.0f, (float)(int)y2[c], fmaf(256.0f, (float)(int)y1[c], (float)(int)y0[c]));
                        }
                        dst[k] = make_float4(f[0], f[1], f[2], f[3]);
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&S.ffree[ev.buf]));  // the accumulator is read
            // cells in 32-bit plane coordinates (0 .. G - 1; G <= 46340, so r G + c fits)
            const int slab = ev.key / tiles2;
            const int rem = ev.key - slab * tiles2;
            const int t1 = rem / g.ntile2, t2 = rem - t1 * g.ntile2;
            const float inv_scale = ev.inv * (1.0f / kAScale);
            const int k2 = lane & 7;
            const int last = (int)(g.G - 1);
            const int gi = (int)g.G;
            const int c = t2 * g.T2 + 2 * k2;        // this lane's first cell column
            const int r0 = t1 * g.T + 8 * q;         // the warp's first window row
            float2* const plane = P.planes + ((long long)(slab - P.slab_lo) * P.K + P.term) * GG;
#pragma unroll
            for (int it = 0; it < 2; ++it) {
                const int jrow = 4 * it + (lane >> 3);
                float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
                for (int dd = 0; dd < 3; ++dd) {
                    const float4 u = reinterpret_cast<const float4*>(stage + (8 * dd + jrow) * kEpiStride)[k2];
                    v.x += u.x;
                    v.y += u.y;
                    v.z += u.z;
                    v.w += u.w;
                }
                const int r = r0 + jrow;
                if (r <= last && c <= last && (v.x != 0.0f || v.y != 0.0f || v.z != 0.0f || v.w != 0.0f)) {
                    // checkerboard sign of grid cell (gmin + r, gmin + c): 2 gmin is even
                    const float s0 = ((r + c) & 1) ? -inv_scale : inv_scale;
                    const int cell = r * gi + c;
                    float2* p = plane + cell;
                    if (c + 1 <= last && (cell & 1) == 0) {  // two cells, 16-byte aligned
                        red_add_v4(p, s0 * v.x, s0 * v.y, -s0 * v.z, -s0 * v.w);
                    } else {
                        red_add_v2(p, s0 * v.x, s0 * v.y);
                        if (c + 1 <= last) red_add_v2(p + 1, -s0 * v.z, -s0 * v.w);
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

int launch_grid_i8(const SampleRec* d_rec, const float* d_rec_s, const unsigned int* d_offsets,
                   const unsigned int* d_kb_offsets, int n_keys, int key_lo, int key_hi, int slab_lo, int K,
                   const GridGeom& g, const EsPoly& poly, float2* d_planes, const unsigned int* d_keymax,
                   unsigned int* d_status, int sm_count, cudaStream_t st) {
    if (key_lo < 0 || key_hi > n_keys || key_lo >= key_hi) {
        set_error("integer tensor-core gridder: bad key range");
        return SVDI_ERR_INTERNAL;
    }
    if (K < 1 || (K > 1 && !d_rec_s)) {
        set_error("integer tensor-core gridder: K > 1 needs the records' Chebyshev arguments");
        return SVDI_ERR_INTERNAL;
    }
    if (g.W > 8 || (g.W & 1) || g.T != kI8TileRows || g.T2 != kI8TileCols || g.G > 46340) {
        set_error("integer tensor-core gridder: needs even support <= 8, 24 x 8 tiles and a grid of at most 46340");
        return SVDI_ERR_UNSUPPORTED;
    }
    if (reinterpret_cast<uintptr_t>(d_rec) % 16 != 0) {
        set_error("integer tensor-core gridder: records must be 16-byte aligned");
        return SVDI_ERR_INTERNAL;
    }
    SVDI_TRY(ensure_dynamic_smem((const void*)k_grid_i8<false>, kSmemBytes, true));
    if (K > 1) SVDI_TRY(ensure_dynamic_smem((const void*)k_grid_i8<true>, kSmemBytes, true));
    int per_sm = 0;
    SVDI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_grid_i8<false>, kThreads, kSmemBytes));
    if (per_sm < 1) {
        set_error("integer tensor-core gridder: kernel does not fit on an SM");
        return SVDI_ERR_UNSUPPORTED;
    }
    // d_status: [0] give-up flags, [2] the work counter; one launch per Chebyshev term
    for (int term = 0; term < K; ++term) {
        SVDI_CUDA(cudaMemsetAsync(d_status + 2, 0, sizeof(unsigned int), st));
        I8Params P{d_rec,  d_offsets, d_kb_offsets, d_keymax, d_planes, d_status, d_status + 2,
                   d_rec_s, key_lo,    key_hi,       slab_lo,  K,        term};
        // two CTAs per SM (two MMA-issuing threads), each with 256 of the SM's 512 TMEM columns
        if (term == 0) k_grid_i8<false><<<2 * sm_count, kThreads, kSmemBytes, st>>>(P, g, poly);
        else k_grid_i8<true><<<2 * sm_count, kThreads, kSmemBytes, st>>>(P, g, poly);
        SVDI_LAUNCHED();
    }
    return SVDI_OK;
}

}  // namespace svdi
