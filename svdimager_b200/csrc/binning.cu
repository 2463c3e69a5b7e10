// Tile binning of visibility samples: a counting sort of samples by (w-slab, grid tile).
//
// The reference grids every sample straight into global memory with float atomics
// (SVDIntegratedImager.cu:1218-1293, 64 * K * 2 atomics per sample). Here samples are first
// binned by the tile that holds the origin of their ES footprint, so that each tile is gridded in
// shared memory by one CTA. The binning contract is bit-exact and shared with the CPU oracle:
//
//   p      = r * (cell_size * G)                FP64 (or the reference's FP32 rounding)
//   Q      = floor(p * 2^24)                    position quantised to 2^-24 cells
//   cell   = Q >> 24, frac = Q & (2^24 - 1)
//   lo     = frac ? cell - (W/2 - 1) : cell - W/2   (= ceil(p - W/2)),  hi = cell + W/2
//   clip   lo, hi to [-G/2, (G-1)/2] (SVDIntegratedImager.cu:1261-1267); drop if lo > hi
//          (strict mode: drop if the footprint leaves the grid)
//   tile1  = (lo1 + G/2) / T1, tile2 = (lo2 + G/2) / T2 (tiles may be rectangular)
//   slab   = clamp(floor((r3 - r3_min) / width), 0, nslab - 1)
//   key    = (slab * ntile1 + tile1) * ntile2 + tile2
#include "binning_rules.cuh"
#include "svdi_internal.cuh"

namespace svdi {

namespace {

using namespace binrules;

constexpr int kThreads = 256;
constexpr int kPerThread = 8;                       // samples per thread per scatter chunk
constexpr int kChunk = kThreads * kPerThread;       // samples per scatter block
constexpr int kSmemKeyLimit = 24576;                // keys aggregated in shared memory

// Per-block shared-memory histogram (warp-aggregated), flushed once per block.
__global__ void __launch_bounds__(kThreads) k_histogram(SampleSource src, GridGeom g, SlabParams sp,
                                                       unsigned int* __restrict__ counts, int n_keys,
                                                       unsigned long long* __restrict__ dropped,
                                                       const DevPlan* __restrict__ plan) {
    if (plan) sp = plan->sp;
    extern __shared__ unsigned int sh[];
    const bool use_smem = n_keys <= kSmemKeyLimit;
    if (use_smem) {
        for (int k = threadIdx.x; k < n_keys; k += kThreads) sh[k] = 0;
        __syncthreads();
    }
    unsigned int ndrop = 0;
    const int lane = threadIdx.x & 31;
    const long long n = src.n;
    const long long stride = (long long)gridDim.x * kThreads;
    const long long n_round = ((n + stride - 1) / stride) * stride;
    for (long long idx = blockIdx.x * (long long)kThreads + threadIdx.x; idx < n_round; idx += stride) {
        int key = -2;
        if (idx < n) {
            key = sample_key(src, idx, g, sp).key;
            if (key < 0) ++ndrop;
        }
        const unsigned int peers = __match_any_sync(0xffffffffu, key);
        const int leader = __ffs(peers) - 1;
        if (key >= 0 && lane == leader) {
            const unsigned int c = __popc(peers);
            if (use_smem) atomicAdd(&sh[key], c);
            else atomicAdd(&counts[key], c);
        }
    }
    for (int o = 16; o > 0; o >>= 1) ndrop += __shfl_xor_sync(0xffffffffu, ndrop, o);
    if (lane == 0 && ndrop) atomicAdd(dropped, (unsigned long long)ndrop);
    if (use_smem) {
        __syncthreads();
        for (int k = threadIdx.x; k < n_keys; k += kThreads)
            if (sh[k]) atomicAdd(&counts[k], sh[k]);
    }
}

// Exclusive scan of the key counts (one block): offsets[0..n_keys], cursor = offsets. With
// kb_offsets, also the exclusive scan of ceil(count / kb_size): the K-blocks of kb_size records of
// one key each that the tensor-core gridder splits evenly over its CTAs. With chunk_key, for every
// chunk of chunk_size records the key its first record belongs to.
// The keys go through shared memory in tiles of kScanTile (coalesced loads and stores), each thread
// scanning kScanPer consecutive keys of a tile and the block combining the 1024 thread sums with warp
// shuffles; a running carry links the tiles.
constexpr int kScanPer = 4;               // keys (or chunks) per thread and tile
constexpr int kScanTile = kScanPer * 1024;

// Inclusive block-wide scan (sum or max) of one value per thread of a 1024-thread block; `tmp`
// holds 32 words of shared memory. Returns this thread's inclusive result and the block total.
template <bool kMax>
__device__ __forceinline__ unsigned int block_scan(unsigned int v, unsigned int* tmp, unsigned int& total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = kMax ? max(v, u) : v + u;
    }
    if (lane == 31) tmp[w] = v;
    __syncthreads();
    if (w == 0) {
        unsigned int x = tmp[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int u = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x = kMax ? max(x, u) : x + u;
        }
        tmp[lane] = x;
    }
    __syncthreads();
    if (w > 0) v = kMax ? max(v, tmp[w - 1]) : v + tmp[w - 1];
    total = tmp[31];
    __syncthreads();
    return v;
}

__global__ void __launch_bounds__(1024) k_scan(const unsigned int* __restrict__ counts, int n_keys,
                                              unsigned int* __restrict__ offsets,
                                              unsigned int* __restrict__ cursor,
                                              unsigned int* __restrict__ kb_offsets, int kb_size,
                                              unsigned int* __restrict__ chunk_key, int chunk_size) {
    __shared__ __align__(16) unsigned int tile[kScanTile];
    __shared__ __align__(16) unsigned int ktile[kScanTile];
    __shared__ unsigned int tmp[32];
    const int t = threadIdx.x;
    unsigned int carry = 0, kcarry = 0;
    if (chunk_key) {  // chunks are marked below: clear the table first (needs the record total)
        unsigned int sum = 0, total = 0;
        for (int k = t; k < n_keys; k += 1024) sum += counts[k];
        block_scan<false>(sum, tmp, total);
        const unsigned int n_chunks = (total + chunk_size - 1) / chunk_size;
        for (unsigned int ch = t; ch < n_chunks; ch += 1024) chunk_key[ch] = 0u;
        __syncthreads();
    }
    for (int base = 0; base < n_keys; base += kScanTile) {
        const int n = min(kScanTile, n_keys - base);
        for (int i = t; i < kScanTile; i += 1024) tile[i] = i < n ? counts[base + i] : 0u;
        __syncthreads();
        unsigned int c[kScanPer], s = 0, ks = 0;
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) {
            c[k] = tile[kScanPer * t + k];
            s += c[k];
            ks += (c[k] + kb_size - 1) / kb_size;
        }
        unsigned int tot = 0, ktot = 0;
        const unsigned int incl = block_scan<false>(s, tmp, tot);
        const unsigned int kincl = kb_offsets ? block_scan<false>(ks, tmp, ktot) : 0u;
        unsigned int run = carry + incl - s, krun = kcarry + kincl - ks;
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) {
            const int key = base + kScanPer * t + k;
            if (chunk_key && c[k] && key < n_keys) {  // the first chunk that starts inside this key's records
                const unsigned int ch = (run + chunk_size - 1) / chunk_size;
                if ((unsigned long long)ch * chunk_size < (unsigned long long)run + c[k]) chunk_key[ch] = (unsigned int)key;
            }
            tile[kScanPer * t + k] = run;
            run += c[k];
            ktile[kScanPer * t + k] = krun;
            krun += (c[k] + kb_size - 1) / kb_size;
        }
        __syncthreads();
        for (int i = t; i < n; i += 1024) {
            offsets[base + i] = tile[i];
            cursor[base + i] = tile[i];
            if (kb_offsets) kb_offsets[base + i] = ktile[i];
        }
        carry += tot;
        kcarry += ktot;
        __syncthreads();
    }
    if (t == 0) {
        offsets[n_keys] = carry;
        if (kb_offsets) kb_offsets[n_keys] = kcarry;
    }
    if (!chunk_key) return;
    // chunks without a mark start inside the key of the last mark before them: a running maximum
    // (keys increase along the records), in tiles with a carry
    __syncthreads();
    const unsigned int n_chunks = (carry + chunk_size - 1) / chunk_size;
    unsigned int mcarry = 0;
    for (unsigned int base = 0; base < n_chunks; base += kScanTile) {
        const unsigned int n = min((unsigned int)kScanTile, n_chunks - base);
        for (unsigned int i = t; i < (unsigned int)kScanTile; i += 1024) tile[i] = i < n ? chunk_key[base + i] : 0u;
        __syncthreads();
        unsigned int v[kScanPer], m = 0;
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) {
            m = max(m, tile[kScanPer * t + k]);
            v[k] = m;
        }
        unsigned int tot = 0;
        ktile[t] = block_scan<true>(m, tmp, tot);  // inclusive maximum over threads 0..t
        __syncthreads();
        const unsigned int before = max(mcarry, t ? ktile[t - 1] : 0u);
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) tile[kScanPer * t + k] = max(before, v[k]);
        __syncthreads();
        for (unsigned int i = t; i < n; i += 1024) chunk_key[base + i] = tile[i];
        mcarry = max(mcarry, tot);
        __syncthreads();
    }
}

// NaN or +-Inf: all exponent bits set
__device__ __forceinline__ unsigned int nonfinite2(float a, float b) {
    return ((__float_as_uint(a) & 0x7f800000u) == 0x7f800000u) | ((__float_as_uint(b) & 0x7f800000u) == 0x7f800000u);
}

// Adds the warp's non-finite record count to *counter (one atomic per warp that saw any).
__device__ __forceinline__ void flush_nonfinite(unsigned long long* counter, unsigned int nbad) {
    if (!counter || !__any_sync(0xffffffffu, nbad != 0)) return;
    for (int o = 16; o > 0; o >>= 1) nbad += __shfl_xor_sync(0xffffffffu, nbad, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(counter, (unsigned long long)nbad);
}

// Scatter: block-aggregated reservation of output ranges per key, then 16-byte record writes.
__global__ void __launch_bounds__(kThreads) k_scatter(SampleSource src, GridGeom g, SlabParams sp,
                                                     unsigned int* __restrict__ cursor, int n_keys,
                                                     SampleRec* __restrict__ rec, float* __restrict__ rec_s,
                                                     unsigned int* __restrict__ vmax,
                                                     unsigned int* __restrict__ keymax,
                                                     const DevPlan* __restrict__ plan) {
    if (plan) {
        sp = plan->sp;
        src.inv_det = plan->inv_det;
    }
    extern __shared__ unsigned int sh[];  // [n_keys] counts, then [n_keys] bases
    unsigned int* cnt = sh;
    unsigned int* base = sh + n_keys;
    const bool use_smem = n_keys <= kSmemKeyLimit / 2;
    const int lane = threadIdx.x & 31;
    const long long n = src.n;
    float vm = 0.0f;  // max |record value| written by this thread
    unsigned int nbad = 0;  // non-finite records written by this thread
    for (long long c0 = (long long)blockIdx.x * kChunk; c0 < n; c0 += (long long)gridDim.x * kChunk) {
        KeyRec kr[kPerThread];
        unsigned int rank[kPerThread];
        if (use_smem) {
            for (int k = threadIdx.x; k < n_keys; k += kThreads) cnt[k] = 0;
            __syncthreads();
        }
#pragma unroll
        for (int i = 0; i < kPerThread; ++i) {
            const long long idx = c0 + i * kThreads + threadIdx.x;
            kr[i].key = -2;
            if (idx < n) kr[i] = sample_key(src, idx, g, sp);
            const int key = kr[i].key;
            const unsigned int peers = __match_any_sync(0xffffffffu, key);
            const int leader = __ffs(peers) - 1;
            const unsigned int before = __popc(peers & ((1u << lane) - 1u));
            unsigned int b0 = 0;
            if (key >= 0 && lane == leader)
                b0 = use_smem ? atomicAdd(&cnt[key], __popc(peers)) : atomicAdd(&cursor[key], __popc(peers));
            b0 = __shfl_sync(0xffffffffu, b0, leader);
            rank[i] = b0 + before;
        }
        if (use_smem) {
            __syncthreads();
            for (int k = threadIdx.x; k < n_keys; k += kThreads) {
                const unsigned int c = cnt[k];
                base[k] = c ? atomicAdd(&cursor[k], c) : 0u;
            }
            __syncthreads();
        }
#pragma unroll
        for (int i = 0; i < kPerThread; ++i) {
            const long long idx = c0 + i * kThreads + threadIdx.x;
            const int key = kr[i].key;
            if (key < 0) continue;
            const unsigned int pos = use_smem ? base[key] + rank[i] : rank[i];
            SampleRec r;
            r.xq = kr[i].xq;
            r.yq = kr[i].yq;
            r.vre = __fmul_rn(src.vr[idx], src.inv_det);
            r.vim = __fmul_rn(src.vi[idx], src.inv_det);
            rec[pos] = r;
            if (rec_s) rec_s[pos] = kr[i].s;
            nbad += nonfinite2(r.vre, r.vim);
            const float m = fmaxf(fabsf(r.vre), fabsf(r.vim));
            vm = fmaxf(vm, m);
            if (keymax && m > 0.0f) atomicMax(&keymax[key], __float_as_uint(m));
        }
        if (use_smem) __syncthreads();
    }
    flush_nonfinite(src.nonfinite, nbad);
    if (vmax) {  // non-negative floats order like their bit patterns
        const unsigned int mb = __reduce_max_sync(0xffffffffu, __float_as_uint(vm));
        if (lane == 0 && mb) atomicMax(vmax, mb);
    }
}

// Separable sources (r = s[chan] q[row], idx = row + chan R). A warp takes units of kUnitRows
// rows x one chunk of `lpr` channels (lpr a power of two <= 32): lane -> (row kUnitRows-subset
// lane / lpr, channel lane % lpr), so consecutive lanes hold consecutive channels of one row. The
// channels of a baseline mostly share a tile, so match groups are large: one shared-memory or
// global atomic per group, and a group's records land in consecutive slots. No 64-bit division.
constexpr int kUnitRows = 16;
static_assert(32 / 2 <= kUnitRows, "every lane must take part in each row step");

struct SepMap {
    int lpr;       // lanes per row (channels per chunk)
    int nch;       // channel chunks
    int nrt;       // row tiles of kUnitRows
    int C;
};

__device__ inline void unit_of(long long u, const SepMap& m, int& rt, int& ch) {
    rt = (int)(u / m.nch);
    ch = (int)(u - (long long)rt * m.nch);
}

__global__ void __launch_bounds__(kThreads) k_histogram_sep(SampleSource src, SepMap m, GridGeom g, SlabParams sp,
                                                           unsigned int* __restrict__ counts, int n_keys,
                                                           unsigned long long* __restrict__ dropped,
                                                           const DevPlan* __restrict__ plan) {
    if (plan) sp = plan->sp;
    extern __shared__ unsigned int sh[];
    const bool use_smem = n_keys <= kSmemKeyLimit;
    if (use_smem) {
        for (int k = threadIdx.x; k < n_keys; k += kThreads) sh[k] = 0;
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    const int rps = 32 / m.lpr, sub = lane / m.lpr, coff = lane % m.lpr;
    const long long nunits = (long long)m.nrt * m.nch;
    const long long nwarps = (long long)gridDim.x * (kThreads / 32);
    unsigned int ndrop = 0;
    for (long long u = (long long)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5); u < nunits; u += nwarps) {
        int rt, ch;
        unit_of(u, m, rt, ch);
        const int c = ch * m.lpr + coff;
        const bool cvalid = c < m.C;
        const double sc = cvalid ? src.s[c] : 0.0;
        for (int i = sub; i < kUnitRows; i += rps) {
            const long long row = (long long)rt * kUnitRows + i;
            int key = -2;
            if (cvalid && row < src.R) {
                const double* q = src.q + row * 3;
                key = row_chan_key(sc, q[0], q[1], q[2], g, sp).key;
                if (key < 0) ++ndrop;
            }
            const unsigned int peers = __match_any_sync(0xffffffffu, key);
            if (key >= 0 && lane == __ffs(peers) - 1) {
                if (use_smem) atomicAdd(&sh[key], __popc(peers));
                else atomicAdd(&counts[key], __popc(peers));
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) ndrop += __shfl_xor_sync(0xffffffffu, ndrop, o);
    if (lane == 0 && ndrop) atomicAdd(dropped, (unsigned long long)ndrop);
    if (use_smem) {
        __syncthreads();
        for (int k = threadIdx.x; k < n_keys; k += kThreads)
            if (sh[k]) atomicAdd(&counts[k], sh[k]);
    }
}

// Scatter for separable sources: per unit, the warp stages the unit's collapsed visibilities in
// shared memory with row-contiguous loads, then writes each group's records to the slots one
// global atomic on the key's cursor reserved.
constexpr int kVisPitch = kUnitRows + 1;   // float2 pitch of a staged channel (bank-conflict free)

__global__ void __launch_bounds__(kThreads) k_scatter_sep(SampleSource src, SepMap m, GridGeom g, SlabParams sp,
                                                         unsigned int* __restrict__ cursor,
                                                         SampleRec* __restrict__ rec, float* __restrict__ rec_s,
                                                         unsigned int* __restrict__ vmax,
                                                         unsigned int* __restrict__ keymax,
                                                         const DevPlan* __restrict__ plan) {
    if (plan) {
        sp = plan->sp;
        src.inv_det = plan->inv_det;
    }
    __shared__ float2 stage[kThreads / 32][32 * kVisPitch];
    float2* my = stage[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int rps = 32 / m.lpr, sub = lane / m.lpr, coff = lane % m.lpr;
    const long long nunits = (long long)m.nrt * m.nch;
    const long long nwarps = (long long)gridDim.x * (kThreads / 32);
    const long long R = src.R;
    float vm = 0.0f;
    unsigned int nbad = 0;
    for (long long u = (long long)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5); u < nunits; u += nwarps) {
        int rt, ch;
        unit_of(u, m, rt, ch);
        const long long row0 = (long long)rt * kUnitRows;
        const int c0 = ch * m.lpr;
        // stage: lanes 0-15 and 16-31 read kUnitRows consecutive rows of two channels
        __syncwarp();
        for (int k = 0; k < m.lpr; k += 2) {
            const int cc = k + (lane >> 4);
            const long long row = row0 + (lane & 15);
            float2 v = make_float2(0.0f, 0.0f);
            if (c0 + cc < m.C && row < R) {
                const long long idx = row + (long long)(c0 + cc) * R;
                v = make_float2(src.vr[idx], src.vi[idx]);
            }
            my[cc * kVisPitch + (lane & 15)] = v;
        }
        __syncwarp();
        const int c = c0 + coff;
        const bool cvalid = c < m.C;
        const double sc = cvalid ? src.s[c] : 0.0;
        for (int i = sub; i < kUnitRows; i += rps) {
            const long long row = row0 + i;
            KeyRec kr;
            kr.key = -2;
            if (cvalid && row < R) {
                const double* q = src.q + row * 3;
                kr = row_chan_key(sc, q[0], q[1], q[2], g, sp);
            }
            const int key = kr.key;
            const unsigned int peers = __match_any_sync(0xffffffffu, key);
            const int leader = __ffs(peers) - 1;
            unsigned int b0 = 0;
            if (key >= 0 && lane == leader) b0 = atomicAdd(&cursor[key], __popc(peers));
            b0 = __shfl_sync(0xffffffffu, b0, leader);
            if (key >= 0) {
                const unsigned int pos = b0 + __popc(peers & ((1u << lane) - 1u));
                const float2 v = my[coff * kVisPitch + i];
                SampleRec r;
                r.xq = kr.xq;
                r.yq = kr.yq;
                r.vre = __fmul_rn(v.x, src.inv_det);
                r.vim = __fmul_rn(v.y, src.inv_det);
                rec[pos] = r;
                if (rec_s) rec_s[pos] = kr.s;
                nbad += nonfinite2(r.vre, r.vim);
                const float m = fmaxf(fabsf(r.vre), fabsf(r.vim));
                vm = fmaxf(vm, m);
                if (keymax) {  // the group's maximum, one atomic per group
                    const unsigned int gm = __reduce_max_sync(peers, __float_as_uint(m));
                    if (lane == leader && gm) atomicMax(&keymax[key], gm);
                }
            }
        }
    }
    flush_nonfinite(src.nonfinite, nbad);
    if (vmax) {  // non-negative floats order like their bit patterns
        const unsigned int mb = __reduce_max_sync(0xffffffffu, __float_as_uint(vm));
        if (lane == 0 && mb) atomicMax(vmax, mb);
    }
}

SepMap sep_map(const SampleSource& src) {
    SepMap m{};
    m.C = (int)(src.n / src.R);
    m.lpr = 2;   // >= 2: then 32 / lpr <= kUnitRows and every lane runs the same row loop
    while (m.lpr < 32 && m.lpr < m.C) m.lpr <<= 1;
    m.nch = (m.C + m.lpr - 1) / m.lpr;
    m.nrt = (int)((src.R + kUnitRows - 1) / kUnitRows);
    return m;
}

// Separable kernels need whole rows x channels and 32-bit unit and row counts.
bool use_sep(const SampleSource& src) {
    return !src.bin && src.R > 0 && src.n % src.R == 0 && src.n / src.R <= (1LL << 20) &&
           (src.R + kUnitRows - 1) / kUnitRows * ((src.n / src.R + 31) / 32) < (1LL << 31);
}

}  // namespace

int launch_histogram(const SampleSource& src, const GridGeom& g, const SlabParams& sp,
                     unsigned int* d_counts, int n_keys, unsigned long long* d_dropped,
                     cudaStream_t st, const DevPlan* d_plan) {
    const size_t smem = n_keys <= kSmemKeyLimit ? (size_t)n_keys * 4 : 0;
    if (use_sep(src)) {
        SVDI_TRY(ensure_dynamic_smem((const void*)k_histogram_sep, smem));
        const SepMap m = sep_map(src);
        const long long units = (long long)m.nrt * m.nch;
        long long blocks = (units + kThreads / 32 - 1) / (kThreads / 32);
        if (blocks > 4LL * current_sm_count()) blocks = 4LL * current_sm_count();   // a few units per warp: the shared histogram is flushed once
        if (blocks < 1) blocks = 1;
        k_histogram_sep<<<(int)blocks, kThreads, smem, st>>>(src, m, g, sp, d_counts, n_keys, d_dropped, d_plan);
        SVDI_LAUNCHED();
        return SVDI_OK;
    }
    SVDI_TRY(ensure_dynamic_smem((const void*)k_histogram, smem));
    long long blocks = (src.n + kThreads - 1) / kThreads;
    if (blocks > 8LL * current_sm_count()) blocks = 8LL * current_sm_count();
    if (blocks < 1) blocks = 1;
    k_histogram<<<(int)blocks, kThreads, smem, st>>>(src, g, sp, d_counts, n_keys, d_dropped, d_plan);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

int launch_scan(const unsigned int* d_counts, int n_keys, unsigned int* d_offsets,
                unsigned int* d_cursor, cudaStream_t st, unsigned int* d_kb_offsets, int kb_size,
                unsigned int* d_chunk_key, int chunk_size) {
    k_scan<<<1, 1024, 0, st>>>(d_counts, n_keys, d_offsets, d_cursor, d_kb_offsets, kb_size, d_chunk_key, chunk_size);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

int launch_scatter(const SampleSource& src, const GridGeom& g, const SlabParams& sp,
                   unsigned int* d_cursor, int n_keys, SampleRec* d_rec, float* d_rec_s,
                   unsigned int* d_vmax, cudaStream_t st, unsigned int* d_keymax, const DevPlan* d_plan) {
    if (use_sep(src)) {
        const SepMap m = sep_map(src);
        const long long units = (long long)m.nrt * m.nch;
        long long blocks = (units + kThreads / 32 - 1) / (kThreads / 32);
        if (blocks > 8LL * current_sm_count()) blocks = 8LL * current_sm_count();
        if (blocks < 1) blocks = 1;
        k_scatter_sep<<<(int)blocks, kThreads, 0, st>>>(src, m, g, sp, d_cursor, d_rec, d_rec_s, d_vmax, d_keymax,
                                                        d_plan);
        SVDI_LAUNCHED();
        return SVDI_OK;
    }
    const size_t smem = n_keys <= kSmemKeyLimit / 2 ? (size_t)n_keys * 8 : 0;
    SVDI_TRY(ensure_dynamic_smem((const void*)k_scatter, smem));
    long long blocks = (src.n + kChunk - 1) / kChunk;
    if (blocks > 16LL * current_sm_count()) blocks = 16LL * current_sm_count();
    if (blocks < 1) blocks = 1;
    k_scatter<<<(int)blocks, kThreads, smem, st>>>(src, g, sp, d_cursor, n_keys, d_rec, d_rec_s, d_vmax, d_keymax,
                                                   d_plan);
    SVDI_LAUNCHED();
    return SVDI_OK;
}

}  // namespace svdi
