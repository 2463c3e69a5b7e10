// probe_tcgen05_mma: issue and completion rates of the skinny tcgen05.mma shapes the tensor-core
// gridders use, with shared-memory operands in the MN-major no-swizzle layout, and an exact check of
// that layout (FP16 and unsigned x signed 8-bit operands against a host product).
//
// For each shape it reports, per K-block of 32 samples (one 8-bit MMA of K = 32, or two FP16 MMAs
// of K = 16): the issuing thread's clock cycles in a loop of back-to-back MMAs into one accumulator,
// the cycles until their commit arrives, per CTA and per SM, and the operand bytes the tensor core
// read per SM clock. The issuer variant runs 1, 2 or 4 issuing warps per CTA into their own
// accumulators with precomputed descriptors. Every wait is bounded (0.5 s) and reported.
//
// Output: one line per measurement; exit status 1 if a layout check or a wait failed.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#define CK(x)                                                                                 \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess) {                                                              \
            std::printf("CUDA error %s at %s:%d: %s\n", #x, __FILE__, __LINE__, cudaGetErrorString(e_)); \
            std::exit(2);                                                                     \
        }                                                                                     \
    } while (0)

namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long gns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ bool mbar_wait(uint32_t addr, uint32_t parity) {  // bounded: about 0.5 s
    const unsigned long long t0 = gns();
    for (unsigned int it = 0; it < (1u << 26); ++it) {
        if (mbar_try(addr, parity)) return true;
        if ((it & 63u) == 63u && gns() - t0 > 500000000ull) return false;
    }
    return false;
}
__device__ __forceinline__ void mma_f16(uint32_t d, unsigned long long a, unsigned long long b, uint32_t idesc,
                                        uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_i8(uint32_t d, unsigned long long a, unsigned long long b, uint32_t idesc,
                                       uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
// MN-major, no swizzle: the next 8 K at +128 bytes (LBO), the next 16 bytes of M / N at +512 (SBO)
__device__ __forceinline__ unsigned long long sdesc(uint32_t addr) {
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((128ull >> 4) << 16) | ((512ull >> 4) << 32) | (1ull << 46);
}

struct Shape {
    int kind;  // 0: FP16 (two K = 16 MMAs per K-block), 1: u8 x s8 (one K = 32 MMA)
    int M, N;
    int a_bytes, b_bytes;  // one K-block of 32 samples
    int slots;             // K-block operand slots cycled through
    uint32_t idesc;
};

__device__ __forceinline__ void issue_kblock(const Shape& c, uint32_t d, unsigned long long a, unsigned long long b,
                                             uint32_t acc) {
    if (c.kind == 0) {
        mma_f16(d, a, b, c.idesc, acc);
        mma_f16(d, a + 16, b + 16, c.idesc, 1u);  // second K half, +256 bytes
    } else {
        mma_i8(d, a, b, c.idesc, acc);
    }
}

// `issuers` warps (lane 0 each) issue n_kb / issuers K-blocks into their own accumulators (columns
// w * N). Slots are filled from src (src_bytes, wrapped). Block 0 optionally reads the first
// accumulator back (M = 128 only).
// commit_every > 0: the issuer also commits its MMAs to a second mbarrier after every commit_every
// K-blocks (as a pipeline frees a stage), without waiting on it.
__global__ void __launch_bounds__(128) k_probe(Shape c, int n_kb, int issuers, const unsigned char* __restrict__ src,
                                               int src_bytes, unsigned long long* cyc, int* status, int* out,
                                               int commit_every) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) unsigned long long bar[4];
    __shared__ __align__(8) unsigned long long stage_bar[4];
    __shared__ uint32_t tbase;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int slot_bytes = (c.a_bytes + c.b_bytes + 1023) & ~1023;
    for (int i = tid; i < c.slots * slot_bytes; i += 128) sm[i] = src[i % src_bytes];
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tbase)), "r"(256)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int w = 0; w < 4; ++w) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bar[w])), "r"(1) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&stage_bar[w])), "r"(1) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tbase;
    if (warp < issuers && lane == 0) {
        unsigned long long ad[8], bd[8];
        const uint32_t base = smem_u32(sm);
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            const uint32_t a = base + (uint32_t)((s % c.slots) * slot_bytes);
            ad[s] = sdesc(a);
            bd[s] = sdesc(a + (uint32_t)c.a_bytes);
        }
        const uint32_t d = tmem + (uint32_t)(warp * c.N);
        const int mine = n_kb / issuers;
        const unsigned long long t0 = clock64();
        int until_commit = commit_every;  // K-blocks left before the next commit (a countdown: no division)
        for (int i = 0; i < mine; i += 8) {
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                if (i + s < mine) issue_kblock(c, d, ad[s], bd[s], (i + s) > 0 ? 1u : 0u);
                if (commit_every > 0 && --until_commit == 0) {
                    commit(smem_u32(&stage_bar[warp]));
                    until_commit = commit_every;
                }
            }
        }
        const unsigned long long t1 = clock64();
        commit(smem_u32(&bar[warp]));
        const bool ok = mbar_wait(smem_u32(&bar[warp]), 0);
        const unsigned long long t2 = clock64();
        if (!ok) atomicOr(status, 1);
        if (blockIdx.x == 0 && warp == 0) {
            cyc[0] = t1 - t0;
            cyc[1] = t2 - t0;
        }
        atomicMax(&cyc[2], t2 - t0);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (blockIdx.x == 0 && out != nullptr && c.M == 128) {
        for (int col = 0; col < c.N; col += 8) {  // warp w: TMEM lanes 32w .. 32w + 31
            uint32_t r[8];
            const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)col;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            for (int j = 0; j < 8; ++j) out[(32 * warp + lane) * c.N + col + j] = (int)r[j];
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
}

uint32_t idesc_of(int kind, int M, int N) {
    uint32_t d = (1u << 15) | (1u << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
    if (kind == 0) d |= (1u << 4);                 // F32 accumulator, F16 A and B
    else d |= (2u << 4) | (0u << 7) | (1u << 10);  // S32 accumulator, A unsigned 8-bit, B signed 8-bit
    return d;
}
int off_i8(int mn, int k) { return (mn % 16) + (k % 8) * 16 + (k / 8) * 128 + (mn / 16) * 512; }
int off_f16(int mn, int k) { return (mn % 8) * 2 + (k % 8) * 16 + (k / 8) * 128 + (mn / 8) * 512; }

Shape shape(int kind, int M, int N, int slots) {
    Shape c;
    c.kind = kind;
    c.M = M;
    c.N = N;
    c.slots = slots;
    c.a_bytes = kind == 0 ? M * 64 : M * 32;
    c.b_bytes = kind == 0 ? N * 64 : N * 32;
    c.idesc = idesc_of(kind, M, N);
    return c;
}

}  // namespace

int main() {
    CK(cudaSetDevice(0));
    cudaDeviceProp p;
    CK(cudaGetDeviceProperties(&p, 0));
    const int SM = p.multiProcessorCount;
    std::printf("device %s, %d SMs\n", p.name, SM);
    unsigned long long* d_cyc;
    int *d_status, *d_out;
    unsigned char* d_src;
    const int src_bytes = 1 << 20;
    CK(cudaMalloc(&d_cyc, 3 * sizeof(unsigned long long)));
    CK(cudaMalloc(&d_status, sizeof(int)));
    CK(cudaMalloc(&d_out, 128 * 256 * sizeof(int)));
    CK(cudaMalloc(&d_src, src_bytes));
    CK(cudaFuncSetAttribute(k_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    int failures = 0;

    // ---- layout checks: 4 K-blocks accumulated, exact against the host
    for (const Shape& c0 : {shape(0, 128, 64, 4), shape(1, 128, 96, 4)}) {
        Shape c = c0;
        const int slot_bytes = (c.a_bytes + c.b_bytes + 1023) & ~1023;
        std::vector<unsigned char> h(src_bytes, 0);
        std::vector<double> A(4 * c.M * 32), B(4 * c.N * 32);
        srand(7);
        for (int s = 0; s < 4; ++s) {
            unsigned char* sl = h.data() + s * slot_bytes;
            for (int m = 0; m < c.M; ++m)
                for (int k = 0; k < 32; ++k) {
                    int v;
                    if (c.kind == 0) {
                        v = rand() % 17 - 8;
                        const __half hv = __float2half((float)v);
                        std::memcpy(sl + off_f16(m, k), &hv, 2);
                    } else {
                        v = rand() % 256;
                        sl[off_i8(m, k)] = (unsigned char)v;
                    }
                    A[(s * c.M + m) * 32 + k] = v;
                }
            for (int n = 0; n < c.N; ++n)
                for (int k = 0; k < 32; ++k) {
                    int v;
                    if (c.kind == 0) {
                        v = rand() % 17 - 8;
                        const __half hv = __float2half((float)v);
                        std::memcpy(sl + c.a_bytes + off_f16(n, k), &hv, 2);
                    } else {
                        v = rand() % 256 - 128;
                        sl[c.a_bytes + off_i8(n, k)] = (unsigned char)(signed char)v;
                    }
                    B[(s * c.N + n) * 32 + k] = v;
                }
        }
        CK(cudaMemcpy(d_src, h.data(), src_bytes, cudaMemcpyHostToDevice));
        CK(cudaMemset(d_cyc, 0, 3 * sizeof(unsigned long long)));
        CK(cudaMemset(d_status, 0, sizeof(int)));
        CK(cudaMemset(d_out, 0, 128 * 256 * sizeof(int)));
        k_probe<<<1, 128, 4 * slot_bytes>>>(c, 4, 1, d_src, src_bytes, d_cyc, d_status, d_out, 0);
        CK(cudaGetLastError());
        CK(cudaDeviceSynchronize());
        int st;
        CK(cudaMemcpy(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost));
        std::vector<int> o(128 * 256);
        CK(cudaMemcpy(o.data(), d_out, o.size() * sizeof(int), cudaMemcpyDeviceToHost));
        int bad = 0;
        for (int m = 0; m < c.M; ++m)
            for (int n = 0; n < c.N; ++n) {
                double ref = 0;
                for (int s = 0; s < 4; ++s)
                    for (int k = 0; k < 32; ++k) ref += A[(s * c.M + m) * 32 + k] * B[(s * c.N + n) * 32 + k];
                double got;
                if (c.kind == 0) {
                    float f;
                    std::memcpy(&f, &o[m * c.N + n], 4);
                    got = f;
                } else {
                    got = o[m * c.N + n];
                }
                if (got != ref) ++bad;
            }
        std::printf("layout check %s M %d N %d: wait status %d, mismatched cells %d of %d\n", c.kind == 0 ? "f16" : "u8xs8",
                    c.M, c.N, st, bad, c.M * c.N);
        if (st || bad) ++failures;
    }

    // ---- rates
    std::vector<unsigned char> fill(src_bytes);
    for (int i = 0; i < src_bytes; ++i) fill[i] = (unsigned char)(i * 37 + 11);
    CK(cudaMemcpy(d_src, fill.data(), src_bytes, cudaMemcpyHostToDevice));
    for (const Shape& c : {shape(0, 128, 64, 8), shape(1, 128, 64, 8), shape(1, 128, 96, 8), shape(1, 128, 144, 8),
                           shape(1, 128, 240, 6)}) {
        const int slot_bytes = (c.a_bytes + c.b_bytes + 1023) & ~1023;
        const int smem = c.slots * slot_bytes;
        for (int issuers = 1; issuers <= 4; issuers *= 2) {
            if (issuers * c.N > 256) continue;
            for (int per_sm = 1; per_sm <= 2; ++per_sm) {
                const int n_kb = 4096;
                // per_sm 1: enough shared memory that only one CTA fits an SM; per_sm 2: two, not three
                const int req = std::max(smem, per_sm == 1 ? 120 * 1024 : 80 * 1024);
                if (per_sm == 2 && 2 * (req + 1024 + 256) > 228 * 1024) continue;
                CK(cudaMemset(d_cyc, 0, 3 * sizeof(unsigned long long)));
                CK(cudaMemset(d_status, 0, sizeof(int)));
                k_probe<<<SM * per_sm, 128, req>>>(c, n_kb, issuers, d_src, src_bytes, d_cyc, d_status, nullptr, 0);
                CK(cudaGetLastError());
                CK(cudaDeviceSynchronize());
                unsigned long long cy[3];
                int st;
                CK(cudaMemcpy(cy, d_cyc, sizeof(cy), cudaMemcpyDeviceToHost));
                CK(cudaMemcpy(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost));
                const double per_cta = (double)cy[2] / n_kb;  // slowest issuer's clk per CTA K-block
                const double per_sm_kb = per_cta / per_sm;
                std::printf(
                    "rate %s M %d N %3d issuers %d CTAs/SM %d: issuer %.1f clk per own K-block, %.1f clk per "
                    "K-block per CTA, %.1f per SM, %.1f operand B/clk/SM, wait status %d\n",
                    c.kind == 0 ? "f16 " : "u8s8", c.M, c.N, issuers, per_sm, (double)cy[0] / (n_kb / issuers), per_cta,
                    per_sm_kb, (c.a_bytes + c.b_bytes) / per_sm_kb, st);
                if (st) ++failures;
            }
        }
    }
    // ---- a commit (tcgen05.commit to an mbarrier, not waited on) after every 1, 4 or 16 K-blocks
    for (const Shape& c : {shape(1, 128, 96, 8), shape(0, 128, 64, 8)}) {
        const int slot_bytes = (c.a_bytes + c.b_bytes + 1023) & ~1023;
        const int req = std::max(c.slots * slot_bytes, 80 * 1024);
        for (int every : {0, 16, 4, 1}) {
            const int n_kb = 4096;
            CK(cudaMemset(d_cyc, 0, 3 * sizeof(unsigned long long)));
            CK(cudaMemset(d_status, 0, sizeof(int)));
            k_probe<<<SM * 2, 128, req>>>(c, n_kb, 1, d_src, src_bytes, d_cyc, d_status, nullptr, every);
            CK(cudaGetLastError());
            CK(cudaDeviceSynchronize());
            unsigned long long cy[3];
            int st;
            CK(cudaMemcpy(cy, d_cyc, sizeof(cy), cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost));
            std::printf("commit %s M %d N %3d, commit every %2d K-blocks (0: none), 2 CTAs/SM: issuer %.1f clk per K-block, "
                        "%.1f clk per K-block per CTA to completion, wait status %d\n",
                        c.kind == 0 ? "f16 " : "u8s8", c.M, c.N, every, (double)cy[0] / n_kb, (double)cy[2] / n_kb, st);
            if (st) ++failures;
        }
    }
    std::printf("%s\n", failures ? "FAILED" : "done");
    return failures ? 1 : 0;
}
