// Synchronisation and tensor-memory helpers shared by the tcgen05 gridders (gridder_tc.cu,
// gridder_i8.cu): mbarriers with bounded waits, bulk copies from this GPU's global memory into
// shared memory (no multicast), tcgen05 fences, MMA issue and commit, TMEM loads.
#pragma once

#include <cstdint>

#include "svdi_internal.cuh"

namespace svdi {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Deadline of a bounded poll loop: the clock starts at the first check, so a loop that ends at once
// reads no timer; expired() turns true about one second later.
struct PollClock {
    unsigned long long t0 = 0;
    __device__ __forceinline__ bool expired() {
        const unsigned long long now = global_ns();
        if (t0 == 0) {
            t0 = now;
            return false;
        }
        return now - t0 > 1000000000ull;
    }
};

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

__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t addr) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(addr) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t addr, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(addr), "r"(bytes) : "memory");
}
// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from this GPU's global
// memory into this CTA's shared memory, completing on the mbarrier at `mbar` (no multicast).
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v) {
    asm volatile("st.release.cta.shared::cta.u32 [%0], %1;" ::"r"(smem_u32(p)), "r"(v) : "memory");
}

// Bounded waits (about one second of global time) that also give up when another thread of the
// CTA has given up (*abort != 0). They return false on either.
__device__ inline bool mbar_wait(uint32_t addr, uint32_t parity, const volatile int* abort) {
    if (mbar_try(addr, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (unsigned int it = 1; it < (1u << 28); ++it) {
        if (mbar_try(addr, parity)) return true;
        if ((it & 63u) == 0 && (*abort || global_ns() - t0 > 1000000000ull)) return false;
    }
    return false;
}
__device__ inline bool wait_at_least(const unsigned int* p, unsigned int target, const volatile int* abort) {
    if (ld_acquire(p) >= target) return true;
    const unsigned long long t0 = global_ns();
    for (unsigned int it = 1; it < (1u << 28); ++it) {
        __nanosleep(64);
        if (ld_acquire(p) >= target) return true;
        if ((it & 15u) == 0 && (*abort || global_ns() - t0 > 1000000000ull)) return false;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, unsigned long long a, unsigned long long b, uint32_t accum,
                                        uint32_t idesc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accum)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

// 8 consecutive TMEM columns of this thread's lane (the wait is separate: issue several, then wait).
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void red_add_v2(float2* addr, float a, float b) {
    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(addr), "f"(a), "f"(b) : "memory");
}

// Exact ES kernel psi(x) = exp(beta (sqrt(1 - x^2) - 1)) written without cancellation.
__device__ __forceinline__ float es_exact(float beta, float x) {
    if (fabsf(x) > 1.0f) return 0.0f;
    return expf(-beta * x * x / (1.0f + sqrtf((1.0f - x) * (1.0f + x))));
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, unsigned long long a, unsigned long long b, uint32_t accum,
                                       uint32_t idesc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accum)
        : "memory");
}

// One K-block of a tile key: records [pos, pos + cnt) of the binned record array.
struct KBMeta {
    int key;            // tile key of the K-block
    unsigned int pos;   // first record
    int cnt;            // records (1..32)
    float scale;        // per-key fixed-point scale of the integer gridder (0 elsewhere)
    float inv_scale;    // 1 / scale (0 with it)
};

// Fixed-point scale of a key whose largest |value| is vmax: 0.999 2^(22 - e) with vmax < 2^e, so
// that |w v| * scale < 2^22 for |w| <= 1; 0 when the key holds no finite non-zero value.
__device__ __forceinline__ float key_fixed_scale(float vmax) {
    if (!(vmax > 0.0f && vmax < 3.0e38f)) return 0.0f;
    int ex;
    frexpf(vmax, &ex);  // vmax = f 2^ex, f in [0.5, 1)
    return ldexpf(0.999f, max(-100, min(100, 22 - ex)));
}

// The K-blocks of keys [key_lo, key_hi) are handed out in chunks of kChunkKB from a global
// counter (dynamic balance: CTAs whose tiles cost more take fewer chunks). K-block m of key k
// covers records [offsets[k] + kKB m, min(offsets[k + 1], offsets[k] + kKB (m + 1))).
// The warp publishes up to 32 K-blocks at a time, one per lane: lane l holds offsets, kb_offsets
// and keymax of key kc + l of the current 32-key window (the next window is loaded one ahead), a
// lane finds its K-block's key by a binary search over the window's kb_offsets (shuffles), writes
// the descriptor and issues the bulk copy of the K-block's records (one contiguous run of 16-byte
// records from this GPU's global memory, no multicast) on the record slot's mbarrier. At most
// kRecSlots K-blocks are published ahead of `consumed`.
// Run by one warp (`lane` its lane); S and P are the kernel's shared state and parameters (members
// meta, rec_full, published, consumed, sched_done; offsets, kb_offsets, key_lo, key_hi, work, rec,
// status), rec_smem the record slots, [kb_lo, kb_hi) the K-blocks of the key range; keymax (may be
// null) the per-key max |value| from which each K-block's scale is set; open (may be null, kMetaRing
// bytes) receives per published K-block 1 when it starts an accumulation interval -- its key differs
// from the previous published K-block's, or it is the first of its chunk -- and 0 otherwise.
template <int kKB, int kMetaRing, int kRecSlots, int kChunkKB, class Shared, class Params>
__device__ void schedule_kblocks(Shared& S, const Params& P, unsigned char* rec_smem, unsigned int kb_lo,
                                 unsigned int kb_hi, const unsigned int* keymax, unsigned char* open,
                                 const volatile int* abort_flag, int lane) {
    static_assert(kRecSlots <= 32 && kRecSlots <= kMetaRing, "one lane per K-block published at once");
    struct Window {
        unsigned int off, kbo, km;  // this lane's key
        unsigned int off_e, kbo_e;  // key kc + 32 (clamped to key_hi)
    };
    auto fetch = [&](int base) {
        Window w;
        const int k = min(base + lane, P.key_hi);
        w.off = P.offsets[k];
        w.kbo = P.kb_offsets[k];
        w.km = keymax ? keymax[min(k, P.key_hi - 1)] : 0u;
        const int ke = min(base + 32, P.key_hi);
        w.off_e = P.offsets[ke];
        w.kbo_e = P.kb_offsets[ke];
        return w;
    };
    unsigned int published = 0;
    int prev_key = -1;  // key of the last K-block published (warp-uniform)
    bool ok = true;
    for (;;) {
        // next chunk of K-blocks
        unsigned int c = 0;
        if (lane == 0) c = atomicAdd(P.work, 1u);
        c = __shfl_sync(0xffffffffu, c, 0);
        const unsigned long long kb0l = (unsigned long long)kb_lo + (unsigned long long)c * kChunkKB;
        if (kb0l >= kb_hi) break;
        const unsigned int kb0 = (unsigned int)kb0l, kb1 = min(kb_hi, kb0 + (unsigned int)kChunkKB);
        // its first key: the last key with kb_offsets[key] <= kb0 (32 probes per round)
        int lo = P.key_lo, hi = P.key_hi;
        while (hi - lo > 1) {
            const int step = (hi - lo + 31) / 32;
            const int probe = lo + lane * step;
            const bool le = probe < hi && P.kb_offsets[probe] <= kb0;
            const unsigned int bal = __ballot_sync(0xffffffffu, le);
            const int lmax = 31 - __clz(bal);  // lane 0 always qualifies (kb_offsets[lo] <= kb0)
            const int nlo = lo + lmax * step;
            hi = min(hi, nlo + step);
            lo = nlo;
        }
        int kc = lo;  // window [kc, kc + 32): kb_offsets[kc] <= g for the next K-block g
        Window cur = fetch(kc), nxt = fetch(kc + 32);
        unsigned int g = kb0;
        while (g < kb1) {
            int cons = 0;
            if (lane == 0) cons = (int)ld_acquire(&S.consumed);
            cons = __shfl_sync(0xffffffffu, cons, 0);
            const int room = cons + kRecSlots - (int)published;  // record slots free
            if (room <= 0) {
                if (lane == 0) ok = wait_at_least(&S.consumed, (unsigned int)cons + 1, abort_flag);
                ok = __shfl_sync(0xffffffffu, (int)ok, 0);
                if (!ok) break;  // the waiting role reports the failure
                continue;
            }
            while (g >= cur.kbo_e && kc + 32 < P.key_hi) {  // the window ends before g: move it on
                kc += 32;
                cur = nxt;
                nxt = fetch(kc + 32);
            }
            const unsigned int n = min(min((unsigned int)room, kb1 - g), cur.kbo_e - g);
            // lane i: K-block g + i, key kc + ci with ci the last window entry with kb_offsets <= g + i
            const unsigned int gi = g + (unsigned int)lane;
            int ci = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                const unsigned int v = __shfl_sync(0xffffffffu, cur.kbo, (ci + step) & 31);
                if (ci + step < 32 && v <= gi) ci += step;
            }
            const unsigned int kbo_k = __shfl_sync(0xffffffffu, cur.kbo, ci);
            const unsigned int ka = __shfl_sync(0xffffffffu, cur.off, ci);
            const unsigned int kn = __shfl_sync(0xffffffffu, cur.off, (ci + 1) & 31);
            const unsigned int km = __shfl_sync(0xffffffffu, cur.km, ci);
            if ((unsigned int)lane < n) {
                const unsigned int kend = ci < 31 ? kn : cur.off_e;
                const unsigned int pos = ka + (unsigned int)kKB * (gi - kbo_k);
                const unsigned int cnt = min((unsigned int)kKB, kend - pos);
                const unsigned int idx = published + (unsigned int)lane;
                const float sc = keymax ? key_fixed_scale(__uint_as_float(km)) : 0.0f;
                S.meta[idx % kMetaRing] = KBMeta{kc + ci, pos, (int)cnt, sc, sc > 0.0f ? 1.0f / sc : 0.0f};
                const uint32_t bar = smem_u32(&S.rec_full[idx % kRecSlots]);
                mbar_arrive_expect_tx(bar, cnt * 16u);
                bulk_g2s(smem_u32(rec_smem + (idx % kRecSlots) * kKB * 16), P.rec + pos, cnt * 16u, bar);
            }
            if (open) {  // interval starts: a key change, or the first K-block of the chunk
                const int key_i = kc + ci;
                int key_p = __shfl_up_sync(0xffffffffu, key_i, 1);
                if (lane == 0) key_p = prev_key;
                if ((unsigned int)lane < n)
                    open[(published + (unsigned int)lane) % kMetaRing] = (key_i != key_p || gi == kb0) ? 1 : 0;
                prev_key = __shfl_sync(0xffffffffu, key_i, (int)n - 1);
            }
            published += n;
            g += n;
            __syncwarp();
            if (lane == 0) st_release(&S.published, published);
        }
        if (!ok) break;
    }
    if (ok && lane == 0) st_release(&S.sched_done, published + 1);
    // no record copy of this CTA may still be in flight when it exits: wait for the last copy of
    // every slot (the producers normally consumed them all already)
    if (lane == 0) {
        const volatile int never = 0;
        for (unsigned int s = 0; s < (unsigned int)kRecSlots && s < published; ++s) {
            const unsigned int uses = (published - s + kRecSlots - 1) / kRecSlots;
            if (!mbar_wait(smem_u32(&S.rec_full[s]), (uint32_t)((uses - 1) & 1u), &never)) atomicOr(P.status, 16u);
        }
    }
}

}  // namespace tc
}  // namespace svdi
