// probe_shared_red: throughput of shared-memory integer reductions as the FP32 gridder issues them
// (red.shared.add.u32 on two 32-bit planes, one cell per lane, conflict-free) against one
// red.shared.add.u64 of the same pair packed into 64 bits. Reports cell updates per SM clock and
// reduction warp instructions per SM clock at 1, 2 and 4 CTAs (8 warps each) per SM.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>

#define CK(x)                                                                                 \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess) {                                                              \
            std::printf("CUDA error %s at %s:%d: %s\n", #x, __FILE__, __LINE__, cudaGetErrorString(e_)); \
            std::exit(2);                                                                     \
        }                                                                                     \
    } while (0)

namespace {

template <int MODE>
__global__ void __launch_bounds__(256) k_red(int iters, unsigned long long* cyc, unsigned int* sink) {
    __shared__ __align__(16) unsigned long long acc[2048];  // 16 KB: two 8 KB planes, or 2048 pairs
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < 2048; i += 256) acc[i] = 0;
    __syncthreads();
    const unsigned int base = (unsigned int)__cvta_generic_to_shared(acc);
    unsigned int v = tid * 977u + 1u;
    const unsigned long long t0 = clock64();
    for (int it = 0; it < iters; ++it) {
        const unsigned int cell = (unsigned int)((warp * 64 + (it & 15) * 4 + lane) & 2047);
        v = v * 1664525u + 1013904223u;
        if (MODE == 0) {  // two 32-bit reductions: real plane, imaginary plane 8 KB further
            const unsigned int a = base + cell * 4u;
            asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
            asm volatile("red.shared.add.u32 [%0+8192], %1;" ::"r"(a), "r"(v ^ 0x5555u) : "memory");
        } else {  // one 64-bit reduction of the packed pair
            const unsigned int a = base + cell * 8u;
            const unsigned long long pv = ((unsigned long long)(v ^ 0x5555u) << 32) | v;
            asm volatile("red.shared.add.u64 [%0], %1;" ::"r"(a), "l"(pv) : "memory");
        }
    }
    __syncthreads();
    const unsigned long long t1 = clock64();
    if (tid == 0) atomicAdd(cyc, t1 - t0);
    if (tid < 4) sink[blockIdx.x * 4 + tid] = (unsigned int)acc[tid];
}

}  // namespace

int main() {
    CK(cudaSetDevice(0));
    cudaDeviceProp p;
    CK(cudaGetDeviceProperties(&p, 0));
    const int SM = p.multiProcessorCount;
    unsigned long long* d_cyc;
    unsigned int* d_sink;
    CK(cudaMalloc(&d_cyc, 8));
    CK(cudaMalloc(&d_sink, 4 * 4 * SM * sizeof(unsigned int)));
    const int iters = 4096;
    std::printf("device %s, %d SMs\n", p.name, SM);
    for (int per_sm = 1; per_sm <= 4; per_sm *= 2) {
        for (int mode = 0; mode < 2; ++mode) {
            CK(cudaMemset(d_cyc, 0, 8));
            if (mode == 0) k_red<0><<<SM * per_sm, 256>>>(iters, d_cyc, d_sink);
            else k_red<1><<<SM * per_sm, 256>>>(iters, d_cyc, d_sink);
            CK(cudaGetLastError());
            CK(cudaDeviceSynchronize());
            unsigned long long cy;
            CK(cudaMemcpy(&cy, d_cyc, 8, cudaMemcpyDeviceToHost));
            const double per_cta = (double)cy / (SM * per_sm);
            std::printf("CTAs/SM %d, %s: %.2f cell updates per clk per SM, %.2f reduction warp instructions per clk per SM\n",
                        per_sm, mode == 0 ? "2 x red.shared.add.u32" : "1 x red.shared.add.u64",
                        per_sm * 256.0 * iters / per_cta, per_sm * 8.0 * iters * (mode == 0 ? 2 : 1) / per_cta);
        }
    }
    std::printf("done\n");
    return 0;
}
