// cufsp_reduce.cuh -- deterministic block/grid reductions for the streaming vector kernels.
//
// Every CTA reduces its per-thread partial sums (warp shuffles, then a fixed-order pass over
// the warps), writes one partial per output to global memory, and the last CTA to finish
// (completion counter) sums the per-CTA partials in a fixed order.  Results therefore do not
// depend on CTA scheduling, unlike floating-point atomics.
#pragma once
#include <cuda_runtime.h>

namespace cufsp {

constexpr int kRedThreads = 256;
constexpr int kRedWarps = kRedThreads / 32;

// Shared-memory layout needed by grid_reduce<KP>: (kRedWarps * KP + KP) doubles.
template <int KP>
struct RedSmem {
    double warp_part[kRedWarps][KP];
    double final_[KP];
    int is_last;
};

// Second half of a grid reduction: this CTA's totals for outputs 0..K-1 are already in
// partials[blockIdx.x * KP + k].  Returns `true` in every thread of the last CTA to arrive, with the
// grid totals in sm.final_[0..K-1] (visible after the call); sm.warp_part is reused as scratch.
template <int KP>
__device__ __forceinline__ bool grid_finish(int K, double *__restrict__ partials, unsigned int *__restrict__ counter,
                                            RedSmem<KP> &sm) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int prev = atomicAdd(counter, 1u);
        sm.is_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!sm.is_last) return false;
    __threadfence();
    // Last CTA: thread t handles output k = t % KP for the CTA group g = t / KP (fixed order);
    // the warp_part array (kRedWarps * KP doubles) holds the G <= kRedWarps group sums.
    constexpr int G = (kRedThreads / KP) < kRedWarps ? (kRedThreads / KP) : kRedWarps;
    static_assert(G >= 1, "KP must not exceed the CTA size");
    double *grp = &sm.warp_part[0][0];
    const int k = threadIdx.x % KP, g = threadIdx.x / KP;
    __syncthreads();
    if (g < G) {
        double v = 0.0;
        if (k < K) {
            const volatile double *vp = partials;
            for (int c = g; c < (int)gridDim.x; c += G) v += vp[(size_t)c * KP + k];
        }
        grp[g * KP + k] = v;
    }
    __syncthreads();
    for (int kk = threadIdx.x; kk < K; kk += blockDim.x) {
        double v = 0.0;
        for (int gg = 0; gg < G; ++gg) v += grp[gg * KP + kk];
        sm.final_[kk] = v;
    }
    if (threadIdx.x == 0) *counter = 0u;  // ready for the next launch on this stream
    __syncthreads();
    return true;
}

// acc[0..K-1] hold this thread's partial sums (K <= KP).  On return, `true` in every thread of
// the last CTA, with the grid totals in sm.final_[0..K-1] (visible after the call).
template <int KP>
__device__ __forceinline__ bool grid_reduce(double (&acc)[KP], int K, double *__restrict__ partials,
                                            unsigned int *__restrict__ counter, RedSmem<KP> &sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < KP; ++k) {
        if (k < K) {
            double v = acc[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) sm.warp_part[warp][k] = v;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        double v = 0.0;
        for (int w = 0; w < kRedWarps; ++w) v += sm.warp_part[w][k];
        partials[(size_t)blockIdx.x * KP + k] = v;
    }
    return grid_finish<KP>(K, partials, counter, sm);
}

}  // namespace cufsp
