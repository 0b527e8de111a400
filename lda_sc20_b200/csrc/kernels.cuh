// kernels.cuh -- sm_100a kernels of the collapsed-Gibbs sweep.
//
// Every float operation below is an explicit round-to-nearest intrinsic, so the compiler
// cannot contract or reorder it.  The sampling arithmetic (summation orders, bin order,
// tie rules) is the specification the CPU oracle restates; the CUDA path and the oracle
// therefore draw identical topics for identical (seed, iteration, token).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sweep_body.cuh"

namespace lda {
namespace dev {

// Word-topic rebuild: warp per word tile, topic totals privatised per CTA.
__global__ void __launch_bounds__(256) k_wt_build(WtArgs a) {
    extern __shared__ uint32_t smu[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* nk = smu;
    uint32_t* hist = smu + (size_t)a.K * (1 + wid);
    for (int i = threadIdx.x; i < a.K * (warps + 1); i += blockDim.x) smu[i] = 0u;
    __syncthreads();
    for (;;) {
        int tile = 0;
        if (lane == 0) tile = (int)atomicAdd(a.tile_counter, 1u);
        tile = __shfl_sync(FULL, tile, 0);
        if (tile >= a.ntiles) break;
        const int4 t = a.tiles[tile];
        wt_tile(a, t, hist, nk, lane);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < a.K; k += blockDim.x) {
        const uint32_t v = nk[k];
        if (v) atomicAdd(a.n_k + k, (int)v);
    }
}

// Word statistics: warp per word.
__global__ void __launch_bounds__(256) k_word_stats(StatsArgs a) {
    extern __shared__ float smf[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* r = smf;
    float* col = smf + (size_t)a.K * (1 + wid);
    fill_recip(r, a.n_k, a.K, a.Vbeta);
    __syncthreads();
    for (int w = blockIdx.x * warps + wid; w < a.V; w += gridDim.x * warps) {
        word_stats_word(a, w, r, col, lane);
    }
}

// Doc-topic rebuild: warp per doc of one chunk.
__global__ void __launch_bounds__(256) k_dt_build(DtArgs a) {
    extern __shared__ uint32_t smu[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = a.K + dt_bit_words(a.K);
    uint32_t* hist = smu + (size_t)per * wid;
    uint32_t* bits = hist + a.K;
    for (int i = threadIdx.x; i < per * warps; i += blockDim.x) smu[i] = 0u;
    __syncthreads();
    for (uint32_t d = a.d_begin + blockIdx.x * warps + wid; d < a.d_end; d += gridDim.x * warps) {
        dt_doc(a, d, hist, bits, lane);
    }
}

// Sampler: warp per tile, tiles taken from an atomic counter.
template <bool LL, int QB = 1>
__global__ void __launch_bounds__(256, LDA_SAMPLE_MIN_BLOCKS) k_sample_t(SampleArgs a) {
    extern __shared__ float smf[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* r = smf;
    float* col = smf + a.K + (size_t)col_words(a.K) * wid;
    uint32_t* ctr = reinterpret_cast<uint32_t*>(smf + a.K + (size_t)col_words(a.K) * warps) + C_NUM * wid;
    fill_recip(r, a.n_k, a.K, a.Vbeta);
    if (lane < C_NUM) ctr[lane] = 0u;
    __syncthreads();
    for (;;) {
        int tile = 0;
        if (lane == 0) tile = (int)atomicAdd(a.tile_counter, 1u);
        tile = __shfl_sync(FULL, tile, 0);
        if (tile >= a.ntiles) break;
        const int4 t = a.tiles[tile];
        sample_tile<LL, QB>(a, tile, t, a.iter, r, col, ctr, lane);
    }
    __syncwarp();
    if (lane < C_NUM && ctr[lane]) atomicAdd(a.ctr + lane, (unsigned long long)ctr[lane]);
}

// Fixed-order FP64 reduction of the per-tile LL partials (one CTA of 1024 threads).
// Replaces LDATrainPerplexityReduce (EZLDA/utility.cu:2106-2151).
__global__ void __launch_bounds__(1024) k_ll_reduce(const double* __restrict__ in, int n, double* out) {
    __shared__ double s[1024];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += in[i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int h = blockDim.x >> 1; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

}  // namespace dev
}  // namespace lda
