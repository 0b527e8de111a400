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
    const int per = a.K + wt_bit_words(a.K);
    uint32_t* nk = smu;
    uint32_t* hist = smu + a.K + (size_t)per * wid;
    uint32_t* bits = hist + a.K;
    for (int i = threadIdx.x; i < a.K + per * warps; i += blockDim.x) smu[i] = 0u;
    __syncthreads();
    for (;;) {
        int tile = 0;
        if (lane == 0) tile = (int)atomicAdd(a.tile_counter, 1u);
        tile = __shfl_sync(FULL, tile, 0);
        if (tile >= a.ntiles) break;
        const int4 t = a.tiles[tile];
        wt_tile(a, t, hist, bits, nk, lane);
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

// ------------------------------------------------------------------ large K
// Above kLargeK topics a per-warp word column (4K bytes) leaves few warps on an SM, so
// the sampler splits a chunk's tiles by kind.  Dense words: one CTA per tile, its warps
// share one column in shared memory and take the tile's 32-token groups in turn.  Sparse
// words: warp per tile with no column at all (ColBits).  Both run the same per-group code
// (sample_groups) on the same values as the per-warp column, so results are unchanged.
// The threshold is kLargeK (sweep_body.cuh).

// Sparse-word view without a column: the word's topics as a bitmap in shared memory, with
// the number of set bits before each 32-topic word; a topic's count is read from the
// word's row (ascending k), and phi_k is formed exactly as build_column forms it.
struct ColBits {
    const uint32_t* bits;  // ceil(K/32) words
    const uint16_t* pre;   // set bits before each word
    const uint32_t* ent;   // the word's row, (k << 16) | count
    const float* r;
    float beta;
    int maxK;
    __device__ __forceinline__ float operator()(int k) const {
        if (k == maxK) return 0.0f;
        const uint32_t b = bits[k >> 5], m = 1u << (k & 31);
        if (b & m) {
            const uint32_t e = __ldg(ent + pre[k >> 5] + __popc(b & (m - 1u)));
            return fmul(fadd(u2f(e & 0xffffu), beta), r[k]);
        }
        return fmul(beta, r[k]);
    }
};

__host__ __device__ __forceinline__ int large_bit_words(int K) { return (K + 31) >> 5; }
__host__ __device__ __forceinline__ int large_pre_words(int K) { return ((K + 31) >> 5) + 1 & ~1; }

// Shared memory of the sparse-word kernel: r[K], then per warp the bitmap, then per warp
// the prefix counts (uint16, an even number per warp), then per warp the counter row.
__host__ __device__ __forceinline__ size_t sparse_large_smem(int K, int warps) {
    return (size_t)K * 4 + (size_t)warps * (large_bit_words(K) * 4 + large_pre_words(K) * 2 + C_NUM * 4);
}

// Shared memory of the dense-word kernel: the shared column, the warps' counter rows and
// their LL partials (the reciprocals are formed while the column is built).
__host__ __device__ __forceinline__ size_t dense_large_smem(int K, int warps) {
    return (((size_t)col_words(K) * 4 + (size_t)warps * C_NUM * 4 + 7) & ~(size_t)7) + (size_t)warps * 8;
}

#ifndef LDA_DENSE_LARGE_MIN_BLOCKS
#define LDA_DENSE_LARGE_MIN_BLOCKS 4
#endif

template <bool LL, int QB>
__global__ void __launch_bounds__(256, LDA_SAMPLE_MIN_BLOCKS) k_sample_sparse_large(SampleArgs a) {
    extern __shared__ float smf[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bw = large_bit_words(a.K), pw = large_pre_words(a.K);
    float* r = smf;
    uint32_t* bits = reinterpret_cast<uint32_t*>(smf + a.K) + (size_t)bw * wid;
    uint16_t* pre = reinterpret_cast<uint16_t*>(reinterpret_cast<uint32_t*>(smf + a.K) + (size_t)bw * warps) +
                    (size_t)pw * wid;
    uint32_t* ctr = reinterpret_cast<uint32_t*>(reinterpret_cast<uint16_t*>(reinterpret_cast<uint32_t*>(smf + a.K) +
                                                                            (size_t)bw * warps) +
                                                (size_t)pw * warps) +
                    C_NUM * wid;
    fill_recip(r, a.n_k, a.K, a.Vbeta);
    for (int i = lane; i < bw; i += 32) bits[i] = 0u;
    if (lane < C_NUM) ctr[lane] = 0u;
    __syncthreads();
    for (;;) {
        int tile = 0;
        if (lane == 0) tile = (int)atomicAdd(a.tile_counter, 1u);
        tile = __shfl_sync(FULL, tile, 0);
        if (tile >= a.ntiles) break;
        const int4 t = a.tiles[tile];
        const int w = t.x;
        const int s = w - a.Vd;
        const uint32_t* ent = a.swt_ent + __ldg(a.swt_off + s);
        const uint32_t nnz_w = __ldg(a.swt_nnz + s);
        for (uint32_t e = lane; e < nnz_w; e += 32) {
            const uint32_t k = __ldg(ent + e) >> 16;
            atomicOr(&bits[k >> 5], 1u << (k & 31u));
        }
        __syncwarp();
        uint32_t carry = 0;
        for (int wb = 0; wb < bw; wb += 32) {
            const int i = wb + lane;
            const uint32_t c = i < bw ? (uint32_t)__popc(bits[i]) : 0u;
            uint32_t incl = c;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t v = __shfl_up_sync(FULL, incl, off);
                if (lane >= off) incl += v;
            }
            if (i < bw) pre[i] = (uint16_t)(carry + incl - c);
            carry += __shfl_sync(FULL, incl, 31);
        }
        if (lane == 0) {
            ctr[C_WNNZ] += nnz_w;
            ctr[C_TSPARSE] += 1u;
        }
        const int maxK = (int)(__ldg(a.st_top2 + w) & 0xffffu);
        const float4 ph = __ldg(a.st_phi + w);
        const float QL = __ldg(a.st_ql + (size_t)w * 32 + lane);
        const float QP = warp_ks_scan(QL, lane);
        const float Q = __shfl_sync(FULL, QP, 31);
        __syncwarp();
        const ColBits view{bits, pre, ent, r, a.beta, maxK};
        double ll = sample_groups<LL, QB>(a, (uint32_t)t.y, (uint32_t)t.z, 0u, 32u, a.iter, maxK, ph, QL, QP, Q, view,
                                          ctr, lane);
        if (LL) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) ll += __shfl_xor_sync(FULL, ll, off);
            if (lane == 0) a.tile_ll[tile] = ll;
        }
        __syncwarp();
        for (uint32_t e = lane; e < nnz_w; e += 32) bits[(__ldg(ent + e) >> 16) >> 5] = 0u;
        __syncwarp();
    }
    __syncwarp();
    if (lane < C_NUM && ctr[lane]) atomicAdd(a.ctr + lane, (unsigned long long)ctr[lane]);
}

template <bool LL, int QB>
__global__ void __launch_bounds__(256, LDA_DENSE_LARGE_MIN_BLOCKS) k_sample_dense_large(SampleArgs a) {
    extern __shared__ float smf[];
    __shared__ int s_tile;
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* col = smf;
    uint32_t* ctr_all = reinterpret_cast<uint32_t*>(col + col_words(a.K));
    uint32_t* ctr = ctr_all + C_NUM * wid;
    double* wll = reinterpret_cast<double*>(
        (reinterpret_cast<uintptr_t>(ctr_all + C_NUM * warps) + 7) & ~(uintptr_t)7);
    if (lane < C_NUM) ctr[lane] = 0u;
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) s_tile = (int)atomicAdd(a.tile_counter, 1u);
        __syncthreads();
        const int tile = s_tile;
        if (tile >= a.ntiles) break;
        const int4 t = a.tiles[tile];
        const int w = t.x;
        const int* wrow = a.dwt + (size_t)w * a.K;
        // phi_k = ((float)n_wk + beta) * r_k with r_k = 1 / ((float)n_k + V*beta), the values
        // fill_recip and build_column form
        for (int k = threadIdx.x; k < a.K; k += blockDim.x) {
            const float rk = __fdiv_rn(1.0f, fadd(__int2float_rn(__ldg(a.n_k + k)), a.Vbeta));
            col[col_skew(k)] = fmul(fadd(__int2float_rn(__ldg(wrow + k)), a.beta), rk);
        }
        const int maxK = (int)(__ldg(a.st_top2 + w) & 0xffffu);
        __syncthreads();
        if (threadIdx.x == 0) {
            col[col_skew(maxK)] = 0.0f;
            ctr[C_TDENSE] += 1u;
        }
        __syncthreads();
        const float4 ph = __ldg(a.st_phi + w);
        const float QL = __ldg(a.st_ql + (size_t)w * 32 + lane);
        const float QP = warp_ks_scan(QL, lane);
        const float Q = __shfl_sync(FULL, QP, 31);
        double ll = sample_groups<LL, QB>(a, (uint32_t)t.y, (uint32_t)t.z, 32u * wid, 32u * warps, a.iter, maxK, ph, QL,
                                          QP, Q, ColShared{col}, ctr, lane);
        if (LL) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) ll += __shfl_xor_sync(FULL, ll, off);
            if (lane == 0) wll[wid] = ll;
        }
        __syncthreads();
        if (LL && threadIdx.x == 0) {
            double sum = 0.0;
            for (int i = 0; i < warps; ++i) sum += wll[i];
            a.tile_ll[tile] = sum;
        }
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
