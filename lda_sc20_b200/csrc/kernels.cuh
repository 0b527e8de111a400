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

// Word-topic rebuild: warp per word tile, topic totals privatised per CTA.  P16: 16-bit
// histogram counts (a dense tile holds at most 16,384 tokens and a sparse word fewer than
// 65,536, so every count fits).
template <bool P16>
__global__ void __launch_bounds__(256) k_wt_build(WtArgs a) {
    extern __shared__ uint32_t smu[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int hw = Hist<P16>::words(a.K);
    const int per = hw + wt_bit_words(a.K);
    uint32_t* nk = smu;
    const Hist<P16> hist{smu + a.K + (size_t)per * wid};
    uint32_t* bits = hist.h + hw;
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

// ---------------------------------------------------------------- large-K rebuilds
// Above kLargeK topics a warp-private K-sized histogram leaves one 8-warp CTA per SM, and
// the rebuilds wait on their gathers with little else to run (halving the histogram's
// size to 16-bit counts halved both rebuilds' time).  These kernels share one histogram
// across the CTA's 256 threads and take one unit at a time (a word tile, a doc), so that
// eight CTAs per SM keep 64 warps of gathers in flight.  Their rows, counts, metadata and
// errors are those of k_wt_build / k_dt_build, bit for bit; the topic totals come from
// k_topic_totals.
constexpr int kRebuildThreads = 256;
constexpr int kSmoothMaxRounds = 2048;  // rounds of 32 topics in the smoothing table (K <= 65,536)

// Exclusive scan of one value per thread across the CTA; *total gets the sum.  wsum holds
// a word per warp.  Every thread of the CTA calls it.
__device__ __forceinline__ uint32_t cta_exclusive_scan(uint32_t v, uint32_t* wsum, uint32_t* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t t = __shfl_up_sync(FULL, incl, off);
        if (lane >= off) incl += t;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    uint32_t before = 0, tot = 0;
    for (int i = 0; i < nw; ++i) {
        const uint32_t x = wsum[i];
        before += i < wid ? x : 0u;
        tot += x;
    }
    *total = tot;
    __syncthreads();
    return before + incl - v;
}

// Adds topics topic_of(i), i in [0, n), to the CTA's histogram (16-bit counts) and sets
// the bit of each topic whose count leaves zero; a topic >= K sets *err and is skipped.
// Four 256-token steps of loads are in flight per thread.  n is uniform across the CTA.
template <class F>
__device__ __forceinline__ void cta_hist(uint32_t n, const F& topic_of, const Hist<true>& hist, uint32_t* bits, int K,
                                         int* err) {
    for (uint32_t base = 0; base < n; base += 4u * kRebuildThreads) {
        uint32_t k[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const uint32_t i = base + (uint32_t)(s * kRebuildThreads) + threadIdx.x;
            k[s] = i < n ? topic_of(i) : 0xffffffffu;
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (base + (uint32_t)(s * kRebuildThreads) >= n) break;
            bool valid = k[s] != 0xffffffffu;
            uint32_t kk = k[s];
            if (valid && kk >= (uint32_t)K) {
                atomicOr(err, 1);
                valid = false;
                kk = 0xfffffffeu;
            }
            if (valid) hist_token(hist, bits, kk);
        }
    }
}

// Walks the CTA's bitmap (bw words) in ascending topic order: thread t takes words
// [t R, t R + R), R = ceil(bw / threads), an exclusive scan of their popcounts places
// its entries, and emit(k, count, position) is called for each non-zero topic; bits and
// counts are cleared.  Returns the number of non-zero topics.
template <class E>
__device__ __forceinline__ uint32_t cta_compact(int bw, const Hist<true>& hist, uint32_t* bits, uint32_t* wsum,
                                                const E& emit) {
    const int R = (bw + blockDim.x - 1) / blockDim.x;
    const int w0 = min(bw, (int)threadIdx.x * R), w1 = min(bw, w0 + R);
    uint32_t c = 0;
    for (int wi = w0; wi < w1; ++wi) c += (uint32_t)__popc(bits[wi]);
    uint32_t total;
    uint32_t p = cta_exclusive_scan(c, wsum, &total);
    for (int wi = w0; wi < w1; ++wi) {
        uint32_t m = bits[wi];
        if (m) bits[wi] = 0u;
        while (m) {
            const uint32_t k = (uint32_t)wi * 32u + (uint32_t)(__ffs(m) - 1);
            m &= m - 1u;
            emit(k, hist.get(k), p++);
            hist.clear(k);
        }
    }
    return total;
}

// Word-topic rows above kLargeK topics: CTA per word tile (a dense word's chunk segment
// of up to 16,384 tokens, or a sparse word over all chunks).  Shared memory: the
// histogram, the bitmap, then a sparse word's chunk segments ([C] offsets, [C + 1] prefix
// counts).  Topic totals are not accumulated here (k_topic_totals).
__global__ void __launch_bounds__(kRebuildThreads, 8) k_wt_build_cta(WtArgs a) {
    extern __shared__ uint32_t smu[];
    __shared__ uint32_t wsum[kRebuildThreads / 32];
    __shared__ int s_tile;
    const int hw = Hist<true>::words(a.K), bw = wt_bit_words(a.K);
    const Hist<true> hist{smu};
    uint32_t* bits = smu + hw;
    uint32_t* so = bits + bw;
    uint32_t* pre = so + a.C;
    const int lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < hw + bw; i += blockDim.x) smu[i] = 0u;
    for (;;) {
        __syncthreads();  // the previous tile is done with the shared state
        if (threadIdx.x == 0) s_tile = (int)atomicAdd(a.tile_counter, 1u);
        __syncthreads();
        const int tile = s_tile;
        if (tile >= a.ntiles) break;
        const int4 t = a.tiles[tile];
        const int w = t.x;
        if (t.w & 1) {
            const uint16_t* z = a.z + (uint32_t)t.y;
            cta_hist((uint32_t)t.z, [&](uint32_t i) { return (uint32_t)__ldg(z + i); }, hist, bits, a.K, a.err);
        } else {
            // the word's segment in every chunk, and their prefix counts
            if (threadIdx.x < 32) {
                uint32_t carry = 0;
                if (lane == 0) pre[0] = 0u;
                for (int c0 = 0; c0 < a.C; c0 += 32) {
                    const int c = c0 + lane;
                    uint32_t cnt = 0;
                    if (c < a.C) {
                        const size_t idx = (size_t)c * a.V + w;
                        so[c] = __ldg(a.seg_off + idx);
                        cnt = __ldg(a.seg_cnt + idx);
                    }
                    uint32_t incl = cnt;
#pragma unroll
                    for (int off = 1; off < 32; off <<= 1) {
                        const uint32_t v = __shfl_up_sync(FULL, incl, off);
                        if (lane >= off) incl += v;
                    }
                    if (c < a.C) pre[c + 1] = carry + incl;
                    carry += __shfl_sync(FULL, incl, 31);
                }
            }
            __syncthreads();
            const int C = a.C;
            cta_hist(pre[C], [&](uint32_t i) {
                // the chunk holding the word's i-th token: the last c with pre[c] <= i
                int lo = 0, hi = C - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (pre[mid] <= i) lo = mid; else hi = mid - 1;
                }
                return (uint32_t)__ldg(a.z + so[lo] + (i - pre[lo]));
            }, hist, bits, a.K, a.err);
        }
        __syncthreads();
        if (t.w & 1) {
            int* row = a.dwt + (size_t)w * a.K;
            cta_compact(bw, hist, bits, wsum, [&](uint32_t k, uint32_t h, uint32_t) { atomicAdd(row + k, (int)h); });
        } else {
            const int s = w - a.Vd;
            uint32_t* out = a.swt_ent + a.swt_off[s];
            const uint32_t nnz = cta_compact(bw, hist, bits, wsum,
                                             [&](uint32_t k, uint32_t h, uint32_t p) { out[p] = (k << 16) | h; });
            if (threadIdx.x == 0) a.swt_nnz[s] = nnz;
        }
    }
}

// Rows of small sparse words above kLargeK topics (at most kSmallSparse tokens, over at
// most 32 chunks): warp per word, without a histogram.  The warp holds the word's topics
// in registers (up to 8 per lane), marks them in a bitmap, gives each topic its rank among
// the word's distinct topics (the popcount prefix of the bitmap), counts per rank, and
// writes the row ascending k.  Per warp: bitmap (bw words), prefix (bw uint16) and counts
// (kSmallSparse words).  Rows equal k_wt_build_cta's.
constexpr int kSmallSparse = 256;
__host__ __device__ __forceinline__ size_t wt_small_warp_words(int K) {
    const size_t bw = (size_t)(K + 31) >> 5;
    return bw + ((bw + 1) >> 1) + kSmallSparse;
}
__global__ void __launch_bounds__(256) k_wt_sparse_small(WtArgs a) {
    extern __shared__ uint32_t smu[];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bw = wt_bit_words(a.K);
    uint32_t* bits = smu + wt_small_warp_words(a.K) * wid;
    uint16_t* pre = reinterpret_cast<uint16_t*>(bits + bw);
    uint32_t* cnt = bits + bw + ((bw + 1) >> 1);
    for (int i = lane; i < bw; i += 32) bits[i] = 0u;
    for (int i = lane; i < kSmallSparse; i += 32) cnt[i] = 0u;
    __syncwarp();
    for (;;) {
        int tile = 0;
        if (lane == 0) tile = (int)atomicAdd(a.tile_counter, 1u);
        tile = __shfl_sync(FULL, tile, 0);
        if (tile >= a.ntiles) break;
        const int w = a.tiles[tile].x;
        // lane c: chunk c's segment of the word, as z index minus the segment's first rank
        uint32_t so = 0, sc = 0;
        if (lane < a.C) {
            const size_t idx = (size_t)lane * a.V + w;
            so = __ldg(a.seg_off + idx);
            sc = __ldg(a.seg_cnt + idx);
        }
        uint32_t incl = sc;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t v = __shfl_up_sync(FULL, incl, off);
            if (lane >= off) incl += v;
        }
        const uint32_t base_l = so - (incl - sc);
        const uint32_t n = min(__shfl_sync(FULL, incl, 31), (uint32_t)kSmallSparse);
        uint32_t k[kSmallSparse / 32];
#pragma unroll
        for (int j = 0; j < kSmallSparse / 32; ++j) {
            const uint32_t i = 32u * (uint32_t)j + (uint32_t)lane;
            k[j] = 0xffffffffu;
            if (32u * (uint32_t)j >= n) continue;  // uniform
            // the first lane whose inclusive prefix exceeds i
            const uint32_t ii = i < n ? i : n - 1;
            int c = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const uint32_t v = __shfl_sync(FULL, incl, c + step - 1);
                if (v <= ii) c += step;
            }
            const uint32_t b = __shfl_sync(FULL, base_l, c);
            if (i < n) {
                uint32_t kk = (uint32_t)__ldg(a.z + b + i);
                if (kk >= (uint32_t)a.K) {
                    atomicOr(a.err, 1);
                    kk = 0xffffffffu;
                }
                k[j] = kk;
            }
        }
#pragma unroll
        for (int j = 0; j < kSmallSparse / 32; ++j)
            if (k[j] != 0xffffffffu) atomicOr(&bits[k[j] >> 5], 1u << (k[j] & 31u));
        __syncwarp();
        uint32_t carry = 0;
        for (int wb = 0; wb < bw; wb += 32) {
            const int wi = wb + lane;
            const uint32_t c = wi < bw ? (uint32_t)__popc(bits[wi]) : 0u;
            uint32_t inc = c;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t v = __shfl_up_sync(FULL, inc, off);
                if (lane >= off) inc += v;
            }
            if (wi < bw) pre[wi] = (uint16_t)(carry + inc - c);
            carry += __shfl_sync(FULL, inc, 31);
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < kSmallSparse / 32; ++j) {
            const uint32_t kk = k[j];
            if (kk != 0xffffffffu) {
                const uint32_t m = bits[kk >> 5];
                atomicAdd(&cnt[pre[kk >> 5] + __popc(m & ((1u << (kk & 31u)) - 1u))], 1u);
            }
        }
        __syncwarp();
        const int s = w - a.Vd;
        uint32_t* out = a.swt_ent + a.swt_off[s];
        for (int wb = 0; wb < bw; wb += 32) {
            const int wi = wb + lane;
            uint32_t m = wi < bw ? bits[wi] : 0u;
            if (m) {
                bits[wi] = 0u;
                uint32_t p = pre[wi];
                while (m) {
                    const uint32_t kk = (uint32_t)wi * 32u + (uint32_t)(__ffs(m) - 1);
                    m &= m - 1u;
                    out[p] = (kk << 16) | cnt[p];
                    cnt[p] = 0u;
                    ++p;
                }
            }
        }
        if (lane == 0) a.swt_nnz[s] = carry;
        __syncwarp();
    }
}

// Topic totals n_k of the word tiles a.tiles (all words, or a word range): warp per tile,
// counts privatised per CTA in shared memory (K words) and flushed once; without SHARED
// (K words beyond the shared memory) the warps add to n_k directly.
template <bool SHARED>
__global__ void __launch_bounds__(256) k_topic_totals(WtArgs a) {
    extern __shared__ uint32_t smu[];
    const int lane = threadIdx.x & 31;
    if (SHARED) {
        for (int i = threadIdx.x; i < a.K; i += blockDim.x) smu[i] = 0u;
        __syncthreads();
    }
    auto add = [&](const uint16_t* z, uint32_t n) {
        for (uint32_t base = 0; base < n; base += 128) {
            uint32_t k[4];
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const uint32_t i = base + 32u * s + lane;
                k[s] = i < n ? (uint32_t)__ldg(z + i) : 0xffffffffu;
            }
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                if (base + 32u * s >= n) break;
                // a topic >= K is reported by the rebuild; it is not counted here
                const bool valid = k[s] < (uint32_t)a.K;
                const uint32_t kk = valid ? k[s] : 0xfffffffeu;
                if (valid && SHARED) atomicAdd(smu + kk, 1u);
                if (valid && !SHARED) atomicAdd(a.n_k + kk, 1);
            }
        }
    };
    for (;;) {
        int tile = 0;
        if (lane == 0) tile = (int)atomicAdd(a.tile_counter, 1u);
        tile = __shfl_sync(FULL, tile, 0);
        if (tile >= a.ntiles) break;
        const int4 t = a.tiles[tile];
        if (t.w & 1) {
            add(a.z + (uint32_t)t.y, (uint32_t)t.z);
        } else {
            for (int c0 = 0; c0 < a.C; c0 += 32) {
                const int c = c0 + lane;
                uint32_t so = 0, sc = 0;
                if (c < a.C) {
                    const size_t idx = (size_t)c * a.V + t.x;
                    so = __ldg(a.seg_off + idx);
                    sc = __ldg(a.seg_cnt + idx);
                }
                const int nc = min(32, a.C - c0);
                for (int j = 0; j < nc; ++j) {
                    const uint32_t o = __shfl_sync(FULL, so, j), n = __shfl_sync(FULL, sc, j);
                    if (n) add(a.z + o, n);
                }
            }
        }
    }
    if (SHARED) {
        __syncthreads();
        for (int k = threadIdx.x; k < a.K; k += blockDim.x) {
            const uint32_t v = smu[k];
            if (v) atomicAdd(a.n_k + k, (int)v);
        }
    }
}

// Doc rows above kLargeK topics: CTA per doc (the doc's tokens spread over the CTA's
// threads), the histogram and bitmap shared.  Rows are ascending k with topic keys.  (Up
// to 2048 topics the warp-per-doc kernel is faster: 1.35 against 1.59 ms per sweep on the
// K=1024 corpus, where a warp's histogram is small enough for 64 warps per SM.)
__global__ void __launch_bounds__(kRebuildThreads, 8) k_dt_build_cta(DtArgs a) {
    extern __shared__ uint32_t smu[];
    __shared__ uint32_t wsum[kRebuildThreads / 32];
    const int hw = Hist<true>::words(a.K), bw = dt_bit_words(a.K);
    const Hist<true> hist{smu};
    uint32_t* bits = smu + hw;
    for (int i = threadIdx.x; i < hw + bw; i += blockDim.x) smu[i] = 0u;
    for (uint32_t d = a.d_begin + blockIdx.x; d < a.d_end; d += gridDim.x) {
        __syncthreads();  // the previous doc is done with the shared state
        const uint32_t b = __ldg(a.doc_off + d), n = __ldg(a.doc_off + d + 1) - b;
        if (n <= a.small_max) continue;  // k_dt_build_small's doc
        const uint32_t* dpos = a.dtok_pos + (b - a.tok_base);
        const uint32_t* dword = a.dtok_word + (b - a.tok_base);
        const uint16_t* z = a.z;
        cta_hist(n, [&](uint32_t i) { return (uint32_t)__ldg(z + __ldg(dpos + i)); }, hist, bits, a.K, a.err);
        __syncthreads();
        for (uint32_t base = 0; base < n; base += 4u * kRebuildThreads) {
            uint32_t pos[4], t2[4];
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const uint32_t i = base + (uint32_t)(s * kRebuildThreads) + threadIdx.x;
                pos[s] = i < n ? __ldg(dpos + i) : 0xffffffffu;
                t2[s] = i < n ? __ldg(dword + i) : 0u;
            }
#pragma unroll
            for (int s = 0; s < 4; ++s) t2[s] = pos[s] != 0xffffffffu ? __ldg(a.st_top2 + t2[s]) : 0u;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                if (pos[s] == 0xffffffffu) continue;
                const uint32_t k1 = t2[s] & 0xffffu, k2 = t2[s] >> 16;
                const uint32_t c1 = k1 < (uint32_t)a.K ? hist.get(k1) : 0u, c2 = k2 < (uint32_t)a.K ? hist.get(k2) : 0u;
                a.meta[pos[s] - a.tok_base] = (c2 << 16) | c1;
            }
        }
        __syncthreads();
        uint32_t* out = a.dt_ent + (__ldg(a.dt_off + d) - a.dt_base);
        const uint32_t nnz =
            cta_compact(bw, hist, bits, wsum, [&](uint32_t k, uint32_t h, uint32_t p) { out[p] = (k << 16) | h; });
        if (threadIdx.x == 0) a.dt_nnz[d] = nnz;
    }
}

// Doc rows above kLargeK topics for docs of at most a.small_max (<= kSmallDoc) tokens:
// warp per doc, without a histogram (as k_wt_sparse_small builds small words' rows).  The
// warp holds the doc's topics in registers, marks them in a bitmap, ranks each topic among
// the doc's distinct topics by the bitmap's popcount prefix and counts per rank; a topic's
// count is then one bitmap test and one lookup, for the tokens' metadata and the row.
// Rows, metadata and errors equal k_dt_build_cta's.
constexpr int kSmallDoc = 384;
__host__ __device__ __forceinline__ size_t dt_small_warp_words(int K) {
    const size_t bw = (size_t)(K + 31) >> 5;
    return bw + ((bw + 1) >> 1) + kSmallDoc;
}
#ifndef LDA_DT_SMALL_MIN_BLOCKS
#define LDA_DT_SMALL_MIN_BLOCKS 6
#endif
__global__ void __launch_bounds__(256, LDA_DT_SMALL_MIN_BLOCKS) k_dt_build_small(DtArgs a) {
    extern __shared__ uint32_t smu[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bw = dt_bit_words(a.K);
    uint32_t* bits = smu + dt_small_warp_words(a.K) * wid;
    uint16_t* pre = reinterpret_cast<uint16_t*>(bits + bw);
    uint32_t* cnt = bits + bw + ((bw + 1) >> 1);
    for (int i = lane; i < bw; i += 32) bits[i] = 0u;
    for (int i = lane; i < kSmallDoc; i += 32) cnt[i] = 0u;
    __syncwarp();
    // the doc's count of topic k (bits, pre and cnt complete)
    auto count_of = [&](uint32_t k) -> uint32_t {
        if (k >= (uint32_t)a.K) return 0u;
        const uint32_t m = bits[k >> 5], sh = k & 31u;
        return (m >> sh) & 1u ? cnt[pre[k >> 5] + __popc(m & ((1u << sh) - 1u))] : 0u;
    };
    for (uint32_t d = a.d_begin + blockIdx.x * warps + wid; d < a.d_end; d += gridDim.x * warps) {
        const uint32_t b = __ldg(a.doc_off + d), n = __ldg(a.doc_off + d + 1) - b;
        if (n > a.small_max) continue;  // k_dt_build_cta's doc
        const uint32_t* dpos = a.dtok_pos + (b - a.tok_base);
        const uint32_t* dword = a.dtok_word + (b - a.tok_base);
        uint32_t k[kSmallDoc / 32];
#pragma unroll
        for (int j = 0; j < kSmallDoc / 32; ++j) {
            const uint32_t i = 32u * (uint32_t)j + (uint32_t)lane;
            k[j] = i < n ? __ldg(dpos + i) : 0xffffffffu;
        }
#pragma unroll
        for (int j = 0; j < kSmallDoc / 32; ++j) {
            if (k[j] == 0xffffffffu) continue;
            uint32_t kk = (uint32_t)__ldg(a.z + k[j]);
            if (kk >= (uint32_t)a.K) {
                atomicOr(a.err, 1);
                kk = 0xffffffffu;
            }
            k[j] = kk;
        }
#pragma unroll
        for (int j = 0; j < kSmallDoc / 32; ++j)
            if (k[j] != 0xffffffffu) atomicOr(&bits[k[j] >> 5], 1u << (k[j] & 31u));
        __syncwarp();
        uint32_t carry = 0;
        for (int wb = 0; wb < bw; wb += 32) {
            const int wi = wb + lane;
            const uint32_t c = wi < bw ? (uint32_t)__popc(bits[wi]) : 0u;
            uint32_t inc = c;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t v = __shfl_up_sync(FULL, inc, off);
                if (lane >= off) inc += v;
            }
            if (wi < bw) pre[wi] = (uint16_t)(carry + inc - c);
            carry += __shfl_sync(FULL, inc, 31);
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < kSmallDoc / 32; ++j) {
            const uint32_t kk = k[j];
            if (kk != 0xffffffffu) {
                const uint32_t m = bits[kk >> 5];
                atomicAdd(&cnt[pre[kk >> 5] + __popc(m & ((1u << (kk & 31u)) - 1u))], 1u);
            }
        }
        __syncwarp();
        // each token's counts of its word's max and 2nd topics
        for (uint32_t base = 0; base < n; base += 32) {
            const uint32_t i = base + (uint32_t)lane;
            if (i < n) {
                const uint32_t pos = __ldg(dpos + i), t2 = __ldg(a.st_top2 + __ldg(dword + i));
                a.meta[pos - a.tok_base] = (count_of(t2 >> 16) << 16) | count_of(t2 & 0xffffu);
            }
        }
        __syncwarp();
        uint32_t* out = a.dt_ent + (__ldg(a.dt_off + d) - a.dt_base);
        for (int wb = 0; wb < bw; wb += 32) {
            const int wi = wb + lane;
            uint32_t m = wi < bw ? bits[wi] : 0u;
            if (m) {
                bits[wi] = 0u;
                uint32_t p = pre[wi];
                while (m) {
                    const uint32_t kk = (uint32_t)wi * 32u + (uint32_t)(__ffs(m) - 1);
                    m &= m - 1u;
                    out[p] = (kk << 16) | cnt[p];
                    cnt[p] = 0u;
                    ++p;
                }
            }
        }
        if (lane == 0) a.dt_nnz[d] = carry;
        __syncwarp();
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
    for (int w = a.wlo + blockIdx.x * warps + wid; w < a.V; w += gridDim.x * warps) {
        word_stats_word(a, w, r, col, lane);
    }
}

// Word statistics of dense words above kLargeK topics: warp per word, phi formed on the fly
// from the word's count row and the CTA's reciprocals (no K-wide column per warp, which
// left 4 warps per SM at K=10,000).  Results equal k_word_stats'.
__global__ void __launch_bounds__(256) k_word_stats_dense_rows(StatsArgs a) {
    extern __shared__ float smf[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* r = smf;
    fill_recip(r, a.n_k, a.K, a.Vbeta);
    __syncthreads();
    for (int w = a.wlo + blockIdx.x * warps + wid; w < a.V; w += gridDim.x * warps)
    {
        const DenseRowPhi phi{a.dwt + (size_t)w * a.K, r, a.beta};
        const int k1 = word_stats_from(a, w, phi, lane);
        if (a.qtab) word_qtab(a, w, k1, phi, lane);
    }
}

// Doc-topic rebuild: warp per doc of one chunk.  P16: 16-bit histogram counts (a doc has
// at most 65,535 tokens).
template <bool P16>
__global__ void __launch_bounds__(256) k_dt_build(DtArgs a) {
    extern __shared__ uint32_t smu[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int hw = Hist<P16>::words(a.K);
    const int per = hw + dt_bit_words(a.K);
    const Hist<P16> hist{smu + (size_t)per * wid};
    uint32_t* bits = hist.h + hw;
    for (int i = threadIdx.x; i < per * warps; i += blockDim.x) smu[i] = 0u;
    __syncthreads();
    for (uint32_t d = a.d_begin + blockIdx.x * warps + wid; d < a.d_end; d += gridDim.x * warps) {
        dt_doc(a, d, hist, bits, lane);
    }
}

// Sampler: warp per tile, tiles taken from an atomic counter.  SKEWKEYS: the doc rows'
// keys are word-column slot indices (the trainer's rows up to kLargeK topics).
template <bool LL, int QB = 1, bool SKEWKEYS = true>
__global__ void __launch_bounds__(32 * kSampleWarps, LL ? LDA_SAMPLE_LL_MIN_BLOCKS
                                                       : (QB == 1 ? LDA_SAMPLE_MIN_BLOCKS : LDA_SAMPLE_QB_MIN_BLOCKS))
k_sample_t(SampleArgs a) {
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
        sample_tile<LL, QB, SKEWKEYS>(a, tile, t, a.iter, r, col, ctr, lane);
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
    using Entry = uint32_t;  // a doc-row entry: (k << 16) | count
    const uint32_t* bits;  // ceil(K/32) words
    const uint16_t* pre;   // set bits before each word
    const uint32_t* ent;   // the word's row, (k << 16) | count
    const float* r;        // reciprocals in the skewed layout: r_k at col_skew(k)
    float beta;
    int maxK;
    // Branch-free: (0 + beta) is beta exactly, so one formula gives phi_k for topics in
    // and out of the word, and only the count's load is predicated.  The branch it replaces
    // kept the four batched row lookups of lane_mass apart (K=10,000 corpus: samplers
    // 115.7 -> 109.5 ms per sweep, the same topics).
    __device__ __forceinline__ float operator()(int k) const {
        const uint32_t b = bits[k >> 5], m = 1u << (k & 31);
        const float rk = r[col_skew(k)];
        uint32_t e = 0u;
        if (b & m) e = __ldg(ent + pre[k >> 5] + __popc(b & (m - 1u)));
        const float phi = fmul(fadd(u2f(e & 0xffffu), beta), rk);
        return k == maxK ? 0.0f : phi;
    }
    __device__ __forceinline__ float row(uint32_t key) const { return (*this)((int)key); }
    __device__ __forceinline__ int topic(uint32_t key) const { return (int)key; }
    __device__ __forceinline__ uint32_t key(uint32_t e) const { return e >> 16; }
    __device__ __forceinline__ float cnt(uint32_t e) const { return u2f(e & 0xffffu); }
};

__host__ __device__ __forceinline__ int large_bit_words(int K) { return (K + 31) >> 5; }
__host__ __device__ __forceinline__ int large_pre_words(int K) { return ((K + 31) >> 5) + 1 & ~1; }

// Shared memory of the sparse-word kernel: the reciprocals in the skewed column layout
// (col_words(K) floats: a Q round's 32 topics k, k + 32, ... then sit in 32 banks), then
// per warp the bitmap, then per warp the prefix counts (uint16, an even number per warp),
// then per warp the counter row.
__host__ __device__ __forceinline__ size_t sparse_large_smem(int K, int warps) {
    return (size_t)col_words(K) * 4 + (size_t)warps * (large_bit_words(K) * 4 + large_pre_words(K) * 2 + C_NUM * 4);
}

// Shared memory of the dense-word kernel: the shared column, the warps' counter rows and
// their LL partials (the reciprocals are formed while the column is built).
#ifndef LDA_QTAB
#define LDA_QTAB 1
#endif
// Shared memory of the dense-word sampler: the word column, the warps' counter rows, their
// LL partials and (when qtab_rounds(K) > 0) the Q-round table of 32 x R float2.
__host__ __device__ __forceinline__ size_t dense_large_smem(int K, int warps) {
    return (((size_t)col_words(K) * 4 + (size_t)warps * C_NUM * 4 + 7) & ~(size_t)7) + (size_t)warps * 8 +
           (LDA_QTAB ? (size_t)32 * qtab_rounds(K) * sizeof(float2) : 0);
}

#ifndef LDA_DENSE_LARGE_MIN_BLOCKS
#define LDA_DENSE_LARGE_MIN_BLOCKS 4
#endif

// How the large-K samplers issue a doc row's loads (lane_mass ROWM): four steps together,
// since at large K a third of the rows' bytes miss L2 (K=10,000 corpus: 148.3 -> 133.6
// ms of sampling per sweep; at K=1024 the same batching loses).
#ifndef LDA_LARGE_ROW_MODE
#define LDA_LARGE_ROW_MODE 1
#endif

// The sparse-word sampler keeps each word's Qw rounds' table in registers (lane r: round
// r), so a Q draw evaluates the one round that holds its target instead of walking them.
template <bool LL, int QB>
__global__ void __launch_bounds__(256, LDA_SPARSE_LARGE_MIN_BLOCKS) k_sample_sparse_large(SampleArgs a) {
    extern __shared__ float smf[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bw = large_bit_words(a.K), pw = large_pre_words(a.K);
    float* r = smf;
    float* rend = smf + col_words(a.K);
    uint32_t* bits = reinterpret_cast<uint32_t*>(rend) + (size_t)bw * wid;
    uint16_t* pre = reinterpret_cast<uint16_t*>(reinterpret_cast<uint32_t*>(rend) + (size_t)bw * warps) +
                    (size_t)pw * wid;
    uint32_t* ctr = reinterpret_cast<uint32_t*>(reinterpret_cast<uint16_t*>(reinterpret_cast<uint32_t*>(rend) +
                                                                            (size_t)bw * warps) +
                                                (size_t)pw * warps) +
                    C_NUM * wid;
    for (int k = threadIdx.x; k < a.K; k += blockDim.x)
        r[col_skew(k)] = __fdiv_rn(1.0f, fadd(__int2float_rn(a.n_k[k]), a.Vbeta));
    for (int i = lane; i < bw; i += 32) bits[i] = 0u;
    if (lane < C_NUM) ctr[lane] = 0u;
    __syncthreads();
    // the next tile is claimed when a tile starts, so that the claim's round trip overlaps
    // the tile's work
    int tile = 0;
    if (lane == 0) tile = (int)atomicAdd(a.tile_counter, 1u);
    tile = __shfl_sync(FULL, tile, 0);
    for (;;) {
        if (tile >= a.ntiles) break;
        int next = 0;
        if (lane == 0) next = (int)atomicAdd(a.tile_counter, 1u);
        const int4 t = a.tiles[tile];
        const int w = t.x;
        const int s = w - a.Vd;
        const uint32_t* ent = a.swt_ent + __ldg(a.swt_off + s);
        const uint32_t nnz_w = __ldg(a.swt_nnz + s);
        // the word's statistics, loaded before the bitmap work so that their loads overlap it
        const int maxK = (int)(__ldg(a.st_top2 + w) & 0xffffu);
        const float4 ph = __ldg(a.st_phi + w);
        const float QL = __ldg(a.st_ql + (size_t)w * 32 + lane);
        // the word's topics into the bitmap; pre[j] = the rank of the first of the word's
        // topics in bitmap word j (the entries ascend, so that is the entry's index).  Only
        // words with a set bit are ever read, so the others are left as they are.
        for (uint32_t e = lane; e < nnz_w; e += 32) {
            const uint32_t k = __ldg(ent + e) >> 16;
            atomicOr(&bits[k >> 5], 1u << (k & 31u));
            if (e == 0 || (__ldg(ent + e - 1) >> 21) != (k >> 5)) pre[k >> 5] = (uint16_t)e;
        }
        __syncwarp();
        if (lane == 0) {
            ctr[C_WNNZ] += nnz_w;
            ctr[C_TSPARSE] += 1u;
        }
        const float QP = warp_ks_scan(QL, lane);
        const float Q = __shfl_sync(FULL, QP, 31);
        __syncwarp();
        const ColBits view{bits, pre, ent, r, a.beta, maxK};
        SplitQ sq{ent, nnz_w, __shfl_sync(FULL, QL, 0), a.smooth, r, true};
        split_q_table(sq, maxK, a.alpha, lane);
        double ll = sample_groups<LL, QB, true, LDA_LARGE_ROW_MODE>(a, (uint32_t)t.y, (uint32_t)t.z, 0u, 32u, a.iter,
                                                                    maxK, ph, QL, QP, Q, view, ctr, lane, nullptr, 0,
                                                                    &sq);
        if (LL) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) ll += __shfl_xor_sync(FULL, ll, off);
            if (lane == 0) a.tile_ll[tile] = ll;
        }
        __syncwarp();
        for (uint32_t e = lane; e < nnz_w; e += 32) bits[(__ldg(ent + e) >> 16) >> 5] = 0u;
        __syncwarp();
        tile = __shfl_sync(FULL, next, 0);
    }
    __syncwarp();
    if (lane < C_NUM && ctr[lane]) atomicAdd(a.ctr + lane, (unsigned long long)ctr[lane]);
}

template <bool LL, int QB>
__global__ void __launch_bounds__(256, LDA_DENSE_LARGE_MIN_BLOCKS) k_sample_dense_large(SampleArgs a) {
    extern __shared__ float smf[];
    __shared__ int s_tile;
    __shared__ uint32_t s_group;  // plain sweeps: the tile's next 32-token group
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* col = smf;
    uint32_t* ctr_all = reinterpret_cast<uint32_t*>(col + col_words(a.K));
    uint32_t* ctr = ctr_all + C_NUM * wid;
    double* wll = reinterpret_cast<double*>(
        (reinterpret_cast<uintptr_t>(ctr_all + C_NUM * warps) + 7) & ~(uintptr_t)7);
    const int qr = LDA_QTAB ? qtab_rounds(a.K) : 0;
    float2* qtab = reinterpret_cast<float2*>(wll + warps);
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
        // the count row is read once per tile and chunk (800 MB per chunk on the K=10,000
        // corpus): evict_first, so that it displaces fewer of the chunk's doc rows in L2
        // (that corpus: samplers 116.1 -> 115.6 ms per sweep)
        const uint64_t spol = l2_stream_policy();
        for (int k = threadIdx.x; k < a.K; k += blockDim.x) {
            const float rk = a.recip ? __ldg(a.recip + k) : __fdiv_rn(1.0f, fadd(__int2float_rn(__ldg(a.n_k + k)), a.Vbeta));
            const int c = ldg_hint(wrow + k, spol);
            col[col_skew(k)] = fmul(fadd(__int2float_rn(c), a.beta), rk);
        }
        const int maxK = (int)(__ldg(a.st_top2 + w) & 0xffffu);
        __syncthreads();
        if (threadIdx.x == 0) {
            col[col_skew(maxK)] = 0.0f;
            ctr[C_TDENSE] += 1u;
            s_group = 0u;
        }
        __syncthreads();
        if (qr && a.qtab_g) {
            // the word's Q-round table, built by the word statistics
            const float2* src = a.qtab_g + (size_t)w * 32 * qr;
            for (int i = threadIdx.x; i < 32 * qr; i += blockDim.x) qtab[i] = __ldg(src + i);
            __syncthreads();
        } else if (qr) {
            // the Q-round table of this word: for lane slot ls and round r, the KS total and the
            // largest KS prefix of alpha * colz(ls + 32 * (32 r + l)), l = 0..31 (slots past the
            // lane's last topic add 0), the terms and scan of warp_level2_rounds
            const ColShared cv{col};
            for (int job = wid; job < 32 * qr; job += warps) {
                const int ls = job / qr, r = job - ls * qr;
                const uint32_t n = (uint32_t)((a.K - ls + 31) / 32), i = 32u * (uint32_t)r + (uint32_t)lane;
                const float term = i < n ? fmul(a.alpha, cv(ls + 32 * (int)i)) : 0.0f;
                const float ks = warp_ks_scan(term, lane);
                float mx = ks;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, off));
                const float tot = __shfl_sync(FULL, ks, 31);
                if (lane == 0) qtab[job] = make_float2(tot, mx);
            }
            __syncthreads();
            // per lane slot: the carry before each round (the fadd chain of the round
            // totals) and the round's threshold carry + largest prefix
            if (threadIdx.x < 32) {
                float carry = 0.0f;
                for (int r = 0; r < qr; ++r) {
                    const float2 tm = qtab[threadIdx.x * qr + r];
                    qtab[threadIdx.x * qr + r] = make_float2(carry, fadd(carry, tm.y));
                    carry = fadd(carry, tm.x);
                }
            }
            __syncthreads();
        }
        const float4 ph = __ldg(a.st_phi + w);
        const float QL = __ldg(a.st_ql + (size_t)w * 32 + lane);
        const float QP = warp_ks_scan(QL, lane);
        const float Q = __shfl_sync(FULL, QP, 31);
        double ll = sample_groups<LL, QB, false, LDA_LARGE_ROW_MODE>(a, (uint32_t)t.y, (uint32_t)t.z, 32u * wid,
                                                                     32u * warps, a.iter, maxK, ph, QL, QP, Q,
                                                                     ColShared{col}, ctr, lane, qr ? qtab : nullptr, qr,
                                                                     nullptr, LL ? nullptr : &s_group);
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

// ------------------------------------------------------------ large-K word statistics
// For K > kLargeK a sparse word's column is beta * r_k except at its own few topics, so its
// statistics need no column: the top three come from its own topics and the first three
// other topics of the CTA's list of topics in decreasing beta * r_k (ties to the lower k),
// and its split Q from its own entries and the smoothing table (Qw in st_ql slot 0, Qs in
// slot 1).  Dense words keep k_word_stats.
constexpr int kOrderList = 64;

// (v, k) ranks above (a, i): larger value, ties to the lower topic.
__device__ __forceinline__ bool ranks_above(float v, int k, float a, int i) { return v > a || (v == a && k < i); }

__device__ __forceinline__ void top3_insert(float v, int k, float& a1, int& i1, float& a2, int& i2, float& a3, int& i3) {
    if (ranks_above(v, k, a1, i1)) {
        a3 = a2; i3 = i2;
        a2 = a1; i2 = i1;
        a1 = v; i1 = k;
    } else if (ranks_above(v, k, a2, i2)) {
        a3 = a2; i3 = i2;
        a2 = v; i2 = k;
    } else if (ranks_above(v, k, a3, i3)) {
        a3 = v; i3 = k;
    }
}

// Shared memory of the sparse-word statistics: the order list, then per warp the bitmap.
// The reciprocals are read from the global table (k_recip), so that the CTA does not
// hold K of them and eight CTAs fit per SM.
__host__ __device__ __forceinline__ size_t stats_sparse_smem(int K, int warps) {
    return kOrderList * 4 + (size_t)warps * (large_bit_words(K) * 4);
}

// The first kOrderList topics by (beta * r_k desc, k asc), by repeated CTA-wide arg-max
// over the global reciprocal table (k_recip); one CTA.
__global__ void __launch_bounds__(256) k_sparse_order(StatsArgs a, int* order) {
    __shared__ float red_v[8];
    __shared__ int red_k[8];
    __shared__ int pick;
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float* __restrict__ r = a.recip;
    const int L = min(kOrderList, a.K);
    float pv = __int_as_float(0x7f800000);  // the previous pick; the next is the best ranked after it
    int pk = -1;
    for (int n = 0; n < L; ++n) {
        float bv = -1.0f;
        int bk = 0x7fffffff;
        for (int k = threadIdx.x; k < a.K; k += blockDim.x) {
            const float v = fmul(a.beta, r[k]);
            if (ranks_above(pv, pk, v, k) && ranks_above(v, k, bv, bk)) { bv = v; bk = k; }
        }
        warp_argmax(bv, bk);
        if (lane == 0) { red_v[wid] = bv; red_k[wid] = bk; }
        __syncthreads();
        if (threadIdx.x == 0) {
            float v = red_v[0];
            int k = red_k[0];
            for (int i = 1; i < warps; ++i)
                if (ranks_above(red_v[i], red_k[i], v, k)) { v = red_v[i]; k = red_k[i]; }
            order[n] = k;
            pick = k;
        }
        __syncthreads();
        pk = pick;
        pv = fmul(a.beta, r[pk]);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_word_stats_sparse_large(StatsArgs a) {
    extern __shared__ float smf[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bw = large_bit_words(a.K);
    const float* __restrict__ r = a.recip;
    int* order = reinterpret_cast<int*>(smf);
    uint32_t* bits = reinterpret_cast<uint32_t*>(order + kOrderList) + (size_t)bw * wid;
    const int L = min(kOrderList, a.K);
    for (int i = threadIdx.x; i < L; i += blockDim.x) order[i] = __ldg(a.order + i);
    for (int i = lane; i < bw; i += 32) bits[i] = 0u;
    __syncthreads();
    for (int w = max(a.Vd, a.wlo) + blockIdx.x * warps + wid; w < a.V; w += gridDim.x * warps) {
        const int s = w - a.Vd;
        const uint32_t* ent = a.swt_ent + __ldg(a.swt_off + s);
        const uint32_t nnz = __ldg(a.swt_nnz + s);
        float a1 = -1.0f, a2 = -1.0f, a3 = -1.0f;
        int i1 = 0x7fffffff, i2 = 0x7fffffff, i3 = 0x7fffffff;
        for (uint32_t e = lane; e < nnz; e += 32) {
            const uint32_t en = __ldg(ent + e);
            const int k = (int)(en >> 16);
            atomicOr(&bits[k >> 5], 1u << (k & 31));
            top3_insert(fmul(fadd(u2f(en & 0xffffu), a.beta), r[k]), k, a1, i1, a2, i2, a3, i3);
        }
        __syncwarp();
        // the best three topics outside the word: the first three of the CTA's order that
        // the word lacks (lane j looks at entry j), or, if the list runs out, every topic
        int found = 0, o0 = 0, o1 = 0, o2 = 0;
        for (int b = 0; b < L && found < 3; b += 32) {
            const int j = b + lane;
            const int kj = j < L ? order[j] : 0;
            const bool out = j < L && !((bits[kj >> 5] >> (kj & 31)) & 1u);
            for (unsigned m = __ballot_sync(FULL, out); m && found < 3; m &= m - 1u) {
                const int k = __shfl_sync(FULL, kj, __ffs(m) - 1);
                if (found == 0) o0 = k;
                else if (found == 1) o1 = k;
                else o2 = k;
                ++found;
            }
        }
        if (found == 3) {
            if (lane == 0) {
                top3_insert(fmul(a.beta, r[o0]), o0, a1, i1, a2, i2, a3, i3);
                top3_insert(fmul(a.beta, r[o1]), o1, a1, i1, a2, i2, a3, i3);
                top3_insert(fmul(a.beta, r[o2]), o2, a1, i1, a2, i2, a3, i3);
            }
        } else {
            for (int k = lane; k < a.K; k += 32)
                if (!((bits[k >> 5] >> (k & 31)) & 1u)) top3_insert(fmul(a.beta, r[k]), k, a1, i1, a2, i2, a3, i3);
        }
        float v[3];
        int kk[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            float bv = a1;
            int bk = i1;
            warp_argmax(bv, bk);
            v[q] = bv;
            kk[q] = bk;
            if (i1 == bk) {
                a1 = a2; i1 = i2;
                a2 = a3; i2 = i3;
                a3 = -1.0f; i3 = 0x7fffffff;
            }
        }
        const int k1 = kk[0];
        // Q = Qw + Qs (the split Q bucket): Qw over the word's own topics in rounds of 32
        // entries (ascending k, the max topic's term 0), Qs = T[K-1] - sm_max
        float carry = 0.0f;
        for (uint32_t base = 0; base < nnz; base += 32) {
            const uint32_t e = base + (uint32_t)lane;
            float term = 0.0f;
            if (e < nnz) {
                const uint32_t en = __ldg(ent + e);
                const int k = (int)(en >> 16);
                if (k != k1) term = fmul(a.alpha, fmul(u2f(en & 0xffffu), r[k]));
            }
            const float P = fadd(carry, warp_ks_scan(term, lane));
            carry = __shfl_sync(FULL, P, 31);
        }
        const float Qw = carry;
        const float Qs = fsub(__ldg(a.smooth + a.K - 1), fmul(a.alpha, fmul(a.beta, r[k1])));
        a.st_ql[(size_t)w * 32 + lane] = lane == 0 ? Qw : (lane == 1 ? Qs : 0.0f);
        if (lane == 0) {
            a.st_top2[w] = ((uint32_t)kk[1] << 16) | (uint32_t)k1;
            a.st_k3[w] = (uint32_t)kk[2];
            a.st_phi[w] = make_float4(v[0], v[1], v[2], fadd(Qw, Qs));
        }
        __syncwarp();
        for (uint32_t e = lane; e < nnz; e += 32) bits[(__ldg(ent + e) >> 16) >> 5] = 0u;
        __syncwarp();
    }
}

// The smoothing table of the split Q bucket (K > kLargeK): T[k] = carry + Kogge-Stone scan
// of sm_k = alpha * (beta * r_k) over rounds of 32 topics, the carry being the previous
// round's last prefix, so T is non-decreasing and T[K-1] is the total.  r_k is formed from
// n_k as fill_recip forms it.  One CTA: its warps scan the rounds in parallel (the scan of
// a round does not depend on the carry), one thread chains the carries, then every T[k] is
// one addition.  T holds each round's scan until the carries are known.
__global__ void __launch_bounds__(1024) k_smooth_table(const int* __restrict__ n_k, int K, float Vbeta, float alpha,
                                                       float beta, float* __restrict__ T) {
    __shared__ float carry_s[kSmoothMaxRounds];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rounds = (K + 31) >> 5;
    for (int rd = wid; rd < rounds; rd += warps) {
        const int k = 32 * rd + lane;
        const float sm = k < K ? fmul(alpha, fmul(beta, __fdiv_rn(1.0f, fadd(__int2float_rn(n_k[k]), Vbeta)))) : 0.0f;
        const float sc = warp_ks_scan(sm, lane);
        if (k < K) T[k] = sc;
        if (lane == 31) carry_s[rd] = sc;  // the round's total for now
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float carry = 0.0f;
        for (int rd = 0; rd < rounds; ++rd) {
            const float tot = carry_s[rd];
            carry_s[rd] = carry;
            carry = fadd(carry, tot);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < K; k += blockDim.x) T[k] = fadd(carry_s[k >> 5], T[k]);
}

// r_k = 1 / ((float)n_k + V*beta), the value fill_recip forms, into a global table.
__global__ void __launch_bounds__(256) k_recip(const int* __restrict__ n_k, int K, float Vbeta, float* r) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < K) r[k] = __fdiv_rn(1.0f, fadd(__int2float_rn(n_k[k]), Vbeta));
}

// Fixed-order FP64 reduction of the per-tile LL partials (one CTA of 1024 threads).
// Replaces LDATrainPerplexityReduce (EZLDA/utility.cu:2106-2151).
__global__ void __launch_bounds__(1024) k_ll_reduce(const double* __restrict__ in, int n, double* out) {
    __shared__ double s[1024];
    const double acc = strided_sum(in, n);
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
