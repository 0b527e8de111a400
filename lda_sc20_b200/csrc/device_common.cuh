// device_common.cuh -- device helpers shared by the sweep and the fold-in kernels.
//
// Every float operation is an explicit round-to-nearest intrinsic, so the compiler cannot
// contract or reorder it; the summation orders below are part of the arithmetic
// specification the CPU oracle restates.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace lda {
namespace dev {

constexpr unsigned FULL = 0xffffffffu;

// Above this many topics the trainer samples with the CTA-per-tile dense-word kernel and
// the column-free sparse-word kernel (kernels.cuh) instead of a column per warp, and a
// sparse word's Q bucket is split into its own topics and a word-independent smoothing
// part (split_q_draw).
constexpr int kLargeK = 2048;

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float u2f(uint32_t x) { return __uint2float_rn(x); }

// Inclusive Kogge-Stone scan over the warp: round `off` adds lane l-off into lane l.
__device__ __forceinline__ float warp_ks_scan(float v, int lane) {
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const float t = __shfl_up_sync(FULL, v, off);
        if (lane >= off) v = fadd(v, t);
    }
    return v;
}

// Thread t's sum of in[t], in[t + blockDim.x], ... in that order (the first stage of the
// fixed-order FP64 LL reductions).  Eight loads are issued before their eight additions.
__device__ __forceinline__ double strided_sum(const double* __restrict__ in, int n) {
    const int st = blockDim.x;
    double acc = 0.0;
    int i = threadIdx.x;
    for (; i + 7 * st < n; i += 8 * st) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = __ldg(in + i + u * st);
#pragma unroll
        for (int u = 0; u < 8; ++u) acc += v[u];
    }
    for (; i < n; i += st) acc += __ldg(in + i);
    return acc;
}

// Philox4x32-10 (Salmon et al., SC'11), first output word.
__device__ __forceinline__ uint32_t philox_x0(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                              uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c1 = lo1;
        c3 = lo0;
        c0 = n0;
        c2 = n2;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c0;
}

// u in [0,1) of token `tok` at sweep `iter` (replaces curand_uniform()/1.00001,
// EZLDA/utility.cu:1353).
__device__ __forceinline__ float token_uniform(uint32_t seed_lo, uint32_t seed_hi, uint32_t iter,
                                               uint32_t tok) {
    const uint32_t x = philox_x0(tok, 0u, iter, 0x4C444131u, seed_lo, seed_hi);
    return u2f(x >> 8) * 0x1p-24f;
}

// A warp-private shared histogram over topics [0, K).  Hist<false>: one 32-bit count per
// topic.  Hist<true>: 16-bit counts, two per 32-bit word (half the shared memory, so twice
// the warps at large K), for counts known to stay below 2^16.  Adds are 32-bit atomics on
// the containing word with the count shifted into its half; they never carry into the
// other half.  Reads and clears use the 16-bit view; the two topics of a word (k, k ^ 1)
// share a bitmap word, so one lane owns both when a histogram is read out and cleared.
template <bool P16>
struct Hist;
template <>
struct Hist<false> {
    uint32_t* h;
    __host__ __device__ static constexpr int words(int K) { return K; }
    __device__ __forceinline__ uint32_t add(uint32_t k, uint32_t c) const { return atomicAdd(h + k, c); }
    __device__ __forceinline__ uint32_t get(uint32_t k) const { return h[k]; }
    __device__ __forceinline__ void clear(uint32_t k) const { h[k] = 0u; }
};
template <>
struct Hist<true> {
    uint32_t* h;
    __host__ __device__ static constexpr int words(int K) { return (K + 1) >> 1; }
    __device__ __forceinline__ uint32_t add(uint32_t k, uint32_t c) const {
        const uint32_t sh = (k & 1u) << 4;
        return (atomicAdd(h + (k >> 1), c << sh) >> sh) & 0xffffu;
    }
    __device__ __forceinline__ uint32_t get(uint32_t k) const { return reinterpret_cast<const uint16_t*>(h)[k]; }
    __device__ __forceinline__ void clear(uint32_t k) const { reinterpret_cast<uint16_t*>(h)[k] = 0; }
};

// One token of topic k into a histogram, and the topic's bit into the bitmap of non-zero
// topics when its count leaves zero.  (Setting the bit for every token instead, so that
// neither atomic's result is waited on, was no faster.)
template <class H>
__device__ __forceinline__ void hist_token(const H& hist, uint32_t* bits, uint32_t k) {
    if (hist.add(k, 1u) == 0u) atomicOr(&bits[k >> 5], 1u << (k & 31u));
}

// Histogram of topics z[start, start + cnt) into the warp's shared `hist`; a topic whose
// count leaves zero also gets its bit in `bits` (ceil(K/32) words).  Four 32-token steps
// of topic loads are in flight together.
template <class H>
__device__ __forceinline__ void hist_segment(const uint16_t* __restrict__ z, uint32_t start, uint32_t cnt,
                                             const H& hist, uint32_t* bits, int K, int lane, int* err) {
    for (uint32_t base = 0; base < cnt; base += 128) {
        uint32_t k[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const uint32_t i = base + 32u * s + lane;
            k[s] = i < cnt ? (uint32_t)__ldg(z + start + i) : 0xffffffffu;
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (base + 32u * s >= cnt) break;
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

// ------------------------------------------------------------ word columns
// The sampler's shared word column stores topic k at k + k/32: the 32 topics k = l,
// l+32, ..., l+992 that one Q-bucket round reads then fall in 32 different banks (a plain
// layout puts them all in bank l).  col_words(K) floats hold a skewed column.
__host__ __device__ __forceinline__ int col_skew(int k) { return k + (k >> 5); }
__host__ __device__ __forceinline__ int col_words(int K) { return (K + (K >> 5) + 4) & ~3; }

// phi_k = ((float)n_wk + beta) * r_k into a warp-private shared row (EZLDA builds the
// same column as WTHead, utility.cu:1257-1269 sparse, :1698-1702 dense); SKEW selects the
// sampler's layout.
template <bool SKEW = false>
__device__ __forceinline__ void build_column(float* col, const float* r, int w, int Vd, int K, float beta,
                                             const int* __restrict__ dwt, const uint32_t* __restrict__ swt_off,
                                             const uint32_t* __restrict__ swt_nnz,
                                             const uint32_t* __restrict__ swt_ent, int lane, uint32_t* nnz_read) {
    if (w < Vd) {
        const int* row = dwt + (size_t)w * K;
        for (int k = lane; k < K; k += 32)
            col[SKEW ? col_skew(k) : k] = fmul(fadd(__int2float_rn(__ldg(row + k)), beta), r[k]);
    } else {
        for (int k = lane; k < K; k += 32) col[SKEW ? col_skew(k) : k] = fmul(beta, r[k]);
        __syncwarp();
        const int s = w - Vd;
        const uint32_t off = __ldg(swt_off + s), nnz = __ldg(swt_nnz + s);
        for (uint32_t e = lane; e < nnz; e += 32) {
            const uint32_t en = __ldg(swt_ent + off + e);
            const uint32_t k = en >> 16;
            col[SKEW ? col_skew((int)k) : (int)k] = fmul(fadd(u2f(en & 0xffffu), beta), r[k]);
        }
        if (nnz_read && lane == 0) *nnz_read += nnz;
    }
    __syncwarp();
}

__device__ __forceinline__ void warp_argmax(float& v, int& k) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_xor_sync(FULL, v, off);
        const int ok = __shfl_xor_sync(FULL, k, off);
        if (ov > v || (ov == v && ok < k)) {
            v = ov;
            k = ok;
        }
    }
}

__device__ __forceinline__ void fill_recip(float* r, const int* __restrict__ n_k, int K, float Vbeta) {
    for (int k = threadIdx.x; k < K; k += blockDim.x) r[k] = __fdiv_rn(1.0f, fadd(__int2float_rn(n_k[k]), Vbeta));
}

// Second-level search over 32-entry rounds: term = weight of slot i, ok = slot may be
// drawn; returns the key of the first ok slot whose carried scan exceeds t2, else the
// last ok slot's key, else `fallback`.  Uniform across the warp.
template <class Slot>
__device__ __forceinline__ int warp_level2(uint32_t n, float t2, int fallback, int lane, Slot slot) {
    float carry = 0.0f;
    int last = -1;
    for (uint32_t base = 0; base < n; base += 32) {
        int key = -1;
        float term = 0.0f;
        bool ok = false;
        if (base + lane < n) slot(base + lane, key, term, ok);
        const float P = fadd(carry, warp_ks_scan(term, lane));
        const unsigned f = __ballot_sync(FULL, ok && t2 < P);
        const unsigned v = __ballot_sync(FULL, ok);
        if (f) return __shfl_sync(FULL, key, __ffs(f) - 1);
        if (v) last = __shfl_sync(FULL, key, 31 - __clz(v));
        carry = __shfl_sync(FULL, P, 31);
    }
    return last >= 0 ? last : fallback;
}

// warp_level2 with QB rounds loaded and scanned together: the rounds' terms and their
// Kogge-Stone scans are independent, only the carry links them, so QB scans run
// interleaved and the rounds are then decided in order with the same additions
// (carry + the round's total equals the round's last prefix).  QB = 1 is warp_level2.
template <int QB, class Slot>
__device__ __forceinline__ int warp_level2_rounds(uint32_t n, float t2, int fallback, int lane, Slot slot) {
    if (QB == 1) return warp_level2(n, t2, fallback, lane, slot);
    float carry = 0.0f;
    int last = -1;
    for (uint32_t base = 0; base < n; base += 32u * QB) {
        float ks[QB];
        int key[QB];
        bool ok[QB];
#pragma unroll
        for (int q = 0; q < QB; ++q) {
            key[q] = -1;
            ks[q] = 0.0f;
            ok[q] = false;
            const uint32_t i = base + 32u * q + lane;
            if (i < n) slot(i, key[q], ks[q], ok[q]);
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
            for (int q = 0; q < QB; ++q) {
                const float t = __shfl_up_sync(FULL, ks[q], off);
                if (lane >= off) ks[q] = fadd(ks[q], t);
            }
        }
        float tot[QB];
#pragma unroll
        for (int q = 0; q < QB; ++q) tot[q] = __shfl_sync(FULL, ks[q], 31);
#pragma unroll
        for (int q = 0; q < QB; ++q) {
            if (base + 32u * q >= n) break;
            const float P = fadd(carry, ks[q]);
            const unsigned f = __ballot_sync(FULL, ok[q] && t2 < P);
            const unsigned v = __ballot_sync(FULL, ok[q]);
            if (f) return __shfl_sync(FULL, key[q], __ffs(f) - 1);
            if (v) last = __shfl_sync(FULL, key[q], 31 - __clz(v));
            carry = fadd(carry, tot[q]);
        }
    }
    return last >= 0 ? last : fallback;
}

// First k in [lo, hi) with x < T[k] for a non-decreasing table T in global memory, else
// -1; uniform across the warp.  A 32-way search: each round the lanes probe the ends of 32
// equal segments of the range, and a ballot keeps the first segment whose end exceeds x
// (the answer lies in it, since every entry before its start is <= x).
__device__ __forceinline__ int warp_first_above(const float* __restrict__ T, int lo, int hi, float x, int lane) {
    if (lo >= hi || !(x < __ldg(T + hi - 1))) return -1;
    while (hi - lo > 32) {
        const int step = (hi - lo + 31) >> 5;
        const int p = min(lo + (lane + 1) * step - 1, hi - 1);
        const unsigned b = __ballot_sync(FULL, x < __ldg(T + p));  // lane 31 probes hi - 1
        const int f = __ffs(b) - 1;
        const int nlo = f == 0 ? lo : min(lo + f * step - 1, hi - 1) + 1;
        hi = min(lo + (f + 1) * step - 1, hi - 1) + 1;
        lo = nlo;
    }
    const int p = lo + lane;
    const unsigned b = __ballot_sync(FULL, p < hi && x < __ldg(T + p));
    return lo + __ffs(b) - 1;
}

// Rounds of the Q-bucket search of one lane slot ls whose (round total, largest lane
// prefix) pairs the dense-word sampler keeps per tile: R = ceil(ceil(K/32) / 32) rounds of
// 32 slots, for 2 <= R <= 16 (above that the table is not kept).
__host__ __device__ __forceinline__ int qtab_rounds(int K) {
    const int R = ((K + 31) / 32 + 31) / 32;
    return (R >= 2 && R <= 16) ? R : 0;
}

// warp_level2_rounds (QB = 1 order) with each round's carry and threshold known
// (tab[r] = (carry before round r, carry + the round's largest KS lane prefix), the carry
// being the fadd chain of the round totals).  Round r can hold the crossing only if
// t2 < its threshold; one ballot over the R <= 32 rounds gives every such round, and they
// are evaluated in order with the same carry the round-by-round walk reaches, so the
// topic is the one warp_level2_rounds finds.  Returns -1 when no evaluated round crosses;
// the caller then runs the full search, which also finds the fallback topic.
template <class Slot>
__device__ __forceinline__ int warp_level2_table(uint32_t n, float t2, int lane, Slot slot, const float2* tab) {
    const uint32_t R = (n + 31u) >> 5;
    for (unsigned b = __ballot_sync(FULL, (uint32_t)lane < R && t2 < tab[lane < (int)R ? lane : 0].y); b;
         b &= b - 1u) {
        const uint32_t r = (uint32_t)(__ffs(b) - 1);
        const float carry = tab[r].x;
        int key = -1;
        float ks = 0.0f;
        bool ok = false;
        const uint32_t i = 32u * r + lane;
        if (i < n) slot(i, key, ks, ok);
        ks = warp_ks_scan(ks, lane);
        const unsigned f = __ballot_sync(FULL, ok && t2 < fadd(carry, ks));
        if (f) return __shfl_sync(FULL, key, __ffs(f) - 1);
    }
    return -1;
}

// Doc-row entries are (key << 16) | count.  Up to kLargeK topics the trainer's rows carry
// the word column's slot index col_skew(k) as the key, so a lookup needs no index
// arithmetic; above kLargeK, and in rows a caller supplies, the key is the topic k.
// col_skew is k + k/32, so k = s - s/33 inverts it (s = 33a + b with b < 32).
__host__ __device__ __forceinline__ int col_unskew(int s) { return s - s / 33; }

// The sampler's view of the tile's word column: colz(k) = phi_k of the word with its max
// topic zeroed; row(key) the same for a doc-row key and topic(key) the key's topic.
// ColSharedT reads a column built in shared memory (skewed layout, with the max topic's
// slot already zeroed); SKEWKEYS: the rows' keys are slot indices.
template <bool SKEWKEYS>
struct ColSharedT {
    using Entry = uint32_t;  // a doc-row entry: (key << 16) | count
    const float* col;
    __device__ __forceinline__ float operator()(int k) const { return col[col_skew(k)]; }
    __device__ __forceinline__ float row(uint32_t key) const { return col[SKEWKEYS ? (int)key : col_skew((int)key)]; }
    __device__ __forceinline__ int topic(uint32_t key) const { return SKEWKEYS ? col_unskew((int)key) : (int)key; }
    __device__ __forceinline__ uint32_t key(uint32_t e) const { return e >> 16; }
    __device__ __forceinline__ float cnt(uint32_t e) const { return u2f(e & 0xffffu); }
};
using ColShared = ColSharedT<false>;

// An L2 policy for loads of data read once per pass (evict_first), and a load with it.
__device__ __forceinline__ uint64_t l2_stream_policy() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ int ldg_hint(const int* p, uint64_t pol) {
    int v;
    asm("ld.global.nc.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}

// Serial per-lane sum over the lane's entries l, l + 32, l + 64, ... of a doc row of nnz
// entries (one fmaf chain).  A warp's loads of one step then read 32 consecutive entries,
// one or two 128-byte lines, where contiguous per-lane blocks would touch one line per
// lane block.
// ROWM 1: the loads of four steps at a time are issued before their use (rows that often
// miss L2, at large K); ROWM 0: two steps at a time.
template <int ROWM = 0, class View>
__device__ __forceinline__ float lane_mass(const typename View::Entry* __restrict__ row, uint32_t lane, uint32_t nnz,
                                           const View& colz, float acc = 0.0f) {
    using E = typename View::Entry;
    // Loop bounds are warp-uniform: `full` steps in which every lane has an entry, taken in
    // batches, then the lane's last steps together with the partial step.  Bounds per lane
    // would send the lanes of one warp through different batches, and the warp would issue
    // each of them (K=1024 corpus: sampler 10.38 -> 9.93 ms per sweep, the same sums).
    const uint32_t full = nnz >> 5;
    const E* __restrict__ p = row + lane;
    uint32_t s = 0;
    if (ROWM == 1) {
        for (; s + 4u <= full; s += 4u) {
            const E e0 = __ldg(p + 32u * s), e1 = __ldg(p + 32u * s + 32u), e2 = __ldg(p + 32u * s + 64u),
                    e3 = __ldg(p + 32u * s + 96u);
            acc = ffma(colz.cnt(e0), colz.row(colz.key(e0)), acc);
            acc = ffma(colz.cnt(e1), colz.row(colz.key(e1)), acc);
            acc = ffma(colz.cnt(e2), colz.row(colz.key(e2)), acc);
            acc = ffma(colz.cnt(e3), colz.row(colz.key(e3)), acc);
        }
        // the lane's last steps (up to three full ones and the partial one): their loads
        // issued together, so that a row of up to 256 entries costs two rounds of loads
        const uint32_t nl = full + (lane < (nnz & 31u) ? 1u : 0u);
        if (s < full + ((nnz & 31u) ? 1u : 0u)) {
            E e[4];
#pragma unroll
            for (uint32_t j = 0; j < 4u; ++j) e[j] = s + j < nl ? __ldg(p + 32u * (s + j)) : E{};
#pragma unroll
            for (uint32_t j = 0; j < 4u; ++j)
                if (s + j < nl) acc = ffma(colz.cnt(e[j]), colz.row(colz.key(e[j])), acc);
        }
        return acc;
    }
    for (; s + 2u <= full; s += 2u) {
        const E e0 = __ldg(p + 32u * s), e1 = __ldg(p + 32u * s + 32u);
        acc = ffma(colz.cnt(e0), colz.row(colz.key(e0)), acc);
        acc = ffma(colz.cnt(e1), colz.row(colz.key(e1)), acc);
    }
    // the last full step (if any) and the lanes of the partial step, loads issued together
    const bool one = s < full, tail = lane < (nnz & 31u);
    E e0{}, e1{};
    if (one) e0 = __ldg(p + 32u * s);
    if (tail) e1 = __ldg(p + 32u * full);
    if (one) acc = ffma(colz.cnt(e0), colz.row(colz.key(e0)), acc);
    if (tail) acc = ffma(colz.cnt(e1), colz.row(colz.key(e1)), acc);
    return acc;
}

// The S-bucket draw among lane ls's entries ls, ls + 32, ... of the row: their serial
// partial sums (the fmaf chain of lane_mass) are compared with t2; the first entry with
// colz > 0 whose partial sum exceeds t2 wins, else the last entry with colz > 0, else
// `fallback`.  Each entry of the lane sits on its own 128-byte line, so the loads of four
// entries are issued before any of them is used.
template <class View>
__device__ __forceinline__ int lane_draw(const typename View::Entry* __restrict__ row, uint32_t ls, uint32_t nnz,
                                         const View& colz, float t2, int fallback) {
    using E = typename View::Entry;
    float acc = 0.0f;
    int last = -1;
    for (uint32_t q = ls; q < nnz; q += 128u) {
        E e[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) e[s] = q + 32u * s < nnz ? __ldg(row + q + 32u * s) : E{};
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (q + 32u * s >= nnz) break;
            const uint32_t key = colz.key(e[s]);
            const float cz = colz.row(key);
            acc = ffma(colz.cnt(e[s]), cz, acc);
            if (cz > 0.0f) {
                last = (int)key;
                if (t2 < acc) return colz.topic(key);
            }
        }
    }
    return last >= 0 ? colz.topic((uint32_t)last) : fallback;
}


}  // namespace dev
}  // namespace lda
