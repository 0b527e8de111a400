// sweep_body.cuh -- per-unit bodies of the sweep kernels (one word tile, one word, one
// doc, one sampler tile), shared by the single-corpus kernels and the batched ones.
//
// Every float operation below is an explicit round-to-nearest intrinsic, so the compiler
// cannot contract or reorder it.  The sampling arithmetic (summation orders, bin order,
// tie rules) is the specification the CPU oracle restates; the CUDA path and the oracle
// therefore draw identical topics for identical (seed, iteration, token).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"

namespace lda {
namespace dev {

// ---------------------------------------------------------------- WT rebuild
// Warp per word tile: the tile's topics are histogrammed in a warp-private shared row
// with one shared atomic per token (aggregating a warp's equal topics with
// __match_any_sync first made the rebuild 2.6x slower).  Dense tiles add their row into the dense
// word-topic matrix; a sparse word (one tile over all chunks) is compacted to
// (k<<16 | count) ascending k.  Topic totals n_k are privatised per CTA and flushed once.
// Replaces WTDen_Update_Kernel, WT_Update_Kernel, sparseMatrixAdd and
// WTDen_Sum_Update_Kernel (EZLDA/utility.cu:1067-1102, :10-76, :1132-1204, :1104-1126).
struct WtArgs {
    const int4* tiles;  // {word, start, count, dense}
    int ntiles;
    unsigned* tile_counter;
    const uint16_t* z;
    int K, V, Vd, C;
    const uint32_t* seg_off;  // [C*V]
    const uint32_t* seg_cnt;  // [C*V]
    int* dwt;                 // [Vd*K]
    const uint32_t* swt_off;  // [V-Vd]
    uint32_t* swt_nnz;
    uint32_t* swt_ent;
    int* n_k;
    int* err;
};

// One word tile: histogram its topics in the warp's shared row `hist` (K words) with the
// bitmap of its non-zero topics in `bits` (ceil(K/32) words), both zero on entry and on
// exit, and add it to the dense row or write the sparse row (ascending k, placed by a
// prefix scan of the bitmap words' popcounts); topic totals go to `nk` (a CTA-private
// shared array, or the model's global totals).
__device__ __forceinline__ int wt_bit_words(int K) { return (K + 31) >> 5; }

template <class H>
__device__ __forceinline__ void wt_tile(const WtArgs& a, const int4 t, const H& hist, uint32_t* bits, unsigned* nk,
                                        int lane) {
    const int w = t.x;
    if (t.w & 1) {
        hist_segment(a.z, (uint32_t)t.y, (uint32_t)t.z, hist, bits, a.K, lane, a.err);
    } else {
        // a sparse word's segments in every chunk: lane c loads chunk c's offset and count
        for (int c0 = 0; c0 < a.C; c0 += 32) {
            const int c = c0 + lane;
            uint32_t so = 0, sc = 0;
            if (c < a.C) {
                const size_t idx = (size_t)c * a.V + w;
                so = __ldg(a.seg_off + idx);
                sc = __ldg(a.seg_cnt + idx);
            }
            const int nc = min(32, a.C - c0);
            for (int j = 0; j < nc; ++j) {
                const uint32_t o = __shfl_sync(FULL, so, j), n = __shfl_sync(FULL, sc, j);
                if (n) hist_segment(a.z, o, n, hist, bits, a.K, lane, a.err);
            }
        }
    }
    __syncwarp();
    const int words = wt_bit_words(a.K);
    if (t.w & 1) {
        int* row = a.dwt + (size_t)w * a.K;
        for (int wi = lane; wi < words; wi += 32) {
            uint32_t m = bits[wi];
            if (m) bits[wi] = 0u;
            while (m) {
                const uint32_t k = (uint32_t)wi * 32u + (uint32_t)(__ffs(m) - 1);
                m &= m - 1u;
                const uint32_t h = hist.get(k);
                atomicAdd(row + k, (int)h);
                atomicAdd(nk + k, h);
                hist.clear(k);
            }
        }
    } else {
        const int s = w - a.Vd;
        uint32_t* out = a.swt_ent + a.swt_off[s];
        uint32_t nnz = 0;
        for (int wb = 0; wb < words; wb += 32) {
            const int wi = wb + lane;
            uint32_t m = wi < words ? bits[wi] : 0u;
            const uint32_t c = (uint32_t)__popc(m);
            uint32_t incl = c;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t v = __shfl_up_sync(FULL, incl, off);
                if (lane >= off) incl += v;
            }
            uint32_t p = nnz + incl - c;
            nnz += __shfl_sync(FULL, incl, 31);
            if (m) bits[wi] = 0u;
            while (m) {
                const uint32_t k = (uint32_t)wi * 32u + (uint32_t)(__ffs(m) - 1);
                m &= m - 1u;
                const uint32_t h = hist.get(k);
                out[p++] = (k << 16) | h;
                atomicAdd(nk + k, h);
                hist.clear(k);
            }
        }
        if (lane == 0) a.swt_nnz[s] = nnz;
    }
    __syncwarp();
}

// ---------------------------------------------------------------- word stats
// Warp per word: max / 2nd / 3rd topic of phi (ties to the lower k), phi at those
// topics, and the 32 lane partials of Q = alpha * sum_{k != max} phi_k.  Replaces
// MaxTopicDense_Update_Kernel / MaxTopicSparse_Update_Kernel (EZLDA/utility.cu:305-1062).
struct StatsArgs {
    int V, Vd, K;
    float alpha, beta, Vbeta;
    const int* n_k;
    const int* dwt;
    const uint32_t* swt_off;
    const uint32_t* swt_nnz;
    const uint32_t* swt_ent;
    uint32_t* st_top2;  // (k2 << 16) | maxK
    uint32_t* st_k3;
    float4* st_phi;     // {phi_max, phi_2nd, phi_3rd, Q}
    float* st_ql;       // [V*32]
    const float* smooth = nullptr;  // K > kLargeK: the smoothing table (k_smooth_table)
    int wlo = 0;                    // the words [wlo, V) get statistics (a word range)
    const float* recip = nullptr;   // K > kLargeK: r_k as fill_recip forms it (k_recip)
    const int* order = nullptr;     // K > kLargeK: the sparse words' topic order (k_sparse_order)
    // K > kLargeK: the dense words' Q-round tables (32 lane slots x qrounds float2 per word,
    // the table k_sample_dense_large would build per tile), or null
    float2* qtab = nullptr;
    int qrounds = 0;
};

// Statistics of word w from its column (built into the warp's shared `col`).
// phi_k of dense word w formed on the fly from its count row, the value build_column stores
struct DenseRowPhi {
    const int* row;
    const float* r;
    float beta;
    __device__ __forceinline__ float operator()(int k) const {
        return fmul(fadd(__int2float_rn(__ldg(row + k)), beta), r[k]);
    }
};
struct ColumnPhi {
    const float* col;
    __device__ __forceinline__ float operator()(int k) const { return col[k]; }
};

// The statistics of word w from phi(k), k < K: top three, the lane partials of Q (the
// max topic excluded) and Q.
template <class Phi>
__device__ __forceinline__ int word_stats_from(const StatsArgs& a, int w, const Phi& phi, int lane);

__device__ __forceinline__ void word_stats_word(const StatsArgs& a, int w, const float* r, float* col, int lane) {
    build_column(col, r, w, a.Vd, a.K, a.beta, a.dwt, a.swt_off, a.swt_nnz, a.swt_ent, lane, nullptr);
    word_stats_from(a, w, ColumnPhi{col}, lane);
}

template <class Phi>
__device__ __forceinline__ int word_stats_from(const StatsArgs& a, int w, const Phi& phi, int lane) {
    // the lane's top three by (phi desc, k asc) in one pass (k ascends, so a strictly larger
    // value is needed to displace), then three warp-wide pops of the lanes' heads
    float a1 = -1.0f, a2 = -1.0f, a3 = -1.0f;
    int i1 = 0x7fffffff, i2 = 0x7fffffff, i3 = 0x7fffffff;
    for (int k = lane; k < a.K; k += 32) {
        const float x = phi(k);
        if (x > a1) {
            a3 = a2; i3 = i2;
            a2 = a1; i2 = i1;
            a1 = x; i1 = k;
        } else if (x > a2) {
            a3 = a2; i3 = i2;
            a2 = x; i2 = k;
        } else if (x > a3) {
            a3 = x; i3 = k;
        }
    }
    float v[3];
    int kk[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        float bv = a1;
        int bk = i1;
        warp_argmax(bv, bk);
        v[r] = bv;
        kk[r] = bk;
        if (i1 == bk) {
            a1 = a2; i1 = i2;
            a2 = a3; i2 = i3;
            a3 = -1.0f; i3 = 0x7fffffff;
        }
    }
    const float v1 = v[0], v2 = v[1], v3 = v[2];
    const int k1 = kk[0], k2 = kk[1], k3 = kk[2];
    float ql = 0.0f;
    for (int k = lane; k < a.K; k += 32) if (k != k1) ql = ffma(a.alpha, phi(k), ql);
    const float qp = warp_ks_scan(ql, lane);
    const float Q = __shfl_sync(FULL, qp, 31);
    a.st_ql[(size_t)w * 32 + lane] = ql;
    if (lane == 0) {
        a.st_top2[w] = ((uint32_t)k2 << 16) | (uint32_t)k1;
        a.st_k3[w] = (uint32_t)k3;
        a.st_phi[w] = make_float4(v1, v2, v3, Q);
    }
    __syncwarp();
    return k1;
}

// The Q-round table of dense word w (max topic k1) into a.qtab: for lane slot ls and round
// r, the Kogge-Stone total and largest prefix of alpha * colz(ls + 32 * (32 r + l)),
// l = 0..31 (slots past the lane slot's last topic add 0, colz the column with its max
// topic zeroed), then per lane slot the carries as the fadd chain of the totals: entry
// (ls, r) = (carry before round r, carry + the round's largest prefix).  The values
// k_sample_dense_large forms from its shared column with warp scans; here lane ls scans
// its own slot's 32 terms of a round serially in the same Kogge-Stone order (element l
// adds element l - off at each step off = 1, 2, ..., 16), so that a round's loads read
// 1,024 consecutive topics.
template <class Phi>
__device__ __forceinline__ void word_qtab(const StatsArgs& a, int w, int k1, const Phi& phi, int lane) {
    const int R = a.qrounds;
    float2* tab = a.qtab + (size_t)w * 32 * R;
    const int ls = lane;
    const uint32_t n = (uint32_t)((a.K - ls + 31) / 32);
    float carry = 0.0f;
    for (int r = 0; r < R; ++r) {
        float v[32];
#pragma unroll
        for (int l = 0; l < 32; ++l) {
            const uint32_t i = 32u * (uint32_t)r + (uint32_t)l;
            const int k = ls + 32 * (int)i;
            v[l] = i < n ? fmul(a.alpha, k == k1 ? 0.0f : phi(k)) : 0.0f;
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
            for (int l = 31; l >= off; --l) v[l] = fadd(v[l], v[l - off]);
        }
        float mx = v[0];
#pragma unroll
        for (int l = 1; l < 32; ++l) mx = fmaxf(mx, v[l]);
        tab[ls * R + r] = make_float2(carry, fadd(carry, mx));
        carry = fadd(carry, v[31]);
    }
}

// ---------------------------------------------------------------- DT rebuild
// Warp per doc of one chunk: the doc's topics are gathered through the doc-order ->
// word-sorted map into a warp-private shared histogram, each token's counts of its
// word's max / 2nd topic are scattered to its word-sorted slot, and the histogram is
// compacted to (k<<16 | count) ascending k.  Replaces DT_Update_Kernel
// (EZLDA/utility.cu:79-284).
struct DtArgs {
    uint32_t d_begin, d_end;
    int K;
    const uint32_t* doc_off;    // [D+1] doc-order token offsets
    const uint32_t* dtok_pos;   // [N]
    const uint32_t* dtok_word;  // [N]
    const uint16_t* z;
    const uint32_t* st_top2;
    const uint32_t* dt_off;
    uint32_t* dt_nnz;
    uint32_t* dt_ent;
    uint32_t* meta;             // [N] word-sorted: (n_d,2nd << 16) | n_d,max
    int* err;
    // dtok_pos / dtok_word / meta hold tokens [tok_base, ...) and dt_ent the doc-row
    // entries [dt_base, ...): 0 when the whole corpus is resident, the chunk's first token
    // and first doc-row entry when the chunk is streamed into a slot buffer
    uint32_t tok_base, dt_base;
    // above kLargeK topics: docs of at most small_max tokens are k_dt_build_small's, the
    // rest k_dt_build_cta's (0: all the CTA kernel's)
    uint32_t small_max = 0;
};

// Doc d: its counts in the warp's shared `hist` (K words) and the bitmap of its non-zero
// topics in `bits` (ceil(K/32) words), both zero on entry and on exit; the per-token
// metadata; and the row, compacted from the bitmap: each lane takes 32 topics' bits, an
// exclusive scan of their popcounts places its entries, ascending k.
__device__ __forceinline__ int dt_bit_words(int K) { return (K + 31) >> 5; }

template <class H>
__device__ __forceinline__ void dt_doc(const DtArgs& a, uint32_t d, const H& hist, uint32_t* bits, int lane) {
    const uint32_t b = __ldg(a.doc_off + d), n = __ldg(a.doc_off + d + 1) - b;
    const uint32_t* dpos = a.dtok_pos + (b - a.tok_base);
    const uint32_t* dword = a.dtok_word + (b - a.tok_base);
    // four 32-token steps per pass: their index loads, then their topic gathers, are in
    // flight together
    for (uint32_t base = 0; base < n; base += 128) {
        uint32_t k[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const uint32_t i = base + 32u * s + lane;
            k[s] = i < n ? __ldg(dpos + i) : 0xffffffffu;
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) k[s] = k[s] != 0xffffffffu ? (uint32_t)__ldg(a.z + k[s]) : 0xffffffffu;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            bool valid = k[s] != 0xffffffffu;
            uint32_t kk = k[s];
            if (valid && kk >= (uint32_t)a.K) {
                atomicOr(a.err, 1);
                valid = false;
                kk = 0xfffffffeu;
            }
            if (valid) hist_token(hist, bits, kk);
        }
    }
    __syncwarp();
    for (uint32_t base = 0; base < n; base += 128) {
        uint32_t pos[4], t2[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const uint32_t i = base + 32u * s + lane;
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
    __syncwarp();
    uint32_t* out = a.dt_ent + (__ldg(a.dt_off + d) - a.dt_base);
    const int words = dt_bit_words(a.K);
    uint32_t nnz = 0;
    for (int wb = 0; wb < words; wb += 32) {
        const int wi = wb + lane;
        uint32_t m = wi < words ? bits[wi] : 0u;
        const uint32_t c = (uint32_t)__popc(m);
        uint32_t incl = c;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t t = __shfl_up_sync(FULL, incl, off);
            if (lane >= off) incl += t;
        }
        uint32_t p = nnz + incl - c;
        nnz += __shfl_sync(FULL, incl, 31);
        if (m) bits[wi] = 0u;
        while (m) {
            const uint32_t k = (uint32_t)wi * 32u + (uint32_t)(__ffs(m) - 1);
            m &= m - 1u;
            const uint32_t key = a.K <= kLargeK ? (uint32_t)col_skew((int)k) : k;
            out[p++] = (key << 16) | hist.get(k);
            hist.clear(k);
        }
    }
    if (lane == 0) a.dt_nnz[d] = nnz;
    __syncwarp();
}

// ------------------------------------------------------------------- sampler
// Warp per (word, token range) tile.  The word's phi column (phi_max zeroed) sits in
// warp-private shared memory.  Each 32-token group is screened thread-per-token by the
// max-topic bound.  Tokens the bound does not settle (all tokens in LL mode) are then
// evaluated one at a time by the whole warp, with uniform control flow:
//   S      lane l sums the doc row's entries l, l+32, l+64, ... (coalesced loads); one
//          Kogge-Stone scan gives the lane prefixes; a doc row is evaluated once for
//          consecutive tokens of the same (word, doc) in the tile;
//   bucket a ballot over the lane prefixes picks the lane of an S-bucket draw; the
//          in-lane draw (at most ceil(nnz/32) entries) runs afterwards thread-per-token,
//          all the group's S-bucket tokens at once;
//   Q      a ballot over the per-word lane prefixes of Q, then one topic per lane with a
//          scan and a ballot (topics k = l, l+32, ..., 32 per round, carried).
// Replaces UpdateProbKernelTrainD1, LDAKernelTrainD and LDAKernelTrain
// (EZLDA/utility.cu:2680-3312, :1625-2103, :1217-1611) in one pass, with no
// effective-token list in global memory and no spin lock.
struct SampleArgs {
    const int4* tiles;  // {word, start, count, dense}
    int ntiles;
    unsigned* tile_counter;
    double* tile_ll;
    int K, Vd, ll_mode;
    float alpha, beta, Vbeta;
    double den_add;  // (double)K * (double)alpha
    uint32_t seed_lo, seed_hi, iter;
    const int* n_k;
    const int* dwt;
    const uint32_t* swt_off;
    const uint32_t* swt_nnz;
    const uint32_t* swt_ent;
    const uint32_t* st_top2;
    const float4* st_phi;
    const float* st_ql;
    const uint32_t* tok_doc;
    const uint32_t* meta;
    uint16_t* z;
    const uint32_t* doc_len;
    const uint32_t* dt_off;
    const uint32_t* dt_nnz;
    const uint32_t* dt_ent;
    // tokens, ea, full, sum_nnz, max, s, q, word_nnz, dense tiles, sparse tiles, rows, row entries
    unsigned long long* ctr;
    // tok_doc / meta hold tokens [tok_base, ...) and dt_ent the doc-row entries
    // [dt_base, ...) (non-zero when the chunk is streamed into a slot buffer)
    uint32_t tok_base, dt_base;
    // r_k = 1 / ((float)n_k + V*beta) for k < K, formed once per sweep (the K > kLargeK
    // dense-word sampler reads it instead of dividing for every tile's column)
    const float* recip = nullptr;
    // K > kLargeK: the smoothing table of the split Q bucket (k_smooth_table)
    const float* smooth = nullptr;
    // K > kLargeK: the dense words' Q-round tables (word_qtab), or null
    const float2* qtab_g = nullptr;
};

// The split Q bucket of a sparse word above kLargeK topics: Q = Qw + Qs, Qw over the word's
// own topics, Qs the word-independent smoothing part alpha * beta * sum_{k != max} r_k.
struct SplitQ {
    const uint32_t* ent;  // the word's row (k << 16 | count), ascending k
    uint32_t nnz;
    float Qw;
    const float* T;       // the smoothing table (K entries, non-decreasing)
    const float* r;       // r_k, at col_skew(k) when skew
    bool skew;
    // the Qw rounds' table, lane r holding round r's (carry before it, carry + its largest
    // KS prefix); rounds = 0 when not built (more than 32 rounds, or not wanted)
    int rounds = 0;
    float qcarry = 0.0f, qthr = 0.0f;
    __device__ __forceinline__ float rk(int k) const { return r[skew ? col_skew(k) : k]; }
    // round slot i of the Qw search: alpha * (n_wk * r_k), the max topic's term 0
    __device__ __forceinline__ void slot(uint32_t i, int maxK, float alpha, int& key, float& term, bool& ok) const {
        const uint32_t en = __ldg(ent + i);
        const int k = (int)(en >> 16);
        term = k == maxK ? 0.0f : fmul(alpha, fmul(u2f(en & 0xffffu), rk(k)));
        key = k;
        ok = term > 0.0f;
    }
};

// Builds the Qw rounds' table of a split word (2 to 32 rounds of 32 entries): each
// round's total and largest lane prefix from its Kogge-Stone scan, and the carries as the
// fadd chain of the totals, the values warp_level2 forms round by round.  Warp-uniform.
__device__ __forceinline__ void split_q_table(SplitQ& q, int maxK, float alpha, int lane) {
    const uint32_t R = (q.nnz + 31u) >> 5;
    if (R < 2 || R > 32) return;  // one round: the walk is that round already
    float carry = 0.0f;
    for (uint32_t r = 0; r < R; ++r) {
        int key = -1;
        float term = 0.0f;
        bool ok = false;
        const uint32_t i = 32u * r + (uint32_t)lane;
        if (i < q.nnz) q.slot(i, maxK, alpha, key, term, ok);
        const float ks = warp_ks_scan(term, lane);
        float mx = ks;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, off));
        const float tot = __shfl_sync(FULL, ks, 31);
        if ((uint32_t)lane == r) {
            q.qcarry = carry;
            q.qthr = fadd(carry, mx);
        }
        carry = fadd(carry, tot);
    }
    q.rounds = (int)R;
}

// The Q-bucket draw of a split word for t = target - pS (uniform across the warp): the
// word's own topics first, in rounds of 32 entries (carry + Kogge-Stone scan of
// alpha * (n_wk * r_k), the max topic's term 0; the first entry with a non-zero term whose
// prefix exceeds t, else the last such entry); otherwise smoothing for t' = t - Qw against
// T with the max topic left out: the first k < maxK with t' < T[k] when t' < T[maxK-1],
// else the first k > maxK with t' + sm_max < T[k], else the last topic other than maxK.
__device__ __forceinline__ int split_q_draw(const SplitQ& q, float t, int maxK, int K, float alpha, float beta,
                                            int lane) {
    if (t < q.Qw) {
        auto slot = [&](uint32_t i, int& key, float& term, bool& ok) { q.slot(i, maxK, alpha, key, term, ok); };
        int z = -1;
        if (q.rounds > 0) {
            // the candidate rounds (t below the round's largest prefix), in order
            for (unsigned b = __ballot_sync(FULL, lane < q.rounds && t < q.qthr); b; b &= b - 1u) {
                const uint32_t r = (uint32_t)(__ffs(b) - 1);
                const float carry = __shfl_sync(FULL, q.qcarry, (int)r);
                int key = -1;
                float term = 0.0f;
                bool ok = false;
                const uint32_t i = 32u * r + (uint32_t)lane;
                if (i < q.nnz) slot(i, key, term, ok);
                const float ks = warp_ks_scan(term, lane);
                const unsigned f = __ballot_sync(FULL, ok && t < fadd(carry, ks));
                if (f) {
                    z = __shfl_sync(FULL, key, __ffs(f) - 1);
                    break;
                }
            }
        }
        if (z < 0) z = warp_level2(q.nnz, t, -1, lane, slot);
        if (z >= 0) return z;
    }
    const float t1 = fsub(t, q.Qw);
    if (maxK > 0 && t1 < __ldg(q.T + maxK - 1)) return warp_first_above(q.T, 0, maxK, t1, lane);
    const float t2 = fadd(t1, fmul(alpha, fmul(beta, q.rk(maxK))));
    const int z = warp_first_above(q.T, maxK + 1, K, t2, lane);
    return z >= 0 ? z : (maxK == K - 1 ? K - 2 : K - 1);
}


// Sweep counters live in shared memory (one row per warp, written by lane 0) so they
// cost no registers in the sampling loop.
enum { C_TOK, C_EA, C_FULL, C_NNZ, C_MAX, C_S, C_Q, C_WNNZ, C_TDENSE, C_TSPARSE, C_ROWS, C_RENT, C_NUM };

// Warps per CTA of the K <= 2048 sampler (one shared word column per warp), and the CTAs
// per SM it is compiled for: the register cap is 65536 / (32 * warps * blocks) per
// thread.  The LL-mode kernel (its FP64 term) and the K > 1024 kernel (four Q rounds per
// batch) keep more state live and are compiled for fewer.
// Branch taken by a token (counters only).
enum { BR_NONE = 0, BR_MAX = 1, BR_S = 2, BR_Q = 3 };

#ifndef LDA_SAMPLE_WARPS
#define LDA_SAMPLE_WARPS 8
#endif
constexpr int kSampleWarps = LDA_SAMPLE_WARPS;
#ifndef LDA_SAMPLE_MIN_BLOCKS
#define LDA_SAMPLE_MIN_BLOCKS 5
#endif
#ifndef LDA_SAMPLE_QB_MIN_BLOCKS
#define LDA_SAMPLE_QB_MIN_BLOCKS 4
#endif
#ifndef LDA_SAMPLE_LL_MIN_BLOCKS
#define LDA_SAMPLE_LL_MIN_BLOCKS 5
#endif
#ifndef LDA_SPARSE_LARGE_MIN_BLOCKS
#define LDA_SPARSE_LARGE_MIN_BLOCKS 4
#endif

// The 32-token groups g0, g0 + gstep, ... of the token range [start, start + cnt) of one
// word (column view colz, max topic maxK, phi4 ph, Q partials QL / QP / Q of the word), or,
// with a shared group counter gq, the groups the warp claims from it (32 tokens at a time,
// so that the warps sharing a tile finish it together).  Returns the lane's LL partial (LL
// mode).
template <bool LL, int QB, bool SPLIT = false, int ROWM = 0, class View>
__device__ __forceinline__ double sample_groups(const SampleArgs& a, uint32_t start, uint32_t cnt, uint32_t g0,
                                                uint32_t gstep, uint32_t iter, int maxK, const float4 ph, float QL,
                                                float QP, float Q, const View& colz, uint32_t* ctr, int lane,
                                                const float2* qtab = nullptr, int qrounds = 0,
                                                const SplitQ* sq = nullptr, uint32_t* gq = nullptr) {
    auto claim = [&]() {
        uint32_t v = 0;
        if (lane == 0) v = atomicAdd(gq, 32u);
        return __shfl_sync(FULL, v, 0);
    };
    double ll = 0.0;
    // LL mode: the lane's factors total_t and (n_d + K alpha) as FP64 products, one log of
    // their ratio per 16 tokens (earlier if a product leaves [1e-150, 1e150])
    double ll_num = 1.0, ll_den = 1.0;
    int ll_n = 0;
    using E = typename View::Entry;
    const E* rows = reinterpret_cast<const E*>(a.dt_ent);
    uint32_t cur = 0xffffffffu, nnz = 0;
    const E* row = rows;
    float SL = 0.0f, SP = 0.0f, S = 0.0f;
    unsigned spos = 0u;  // lanes of the current row with a positive sum
    for (uint32_t g = gq ? claim() : g0; g < cnt; g = gq ? claim() : g + gstep) {
        const bool valid = g + lane < cnt;
        const uint32_t tok = start + g + lane;
        uint32_t d = 0xffffffffu, nd = 0, my_nnz = 0, my_off = 0;
        float u = 0.0f, pmax = 0.0f;
        bool ea = false;
        if (valid) {
            d = __ldg(a.tok_doc + (tok - a.tok_base));
            const uint32_t m = __ldg(a.meta + (tok - a.tok_base));
            nd = __ldg(a.doc_len + d);
            my_nnz = __ldg(a.dt_nnz + d);
            my_off = __ldg(a.dt_off + d) - a.dt_base;
            const uint32_t cmax = m & 0xffffu, c2 = m >> 16;
            u = token_uniform(a.seed_lo, a.seed_hi, iter, tok);
            pmax = fmul(fadd(u2f(cmax), a.alpha), ph.x);
            const float shat = ffma(u2f(c2), ph.y, fmul(u2f(nd - cmax - c2), ph.z));
            const float bound = fadd(fadd(pmax, shat), Q);
            ea = fmul(u, bound) < pmax;
        }
        int znew = maxK;
        // per-lane record of this token's evaluation, for the deferred draw and counters
        uint32_t my_ls = 0;
        float my_t2 = 0.0f, my_total = 0.0f;
        int kind = BR_NONE;
        bool evaluated = false;
        const unsigned vmask = __ballot_sync(FULL, valid);
        const unsigned emask = __ballot_sync(FULL, ea);
        const unsigned need0 = LL ? vmask : (vmask & ~emask);
        unsigned need = need0;
        while (need) {
            const int j = __ffs(need) - 1;
            need &= need - 1u;
            const uint32_t dj = __shfl_sync(FULL, d, j);
            if (dj != cur) {
                cur = dj;
                nnz = __shfl_sync(FULL, my_nnz, j);
                row = rows + __shfl_sync(FULL, my_off, j);
                SL = lane_mass<ROWM>(row, (uint32_t)lane, nnz, colz);
                SP = warp_ks_scan(SL, lane);
                S = __shfl_sync(FULL, SP, 31);
                spos = __ballot_sync(FULL, SL > 0.0f);
                evaluated |= (lane == j);
            }
            const float pmj = __shfl_sync(FULL, pmax, j);
            const float uj = __shfl_sync(FULL, u, j);
            const float pS = fadd(pmj, S);
            const float total = fadd(pS, Q);
            if (LL && lane == j) my_total = total;
            if (LL && ((emask >> j) & 1u)) continue;
            const float target = fmul(uj, total);
            if (target < pmj) {
                if (lane == j) kind = BR_MAX;
            } else if (target < pS) {
                const float tt = fsub(target, pmj);
                const unsigned cand = __ballot_sync(FULL, tt < SP && SL > 0.0f);
                const int ls = cand ? __ffs(cand) - 1 : 31 - __clz(spos);
                const float prev = __shfl_sync(FULL, SP, ls > 0 ? ls - 1 : 0);
                if (lane == j) {
                    kind = BR_S;
                    my_ls = (uint32_t)ls;
                    my_t2 = ls > 0 ? fsub(tt, prev) : tt;
                }
            } else {
                const float tt = fsub(target, pS);
                int zq;
                if (SPLIT) {
                    zq = split_q_draw(*sq, tt, maxK, a.K, a.alpha, a.beta, lane);
                } else {
                    const unsigned cand = __ballot_sync(FULL, tt < QP && QL > 0.0f);
                    const unsigned pos = __ballot_sync(FULL, QL > 0.0f);
                    const int ls = cand ? __ffs(cand) - 1 : (pos ? 31 - __clz(pos) : 0);
                    const float prev = __shfl_sync(FULL, QP, ls > 0 ? ls - 1 : 0);
                    const float t2 = ls > 0 ? fsub(tt, prev) : tt;
                    const int K = a.K;
                    const float alpha = a.alpha;
                    const uint32_t n = (uint32_t)((K - ls + 31) / 32);
                    auto slot = [&](uint32_t i, int& key, float& term, bool& ok) {
                        const int k = ls + 32 * (int)i;
                        const float cz = colz(k);
                        key = k;
                        term = fmul(alpha, cz);
                        ok = cz > 0.0f;
                    };
                    zq = qtab ? warp_level2_table(n, t2, lane, slot, qtab + ls * qrounds) : -1;
                    if (zq < 0) zq = warp_level2_rounds<QB>(n, t2, maxK, lane, slot);
                }
                if (lane == j) {
                    kind = BR_Q;
                    znew = zq;
                }
            }
        }
        // each lane's own token's log-likelihood factors, all lanes at once (every lane
        // accumulates only its own tokens, in group order)
        if (LL && valid) {
            ll_num *= (double)my_total;
            ll_den *= (double)nd + a.den_add;
            if (++ll_n == 16 || ll_num < 1e-150 || ll_num > 1e150 || ll_den > 1e150) {
                ll += log(ll_num / ll_den);
                ll_num = ll_den = 1.0;
                ll_n = 0;
            }
        }
        // an S-bucket token's row is its own doc's: the lane holds its offset and length
        if (kind == BR_S) znew = lane_draw(rows + my_off, my_ls, my_nnz, colz, my_t2, maxK);
        if (valid) a.z[tok] = (uint16_t)znew;
        // counters of the group: ballots and warp sums instead of per-token updates
        const bool in_need = (need0 >> lane) & 1u;
        const unsigned sm = __ballot_sync(FULL, kind == BR_S), qm = __ballot_sync(FULL, kind == BR_Q);
        const unsigned xm = __ballot_sync(FULL, kind == BR_MAX), rm = __ballot_sync(FULL, evaluated);
        const uint32_t nnz_full = __reduce_add_sync(FULL, in_need ? my_nnz : 0u);
        const uint32_t nnz_rows = __reduce_add_sync(FULL, evaluated ? my_nnz : 0u);
        if (lane == 0) {
            ctr[C_TOK] += __popc(vmask);
            ctr[C_EA] += __popc(emask);
            ctr[C_FULL] += __popc(need0);
            ctr[C_NNZ] += nnz_full;
            ctr[C_MAX] += __popc(xm) + __popc(emask);
            ctr[C_S] += __popc(sm);
            ctr[C_Q] += __popc(qm);
            ctr[C_ROWS] += __popc(rm);
            ctr[C_RENT] += nnz_rows;
        }
    }
    if (LL && ll_n) ll += log(ll_num / ll_den);
    return ll;
}

// One sampler tile (tile index `tile` of a.tiles, content t) with the word column in the
// warp's shared `col` (col_words(K) floats, skewed layout), the reciprocal table `r` and
// the warp's shared counter row `ctr`.  QB: Q-bucket rounds decided per batch (1 for
// K <= 1024, where a lane has one round of topics).
template <bool LL, int QB = 1, bool SKEWKEYS = true>
__device__ __forceinline__ void sample_tile(const SampleArgs& a, int tile, const int4 t, uint32_t iter,
                                            const float* r, float* col, uint32_t* ctr, int lane) {
    using View = ColSharedT<SKEWKEYS>;
    const int w = t.x;
    const uint32_t start = (uint32_t)t.y, cnt = (uint32_t)t.z;
    __syncwarp();
    uint32_t wnnz = 0;
    build_column<true>(col, r, w, a.Vd, a.K, a.beta, a.dwt, a.swt_off, a.swt_nnz, a.swt_ent, lane, &wnnz);
    if (lane == 0) {
        ctr[C_WNNZ] += wnnz;
        ctr[w < a.Vd ? C_TDENSE : C_TSPARSE] += 1u;
    }
    const int maxK = (int)(__ldg(a.st_top2 + w) & 0xffffu);
    const float4 ph = __ldg(a.st_phi + w);
    const float QL = __ldg(a.st_ql + (size_t)w * 32 + lane);
    const float QP = warp_ks_scan(QL, lane);
    const float Q = __shfl_sync(FULL, QP, 31);
    if (lane == 0) col[col_skew(maxK)] = 0.0f;
    __syncwarp();
    double ll;
    if constexpr (QB > 1) {
        if (a.K > kLargeK && w >= a.Vd) {
            // a sparse word above kLargeK topics: the split Q bucket
            const int s = w - a.Vd;
            const SplitQ sq{a.swt_ent + __ldg(a.swt_off + s), __ldg(a.swt_nnz + s), __shfl_sync(FULL, QL, 0),
                            a.smooth, r, false};
            ll = sample_groups<LL, QB, true>(a, start, cnt, 0u, 32u, iter, maxK, ph, QL, QP, Q, View{col}, ctr,
                                             lane, nullptr, 0, &sq);
        } else {
            ll = sample_groups<LL, QB>(a, start, cnt, 0u, 32u, iter, maxK, ph, QL, QP, Q, View{col}, ctr, lane);
        }
    } else {
        ll = sample_groups<LL, QB>(a, start, cnt, 0u, 32u, iter, maxK, ph, QL, QP, Q, View{col}, ctr, lane);
    }
    if (LL) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) ll += __shfl_xor_sync(FULL, ll, off);
        if (lane == 0) a.tile_ll[tile] = ll;
    }
}

}  // namespace dev
}  // namespace lda
