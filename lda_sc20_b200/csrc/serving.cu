// serving.cu -- fold-in of new documents against a frozen model, with continuous batching.
//
// EZLDA has no inference path.  Fold-in is its sweep with the word-topic side frozen: the
// conditional of a token of word w in a new document d is p(k) ∝ (n_dk+alpha)*phi_wk, with
// phi_wk = (n_wk+beta)/(n_k+V*beta) from the trained counts and n_dk the document's own
// counts at the start of each sweep.  The draw uses the same decomposition and arithmetic
// as the training sampler (max topic / S over the document's row / Q bucket, early accept).
//
// Device layout of a server: a token pool (word + topic per token, each request a
// contiguous range), a theta pool (K floats per request slot) and a request table rebuilt
// every step.  A step runs one sweep for every active request (each at its own sweep
// index); requests that arrive while others run are admitted at the next step when the
// token pool and the slots have room.  Each request's randoms are keyed on (seed, request
// id, sweep, position), so its result does not depend on what it was batched with.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <vector>

#include "common.h"
#include "device_common.cuh"
#include "launch_util.h"

using namespace lda;

namespace lda {
namespace dev {

// Dense phi of every word, phi_wk = ((float)n_wk + beta) * r_k, r_k = 1/((float)n_k + V*beta)
// (the same column the sweep builds per tile).
struct PhiArgs {
    int V, Vd, K;
    float beta, Vbeta;
    const int* n_k;
    const int* dwt;
    const uint32_t* swt_off;
    const uint32_t* swt_nnz;
    const uint32_t* swt_ent;
    float* phi;
};

__global__ void __launch_bounds__(256) k_phi_dense(PhiArgs a) {
    extern __shared__ float smf[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* r = smf;
    fill_recip(r, a.n_k, a.K, a.Vbeta);
    __syncthreads();
    for (int w = blockIdx.x * warps + wid; w < a.V; w += gridDim.x * warps) {
        float* out = a.phi + (size_t)w * a.K;
        if (w < a.Vd) {
            const int* row = a.dwt + (size_t)w * a.K;
            for (int k = lane; k < a.K; k += 32) out[k] = fmul(fadd(__int2float_rn(__ldg(row + k)), a.beta), r[k]);
        } else {
            for (int k = lane; k < a.K; k += 32) out[k] = fmul(a.beta, r[k]);
            __syncwarp();
            const int s = w - a.Vd;
            const uint32_t off = __ldg(a.swt_off + s), nnz = __ldg(a.swt_nnz + s);
            for (uint32_t e = lane; e < nnz; e += 32) {
                const uint32_t en = __ldg(a.swt_ent + off + e);
                out[en >> 16] = fmul(fadd(u2f(en & 0xffffu), a.beta), r[en >> 16]);
            }
        }
        __syncwarp();
    }
}

// Above kLargeK topics the trainer's statistics give a sparse word its split Q bucket
// ({Qw, Qs} in the lane-partial slots); the frozen model has no sparse word rows, so its
// sparse words get the lane partials back, formed from the dense phi rows as k_word_stats
// forms them from a column (serial fmaf of alpha * phi_k over k = l, l+32, ..., k != max),
// with Q their Kogge-Stone total.  Warp per word.
__global__ void __launch_bounds__(256) k_model_lane_q(int V, int Vd, int K, float alpha, const float* __restrict__ phi,
                                                      const uint32_t* __restrict__ top2, float* __restrict__ ql,
                                                      float4* __restrict__ phi4) {
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int w = Vd + blockIdx.x * warps + wid; w < V; w += gridDim.x * warps) {
        const int k1 = (int)(__ldg(top2 + w) & 0xffffu);
        const float* row = phi + (size_t)w * K;
        float acc = 0.0f;
        for (int k = lane; k < K; k += 32)
            if (k != k1) acc = ffma(alpha, __ldg(row + k), acc);
        const float Q = __shfl_sync(FULL, warp_ks_scan(acc, lane), 31);
        ql[(size_t)w * 32 + lane] = acc;
        if (lane == 0) phi4[w].w = Q;
    }
}

// One active request of a step: its tokens sit at [tok_off, tok_off+len) of the pool and
// it is split into items of `item_tokens` tokens, one warp each.  flags: FOLD_INIT (sweep
// 0: sweep-start counts from the Philox initial topics), FOLD_LAST (the last sweep:
// theta); bits 8.. hold the request's item count.
struct FoldReq {
    uint32_t tok_off, len, rid, sweep, flags, slot, pad0, pad1;
};
enum { FOLD_INIT = 1, FOLD_LAST = 2 };

struct FoldArgs {
    int K;
    float alpha, Kalpha;
    uint32_t seed_lo, seed_hi;
    const float* phi;
    const uint32_t* top2;
    const float4* phi4;
    const float* ql;
    const FoldReq* reqs;
    const uint32_t* item_req;  // per item: request index << 16 | item index within the request
    int nitems;
    uint32_t item_tokens;
    const uint32_t* words;
    uint16_t* z0;  // topics after even sweep counts
    uint16_t* z1;  // topics after odd sweep counts
    float* theta;
    unsigned* done;  // per slot: items of the last sweep that finished
};

__device__ __forceinline__ float foldin_uniform(uint32_t seed_lo, uint32_t seed_hi, uint32_t rid, uint32_t sweep,
                                                uint32_t pos) {
    const uint32_t x = philox_x0(pos, rid, sweep, 0x464F4C44u, seed_lo, seed_hi);
    return u2f(x >> 8) * 0x1p-24f;
}

__device__ __forceinline__ uint32_t foldin_init(uint32_t seed_lo, uint32_t seed_hi, uint32_t rid, uint32_t pos,
                                                int K) {
    const uint32_t x = philox_x0(pos, rid, 0xFFFFFFFFu, 0x46494E49u, seed_lo, seed_hi);
    return (uint32_t)(((unsigned long long)x * (unsigned long long)(uint32_t)K) >> 32);
}

// phi of topic k for word row `prow` with the word's max topic zeroed (the sweep's colz).
__device__ __forceinline__ float colz_of(const float* __restrict__ prow, int mk, uint32_t k) {
    return (int)k == mk ? 0.0f : __ldg(prow + k);
}

// Serial fmaf chain over the lane's entries l, l + 32, ... of the document row (in shared
// memory, so a step's 32 reads are conflict-free) with phi gathered from the frozen
// matrix.  The gathers of up to four entries are issued before their products are summed,
// also when the lane has fewer than four left (rows of short requests hold only a few
// entries per lane).
__device__ __forceinline__ float fold_lane_mass(const uint32_t* row, uint32_t lane, uint32_t nnz,
                                                const float* __restrict__ prow, int mk) {
    float acc = 0.0f;
    for (uint32_t q = lane; q < nnz; q += 128u) {
        uint32_t e[4];
        float c[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t i = q + 32u * j;
            e[j] = i < nnz ? row[i] : 0u;
            c[j] = i < nnz ? colz_of(prow, mk, e[j] >> 16) : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (q + 32u * j < nnz) acc = ffma(u2f(e[j] & 0xffffu), c[j], acc);
    }
    return acc;
}

// The S-bucket draw among lane ls's entries ls, ls + 32, ... (the partial sums of
// fold_lane_mass): the first entry with colz > 0 whose partial sum exceeds t2, else the
// last entry with colz > 0, else mk.
__device__ __forceinline__ int fold_lane_draw(const uint32_t* row, uint32_t ls, uint32_t nnz,
                                              const float* __restrict__ prow, int mk, float t2) {
    float acc = 0.0f;
    int last = -1;
    for (uint32_t q = ls; q < nnz; q += 128u) {
        uint32_t e[4];
        float c[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t i = q + 32u * j;
            e[j] = i < nnz ? row[i] : 0u;
            c[j] = i < nnz ? colz_of(prow, mk, e[j] >> 16) : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (q + 32u * j >= nnz) break;
            acc = ffma(u2f(e[j] & 0xffffu), c[j], acc);
            if (c[j] > 0.0f) {
                last = (int)(e[j] >> 16);
                if (t2 < acc) return last;
            }
        }
    }
    return last >= 0 ? last : mk;
}

// Doc-topic counts are at most 65535 (the request length limit), so two topics share a
// 32-bit shared word: topic k is the (k & 1) half of word k >> 1.
__device__ __forceinline__ uint32_t hist_get(const uint32_t* hist, uint32_t k) {
    return (hist[k >> 1] >> ((k & 1u) << 4)) & 0xffffu;
}

// Doc-topic histogram of one request into the warp's shared counts, from the Philox
// initial topics (init) or from a topic array.
__device__ __forceinline__ void fold_hist(uint32_t* hist, const FoldArgs& a, const FoldReq& q,
                                          const uint16_t* zsrc, bool init, int lane) {
    for (uint32_t base = 0; base < q.len; base += 32) {
        const uint32_t pos = base + lane;
        const bool valid = pos < q.len;
        uint32_t k = 0xffffffffu;
        if (valid) {
            k = init ? foldin_init(a.seed_lo, a.seed_hi, q.rid, pos, a.K) : (uint32_t)__ldcg(zsrc + q.tok_off + pos);
            if (k >= (uint32_t)a.K) k = 0;  // topics are written < K; keep the index in bounds
        }
        if (valid) atomicAdd(&hist[k >> 1], 1u << ((k & 1u) << 4));
    }
    __syncwarp();
}

// One sweep of every active request: warp per work item.  The warp rebuilds the request's
// sweep-start doc-topic histogram and its ascending-k row in warp-private shared memory,
// screens each 32-token group thread-per-token by the max-topic bound, evaluates the row
// mass of the tokens it does not settle with the whole warp (lane blocks of the row, phi
// gathered from the frozen matrix, reused while consecutive tokens share a word), and
// finishes S-bucket draws inside the chosen block thread-per-token.  Topics are read from
// one buffer and written to the other, so items of one request can run on any warps in
// any order.  On a request's last sweep the item that finishes last (a per-slot counter)
// writes theta = (n_dk + alpha) / (n_d + K*alpha) of the new topics.
__global__ void __launch_bounds__(256) k_foldin(FoldArgs a) {
    extern __shared__ uint32_t smu[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int hwords = (a.K + 1) >> 1;
    uint32_t* hist = smu + (size_t)(hwords + a.K) * wid;
    uint32_t* row = hist + hwords;
    for (int k = lane; k < hwords; k += 32) hist[k] = 0u;
    __syncwarp();
    for (int r = blockIdx.x * warps + wid; r < a.nitems; r += gridDim.x * warps) {
        const uint32_t ir = __ldg(a.item_req + r);
        const FoldReq it = a.reqs[ir >> 16];
        const uint32_t begin = (ir & 0xffffu) * a.item_tokens;
        const uint16_t* zin = (it.sweep & 1u) ? a.z1 : a.z0;
        uint16_t* zout = (it.sweep & 1u) ? a.z0 : a.z1;
        const uint32_t off = it.tok_off, len = it.len;
        fold_hist(hist, a, it, zin, (it.flags & FOLD_INIT) != 0, lane);
        uint32_t nnz = 0;
        for (int kb = 0; kb < a.K; kb += 32) {
            const int k = kb + lane;
            const uint32_t h = k < a.K ? hist_get(hist, (uint32_t)k) : 0u;
            const unsigned bal = __ballot_sync(FULL, h != 0u);
            if (h) row[nnz + __popc(bal & ((1u << lane) - 1u))] = ((uint32_t)k << 16) | h;
            nnz += (uint32_t)__popc(bal);
        }
        __syncwarp();
        uint32_t cur_w = 0xffffffffu;
        float SL = 0.0f, SP = 0.0f, S = 0.0f;
        const uint32_t end = min(begin + a.item_tokens, len);
        for (uint32_t g = begin; g < end; g += 32) {
            const uint32_t pos = g + lane;
            const bool valid = pos < end;
            uint32_t w = 0;
            int mk = 0;
            float pmax = 0.0f, u = 0.0f, Qw = 0.0f;
            bool ea = false;
            if (valid) {
                w = __ldg(a.words + off + pos);
                const uint32_t t2 = __ldg(a.top2 + w);
                mk = (int)(t2 & 0xffffu);
                const float4 ph = __ldg(a.phi4 + w);
                const uint32_t cmax = hist_get(hist, (uint32_t)mk), c2 = hist_get(hist, t2 >> 16);
                u = foldin_uniform(a.seed_lo, a.seed_hi, it.rid, it.sweep, pos);
                pmax = fmul(fadd(u2f(cmax), a.alpha), ph.x);
                const float shat = ffma(u2f(c2), ph.y, fmul(u2f(len - cmax - c2), ph.z));
                Qw = ph.w;
                ea = fmul(u, fadd(fadd(pmax, shat), Qw)) < pmax;
            }
            int znew = mk;
            bool defer = false;
            uint32_t my_ls = 0;
            float my_t2 = 0.0f;
            unsigned need = __ballot_sync(FULL, valid && !ea);
            while (need) {
                const int j = __ffs(need) - 1;
                need &= need - 1u;
                const uint32_t wj = __shfl_sync(FULL, w, j);
                const int mkj = __shfl_sync(FULL, mk, j);
                const float pmj = __shfl_sync(FULL, pmax, j);
                const float uj = __shfl_sync(FULL, u, j);
                const float Qj = __shfl_sync(FULL, Qw, j);
                const float* prow = a.phi + (size_t)wj * a.K;
                if (wj != cur_w) {
                    cur_w = wj;
                    SL = fold_lane_mass(row, (uint32_t)lane, nnz, prow, mkj);
                    SP = warp_ks_scan(SL, lane);
                    S = __shfl_sync(FULL, SP, 31);
                }
                const float pS = fadd(pmj, S);
                const float total = fadd(pS, Qj);
                const float target = fmul(uj, total);
                if (target < pmj) {
                    // the max topic (znew already holds it)
                } else if (target < pS) {
                    const float tt = fsub(target, pmj);
                    const unsigned cand = __ballot_sync(FULL, tt < SP && SL > 0.0f);
                    const unsigned pos_l = __ballot_sync(FULL, SL > 0.0f);
                    const int ls = cand ? __ffs(cand) - 1 : 31 - __clz(pos_l);
                    const float prev = __shfl_sync(FULL, SP, ls > 0 ? ls - 1 : 0);
                    if (lane == j) {
                        defer = true;
                        my_ls = (uint32_t)ls;
                        my_t2 = ls > 0 ? fsub(tt, prev) : tt;
                    }
                } else {
                    const float tt = fsub(target, pS);
                    const float QL = __ldg(a.ql + (size_t)wj * 32 + lane);
                    const float QP = warp_ks_scan(QL, lane);
                    const unsigned cand = __ballot_sync(FULL, tt < QP && QL > 0.0f);
                    const unsigned pos_l = __ballot_sync(FULL, QL > 0.0f);
                    const int ls = cand ? __ffs(cand) - 1 : (pos_l ? 31 - __clz(pos_l) : 0);
                    const float prev = __shfl_sync(FULL, QP, ls > 0 ? ls - 1 : 0);
                    const float t2 = ls > 0 ? fsub(tt, prev) : tt;
                    const int K = a.K;
                    const float alpha = a.alpha;
                    const uint32_t n = (uint32_t)((K - ls + 31) / 32);
                    const int zq = warp_level2(n, t2, mkj, lane, [&](uint32_t i, int& key, float& term, bool& ok) {
                        const int k = ls + 32 * (int)i;
                        const float cz = colz_of(prow, mkj, (uint32_t)k);
                        key = k;
                        term = fmul(alpha, cz);
                        ok = cz > 0.0f;
                    });
                    if (lane == j) znew = zq;
                }
            }
            if (defer) znew = fold_lane_draw(row, my_ls, nnz, a.phi + (size_t)w * a.K, mk, my_t2);
            if (valid) zout[off + pos] = (uint16_t)znew;
        }
        __syncwarp();
        for (int k = lane; k < hwords; k += 32) hist[k] = 0u;
        __syncwarp();
        if (it.flags & FOLD_LAST) {
            // publish this item's topics, then count it; the last item of the request
            // (whatever warp runs it) sees every other item's topics
            __threadfence();
            __syncwarp();
            unsigned prior = 0;
            if (lane == 0) prior = atomicAdd(a.done + it.slot, 1u);
            prior = __shfl_sync(FULL, prior, 0);
            const unsigned nitems = it.flags >> 8;
            if (prior + 1u == nitems) {
                __threadfence();
                fold_hist(hist, a, it, zout, false, lane);
                float* th = a.theta + (size_t)it.slot * a.K;
                const float den = fadd(u2f(len), a.Kalpha);
                for (int k = lane; k < a.K; k += 32) th[k] = __fdiv_rn(fadd(u2f(hist_get(hist, (uint32_t)k)), a.alpha), den);
                __syncwarp();
                for (int k = lane; k < hwords; k += 32) hist[k] = 0u;
                if (lane == 0) a.done[it.slot] = 0u;
                __syncwarp();
            }
        }
    }
}

}  // namespace dev
}  // namespace lda

#define CUDA_TRY(expr)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (expr);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            cudaGetLastError();                                                                \
            return fail(LDA_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_));         \
        }                                                                                      \
    } while (0)

// ------------------------------------------------------------------ model

struct lda_model {
    int device = 0;
    int K = 0;
    int64_t V = 0;
    float alpha = 0, beta = 0;
    float* phi = nullptr;
    uint32_t* top2 = nullptr;
    float4* phi4 = nullptr;
    float* ql = nullptr;
    int64_t bytes = 0;
    ~lda_model() {
        cudaSetDevice(device);
        cudaFree(phi);
        cudaFree(top2);
        cudaFree(phi4);
        cudaFree(ql);
    }
};

extern "C" int lda_model_from_trainer(lda_trainer* t, int64_t device_budget, lda_model** out) {
    if (!t || !out) return fail(LDA_ERR_ARG, "null argument");
    *out = nullptr;
    int rc;
    // counts and word statistics of the trainer's current topics
    if ((rc = lda_update_wt(t)) || (rc = lda_max_topic(t)) || (rc = lda_trainer_sync(t))) return rc;
    std::unique_ptr<lda_model> m(new lda_model());
    ModelSource src;
    if ((rc = trainer_model_source(t, &src))) return rc;
    m->device = src.device;
    m->K = src.K;
    m->V = src.V;
    m->alpha = src.alpha;
    m->beta = src.beta;
    cudaStream_t stream = (cudaStream_t)src.stream;
    const int64_t need = m->V * m->K * 4 + m->V * (4 + 16 + 128);
    if (device_budget > 0 && need > device_budget)
        return fail(LDA_ERR_DEVICE_MEM, "model needs %lld bytes, budget is %lld", (long long)need, (long long)device_budget);
    CUDA_TRY(cudaSetDevice(m->device));
    cudaError_t e = cudaMalloc(&m->phi, sizeof(float) * (size_t)m->V * m->K);
    if (e == cudaSuccess) e = cudaMalloc(&m->top2, sizeof(uint32_t) * (size_t)m->V);
    if (e == cudaSuccess) e = cudaMalloc(&m->phi4, sizeof(float4) * (size_t)m->V);
    if (e == cudaSuccess) e = cudaMalloc(&m->ql, sizeof(float) * 32 * (size_t)m->V);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(LDA_ERR_DEVICE_MEM, "cudaMalloc of the model failed: %s", cudaGetErrorString(e));
    }
    m->bytes = need;
    dev::PhiArgs a;
    a.V = (int)m->V;
    a.Vd = src.Vd;
    a.K = m->K;
    a.beta = m->beta;
    a.Vbeta = (float)m->V * m->beta;
    a.n_k = src.n_k;
    a.dwt = src.dwt;
    a.swt_off = src.swt_off;
    a.swt_nnz = src.swt_nnz;
    a.swt_ent = src.swt_ent;
    a.phi = m->phi;
    const size_t smem = sizeof(float) * (size_t)m->K;
    CUDA_TRY(raise_smem_limit((const void*)dev::k_phi_dense, smem));
    const int grid = (int)std::min<int64_t>(4096, (m->V + 7) / 8);
    dev::k_phi_dense<<<grid, 256, smem, stream>>>(a);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(m->top2, src.top2, sizeof(uint32_t) * (size_t)m->V, cudaMemcpyDeviceToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(m->phi4, src.phi4, sizeof(float4) * (size_t)m->V, cudaMemcpyDeviceToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(m->ql, src.ql, sizeof(float) * 32 * (size_t)m->V, cudaMemcpyDeviceToDevice, stream));
    if (m->K > dev::kLargeK && m->V > src.Vd) {
        const int grid = (int)std::min<int64_t>(4096, (m->V - src.Vd + 7) / 8);
        dev::k_model_lane_q<<<grid, 256, 0, stream>>>((int)m->V, src.Vd, m->K, m->alpha, m->phi, m->top2, m->ql,
                                                      reinterpret_cast<float4*>(m->phi4));
        CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaStreamSynchronize(stream));
    *out = m.release();
    return LDA_OK;
}

extern "C" int lda_model_info(const lda_model* m, int32_t* K, int64_t* V, int64_t* bytes) {
    if (!m) return fail(LDA_ERR_ARG, "null model");
    if (K) *K = m->K;
    if (V) *V = m->V;
    if (bytes) *bytes = m->bytes;
    return LDA_OK;
}

extern "C" int lda_model_get_phi(const lda_model* m, int32_t w, float* out) {
    if (!m || !out || w < 0 || w >= m->V) return fail(LDA_ERR_ARG, "bad arguments");
    CUDA_TRY(cudaSetDevice(m->device));
    CUDA_TRY(cudaMemcpy(out, m->phi + (size_t)w * m->K, sizeof(float) * m->K, cudaMemcpyDeviceToHost));
    return LDA_OK;
}

extern "C" void lda_model_free(lda_model* m) { delete m; }

// ------------------------------------------------------------------ server

namespace {
using Clock = std::chrono::steady_clock;
double now_s() { return std::chrono::duration<double>(Clock::now().time_since_epoch()).count(); }
constexpr int kRing = 3;      // host item buffers / events
constexpr int kInFlight = 2;  // steps queued on the stream before the host waits
}  // namespace

struct lda_server {
    lda_model* m = nullptr;
    int device = 0;
    cudaStream_t st = nullptr;
    int sweeps = 30, max_active = 0, warps = 8, grid = 0;
    uint32_t item_tokens = 32;
    uint64_t seed = 0;
    int64_t tok_cap = 0, max_items = 0;
    size_t smem = 0;
    uint32_t* d_words = nullptr;
    uint16_t* d_z = nullptr;  // [2][tok_cap]
    float* d_theta = nullptr;
    unsigned* d_done = nullptr;
    dev::FoldReq* d_reqs = nullptr;
    uint32_t* d_items = nullptr;
    dev::FoldReq* h_reqs[kRing] = {};
    uint32_t* h_items[kRing] = {};
    cudaEvent_t ev[kRing] = {};
    uint32_t* h_words = nullptr;
    float* h_theta = nullptr;
    std::map<int64_t, int64_t> free_iv;  // token pool free intervals: offset -> length
    std::vector<int> free_slots;
    struct Pending {
        uint32_t rid;
        std::vector<uint32_t> words;
        double t_submit;
    };
    struct Active {
        uint32_t rid, len;
        int64_t off;
        int sweep, slot;  // sweeps issued so far
        double t_submit;
        int64_t last_step;
    };
    struct Done {
        uint32_t rid;
        std::vector<float> theta;
        double t_submit, t_done;
    };
    std::deque<Pending> queue;
    std::vector<Active> active;
    std::deque<Active> finishing;      // last sweep issued, waiting for its step's event
    std::deque<int64_t> inflight;      // issued steps not yet collected
    std::deque<Done> done;
    int64_t steps = 0, kernel_launches = 0;

    ~lda_server() {
        cudaSetDevice(device);
        if (st) cudaStreamSynchronize(st);
        cudaFree(d_words);
        cudaFree(d_z);
        cudaFree(d_theta);
        cudaFree(d_done);
        cudaFree(d_items);
        cudaFree(d_reqs);
        for (int i = 0; i < kRing; ++i) {
            cudaFreeHost(h_items[i]);
            cudaFreeHost(h_reqs[i]);
            if (ev[i]) cudaEventDestroy(ev[i]);
        }
        cudaFreeHost(h_words);
        cudaFreeHost(h_theta);
        if (st) cudaStreamDestroy(st);
    }

    bool alloc_tokens(int64_t len, int64_t* off) {
        for (auto it = free_iv.begin(); it != free_iv.end(); ++it) {
            if (it->second >= len) {
                *off = it->first;
                const int64_t rest = it->second - len, noff = it->first + len;
                free_iv.erase(it);
                if (rest > 0) free_iv[noff] = rest;
                return true;
            }
        }
        return false;
    }

    void free_tokens(int64_t off, int64_t len) {
        auto it = free_iv.emplace(off, len).first;
        auto nx = std::next(it);
        if (nx != free_iv.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_iv.erase(nx);
        }
        if (it != free_iv.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_iv.erase(it);
            }
        }
    }

    // Retires the requests whose last step is `step` (its event has completed).
    void retire_through(int64_t step, double t) {
        while (!finishing.empty() && finishing.front().last_step <= step) {
            const Active& a = finishing.front();
            Done d;
            d.rid = a.rid;
            d.theta.assign(h_theta + (size_t)a.slot * m->K, h_theta + (size_t)(a.slot + 1) * m->K);
            d.t_submit = a.t_submit;
            d.t_done = t;
            done.push_back(std::move(d));
            free_tokens(a.off, a.len);
            free_slots.push_back(a.slot);
            finishing.pop_front();
        }
    }

    // Collects completed steps: blocking on the oldest while more than `keep` are queued,
    // then every step whose event has already completed.  Returns requests retired.
    int collect(size_t keep, int* rc) {
        const size_t before = done.size();
        while (!inflight.empty()) {
            const int64_t k = inflight.front();
            cudaEvent_t e = ev[k % kRing];
            if (inflight.size() > keep) {
                const cudaError_t err = cudaEventSynchronize(e);
                if (err != cudaSuccess) {
                    cudaGetLastError();
                    *rc = fail(LDA_ERR_CUDA, "fold-in step failed: %s", cudaGetErrorString(err));
                    return 0;
                }
            } else {
                const cudaError_t q = cudaEventQuery(e);
                if (q == cudaErrorNotReady) break;
                if (q != cudaSuccess) {
                    cudaGetLastError();
                    *rc = fail(LDA_ERR_CUDA, "fold-in step failed: %s", cudaGetErrorString(q));
                    return 0;
                }
            }
            inflight.pop_front();
            retire_through(k, now_s());
        }
        return (int)(done.size() - before);
    }
};

extern "C" int lda_server_create(lda_model* m, int64_t max_tokens, int32_t max_active, int32_t sweeps, uint64_t seed,
                                 lda_server** out) {
    if (!m || !out) return fail(LDA_ERR_ARG, "null argument");
    *out = nullptr;
    if (sweeps < 1 || max_active < 1 || max_tokens < 0) return fail(LDA_ERR_ARG, "sweeps and max_active must be >= 1");
    if (max_tokens > ((int64_t)1 << 31)) return fail(LDA_ERR_ARG, "token pool above 2^31 tokens");
    if (max_active > 65535) return fail(LDA_ERR_ARG, "max_active above 65535");
    std::unique_ptr<lda_server> s(new lda_server());
    s->m = m;
    s->device = m->device;
    s->sweeps = sweeps;
    s->max_active = max_active;
    s->seed = seed;
    CUDA_TRY(cudaSetDevice(s->device));
    if (max_tokens == 0) {
        // admission by free HBM: a quarter of the free device memory holds the token pool
        // (4 B word + 2 x 2 B topics per token)
        size_t fr = 0, tot = 0;
        CUDA_TRY(cudaMemGetInfo(&fr, &tot));
        max_tokens = std::min<int64_t>((int64_t)(fr / 4) / 8, (int64_t)1 << 30);
    }
    s->tok_cap = max_tokens;
    s->max_items = (int64_t)max_active + max_tokens / s->item_tokens + 1;
    cudaError_t e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_words, sizeof(uint32_t) * (size_t)max_tokens);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_z, sizeof(uint16_t) * 2 * (size_t)max_tokens);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_theta, sizeof(float) * (size_t)max_active * m->K);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_done, sizeof(unsigned) * (size_t)max_active);
    if (e == cudaSuccess) e = cudaMemset(s->d_done, 0, sizeof(unsigned) * (size_t)max_active);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_items, sizeof(uint32_t) * (size_t)s->max_items);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_reqs, sizeof(dev::FoldReq) * (size_t)max_active);
    for (int i = 0; i < kRing && e == cudaSuccess; ++i) {
        e = cudaMallocHost(&s->h_items[i], sizeof(uint32_t) * (size_t)s->max_items);
        if (e == cudaSuccess) e = cudaMallocHost(&s->h_reqs[i], sizeof(dev::FoldReq) * (size_t)max_active);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_words, sizeof(uint32_t) * (size_t)max_tokens);
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_theta, sizeof(float) * (size_t)max_active * m->K);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(LDA_ERR_DEVICE_MEM, "server allocation failed: %s", cudaGetErrorString(e));
    }
    s->free_iv[0] = max_tokens;
    for (int i = max_active - 1; i >= 0; --i) s->free_slots.push_back(i);
    int max_smem = 0, num_sms = 0, per_sm = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device));
    CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, s->device));
    const int64_t per_warp = 4 * ((int64_t)(m->K + 1) / 2 + m->K);  // packed counts + row
    s->warps = (int)std::min<int64_t>(8, (int64_t)max_smem / per_warp);
    if (s->warps < 1) return fail(LDA_ERR_ARG, "K=%d does not fit in shared memory", m->K);
    s->smem = (size_t)(s->warps * per_warp);
    CUDA_TRY(raise_smem_limit((const void*)dev::k_foldin, s->smem));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)dev::k_foldin, 32 * s->warps, s->smem));
    s->grid = std::max(1, per_sm * num_sms);
    CUDA_TRY(cudaStreamSynchronize(s->st));
    *out = s.release();
    return LDA_OK;
}

extern "C" int lda_server_destroy(lda_server* s) {
    delete s;
    return LDA_OK;
}

extern "C" int lda_server_set_item_tokens(lda_server* s, int32_t n) {
    if (!s || n < 32 || n % 32) return fail(LDA_ERR_ARG, "item size must be a positive multiple of 32");
    if (!s->active.empty() || !s->inflight.empty()) return fail(LDA_ERR_STATE, "server is busy");
    const int64_t need = (int64_t)s->max_active + s->tok_cap / n + 1;
    if (need > s->max_items) {
        CUDA_TRY(cudaSetDevice(s->device));
        CUDA_TRY(cudaStreamSynchronize(s->st));
        cudaFree(s->d_items);
        s->d_items = nullptr;
        for (int i = 0; i < kRing; ++i) {
            cudaFreeHost(s->h_items[i]);
            s->h_items[i] = nullptr;
        }
        s->max_items = 0;
        cudaError_t e = cudaMalloc(&s->d_items, sizeof(uint32_t) * (size_t)need);
        for (int i = 0; i < kRing && e == cudaSuccess; ++i)
            e = cudaMallocHost(&s->h_items[i], sizeof(uint32_t) * (size_t)need);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(LDA_ERR_DEVICE_MEM, "item table allocation failed: %s", cudaGetErrorString(e));
        }
        s->max_items = need;
    }
    s->item_tokens = (uint32_t)n;
    return LDA_OK;
}

extern "C" int lda_server_submit(lda_server* s, uint32_t rid, const int32_t* words, int32_t len) {
    if (!s || !words) return fail(LDA_ERR_ARG, "null argument");
    if (len < 1 || len > 65535) return fail(LDA_ERR_ARG, "request length %d outside [1, 65535]", len);
    if (len > s->tok_cap)
        return fail(LDA_ERR_DEVICE_MEM, "request of %d tokens exceeds the token pool (%lld)", len, (long long)s->tok_cap);
    lda_server::Pending p;
    p.rid = rid;
    p.t_submit = now_s();
    p.words.resize(len);
    for (int32_t i = 0; i < len; ++i) {
        if (words[i] < 0 || words[i] >= s->m->V)
            return fail(LDA_ERR_ARG, "word %d of request %u outside the vocabulary", words[i], rid);
        p.words[i] = (uint32_t)words[i];
    }
    s->queue.push_back(std::move(p));
    return LDA_OK;
}

// Issues one step: admits queued requests that fit (FIFO, by token pool and slots), queues
// one sweep of every active request on the stream, and moves requests whose last sweep it
// is to the finishing list.  Completion is collected by lda_server::collect.
static int server_issue(lda_server* s) {
    CUDA_TRY(cudaSetDevice(s->device));
    int rc = LDA_OK;
    // the host buffers of step `steps` were last used by step `steps - kRing`
    s->collect(kInFlight - 1, &rc);
    if (rc) return rc;
    while (!s->queue.empty() && (int)s->active.size() < s->max_active && !s->free_slots.empty()) {
        auto& p = s->queue.front();
        int64_t off;
        if (!s->alloc_tokens((int64_t)p.words.size(), &off)) break;
        lda_server::Active a;
        a.rid = p.rid;
        a.len = (uint32_t)p.words.size();
        a.off = off;
        a.sweep = 0;
        a.slot = s->free_slots.back();
        s->free_slots.pop_back();
        a.t_submit = p.t_submit;
        a.last_step = -1;
        std::memcpy(s->h_words + off, p.words.data(), sizeof(uint32_t) * a.len);
        CUDA_TRY(cudaMemcpyAsync(s->d_words + off, s->h_words + off, sizeof(uint32_t) * a.len, cudaMemcpyHostToDevice,
                                 s->st));
        s->active.push_back(a);
        s->queue.pop_front();
    }
    if (s->active.empty()) return LDA_OK;
    if (s->max_items == 0) return fail(LDA_ERR_STATE, "the server has no item table (a failed resize)");
    const int64_t k = s->steps;
    uint32_t* items = s->h_items[k % kRing];
    dev::FoldReq* reqs = s->h_reqs[k % kRing];
    int64_t n = 0;
    const uint32_t T = s->item_tokens;
    const int nreq = (int)s->active.size();
    for (int r = 0; r < nreq; ++r) {
        const auto& a = s->active[r];
        const uint32_t nitems = (a.len + T - 1) / T;
        dev::FoldReq& q = reqs[r];
        q.tok_off = (uint32_t)a.off;
        q.len = a.len;
        q.rid = a.rid;
        q.sweep = (uint32_t)a.sweep;
        q.flags = (a.sweep == 0 ? (uint32_t)dev::FOLD_INIT : 0u) |
                  (a.sweep == s->sweeps - 1 ? (uint32_t)dev::FOLD_LAST : 0u) | (nitems << 8);
        q.slot = (uint32_t)a.slot;
        q.pad0 = q.pad1 = 0;
        const uint32_t tag = (uint32_t)r << 16;
        for (uint32_t j = 0; j < nitems; ++j) items[n++] = tag | j;
    }
    CUDA_TRY(cudaMemcpyAsync(s->d_reqs, reqs, sizeof(dev::FoldReq) * (size_t)nreq, cudaMemcpyHostToDevice, s->st));
    CUDA_TRY(cudaMemcpyAsync(s->d_items, items, sizeof(uint32_t) * (size_t)n, cudaMemcpyHostToDevice, s->st));
    dev::FoldArgs fa;
    fa.K = s->m->K;
    fa.alpha = s->m->alpha;
    fa.Kalpha = (float)s->m->K * s->m->alpha;
    fa.seed_lo = (uint32_t)s->seed;
    fa.seed_hi = (uint32_t)(s->seed >> 32);
    fa.phi = s->m->phi;
    fa.top2 = s->m->top2;
    fa.phi4 = s->m->phi4;
    fa.ql = s->m->ql;
    fa.reqs = s->d_reqs;
    fa.item_req = s->d_items;
    fa.nitems = (int)n;
    fa.item_tokens = T;
    fa.words = s->d_words;
    fa.z0 = s->d_z;
    fa.z1 = s->d_z + s->tok_cap;
    fa.theta = s->d_theta;
    fa.done = s->d_done;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(s->grid, (n + s->warps - 1) / s->warps));
    dev::k_foldin<<<grid, 32 * s->warps, s->smem, s->st>>>(fa);
    CUDA_TRY(cudaGetLastError());
    s->kernel_launches++;
    std::vector<lda_server::Active> keep;
    keep.reserve(s->active.size());
    for (auto& a : s->active) {
        if (a.sweep == s->sweeps - 1) {
            CUDA_TRY(cudaMemcpyAsync(s->h_theta + (size_t)a.slot * s->m->K, s->d_theta + (size_t)a.slot * s->m->K,
                                     sizeof(float) * s->m->K, cudaMemcpyDeviceToHost, s->st));
            a.last_step = k;
            a.sweep++;
            s->finishing.push_back(a);
        } else {
            a.sweep++;
            keep.push_back(a);
        }
    }
    s->active.swap(keep);
    CUDA_TRY(cudaEventRecord(s->ev[k % kRing], s->st));
    s->inflight.push_back(k);
    s->steps++;
    return LDA_OK;
}

extern "C" int lda_server_step(lda_server* s, int32_t* n_done) {
    if (!s) return fail(LDA_ERR_ARG, "null server");
    const size_t before = s->done.size();
    int rc;
    if (!s->queue.empty() || !s->active.empty()) {
        if ((rc = server_issue(s))) return rc;
        rc = LDA_OK;
        s->collect(kInFlight, &rc);
    } else {
        rc = LDA_OK;
        s->collect(0, &rc);  // nothing left to issue: wait for the queued steps
    }
    if (rc) return rc;
    if (n_done) *n_done = (int32_t)(s->done.size() - before);
    return LDA_OK;
}

extern "C" int lda_server_poll(lda_server* s, uint32_t* rid, float* theta, double* latency_s) {
    if (!s || !rid) return fail(LDA_ERR_ARG, "null argument");
    if (s->done.empty()) return 0;
    auto& d = s->done.front();
    *rid = d.rid;
    if (theta) std::memcpy(theta, d.theta.data(), sizeof(float) * d.theta.size());
    if (latency_s) *latency_s = d.t_done - d.t_submit;
    s->done.pop_front();
    return 1;
}

extern "C" int lda_server_status(const lda_server* s, int32_t* queued, int32_t* active, int64_t* free_tokens) {
    if (!s) return fail(LDA_ERR_ARG, "null server");
    if (queued) *queued = (int32_t)s->queue.size();
    if (active) *active = (int32_t)(s->active.size() + s->finishing.size());
    if (free_tokens) {
        int64_t f = 0;
        for (auto& kv : s->free_iv) f += kv.second;
        *free_tokens = f;
    }
    return LDA_OK;
}

extern "C" int lda_server_get_topics(lda_server* s, uint32_t rid, uint16_t* out, int32_t len) {
    if (!s || !out) return fail(LDA_ERR_ARG, "null argument");
    for (auto& a : s->active)
        if (a.rid == rid) {
            if ((int32_t)a.len != len) return fail(LDA_ERR_ARG, "request %u has %u tokens", rid, a.len);
            if (a.sweep == 0) return fail(LDA_ERR_STATE, "request %u has not run a sweep yet", rid);
            CUDA_TRY(cudaSetDevice(s->device));
            CUDA_TRY(cudaStreamSynchronize(s->st));
            const uint16_t* z = s->d_z + (size_t)(a.sweep & 1) * s->tok_cap;
            CUDA_TRY(cudaMemcpy(out, z + a.off, sizeof(uint16_t) * a.len, cudaMemcpyDeviceToHost));
            return LDA_OK;
        }
    return fail(LDA_ERR_STATE, "request %u is not active", rid);
}

extern "C" int lda_server_stats(const lda_server* s, int64_t* steps, int64_t* kernel_launches) {
    if (!s) return fail(LDA_ERR_ARG, "null server");
    if (steps) *steps = s->steps;
    if (kernel_launches) *kernel_launches = s->kernel_launches;
    return LDA_OK;
}

// Real-time replay of an arrival schedule on an idle server.
extern "C" int lda_serve_replay(lda_server* s, int32_t n, const int64_t* doc_off, const int32_t* words,
                                const double* arrival_s, double* latency_s, float* theta, double* wall_s) {
    if (!s || !doc_off || !words || !arrival_s || !latency_s || n < 0) return fail(LDA_ERR_ARG, "null argument");
    for (int32_t i = 1; i < n; ++i)
        if (arrival_s[i] < arrival_s[i - 1]) return fail(LDA_ERR_ARG, "arrival times must be non-decreasing");
    if (!s->queue.empty() || !s->active.empty() || !s->finishing.empty() || !s->done.empty())
        return fail(LDA_ERR_STATE, "replay needs an idle server (nothing queued, active or unpolled)");
    const double t0 = now_s();
    int32_t next = 0, finished = 0;
    int rc;
    while (finished < n) {
        const double now = now_s() - t0;
        while (next < n && arrival_s[next] <= now) {
            if ((rc = lda_server_submit(s, (uint32_t)next, words + doc_off[next],
                                        (int32_t)(doc_off[next + 1] - doc_off[next]))))
                return rc;
            s->queue.back().t_submit = t0 + arrival_s[next];  // latency counts from the scheduled arrival
            ++next;
        }
        if (s->queue.empty() && s->active.empty()) {
            rc = LDA_OK;
            if (!s->inflight.empty()) {
                s->collect(s->inflight.size() - 1, &rc);  // wait for the oldest queued step
                if (rc) return rc;
            } else if (next < n) {
                const double wait = arrival_s[next] - (now_s() - t0);
                if (wait > 2e-4) std::this_thread::sleep_for(std::chrono::duration<double>(wait - 1e-4));
            }
        } else {
            if ((rc = server_issue(s))) return rc;
            rc = LDA_OK;
            s->collect(kInFlight, &rc);
            if (rc) return rc;
        }
        while (!s->done.empty()) {
            auto& d = s->done.front();
            if (d.rid < (uint32_t)n) {
                if (theta) std::memcpy(theta + (size_t)d.rid * s->m->K, d.theta.data(), sizeof(float) * s->m->K);
                latency_s[d.rid] = d.t_done - d.t_submit;
                ++finished;
            }
            s->done.pop_front();
        }
    }
    if (wall_s) *wall_s = now_s() - t0;
    return LDA_OK;
}
