// trainer.cu -- device state, stage launches and the C ABI of the sweep.
//
// Driver semantics follow EZLDA/mainKernel.cu:158-380: every count a sweep reads is a
// snapshot of the sweep's starting topics (word-topic counts and n_k rebuilt first, the
// doc-topic rows of each chunk rebuilt from that chunk's topics before it is sampled), and
// new topics are written in place.  Unlike EZLDA, which re-uploads every chunk each
// sweep, the corpus stays resident in HBM (72M tokens use ~1.5 GB of a B200's 180 GB);
// chunks remain the unit of the doc-topic rebuild so that one chunk's doc rows stay
// L2-resident between the rebuild and the sampler.
#include <algorithm>
#include <cstdarg>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "common.h"
#include "kernels.cuh"
#include "launch_util.h"
#include "trainer_internal.h"

using namespace lda;

namespace {

#ifndef LDA_SAMPLE_TILE
#define LDA_SAMPLE_TILE 1024
#endif
constexpr int kSampleTile = LDA_SAMPLE_TILE;  // most tokens per sampler tile (a word's column is rebuilt per tile)
constexpr int kSampleTileMin = 64;            // fewest tokens per tile that a chunk's tile size goes down to
#ifndef LDA_TILES_PER_WARP
#define LDA_TILES_PER_WARP 2
#endif
// A chunk's sampler tiles are sized so that each resident warp gets about this many:
// with fewer, the launch ends with the longest tile while most warps sit idle.
constexpr int kTilesPerWarp = LDA_TILES_PER_WARP;
#ifndef LDA_DENSE_TILE
#define LDA_DENSE_TILE 8192
#endif
constexpr int kDenseTileLarge = LDA_DENSE_TILE;  // dense-word tiles above kLargeK topics (one CTA per tile)
constexpr int kLargeWarps = 8;                // warps per CTA of the large-K sampler kernels
constexpr int kWtTile = 16384;     // tokens per dense word-topic tile
constexpr int kCounters = 16;

struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    int stage = 0;
};

}  // namespace

struct lda_trainer {
    int device = 0;
    cudaStream_t own_stream = nullptr, stream = nullptr;
    int K = 0, Vd = 0, C = 0, warps = 8, num_sms = 0;
    int swarps = 8;  // warps per CTA of the K <= 2048 sampler
    float* recip = nullptr;  // [K] per-sweep reciprocals (K > kLargeK)
    float* smooth = nullptr; // [K] per-sweep smoothing table of the split Q bucket (K > kLargeK)
    int* order = nullptr;    // [dev::kOrderList] per-sweep topic order of the sparse-word statistics (K > kLargeK)
    // K > kLargeK: the dense words' Q-round tables, [Vd][32 * qrounds] float2, built by the
    // word statistics and read by the dense-word sampler (null when dev::qtab_rounds(K) = 0)
    float2* qtab_g = nullptr;
    int qrounds = 0;
    int warps_wt = 8, warps_dt = 8;  // warps per CTA of the word-topic and doc-topic rebuilds
    float alpha = 0, beta = 0, Vbeta = 0;
    uint64_t seed = 0;
    uint32_t iter = 0;
    int64_t N = 0, V = 0, D = 0;
    std::vector<int64_t> chunk_tok, chunk_doc;
    std::vector<int> s_tile_base;  // [C+1]
    // K > kLargeK: a chunk's sampler tiles are its dense-word tiles, then its sparse-word
    // tiles from s_tile_split[chunk] on, each kind sampled by its own kernel
    bool large = false;
    std::vector<int> s_tile_split;  // [C]
    int n_wtiles = 0;

    // device arrays
    uint32_t *tok_doc = nullptr, *meta = nullptr, *dtok_pos = nullptr, *dtok_word = nullptr;
    uint32_t *doc_off = nullptr, *doc_len = nullptr, *dt_off = nullptr, *dt_nnz = nullptr, *dt_ent = nullptr;
    uint16_t* z = nullptr;
    int* dwt = nullptr;
    uint32_t *swt_off = nullptr, *swt_nnz = nullptr, *swt_ent = nullptr;
    int* n_k = nullptr;
    uint32_t *st_top2 = nullptr, *st_k3 = nullptr;
    float4* st_phi = nullptr;
    float* st_ql = nullptr;
    uint32_t *seg_off = nullptr, *seg_cnt = nullptr;
    int4 *s_tiles = nullptr, *w_tiles = nullptr;
    double *tile_ll = nullptr, *ll_dev = nullptr;
    unsigned* tile_ctr = nullptr;         // [3 + 2C]: word-topic tiles, per chunk sampler tiles (two kinds), topic totals, small sparse words
    unsigned long long* ctr = nullptr;    // [kCounters]
    int* err = nullptr;
    double* ll_host = nullptr;            // pinned

    int64_t dt_cap = 0, swt_cap = 0;
    size_t smem_wt = 0, smem_stats = 0, smem_dt = 0, smem_sample = 0, smem_dense = 0, smem_sparse = 0;
    size_t smem_stats_sparse = 0;
    int grid_wt_cta = 0, grid_dt_cta = 0, grid_totals = 0;  // K > kLargeK: the CTA-per-unit rebuilds
    int grid_stats_dense = 0;                                // K > kLargeK: dense-word statistics
    int grid_dt_small = 0;                                   // K > kLargeK: docs of few tokens, warp per doc
    size_t smem_dt_small = 0;
    size_t smem_wt_cta = 0, smem_dt_cta = 0, smem_totals = 0;
    int grid_wt = 0, grid_stats = 0, grid_dt = 0, grid_sample = 0, grid_sample_ll = 0, grid_dense = 0, grid_sparse = 0;
    int grid_stats_sparse = 0;

    std::vector<void*> allocs;
    int64_t bytes = 0, budget = 0;

    bool timing = false;
    std::vector<EventPair> pending, pool;
    lda_stage_timing tm{};

    double last_ll = 0.0;
    int64_t last_ll_tokens = 0;
    bool ll_valid = false;
    std::vector<bool> chunk_sampled_ll;
    int chunk_first = 0, chunk_last = 0;  // sampled chunk range of lda_trainer_iterate
    std::vector<int4> h_stiles, h_wtiles;  // host copies of the tile lists
    // word range of the word-topic rebuild (lda_trainer_set_word_range): its tiles
    int32_t wt_lo = 0, wt_hi = 0;
    int4* w_tiles_rng = nullptr;
    int n_wtiles_rng = 0;
    // K > kLargeK: the last n_wsmall word tiles (n_wsmall_rng of a range's) are sparse words of at
    // most dev::kSmallSparse tokens, built warp per word by k_wt_sparse_small
    int n_wsmall = 0, n_wsmall_rng = 0;
    int grid_wsmall = 0;
    size_t smem_wsmall = 0;

    // streaming: the per-token arrays of the doc-topic rebuild and the sampler (doc of each
    // token, doc-order -> word-sorted map and word, per-token metadata) and the doc rows
    // live in one slot buffer per stream; the static ones are copied in from pinned host
    // memory for every chunk of every sweep
    struct Slot {
        uint32_t *tok_doc = nullptr, *dtok_pos = nullptr, *dtok_word = nullptr, *meta = nullptr, *dt_ent = nullptr;
        int chunk = -1;  // chunk whose static arrays the slot holds (stage entry points)
    };
    bool streaming = false;
    std::vector<cudaStream_t> sstreams;
    std::vector<Slot> slots;
    std::vector<cudaEvent_t> ev_slot;
    std::vector<cudaEvent_t> ev_used;  // above kLargeK: the slot's last chunk has been sampled
    bool stream_down = false;          // above kLargeK: the next streamed sweep takes its chunks in descending order
    cudaEvent_t ev_ready = nullptr;
    // host-buffer sweeps: each chunk's topics are copied back on copy_stream as soon as the
    // chunk is sampled
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_chunk = nullptr, ev_copied = nullptr;
    // asynchronous host-buffer sweeps (lda_iterate_host_async): uploads go on up_stream;
    // ev_down[c] marks chunk c's download of the last such sweep into last_out, and
    // last_seq the stage count right after it (nothing else enqueued since when equal)
    cudaStream_t up_stream = nullptr;
    cudaEvent_t ev_up = nullptr, ev_tail = nullptr;
    std::vector<cudaEvent_t> ev_down;
    bool record_down = false;
    bool copies_pending = false;  // an asynchronous sweep's downloads may still read z
    const uint16_t* last_out = nullptr;
    uint64_t stage_seq = 0, last_seq = ~0ull;
    int last_first = -1, last_last = -1;  // that sweep's chunk range
    // resident sweeps without stage timing run chunk i of the range on work stream i mod 2,
    // so one chunk's doc-topic rebuild and sampling overlap the other's
    cudaStream_t work[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
    // above kLargeK topics a chunk's sparse-word sampler runs on a side stream of the stream
    // that samples its dense words, so that its CTAs fill the dense kernel's tail
    struct Side {
        cudaStream_t parent = nullptr, stream = nullptr;
        cudaEvent_t fork = nullptr, join = nullptr;
    };
    std::vector<Side> sides;
    uint32_t *h_tok_doc = nullptr, *h_dtok_pos = nullptr, *h_dtok_word = nullptr;  // pinned [N]
    std::vector<int64_t> chunk_dt;  // [C+1] first doc-row entry of each chunk
    int64_t max_chunk_tok = 0, max_chunk_dt = 0, h2d_bytes = 0;

    int64_t range_tokens() const { return chunk_tok[chunk_last] - chunk_tok[chunk_first]; }

    ~lda_trainer() {
        if (device >= 0) cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        for (cudaStream_t q : sstreams) {
            cudaStreamSynchronize(q);
            cudaStreamDestroy(q);
        }
        for (cudaEvent_t e : ev_slot) cudaEventDestroy(e);
        for (cudaEvent_t e : ev_used) cudaEventDestroy(e);
        if (ev_ready) cudaEventDestroy(ev_ready);
        if (copy_stream) {
            cudaStreamSynchronize(copy_stream);
            cudaStreamDestroy(copy_stream);
        }
        if (ev_chunk) cudaEventDestroy(ev_chunk);
        if (ev_copied) cudaEventDestroy(ev_copied);
        if (up_stream) {
            cudaStreamSynchronize(up_stream);
            cudaStreamDestroy(up_stream);
        }
        if (ev_up) cudaEventDestroy(ev_up);
        if (ev_tail) cudaEventDestroy(ev_tail);
        for (cudaEvent_t e : ev_down) cudaEventDestroy(e);
        for (int i = 0; i < 2; ++i) {
            if (work[i]) {
                cudaStreamSynchronize(work[i]);
                cudaStreamDestroy(work[i]);
            }
            if (ev_join[i]) cudaEventDestroy(ev_join[i]);
        }
        if (ev_fork) cudaEventDestroy(ev_fork);
        for (Side& s : sides) {
            cudaStreamSynchronize(s.stream);
            cudaStreamDestroy(s.stream);
            cudaEventDestroy(s.fork);
            cudaEventDestroy(s.join);
        }
        cudaFreeHost(h_tok_doc);
        cudaFreeHost(h_dtok_pos);
        cudaFreeHost(h_dtok_word);
        for (void* p : allocs) cudaFree(p);
        if (w_tiles_rng) cudaFree(w_tiles_rng);
        if (ll_host) cudaFreeHost(ll_host);
        for (auto& e : pending) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
        for (auto& e : pool) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
        if (own_stream) cudaStreamDestroy(own_stream);
    }

    template <class T>
    int alloc(T** p, int64_t count) {
        const int64_t b = std::max<int64_t>(count, 1) * (int64_t)sizeof(T);
        if (budget > 0 && bytes + b > budget)
            return fail(LDA_ERR_DEVICE_MEM, "device budget of %lld bytes exceeded (need %lld more, hold %lld)",
                        (long long)budget, (long long)b, (long long)bytes);
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, (size_t)b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(LDA_ERR_DEVICE_MEM, "cudaMalloc of %lld bytes failed: %s", (long long)b, cudaGetErrorString(e));
        }
        allocs.push_back(q);
        bytes += b;
        *p = (T*)q;
        return LDA_OK;
    }

    EventPair* begin_stage(int stage) {
        ++stage_seq;
        if (copies_pending) {
            // work that may write the topics comes after the downloads still reading them
            cudaEventRecord(ev_copied, copy_stream);
            cudaStreamWaitEvent(stream, ev_copied, 0);
            copies_pending = false;
        }
        if (!timing) return nullptr;
        EventPair e;
        if (!pool.empty()) { e = pool.back(); pool.pop_back(); }
        else { cudaEventCreate(&e.a); cudaEventCreate(&e.b); }
        e.stage = stage;
        cudaEventRecord(e.a, stream);
        pending.push_back(e);
        return &pending.back();
    }
    void end_stage() {
        if (!timing || pending.empty()) return;
        cudaEventRecord(pending.back().b, stream);
    }
    void collect_timing() {
        for (auto& e : pending) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e.a, e.b);
            switch (e.stage) {
                case 0: tm.ms_wt += ms; tm.launches_wt++; break;
                case 1: tm.ms_stats += ms; tm.launches_stats++; break;
                case 2: tm.ms_dt += ms; tm.launches_dt++; break;
                case 3: tm.ms_sample += ms; tm.launches_sample++; break;
                case 4: tm.ms_ll += ms; tm.launches_ll++; break;
                default: tm.ms_copy += ms; break;
            }
            pool.push_back(e);
        }
        pending.clear();
    }
};

#define CUDA_TRY(expr)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (expr);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            cudaGetLastError();                                                                \
            return fail(LDA_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_));         \
        }                                                                                      \
    } while (0)

extern "C" const char* lda_version(void) { return "lda_b200 1.0 (sm_100a)"; }

static int occupancy_grid(const void* fn, int threads, size_t smem, int num_sms, int* grid) {
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
    if (per_sm < 1) return fail(LDA_ERR_CUDA, "kernel cannot be resident with %zu bytes of shared memory", smem);
    *grid = per_sm * num_sms;
    return LDA_OK;
}

// The sampler instantiation for (LL mode, K): for K > 1024 a lane's Q-bucket topics span
// several rounds, which are decided four per batch.
static int sample_qb(int K) { return K > 1024 ? 4 : 1; }

// skew: the doc rows' keys are word-column slot indices (the trainer's own rows); the
// allocation-free entry point samples rows whose keys are topics.
static const void* sample_kernel(bool ll, int K, bool skew = true) {
    if (sample_qb(K) == 4) {
        if (skew) return ll ? (const void*)dev::k_sample_t<true, 4, true> : (const void*)dev::k_sample_t<false, 4, true>;
        return ll ? (const void*)dev::k_sample_t<true, 4, false> : (const void*)dev::k_sample_t<false, 4, false>;
    }
    if (skew) return ll ? (const void*)dev::k_sample_t<true, 1, true> : (const void*)dev::k_sample_t<false, 1, true>;
    return ll ? (const void*)dev::k_sample_t<true, 1, false> : (const void*)dev::k_sample_t<false, 1, false>;
}

// K > kLargeK: the dense-word (CTA per tile) and sparse-word (no column) samplers; a lane's
// Q-bucket topics span more than one round there, so four rounds are decided per batch.
static const void* dense_large_kernel(bool ll) {
    return ll ? (const void*)dev::k_sample_dense_large<true, 4> : (const void*)dev::k_sample_dense_large<false, 4>;
}
static const void* sparse_large_kernel(bool ll) {
    return ll ? (const void*)dev::k_sample_sparse_large<true, 4> : (const void*)dev::k_sample_sparse_large<false, 4>;
}

static void launch_sample(bool ll, int K, int grid, int threads, size_t smem, cudaStream_t q, const dev::SampleArgs& a,
                          bool skew = true) {
    if (sample_qb(K) == 4) {
        if (skew) {
            if (ll) dev::k_sample_t<true, 4, true><<<grid, threads, smem, q>>>(a);
            else dev::k_sample_t<false, 4, true><<<grid, threads, smem, q>>>(a);
        } else {
            if (ll) dev::k_sample_t<true, 4, false><<<grid, threads, smem, q>>>(a);
            else dev::k_sample_t<false, 4, false><<<grid, threads, smem, q>>>(a);
        }
    } else {
        if (skew) {
            if (ll) dev::k_sample_t<true, 1, true><<<grid, threads, smem, q>>>(a);
            else dev::k_sample_t<false, 1, true><<<grid, threads, smem, q>>>(a);
        } else {
            if (ll) dev::k_sample_t<true, 1, false><<<grid, threads, smem, q>>>(a);
            else dev::k_sample_t<false, 1, false><<<grid, threads, smem, q>>>(a);
        }
    }
}

extern "C" int lda_trainer_create(const lda_corpus* c, const lda_train_config* cfg, lda_trainer** out) {
    if (!c || !cfg || !out) return fail(LDA_ERR_ARG, "null argument");
    *out = nullptr;
    if (cfg->K < 4 || cfg->K > 65535) return fail(LDA_ERR_ARG, "K=%d outside [4, 65535]", cfg->K);
    if (!(cfg->alpha > 0.f) || !(cfg->beta > 0.f)) return fail(LDA_ERR_ARG, "alpha and beta must be > 0");
    if (cfg->device_budget < 0) return fail(LDA_ERR_ARG, "negative device budget");
    for (int64_t i = 0; i < c->N; ++i)
        if (c->z[i] >= cfg->K) return fail(LDA_ERR_ARG, "initial topic %d of token %lld >= K=%d", c->z[i], (long long)i, cfg->K);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(LDA_ERR_CUDA, "no CUDA device available");
    }
    if (cfg->device < 0 || cfg->device >= ndev) return fail(LDA_ERR_ARG, "device %d of %d", cfg->device, ndev);
    std::unique_ptr<lda_trainer> t(new lda_trainer());
    lda_trainer& T = *t;
    T.device = cfg->device;
    CUDA_TRY(cudaSetDevice(T.device));
    CUDA_TRY(cudaStreamCreateWithFlags(&T.own_stream, cudaStreamNonBlocking));
    T.stream = T.own_stream;
    CUDA_TRY(cudaDeviceGetAttribute(&T.num_sms, cudaDevAttrMultiProcessorCount, T.device));
    int max_smem = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, T.device));
    T.K = cfg->K; T.alpha = cfg->alpha; T.beta = cfg->beta; T.seed = cfg->seed;
    T.N = c->N; T.V = c->V; T.D = c->D; T.C = c->C; T.Vd = c->V_dense;
    if (cfg->num_dense != 0) {
        // words are frequency ranks, so any prefix can take the dense path; sparse rows
        // pack counts in 16 bits
        const int64_t nd = cfg->num_dense < 0 ? 0 : cfg->num_dense;
        if (nd > T.V) return fail(LDA_ERR_ARG, "num_dense %d above the vocabulary (%lld)", cfg->num_dense, (long long)T.V);
        if (nd < T.V && c->word_count[nd] > 65535)
            return fail(LDA_ERR_ARG, "word %lld has %lld tokens: words above 65535 tokens must be dense", (long long)nd,
                        (long long)c->word_count[nd]);
        T.Vd = (int)nd;
    }
    T.Vbeta = (float)T.V * T.beta;
    T.budget = cfg->device_budget;
    T.chunk_tok = c->chunk_tok;
    T.chunk_doc = c->chunk_doc;
    // warps per CTA: (warps + 1) K-wide shared rows must fit
    const int64_t row = (int64_t)T.K * 4;
    T.warps = (int)std::min<int64_t>(8, ((int64_t)max_smem - 2048) / (row + 256) - 1);
    if (T.warps < 1) return fail(LDA_ERR_ARG, "K=%d needs %lld bytes of shared memory per warp (max %d)", T.K, (long long)(2 * row), max_smem);
    auto sample_bytes = [&](int w) { return (size_t)T.K * 4 + (size_t)w * (dev::col_words(T.K) * 4 + 16 * sizeof(uint32_t)); };
    T.large = T.K > dev::kLargeK;
    if (!T.large) {
        T.swarps = dev::kSampleWarps;
        while (T.swarps > 1 && sample_bytes(T.swarps) > (size_t)max_smem) --T.swarps;
        if (sample_bytes(T.swarps) > (size_t)max_smem) return fail(LDA_ERR_ARG, "K=%d does not fit in shared memory", T.K);
        T.smem_sample = sample_bytes(T.swarps);
    } else {
        T.smem_dense = dev::dense_large_smem(T.K, kLargeWarps);
        T.smem_sparse = dev::sparse_large_smem(T.K, kLargeWarps);
        if (T.smem_dense > (size_t)max_smem || T.smem_sparse > (size_t)max_smem)
            return fail(LDA_ERR_ARG, "K=%d does not fit in shared memory (the dense-word sampler needs %zu bytes)", T.K,
                        T.smem_dense);
    }
    T.smem_stats = (size_t)(T.warps + 1) * row;
    // the rebuilds' warp-private histograms hold 16-bit counts, two per word: a dense
    // word-topic tile has kWtTile tokens, a sparse word fewer than 65,536 and a doc at most
    // 65,535 (the corpus layout's limit), so every count fits.  Each rebuild takes as many
    // warps per CTA (up to 8) as its shared memory allows.
    const size_t bitw = (size_t)(T.K + 31) / 32;
    auto wt_bytes = [&](int w) { return ((size_t)T.K + (size_t)w * (dev::Hist<true>::words(T.K) + bitw)) * 4; };
    auto dt_bytes = [&](int w) { return (size_t)w * (dev::Hist<true>::words(T.K) + bitw) * 4; };
    T.warps_wt = 8;
    while (T.warps_wt > 1 && wt_bytes(T.warps_wt) > (size_t)max_smem) --T.warps_wt;
    T.warps_dt = 8;
    while (T.warps_dt > 1 && dt_bytes(T.warps_dt) > (size_t)max_smem) --T.warps_dt;
    if (wt_bytes(T.warps_wt) > (size_t)max_smem || dt_bytes(T.warps_dt) > (size_t)max_smem)
        return fail(LDA_ERR_ARG, "K=%d does not fit in shared memory (count rebuilds)", T.K);
    T.smem_wt = wt_bytes(T.warps_wt);
    T.smem_dt = dt_bytes(T.warps_dt);

    // ---- host-side derived layout
    const int64_t N = T.N, V = T.V, D = T.D, Vs = V - T.Vd;
    std::vector<uint32_t> h32(std::max<int64_t>({N, D + 1, (int64_t)T.C * V, 1}));
    // doc rows: capacity roundup4(min(len, K)) keeps every row 16-byte aligned
    std::vector<uint32_t> hdt_off(D), hdoc_len(D);
    int64_t run = 0;
    for (int64_t d = 0; d < D; ++d) {
        const int64_t len = c->doc_off[d + 1] - c->doc_off[d];
        hdoc_len[d] = (uint32_t)len;
        hdt_off[d] = (uint32_t)run;
        run += (std::min<int64_t>(len, T.K) + 3) & ~int64_t(3);
    }
    T.dt_cap = run;
    if (run >= (int64_t)UINT32_MAX) return fail(LDA_ERR_ARG, "doc-topic storage exceeds 2^32 entries");
    std::vector<uint32_t> hswt_off(std::max<int64_t>(Vs, 1));
    run = 0;
    for (int64_t s = 0; s < Vs; ++s) {
        hswt_off[s] = (uint32_t)run;
        run += std::min<int64_t>(c->word_count[T.Vd + s], T.K);
    }
    T.swt_cap = run;
    // sampler tiles per chunk, largest first (for K > kLargeK: dense-word tiles, then
    // sparse-word tiles, each largest first).  For K <= kLargeK a chunk's tile size is
    // its tokens / (kTilesPerWarp x the sampler's resident warps), rounded up to 32 and
    // kept within [kSampleTileMin, kSampleTile].
    int64_t resident_warps = 0;
    if (!T.large) {
        CUDA_TRY(raise_smem_limit(sample_kernel(false, T.K), T.smem_sample));
        int g = 0, orc = occupancy_grid(sample_kernel(false, T.K), 32 * T.swarps, T.smem_sample, T.num_sms, &g);
        if (orc) return orc;
        resident_warps = (int64_t)g * T.swarps;
    }
    std::vector<int4> st;
    T.s_tile_base.assign(T.C + 1, 0);
    T.s_tile_split.assign(T.C, 0);
    auto by_size = [](const int4& a, const int4& b) { return a.z > b.z; };
    for (int ch = 0; ch < T.C; ++ch) {
        std::vector<int4> ct, cs;
        int64_t tile_ch = kSampleTile;
        if (!T.large) {
            const int64_t per = kTilesPerWarp * std::max<int64_t>(resident_warps, 1);
            const int64_t want = ((T.chunk_tok[ch + 1] - T.chunk_tok[ch] + per - 1) / per + 31) / 32 * 32;
            tile_ch = std::min<int64_t>(kSampleTile, std::max<int64_t>(kSampleTileMin, want));
        }
        for (int64_t w = 0; w < V; ++w) {
            const int64_t n = c->seg_cnt[(size_t)ch * V + w], o = c->seg_off[(size_t)ch * V + w];
            const bool dense = w < T.Vd;
            const int64_t tile = T.large && dense ? kDenseTileLarge : tile_ch;
            for (int64_t p = 0; p < n; p += tile) {
                const int4 v = make_int4((int)w, (int)(o + p), (int)std::min<int64_t>(tile, n - p), dense);
                (T.large && !dense ? cs : ct).push_back(v);
            }
        }
        std::stable_sort(ct.begin(), ct.end(), by_size);
        std::stable_sort(cs.begin(), cs.end(), by_size);
        st.insert(st.end(), ct.begin(), ct.end());
        T.s_tile_split[ch] = (int)st.size();
        st.insert(st.end(), cs.begin(), cs.end());
        T.s_tile_base[ch + 1] = (int)st.size();
    }
    // word-topic tiles: dense segments of every chunk, and one tile per sparse word
    std::vector<int4> wt;
    for (int64_t w = 0; w < V; ++w) {
        if (w < T.Vd) {
            for (int ch = 0; ch < T.C; ++ch) {
                const int64_t n = c->seg_cnt[(size_t)ch * V + w], o = c->seg_off[(size_t)ch * V + w];
                for (int64_t p = 0; p < n; p += kWtTile)
                    wt.push_back(make_int4((int)w, (int)(o + p), (int)std::min<int64_t>(kWtTile, n - p), 1));
            }
        } else if (c->word_count[w] > 0) {
            wt.push_back(make_int4((int)w, 0, (int)c->word_count[w], 0));
        }
    }
    std::stable_sort(wt.begin(), wt.end(), [](const int4& a, const int4& b) { return a.z > b.z; });
    if (T.large && T.C <= 32) {
        // small sparse words last (stable: each part keeps largest first)
        auto big = [&](const int4& x) { return (x.w & 1) || x.z > dev::kSmallSparse; };
        const auto mid = std::stable_partition(wt.begin(), wt.end(), big);
        T.n_wsmall = (int)(wt.end() - mid);
    }
    T.n_wtiles = (int)wt.size();

    // ---- resident or streamed chunks (EZLDA streams every chunk through fixed buffers,
    // EZLDA/mainKernel.cu:203-314; here the corpus stays resident when it fits the budget)
    if (cfg->stream_mode < 0 || cfg->stream_mode > 2) return fail(LDA_ERR_ARG, "stream_mode %d", cfg->stream_mode);
    if (cfg->num_streams < 0 || cfg->num_streams > 64) return fail(LDA_ERR_ARG, "num_streams %d", cfg->num_streams);
    T.chunk_dt.assign(T.C + 1, 0);
    for (int ch = 0; ch < T.C; ++ch) {
        const int64_t d0 = T.chunk_doc[ch], d1 = T.chunk_doc[ch + 1];
        T.chunk_dt[ch] = d0 < D ? hdt_off[d0] : T.dt_cap;
        T.chunk_dt[ch + 1] = d1 < D ? hdt_off[d1] : T.dt_cap;
        T.max_chunk_tok = std::max(T.max_chunk_tok, T.chunk_tok[ch + 1] - T.chunk_tok[ch]);
    }
    for (int ch = 0; ch < T.C; ++ch) T.max_chunk_dt = std::max(T.max_chunk_dt, T.chunk_dt[ch + 1] - T.chunk_dt[ch]);
    {
        // the exact bytes of the resident layout (the allocations below, in resident mode)
        auto nb = [](int64_t n, int64_t size) { return std::max<int64_t>(n, 1) * size; };
        const int64_t ns = (int64_t)st.size(), nw = (int64_t)wt.size();
        const int64_t resident = 4 * nb(N, 4) + nb(T.dt_cap, 4) + nb(N, 2) + nb(D + 1, 4) + 3 * nb(D, 4) +
                                 nb((int64_t)T.Vd * T.K, 4) + 2 * nb(std::max<int64_t>(Vs, 1), 4) + nb(T.swt_cap, 4) +
                                 nb(T.K, 4) + 2 * nb(V, 4) + nb(V, 16) + nb(V * 32, 4) + 2 * nb((int64_t)T.C * V, 4) +
                                 nb(ns, 16) + nb(nw, 16) + nb(ns, 8) + nb(1, 8) + nb(3 + 2 * T.C, 4) + nb(kCounters, 8) + (T.large ? 2 * nb(T.K, 4) + nb(dev::kOrderList, 4) : 0) +
                                 (T.large && dev::qtab_rounds(T.K) > 0 && T.Vd > 0 ? nb((int64_t)T.Vd * 32 * dev::qtab_rounds(T.K), 8) : 0) +
                                 nb(1, 4);
        T.streaming = cfg->stream_mode == 2 || (cfg->stream_mode == 0 && T.budget > 0 && resident > T.budget);
    }
    int rc;
#define ALLOC(p, n) if ((rc = T.alloc(&(p), (n))) != LDA_OK) return rc
    if (!T.streaming) {
        ALLOC(T.tok_doc, N); ALLOC(T.meta, N); ALLOC(T.dtok_pos, N); ALLOC(T.dtok_word, N); ALLOC(T.dt_ent, T.dt_cap);
    } else {
        const int ns = cfg->num_streams > 0 ? cfg->num_streams : 4;
        T.slots.resize(ns);
        for (auto& sl : T.slots) {
            ALLOC(sl.tok_doc, T.max_chunk_tok); ALLOC(sl.dtok_pos, T.max_chunk_tok); ALLOC(sl.dtok_word, T.max_chunk_tok);
            ALLOC(sl.meta, T.max_chunk_tok); ALLOC(sl.dt_ent, T.max_chunk_dt);
        }
        T.sstreams.resize(ns, nullptr);
        T.ev_slot.resize(ns, nullptr);
        T.ev_used.resize(ns, nullptr);
        for (int i = 0; i < ns; ++i) {
            CUDA_TRY(cudaStreamCreateWithFlags(&T.sstreams[i], cudaStreamNonBlocking));
            CUDA_TRY(cudaEventCreateWithFlags(&T.ev_slot[i], cudaEventDisableTiming));
            CUDA_TRY(cudaEventCreateWithFlags(&T.ev_used[i], cudaEventDisableTiming));
        }
        CUDA_TRY(cudaEventCreateWithFlags(&T.ev_ready, cudaEventDisableTiming));
        const size_t nb = sizeof(uint32_t) * (size_t)std::max<int64_t>(N, 1);
        cudaError_t e = cudaMallocHost(&T.h_tok_doc, nb);
        if (e == cudaSuccess) e = cudaMallocHost(&T.h_dtok_pos, nb);
        if (e == cudaSuccess) e = cudaMallocHost(&T.h_dtok_word, nb);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(LDA_ERR_NOMEM, "pinned host staging of %zu bytes failed: %s", 3 * nb, cudaGetErrorString(e));
        }
        for (int64_t i = 0; i < N; ++i) {
            T.h_tok_doc[i] = (uint32_t)c->tok_doc[i];
            T.h_dtok_pos[i] = (uint32_t)c->dtok_pos[i];
            T.h_dtok_word[i] = (uint32_t)c->dtok_word[i];
        }
    }
    ALLOC(T.z, N);
    ALLOC(T.doc_off, D + 1); ALLOC(T.doc_len, D); ALLOC(T.dt_off, D); ALLOC(T.dt_nnz, D);
    ALLOC(T.dwt, (int64_t)T.Vd * T.K); ALLOC(T.swt_off, std::max<int64_t>(Vs, 1)); ALLOC(T.swt_nnz, std::max<int64_t>(Vs, 1));
    ALLOC(T.swt_ent, T.swt_cap);
    ALLOC(T.n_k, T.K); ALLOC(T.st_top2, V); ALLOC(T.st_k3, V); ALLOC(T.st_phi, V); ALLOC(T.st_ql, V * 32);
    ALLOC(T.seg_off, (int64_t)T.C * V); ALLOC(T.seg_cnt, (int64_t)T.C * V);
    ALLOC(T.s_tiles, (int64_t)st.size()); ALLOC(T.w_tiles, (int64_t)wt.size());
    ALLOC(T.tile_ll, (int64_t)st.size()); ALLOC(T.ll_dev, 1);
    ALLOC(T.tile_ctr, 3 + 2 * T.C); ALLOC(T.ctr, kCounters); ALLOC(T.err, 1);
    if (T.large) { ALLOC(T.recip, T.K); ALLOC(T.smooth, T.K); ALLOC(T.order, dev::kOrderList); }
    if (T.large && dev::qtab_rounds(T.K) > 0 && T.Vd > 0) {
        T.qrounds = dev::qtab_rounds(T.K);
        ALLOC(T.qtab_g, (int64_t)T.Vd * 32 * T.qrounds);
    }
#undef ALLOC
    CUDA_TRY(cudaMallocHost(&T.ll_host, sizeof(double)));

    // ---- upload (synchronous: creation is not on the hot path)
    auto up32 = [&](uint32_t* dst, int64_t n, auto getter) -> int {
        for (int64_t i = 0; i < n; ++i) h32[i] = (uint32_t)getter(i);
        CUDA_TRY(cudaMemcpy(dst, h32.data(), sizeof(uint32_t) * (size_t)n, cudaMemcpyHostToDevice));
        return LDA_OK;
    };
    if (!T.streaming) {
        if ((rc = up32(T.tok_doc, N, [&](int64_t i) { return c->tok_doc[i]; }))) return rc;
        if ((rc = up32(T.dtok_pos, N, [&](int64_t i) { return c->dtok_pos[i]; }))) return rc;
        if ((rc = up32(T.dtok_word, N, [&](int64_t i) { return c->dtok_word[i]; }))) return rc;
        CUDA_TRY(cudaMemset(T.meta, 0, sizeof(uint32_t) * (size_t)N));
    }
    if ((rc = up32(T.doc_off, D + 1, [&](int64_t i) { return c->doc_off[i]; }))) return rc;
    if ((rc = up32(T.seg_off, (int64_t)T.C * V, [&](int64_t i) { return c->seg_off[i]; }))) return rc;
    if ((rc = up32(T.seg_cnt, (int64_t)T.C * V, [&](int64_t i) { return c->seg_cnt[i]; }))) return rc;
    CUDA_TRY(cudaMemcpy(T.z, c->z.data(), sizeof(uint16_t) * (size_t)N, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(T.doc_len, hdoc_len.data(), sizeof(uint32_t) * (size_t)D, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(T.dt_off, hdt_off.data(), sizeof(uint32_t) * (size_t)D, cudaMemcpyHostToDevice));
    if (Vs > 0) CUDA_TRY(cudaMemcpy(T.swt_off, hswt_off.data(), sizeof(uint32_t) * (size_t)Vs, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemset(T.swt_nnz, 0, sizeof(uint32_t) * (size_t)std::max<int64_t>(Vs, 1)));
    CUDA_TRY(cudaMemset(T.dt_nnz, 0, sizeof(uint32_t) * (size_t)D));
    // stats start valid (topic 0) so a stage called out of order reads in-range topics
    CUDA_TRY(cudaMemset(T.st_top2, 0, sizeof(uint32_t) * (size_t)V));
    CUDA_TRY(cudaMemset(T.st_k3, 0, sizeof(uint32_t) * (size_t)V));
    CUDA_TRY(cudaMemset(T.st_phi, 0, sizeof(float4) * (size_t)V));
    CUDA_TRY(cudaMemset(T.st_ql, 0, sizeof(float) * 32 * (size_t)V));
    CUDA_TRY(cudaMemset(T.n_k, 0, sizeof(int) * (size_t)T.K));
    CUDA_TRY(cudaMemset(T.err, 0, sizeof(int)));
    CUDA_TRY(cudaMemset(T.ctr, 0, sizeof(unsigned long long) * kCounters));
    CUDA_TRY(cudaMemset(T.tile_ll, 0, sizeof(double) * std::max<size_t>(st.size(), 1)));
    if (!st.empty()) CUDA_TRY(cudaMemcpy(T.s_tiles, st.data(), sizeof(int4) * st.size(), cudaMemcpyHostToDevice));
    if (!wt.empty()) CUDA_TRY(cudaMemcpy(T.w_tiles, wt.data(), sizeof(int4) * wt.size(), cudaMemcpyHostToDevice));
    T.h_stiles = st;
    T.h_wtiles = wt;

    // ---- launch shapes: persistent grids sized by occupancy
    const int threads = 32 * T.warps;
    const void* wt_fn = (const void*)dev::k_wt_build<true>;
    const void* dt_fn = (const void*)dev::k_dt_build<true>;
    for (auto kv : {std::make_pair(wt_fn, T.smem_wt), std::make_pair((const void*)dev::k_word_stats, T.smem_stats),
                    std::make_pair(dt_fn, T.smem_dt)})
        CUDA_TRY(raise_smem_limit(kv.first, kv.second));
    if ((rc = occupancy_grid(wt_fn, 32 * T.warps_wt, T.smem_wt, T.num_sms, &T.grid_wt))) return rc;
    if ((rc = occupancy_grid((const void*)dev::k_word_stats, threads, T.smem_stats, T.num_sms, &T.grid_stats))) return rc;
    if ((rc = occupancy_grid(dt_fn, 32 * T.warps_dt, T.smem_dt, T.num_sms, &T.grid_dt))) return rc;
    if (T.large) {
        // the CTA-per-unit rebuilds: one shared histogram and bitmap (plus a sparse word's
        // chunk segments), and the topic totals' per-CTA counts when K words fit
        const size_t hist_b = ((size_t)dev::Hist<true>::words(T.K) + bitw) * 4;
        T.smem_wt_cta = hist_b + (2 * (size_t)T.C + 1) * 4;
        T.smem_dt_cta = hist_b;
        T.smem_totals = (size_t)T.K * 4 <= (size_t)max_smem ? (size_t)T.K * 4 : 0;
        if (T.smem_wt_cta > (size_t)max_smem)
            return fail(LDA_ERR_ARG, "K=%d with %d chunks does not fit in shared memory (word-topic rebuild)", T.K, T.C);
        const void* tot_fn = T.smem_totals ? (const void*)dev::k_topic_totals<true> : (const void*)dev::k_topic_totals<false>;
        CUDA_TRY(raise_smem_limit((const void*)dev::k_wt_build_cta, T.smem_wt_cta));
        T.smem_dt_small = dev::dt_small_warp_words(T.K) * 4 * 8;
        if (T.smem_dt_small <= (size_t)max_smem) {
            CUDA_TRY(raise_smem_limit((const void*)dev::k_dt_build_small, T.smem_dt_small));
            if ((rc = occupancy_grid((const void*)dev::k_dt_build_small, 256, T.smem_dt_small, T.num_sms, &T.grid_dt_small)))
                return rc;
        }
        T.smem_wsmall = dev::wt_small_warp_words(T.K) * 4 * 8;
        if (T.n_wsmall > 0) {
            if (T.smem_wsmall > (size_t)max_smem) {
                T.n_wsmall = 0;  // the CTA kernel takes every tile
            } else {
                CUDA_TRY(raise_smem_limit((const void*)dev::k_wt_sparse_small, T.smem_wsmall));
                if ((rc = occupancy_grid((const void*)dev::k_wt_sparse_small, 256, T.smem_wsmall, T.num_sms, &T.grid_wsmall)))
                    return rc;
            }
        }
        CUDA_TRY(raise_smem_limit((const void*)dev::k_dt_build_cta, T.smem_dt_cta));
        CUDA_TRY(raise_smem_limit(tot_fn, T.smem_totals));
        if ((rc = occupancy_grid((const void*)dev::k_wt_build_cta, dev::kRebuildThreads, T.smem_wt_cta, T.num_sms,
                                 &T.grid_wt_cta)) ||
            (rc = occupancy_grid((const void*)dev::k_dt_build_cta, dev::kRebuildThreads, T.smem_dt_cta, T.num_sms,
                                 &T.grid_dt_cta)) ||
            (rc = occupancy_grid(tot_fn, 256, T.smem_totals, T.num_sms, &T.grid_totals)))
            return rc;
    }
    if (!T.large) {
        for (bool ll : {false, true}) CUDA_TRY(raise_smem_limit(sample_kernel(ll, T.K), T.smem_sample));
        const int st = 32 * T.swarps;
        if ((rc = occupancy_grid(sample_kernel(false, T.K), st, T.smem_sample, T.num_sms, &T.grid_sample))) return rc;
        if ((rc = occupancy_grid(sample_kernel(true, T.K), st, T.smem_sample, T.num_sms, &T.grid_sample_ll))) return rc;
    } else {
        const int lt = 32 * kLargeWarps;
        int g0 = 0, g1 = 0, g2 = 0, g3 = 0;
        for (bool ll : {false, true}) {
            CUDA_TRY(raise_smem_limit(dense_large_kernel(ll), T.smem_dense));
            CUDA_TRY(raise_smem_limit(sparse_large_kernel(ll), T.smem_sparse));
        }
        if ((rc = occupancy_grid(dense_large_kernel(false), lt, T.smem_dense, T.num_sms, &g0)) ||
            (rc = occupancy_grid(dense_large_kernel(true), lt, T.smem_dense, T.num_sms, &g1)) ||
            (rc = occupancy_grid(sparse_large_kernel(false), lt, T.smem_sparse, T.num_sms, &g2)) ||
            (rc = occupancy_grid(sparse_large_kernel(true), lt, T.smem_sparse, T.num_sms, &g3)))
            return rc;
        T.grid_dense = std::min(g0, g1);
        T.grid_sparse = std::min(g2, g3);
        CUDA_TRY(raise_smem_limit((const void*)dev::k_word_stats_dense_rows, (size_t)T.K * 4));
        if ((rc = occupancy_grid((const void*)dev::k_word_stats_dense_rows, 256, (size_t)T.K * 4, T.num_sms,
                                 &T.grid_stats_dense)))
            return rc;
        T.smem_stats_sparse = dev::stats_sparse_smem(T.K, kLargeWarps);
        CUDA_TRY(raise_smem_limit((const void*)dev::k_word_stats_sparse_large, T.smem_stats_sparse));
        if ((rc = occupancy_grid((const void*)dev::k_word_stats_sparse_large, lt, T.smem_stats_sparse, T.num_sms,
                                 &T.grid_stats_sparse)))
            return rc;
    }
    T.grid_stats = (int)std::max<int64_t>(1, std::min<int64_t>(T.grid_stats, (V + T.warps - 1) / T.warps));
    CUDA_TRY(cudaDeviceSynchronize());
    T.chunk_sampled_ll.assign(T.C, false);
    T.chunk_first = 0;
    T.chunk_last = T.C;
    *out = t.release();
    return LDA_OK;
}

extern "C" int lda_trainer_destroy(lda_trainer* t) {
    delete t;
    return LDA_OK;
}

extern "C" int lda_trainer_set_stream(lda_trainer* t, void* s) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    t->stream = s ? (cudaStream_t)s : t->own_stream;
    return LDA_OK;
}

extern "C" int lda_trainer_get_stream(lda_trainer* t, void** s) {
    if (!t || !s) return fail(LDA_ERR_ARG, "null argument");
    *s = (void*)t->stream;
    return LDA_OK;
}

extern "C" int lda_trainer_set_chunk_range(lda_trainer* t, int32_t first, int32_t last) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    if (first < 0 || last > t->C || first >= last)
        return fail(LDA_ERR_ARG, "chunk range [%d, %d) outside [0, %d)", first, last, t->C);
    t->chunk_first = first;
    t->chunk_last = last;
    t->ll_valid = false;
    return LDA_OK;
}

extern "C" int lda_trainer_set_word_range(lda_trainer* t, int32_t w0, int32_t w1) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    if (w0 < 0 || w1 > t->V || w0 > w1) return fail(LDA_ERR_ARG, "word range [%d, %d) outside [0, %lld)", w0, w1, (long long)t->V);
    CUDA_TRY(cudaSetDevice(t->device));
    CUDA_TRY(cudaStreamSynchronize(t->stream));
    if (t->w_tiles_rng) {
        CUDA_TRY(cudaFree(t->w_tiles_rng));
        t->w_tiles_rng = nullptr;
        t->n_wtiles_rng = 0;
    }
    t->wt_lo = w0;
    t->wt_hi = w1;
    if (w0 == 0 && w1 == t->V) return LDA_OK;  // the whole vocabulary: the trainer's own tiles
    // the range's tiles, in the trainer's largest-first order
    std::vector<int4> r;
    for (const int4& x : t->h_wtiles)
        if (x.x >= w0 && x.x < w1) r.push_back(x);
    CUDA_TRY(cudaMalloc(&t->w_tiles_rng, sizeof(int4) * std::max<size_t>(r.size(), 1)));
    if (!r.empty()) CUDA_TRY(cudaMemcpy(t->w_tiles_rng, r.data(), sizeof(int4) * r.size(), cudaMemcpyHostToDevice));
    t->n_wtiles_rng = (int)r.size();
    t->n_wsmall_rng = 0;
    for (const int4& x : r) t->n_wsmall_rng += t->n_wsmall > 0 && !(x.w & 1) && x.z <= dev::kSmallSparse;
    return LDA_OK;
}

extern "C" int lda_trainer_word_side(lda_trainer* t, lda_word_side* out) {
    if (!t || !out) return fail(LDA_ERR_ARG, "null argument");
    out->n_k = t->n_k;
    out->dense_wt = t->dwt;
    out->sparse_ent = t->swt_ent;
    out->sparse_nnz = t->swt_nnz;
    out->sparse_off = t->swt_off;
    out->top2 = t->st_top2;
    out->k3 = t->st_k3;
    out->phi4 = reinterpret_cast<float*>(t->st_phi);
    out->ql = t->st_ql;
    out->qtab = reinterpret_cast<float*>(t->qtab_g);
    out->qtab_rounds = t->qrounds;
    out->K = t->K;
    out->vocab = t->V;
    out->num_dense = t->Vd;
    out->sparse_capacity = t->swt_cap;
    return LDA_OK;
}

extern "C" int lda_trainer_topics_device(lda_trainer* t, void** ptr, int64_t* count) {
    if (!t || !ptr) return fail(LDA_ERR_ARG, "null argument");
    *ptr = (void*)t->z;
    if (count) *count = t->N;
    return LDA_OK;
}

extern "C" int lda_trainer_stream_info(const lda_trainer* t, int32_t* streaming, int32_t* streams,
                                       int64_t* h2d_bytes) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    if (streaming) *streaming = t->streaming ? 1 : 0;
    if (streams) *streams = (int32_t)t->sstreams.size();
    if (h2d_bytes) *h2d_bytes = t->h2d_bytes;
    return LDA_OK;
}

extern "C" int lda_trainer_device_bytes(const lda_trainer* t, int64_t* b) {
    if (!t || !b) return fail(LDA_ERR_ARG, "null argument");
    *b = t->bytes;
    return LDA_OK;
}

// ------------------------------------------------------------------- stages

static dev::WtArgs wt_args(const lda_trainer* t) {
    dev::WtArgs a;
    a.tiles = t->w_tiles; a.ntiles = t->n_wtiles; a.tile_counter = t->tile_ctr;
    a.z = t->z; a.K = t->K; a.V = (int)t->V; a.Vd = t->Vd; a.C = t->C;
    a.seg_off = t->seg_off; a.seg_cnt = t->seg_cnt;
    a.dwt = t->dwt; a.swt_off = t->swt_off; a.swt_nnz = t->swt_nnz; a.swt_ent = t->swt_ent;
    a.n_k = t->n_k; a.err = t->err;
    return a;
}

static dev::StatsArgs stats_args(const lda_trainer* t) {
    dev::StatsArgs a;
    a.V = (int)t->V; a.Vd = t->Vd; a.K = t->K; a.alpha = t->alpha; a.beta = t->beta; a.Vbeta = t->Vbeta;
    a.n_k = t->n_k; a.dwt = t->dwt; a.swt_off = t->swt_off; a.swt_nnz = t->swt_nnz; a.swt_ent = t->swt_ent;
    a.st_top2 = t->st_top2; a.st_k3 = t->st_k3; a.st_phi = t->st_phi; a.st_ql = t->st_ql;
    a.smooth = t->smooth;
    return a;
}

extern "C" int lda_update_wt(lda_trainer* t) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    CUDA_TRY(cudaSetDevice(t->device));
    t->begin_stage(0);
    CUDA_TRY(cudaMemsetAsync(t->n_k, 0, sizeof(int) * (size_t)t->K, t->stream));
    dev::WtArgs a = wt_args(t);
    if (t->w_tiles_rng) {
        // a word range: its dense rows, its sparse rows and its words' share of n_k
        const int64_t d0 = std::min<int64_t>(t->wt_lo, t->Vd), d1 = std::min<int64_t>(t->wt_hi, t->Vd);
        if (d1 > d0)
            CUDA_TRY(cudaMemsetAsync(t->dwt + d0 * t->K, 0, sizeof(int) * (size_t)(d1 - d0) * t->K, t->stream));
        a.tiles = t->w_tiles_rng;
        a.ntiles = t->n_wtiles_rng;
    } else if (t->Vd > 0) {
        CUDA_TRY(cudaMemsetAsync(t->dwt, 0, sizeof(int) * (size_t)t->Vd * t->K, t->stream));
    }
    CUDA_TRY(cudaMemsetAsync(t->tile_ctr, 0, sizeof(unsigned), t->stream));
    if (t->large) {
        // rows by CTA per tile (small sparse words by warp per word), then the totals over
        // the same tiles
        const int nsmall = t->w_tiles_rng ? t->n_wsmall_rng : t->n_wsmall;
        dev::WtArgs ab = a;
        ab.ntiles = a.ntiles - nsmall;
        if (ab.ntiles > 0) {
            const int grid = std::max(1, std::min(t->grid_wt_cta, ab.ntiles));
            dev::k_wt_build_cta<<<grid, dev::kRebuildThreads, t->smem_wt_cta, t->stream>>>(ab);
            CUDA_TRY(cudaGetLastError());
        }
        if (nsmall > 0) {
            dev::WtArgs as = a;
            as.tiles = a.tiles + ab.ntiles;
            as.ntiles = nsmall;
            as.tile_counter = t->tile_ctr + 2 + 2 * t->C;
            CUDA_TRY(cudaMemsetAsync(as.tile_counter, 0, sizeof(unsigned), t->stream));
            const int grid = std::max(1, std::min(t->grid_wsmall, (nsmall + 7) / 8));
            dev::k_wt_sparse_small<<<grid, 256, t->smem_wsmall, t->stream>>>(as);
            CUDA_TRY(cudaGetLastError());
        }
        dev::WtArgs at = a;
        at.tile_counter = t->tile_ctr + 1 + 2 * t->C;
        CUDA_TRY(cudaMemsetAsync(at.tile_counter, 0, sizeof(unsigned), t->stream));
        const int gt = std::max(1, std::min(t->grid_totals, (a.ntiles + 7) / 8));
        if (t->smem_totals) dev::k_topic_totals<true><<<gt, 256, t->smem_totals, t->stream>>>(at);
        else dev::k_topic_totals<false><<<gt, 256, 0, t->stream>>>(at);
        CUDA_TRY(cudaGetLastError());
    } else {
        const int grid = std::max(1, std::min(t->grid_wt, (a.ntiles + t->warps_wt - 1) / t->warps_wt));
        dev::k_wt_build<true><<<grid, 32 * t->warps_wt, t->smem_wt, t->stream>>>(a);
        CUDA_TRY(cudaGetLastError());
    }
    t->end_stage();
    return LDA_OK;
}

extern "C" int lda_max_topic(lda_trainer* t) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    CUDA_TRY(cudaSetDevice(t->device));
    t->begin_stage(1);
    dev::StatsArgs a = stats_args(t);
    if (t->w_tiles_rng) {
        // a word range: its words' statistics only
        a.wlo = t->wt_lo;
        a.V = t->wt_hi;
    }
    if (!t->large) {
        if (a.V > a.wlo) {
            const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(t->grid_stats, (a.V - a.wlo + t->warps - 1) / t->warps));
            dev::k_word_stats<<<grid, 32 * t->warps, t->smem_stats, t->stream>>>(a);
            CUDA_TRY(cudaGetLastError());
        }
    } else {
        // the sweep's reciprocals (the sparse-word statistics and the dense-word sampler's
        // column builds read them), the smoothing table of the sparse words' split Q bucket,
        // then dense words from their count rows, sparse words from their entries
        dev::k_recip<<<(t->K + 255) / 256, 256, 0, t->stream>>>(t->n_k, t->K, t->Vbeta, t->recip);
        CUDA_TRY(cudaGetLastError());
        dev::k_smooth_table<<<1, 1024, 0, t->stream>>>(t->n_k, t->K, t->Vbeta, t->alpha, t->beta, t->smooth);
        CUDA_TRY(cudaGetLastError());
        dev::StatsArgs ad = a;
        ad.V = std::min(a.V, t->Vd);
        ad.qtab = t->qtab_g;
        ad.qrounds = t->qrounds;
        if (ad.V > ad.wlo) {
            const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(t->grid_stats_dense, (ad.V - ad.wlo + 7) / 8));
            dev::k_word_stats_dense_rows<<<grid, 256, (size_t)t->K * 4, t->stream>>>(ad);
            CUDA_TRY(cudaGetLastError());
        }
        if (a.V > std::max(t->Vd, a.wlo)) {
            // sparse words: the topic order once, then warp per word from the global reciprocals
            dev::StatsArgs as = a;
            as.recip = t->recip;
            as.order = t->order;
            dev::k_sparse_order<<<1, 256, 0, t->stream>>>(as, t->order);
            CUDA_TRY(cudaGetLastError());
            const int64_t ns = a.V - std::max(t->Vd, a.wlo);
            const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(t->grid_stats_sparse, (ns + kLargeWarps - 1) / kLargeWarps));
            dev::k_word_stats_sparse_large<<<grid, 32 * kLargeWarps, t->smem_stats_sparse, t->stream>>>(as);
            CUDA_TRY(cudaGetLastError());
        }
    }
    t->end_stage();
    return LDA_OK;
}

// Buffers holding a chunk's per-token arrays and doc rows: the resident arrays, or the
// chunk's slot when streaming.
struct ChunkBufs {
    const uint32_t *tok_doc, *dtok_pos, *dtok_word;
    uint32_t *meta, *dt_ent;
    uint32_t tok_base, dt_base;
};

static ChunkBufs chunk_bufs(const lda_trainer* t, int chunk, int slot) {
    ChunkBufs b;
    if (!t->streaming) {
        b.tok_doc = t->tok_doc; b.dtok_pos = t->dtok_pos; b.dtok_word = t->dtok_word;
        b.meta = t->meta; b.dt_ent = t->dt_ent;
        b.tok_base = b.dt_base = 0;
    } else {
        const auto& sl = t->slots[slot];
        b.tok_doc = sl.tok_doc; b.dtok_pos = sl.dtok_pos; b.dtok_word = sl.dtok_word;
        b.meta = sl.meta; b.dt_ent = sl.dt_ent;
        b.tok_base = (uint32_t)t->chunk_tok[chunk];
        b.dt_base = (uint32_t)t->chunk_dt[chunk];
    }
    return b;
}

// Streaming: copies a chunk's static per-token arrays into its slot on stream `q`.
static int load_chunk(lda_trainer* t, int chunk, int slot, cudaStream_t q) {
    auto& sl = t->slots[slot];
    const int64_t t0 = t->chunk_tok[chunk], n = t->chunk_tok[chunk + 1] - t0;
    if (n > 0) {
        const size_t nb = sizeof(uint32_t) * (size_t)n;
        CUDA_TRY(cudaMemcpyAsync(sl.tok_doc, t->h_tok_doc + t0, nb, cudaMemcpyHostToDevice, q));
        CUDA_TRY(cudaMemcpyAsync(sl.dtok_pos, t->h_dtok_pos + t0, nb, cudaMemcpyHostToDevice, q));
        CUDA_TRY(cudaMemcpyAsync(sl.dtok_word, t->h_dtok_word + t0, nb, cudaMemcpyHostToDevice, q));
        t->h2d_bytes += 3 * (int64_t)nb;
    }
    sl.chunk = chunk;
    return LDA_OK;
}

static dev::DtArgs dt_args(const lda_trainer* t, int chunk, int slot) {
    const ChunkBufs b = chunk_bufs(t, chunk, slot);
    dev::DtArgs a;
    a.d_begin = (uint32_t)t->chunk_doc[chunk]; a.d_end = (uint32_t)t->chunk_doc[chunk + 1]; a.K = t->K;
    a.doc_off = t->doc_off; a.dtok_pos = b.dtok_pos; a.dtok_word = b.dtok_word; a.z = t->z;
    a.st_top2 = t->st_top2; a.dt_off = t->dt_off; a.dt_nnz = t->dt_nnz; a.dt_ent = b.dt_ent; a.meta = b.meta;
    a.err = t->err;
    a.tok_base = b.tok_base;
    a.dt_base = b.dt_base;
    return a;
}

// The doc-topic rebuild of docs [a.d_begin, a.d_end): warp per doc, or above kLargeK
// topics CTA per doc.
static int launch_dt(const lda_trainer* t, const dev::DtArgs& a, cudaStream_t q) {
    const int64_t nd = a.d_end - a.d_begin;
    if (t->large) {
        // docs of at most kSmallDoc tokens warp per doc, longer ones CTA per doc
        dev::DtArgs as = a;
        as.small_max = t->grid_dt_small > 0 ? (uint32_t)dev::kSmallDoc : 0u;
        if (as.small_max) {
            const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(t->grid_dt_small, (nd + 7) / 8));
            dev::k_dt_build_small<<<grid, 256, t->smem_dt_small, q>>>(as);
            CUDA_TRY(cudaGetLastError());
        }
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(t->grid_dt_cta, nd));
        dev::k_dt_build_cta<<<grid, dev::kRebuildThreads, t->smem_dt_cta, q>>>(as);
    } else {
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(t->grid_dt, (nd + t->warps_dt - 1) / t->warps_dt));
        dev::k_dt_build<true><<<grid, 32 * t->warps_dt, t->smem_dt, q>>>(a);
    }
    CUDA_TRY(cudaGetLastError());
    return LDA_OK;
}

static int dt_launch(lda_trainer* t, int chunk, int slot, cudaStream_t q) {
    return launch_dt(t, dt_args(t, chunk, slot), q);
}

static dev::SampleArgs sample_args(const lda_trainer* t, int chunk, int slot, int ll_mode) {
    const ChunkBufs b = chunk_bufs(t, chunk, slot);
    const int base = t->s_tile_base[chunk], n = t->s_tile_base[chunk + 1] - base;
    dev::SampleArgs a;
    a.tiles = t->s_tiles + base; a.ntiles = n; a.tile_counter = t->tile_ctr + 1 + chunk; a.tile_ll = t->tile_ll + base;
    a.K = t->K; a.Vd = t->Vd; a.ll_mode = ll_mode ? 1 : 0;
    a.alpha = t->alpha; a.beta = t->beta; a.Vbeta = t->Vbeta;
    a.den_add = (double)t->K * (double)t->alpha;
    a.seed_lo = (uint32_t)t->seed; a.seed_hi = (uint32_t)(t->seed >> 32); a.iter = t->iter;
    a.n_k = t->n_k; a.dwt = t->dwt; a.swt_off = t->swt_off; a.swt_nnz = t->swt_nnz; a.swt_ent = t->swt_ent;
    a.st_top2 = t->st_top2; a.st_phi = t->st_phi; a.st_ql = t->st_ql;
    a.tok_doc = b.tok_doc; a.meta = b.meta; a.z = t->z; a.doc_len = t->doc_len;
    a.dt_off = t->dt_off; a.dt_nnz = t->dt_nnz; a.dt_ent = b.dt_ent; a.ctr = t->ctr;
    a.smooth = t->smooth;
    a.qtab_g = t->qtab_g;
    a.tok_base = b.tok_base;
    a.dt_base = b.dt_base;
    a.recip = t->recip;
    return a;
}

static int sample_launch(lda_trainer* t, int chunk, int slot, int ll_mode, cudaStream_t q) {
    const dev::SampleArgs a = sample_args(t, chunk, slot, ll_mode);
    const int n = a.ntiles;
    if (t->large) {
        // dense-word tiles [base, split): one CTA each; sparse-word tiles [split, end)
        const int nd = t->s_tile_split[chunk] - t->s_tile_base[chunk], ns = n - nd;
        dev::SampleArgs ad = a, as = a;
        ad.ntiles = nd;
        as.tiles += nd;
        as.tile_ll += nd;
        as.ntiles = ns;
        as.tile_counter = t->tile_ctr + 1 + t->C + chunk;
        CUDA_TRY(cudaMemsetAsync(ad.tile_counter, 0, sizeof(unsigned), q));
        CUDA_TRY(cudaMemsetAsync(as.tile_counter, 0, sizeof(unsigned), q));
        const bool ll = ll_mode != 0;
        // the sparse-word sampler on the side stream of q, so that its CTAs start as the
        // dense-word kernel's CTAs run out of tiles (both read only this chunk's doc rows)
        lda_trainer::Side* side = nullptr;
        if (nd > 0 && ns > 0) {
            for (auto& s : t->sides)
                if (s.parent == q) side = &s;
            if (!side) {
                lda_trainer::Side s;
                s.parent = q;
                CUDA_TRY(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
                CUDA_TRY(cudaEventCreateWithFlags(&s.fork, cudaEventDisableTiming));
                CUDA_TRY(cudaEventCreateWithFlags(&s.join, cudaEventDisableTiming));
                t->sides.push_back(s);
                side = &t->sides.back();
            }
            CUDA_TRY(cudaEventRecord(side->fork, q));
            CUDA_TRY(cudaStreamWaitEvent(side->stream, side->fork, 0));
        }
        const cudaStream_t qs = side ? side->stream : q;
        if (nd > 0) {
            const int grid = std::max(1, std::min(t->grid_dense, nd));
            if (ll) dev::k_sample_dense_large<true, 4><<<grid, 32 * kLargeWarps, t->smem_dense, q>>>(ad);
            else dev::k_sample_dense_large<false, 4><<<grid, 32 * kLargeWarps, t->smem_dense, q>>>(ad);
            CUDA_TRY(cudaGetLastError());
        }
        if (ns > 0) {
            const int grid = std::max(1, std::min(t->grid_sparse, (ns + kLargeWarps - 1) / kLargeWarps));
            if (ll) dev::k_sample_sparse_large<true, 4><<<grid, 32 * kLargeWarps, t->smem_sparse, qs>>>(as);
            else dev::k_sample_sparse_large<false, 4><<<grid, 32 * kLargeWarps, t->smem_sparse, qs>>>(as);
            CUDA_TRY(cudaGetLastError());
        }
        if (side) {
            CUDA_TRY(cudaEventRecord(side->join, side->stream));
            CUDA_TRY(cudaStreamWaitEvent(q, side->join, 0));
        }
        t->chunk_sampled_ll[chunk] = ll;
        return LDA_OK;
    }
    CUDA_TRY(cudaMemsetAsync(a.tile_counter, 0, sizeof(unsigned), q));
    if (n > 0) {
        const int cap = a.ll_mode ? t->grid_sample_ll : t->grid_sample;
        const int grid = std::max(1, std::min(cap, (n + t->swarps - 1) / t->swarps));
        launch_sample(a.ll_mode != 0, t->K, grid, 32 * t->swarps, t->smem_sample, q, a);
        CUDA_TRY(cudaGetLastError());
    }
    t->chunk_sampled_ll[chunk] = ll_mode != 0;
    return LDA_OK;
}

// Resident chunks [c0, c1) in one doc-topic rebuild launch and one sampler launch (the
// chunks' docs and tiles are contiguous; up to kLargeK topics, one launch samples them all).
static int dt_launch_group(lda_trainer* t, int c0, int c1, cudaStream_t q) {
    dev::DtArgs a = dt_args(t, c0, 0);
    a.d_end = (uint32_t)t->chunk_doc[c1];
    return launch_dt(t, a, q);
}

static int sample_launch_group(lda_trainer* t, int c0, int c1, int ll_mode, cudaStream_t q) {
    int rc;
    if (t->large || c1 - c0 == 1) {
        for (int ch = c0; ch < c1; ++ch)
            if ((rc = sample_launch(t, ch, 0, ll_mode, q))) return rc;
        return LDA_OK;
    }
    dev::SampleArgs a = sample_args(t, c0, 0, ll_mode);
    a.ntiles = t->s_tile_base[c1] - t->s_tile_base[c0];
    CUDA_TRY(cudaMemsetAsync(a.tile_counter, 0, sizeof(unsigned), q));
    if (a.ntiles > 0) {
        const int cap = a.ll_mode ? t->grid_sample_ll : t->grid_sample;
        const int grid = std::max(1, std::min(cap, (a.ntiles + t->swarps - 1) / t->swarps));
        launch_sample(a.ll_mode != 0, t->K, grid, 32 * t->swarps, t->smem_sample, q, a);
        CUDA_TRY(cudaGetLastError());
    }
    for (int ch = c0; ch < c1; ++ch) t->chunk_sampled_ll[ch] = ll_mode != 0;
    return LDA_OK;
}

extern "C" int lda_update_dt(lda_trainer* t, int32_t chunk) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    if (chunk < 0 || chunk >= t->C) return fail(LDA_ERR_ARG, "chunk %d of %d", chunk, t->C);
    CUDA_TRY(cudaSetDevice(t->device));
    int rc;
    const int slot = t->streaming ? chunk % (int)t->slots.size() : 0;
    if (t->streaming) {
        t->begin_stage(5);
        if ((rc = load_chunk(t, chunk, slot, t->stream))) return rc;
        t->end_stage();
    }
    t->begin_stage(2);
    if ((rc = dt_launch(t, chunk, slot, t->stream))) return rc;
    t->end_stage();
    return LDA_OK;
}

extern "C" int lda_sample_chunk(lda_trainer* t, int32_t chunk, int32_t ll_mode) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    if (chunk < 0 || chunk >= t->C) return fail(LDA_ERR_ARG, "chunk %d of %d", chunk, t->C);
    const int slot = t->streaming ? chunk % (int)t->slots.size() : 0;
    if (t->streaming && t->slots[slot].chunk != chunk)
        return fail(LDA_ERR_STATE, "chunk %d is not loaded (run lda_update_dt for it first)", chunk);
    CUDA_TRY(cudaSetDevice(t->device));
    t->begin_stage(3);
    int rc = sample_launch(t, chunk, slot, ll_mode, t->stream);
    if (rc) return rc;
    t->end_stage();
    return LDA_OK;
}

static int perplexity_async(lda_trainer* t) {
    t->begin_stage(4);
    const int base = t->s_tile_base[t->chunk_first], n = t->s_tile_base[t->chunk_last] - base;
    dev::k_ll_reduce<<<1, 1024, 0, t->stream>>>(t->tile_ll + base, n, t->ll_dev);
    CUDA_TRY(cudaGetLastError());
    t->end_stage();
    CUDA_TRY(cudaMemcpyAsync(t->ll_host, t->ll_dev, sizeof(double), cudaMemcpyDeviceToHost, t->stream));
    return LDA_OK;
}

static int finish(lda_trainer* t) {
    CUDA_TRY(cudaStreamSynchronize(t->stream));
    t->collect_timing();
    int herr = 0;
    CUDA_TRY(cudaMemcpy(&herr, t->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) {
        CUDA_TRY(cudaMemset(t->err, 0, sizeof(int)));
        return fail(LDA_ERR_DEVICE, "a kernel found a topic >= K=%d in the topic array (the tokens were skipped)", t->K);
    }
    return LDA_OK;
}

extern "C" int lda_perplexity(lda_trainer* t, double* ll_sum) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    for (int ch = t->chunk_first; ch < t->chunk_last; ++ch)
        if (!t->chunk_sampled_ll[ch]) return fail(LDA_ERR_STATE, "chunk %d was not sampled with ll_mode=1", ch);
    CUDA_TRY(cudaSetDevice(t->device));
    int rc = perplexity_async(t);
    if (rc) return rc;
    if ((rc = finish(t))) return rc;
    t->last_ll = *t->ll_host;
    t->last_ll_tokens = t->range_tokens();
    t->ll_valid = true;
    if (ll_sum) *ll_sum = t->last_ll;
    return LDA_OK;
}

extern "C" int lda_end_sweep(lda_trainer* t) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    t->iter++;
    return LDA_OK;
}

extern "C" int lda_trainer_sync(lda_trainer* t) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    CUDA_TRY(cudaSetDevice(t->device));
    return finish(t);
}

// Copies chunk ch's new topics to host buffer zout on the copy stream once the work
// queued so far on stream q (the chunk's sampling) has finished.
static int copy_back(lda_trainer* t, int ch, cudaStream_t q, uint16_t* zout) {
    const int64_t t0 = t->chunk_tok[ch], n = t->chunk_tok[ch + 1] - t0;
    if (n <= 0) return LDA_OK;
    CUDA_TRY(cudaEventRecord(t->ev_chunk, q));
    CUDA_TRY(cudaStreamWaitEvent(t->copy_stream, t->ev_chunk, 0));
    CUDA_TRY(cudaMemcpyAsync(zout + t0, t->z + t0, sizeof(uint16_t) * (size_t)n, cudaMemcpyDeviceToHost, t->copy_stream));
    if (t->record_down) CUDA_TRY(cudaEventRecord(t->ev_down[ch], t->copy_stream));
    return LDA_OK;
}

// One sweep: the word side (rebuild + statistics) unless the caller has made it current,
// then the chunk range's doc-row rebuilds and sampling, and the sweep's LL.
static int sweep_async(lda_trainer* t, int ll_mode, uint16_t* zout = nullptr, bool word_side_done = false) {
    int rc;
    if (!word_side_done) {
        if (t->w_tiles_rng)
            return fail(LDA_ERR_STATE, "a word range is set: the caller completes the word side and calls lda_trainer_sweep_chunks");
        if ((rc = lda_update_wt(t))) return rc;
        if ((rc = lda_max_topic(t))) return rc;
    }
    // Resident sweeps without host copies take the chunk range in two groups up to kLargeK
    // topics: a group's chunks share one rebuild launch and one sampler launch, so the
    // sampler drains its tail twice per sweep instead of once per chunk (the K=1024 corpus,
    // 8 chunks: 13.51 -> 13.38 ms per sweep; one group of all 8 took 13.78 ms, its
    // rebuild's topics and rows no longer fitting in L2).  Above kLargeK a chunk's rows
    // alone nearly fill L2, and with host copies each chunk's copy waits for its sampling
    // only, so those keep one chunk per launch.
    const int cpl = (zout || t->large) ? 1 : std::max(1, (t->chunk_last - t->chunk_first + 1) / 2);
    if (!t->streaming && (t->timing || t->chunk_last - t->chunk_first < 2 || t->large)) {
        // one stream, so that the stage events time each stage alone.  Resident sweeps above
        // kLargeK topics take this path too: a chunk's doc rows (about 120 MB on the
        // K=10,000 corpus) nearly fill L2, and a second chunk's rebuild and sampling beside
        // them evict the rows the first chunk's sampler reads (that corpus: 131.5 -> 127.5
        // ms per sweep on one stream).
        for (int c0 = t->chunk_first; c0 < t->chunk_last; c0 += cpl) {
            const int c1 = std::min(t->chunk_last, c0 + cpl);
            t->begin_stage(2);
            if ((rc = dt_launch_group(t, c0, c1, t->stream))) return rc;
            t->end_stage();
            t->begin_stage(3);
            if ((rc = sample_launch_group(t, c0, c1, ll_mode, t->stream))) return rc;
            t->end_stage();
            for (int ch = c0; ch < c1; ++ch)
                if (zout && (rc = copy_back(t, ch, t->stream, zout))) return rc;
        }
    } else if (!t->streaming) {
        // chunk i of the range on work stream i mod 2: the next chunk's doc-topic rebuild
        // fills the tail of this chunk's sampling, and the samplings' tails overlap.  Chunks
        // are independent within a sweep (each reads and writes only its own tokens' topics
        // and doc rows).
        if (!t->work[0]) {
            for (int i = 0; i < 2; ++i) {
                CUDA_TRY(cudaStreamCreateWithFlags(&t->work[i], cudaStreamNonBlocking));
                CUDA_TRY(cudaEventCreateWithFlags(&t->ev_join[i], cudaEventDisableTiming));
            }
            CUDA_TRY(cudaEventCreateWithFlags(&t->ev_fork, cudaEventDisableTiming));
        }
        CUDA_TRY(cudaEventRecord(t->ev_fork, t->stream));
        for (int i = 0; i < 2; ++i) CUDA_TRY(cudaStreamWaitEvent(t->work[i], t->ev_fork, 0));
        for (int c0 = t->chunk_first; c0 < t->chunk_last; c0 += cpl) {
            const int c1 = std::min(t->chunk_last, c0 + cpl);
            cudaStream_t q = t->work[((c0 - t->chunk_first) / cpl) & 1];
            if ((rc = dt_launch_group(t, c0, c1, q))) return rc;
            if ((rc = sample_launch_group(t, c0, c1, ll_mode, q))) return rc;
            for (int ch = c0; ch < c1; ++ch)
                if (zout && (rc = copy_back(t, ch, q, zout))) return rc;
        }
        for (int i = 0; i < 2; ++i) {
            CUDA_TRY(cudaEventRecord(t->ev_join[i], t->work[i]));
            CUDA_TRY(cudaStreamWaitEvent(t->stream, t->ev_join[i], 0));
        }
    } else if (t->large) {
        // Above kLargeK topics the chunks are rebuilt and sampled one after another on the
        // trainer's stream (a chunk's rows nearly fill L2, as in resident sweeps).  One slot
        // stream copies, in sampling order, each chunk that no slot holds into the slot
        // whose chunk is needed latest (or not again in this sweep), as soon as that
        // chunk's sampling has ended.  Sweeps alternate the chunk order, so the chunks left
        // in the slots by one sweep are the first the next one samples, with no copy.
        const int S = (int)t->slots.size();
        const int n = t->chunk_last - t->chunk_first;
        const bool down = t->stream_down;
        auto chunk_at = [&](int i) { return down ? t->chunk_last - 1 - i : t->chunk_first + i; };
        cudaStream_t cq = t->sstreams[0];
        CUDA_TRY(cudaEventRecord(t->ev_ready, t->stream));
        CUDA_TRY(cudaStreamWaitEvent(cq, t->ev_ready, 0));
        std::vector<int> used_at(S, -1);  // order position of the slot's last sampling in this sweep
        for (int i = 0; i < n; ++i) {
            const int ch = chunk_at(i);
            int slot = -1;
            for (int k = 0; k < S; ++k)
                if (t->slots[k].chunk == ch) slot = k;
            if (slot < 0) {
                // the slot whose chunk comes latest in the rest of the order (never: n),
                // ties to the one sampled longest ago
                int best_next = -1;
                for (int k = 0; k < S; ++k) {
                    const int held = t->slots[k].chunk;
                    int next = n;
                    if (held >= t->chunk_first && held < t->chunk_last) {
                        const int pos = down ? t->chunk_last - 1 - held : held - t->chunk_first;
                        if (pos > i) next = pos;
                    }
                    if (next > best_next || (next == best_next && used_at[k] < used_at[slot])) {
                        best_next = next;
                        slot = k;
                    }
                }
                if (used_at[slot] >= 0) CUDA_TRY(cudaStreamWaitEvent(cq, t->ev_used[slot], 0));
                if ((rc = load_chunk(t, ch, slot, cq))) return rc;
                CUDA_TRY(cudaEventRecord(t->ev_slot[slot], cq));
                CUDA_TRY(cudaStreamWaitEvent(t->stream, t->ev_slot[slot], 0));
            }
            t->begin_stage(2);
            if ((rc = dt_launch(t, ch, slot, t->stream))) return rc;
            t->end_stage();
            t->begin_stage(3);
            if ((rc = sample_launch(t, ch, slot, ll_mode, t->stream))) return rc;
            t->end_stage();
            if (zout && (rc = copy_back(t, ch, t->stream, zout))) return rc;
            CUDA_TRY(cudaEventRecord(t->ev_used[slot], t->stream));
            used_at[slot] = i;
        }
        t->stream_down = !down;
    } else {
        // chunk i of the range goes to slot / stream i mod S: its copy overlaps the
        // rebuild and sampling of the chunks on the other streams; a slot is reused in
        // stream order.  Chunks are independent within a sweep (each rebuilds its own doc
        // rows from its own topics and writes only its own topics).
        const int S = (int)t->slots.size();
        t->begin_stage(3);
        CUDA_TRY(cudaEventRecord(t->ev_ready, t->stream));
        for (int i = 0; i < S; ++i) CUDA_TRY(cudaStreamWaitEvent(t->sstreams[i], t->ev_ready, 0));
        for (int ch = t->chunk_first; ch < t->chunk_last; ++ch) {
            const int slot = (ch - t->chunk_first) % S;
            cudaStream_t q = t->sstreams[slot];
            if ((rc = load_chunk(t, ch, slot, q))) return rc;
            if ((rc = dt_launch(t, ch, slot, q))) return rc;
            if ((rc = sample_launch(t, ch, slot, ll_mode, q))) return rc;
            if (zout && (rc = copy_back(t, ch, q, zout))) return rc;
        }
        for (int i = 0; i < S; ++i) {
            CUDA_TRY(cudaEventRecord(t->ev_slot[i], t->sstreams[i]));
            CUDA_TRY(cudaStreamWaitEvent(t->stream, t->ev_slot[i], 0));
        }
        t->end_stage();
    }
    if (ll_mode && (rc = perplexity_async(t))) return rc;
    t->iter++;
    return LDA_OK;
}

extern "C" int lda_trainer_iterate(lda_trainer* t, int32_t n, int32_t ll_mode) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    if (n < 0) return fail(LDA_ERR_ARG, "negative iteration count");
    CUDA_TRY(cudaSetDevice(t->device));
    for (int i = 0; i < n; ++i) {
        int rc = sweep_async(t, ll_mode);
        if (rc) return rc;
    }
    int rc = finish(t);
    if (rc) return rc;
    if (ll_mode && n > 0) {
        t->last_ll = *t->ll_host;
        t->last_ll_tokens = t->range_tokens();
        t->ll_valid = true;
    }
    return LDA_OK;
}

extern "C" int lda_trainer_sweep_chunks(lda_trainer* t, int32_t ll_mode) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    CUDA_TRY(cudaSetDevice(t->device));
    int rc = sweep_async(t, ll_mode, nullptr, true);
    if (rc) return rc;
    if ((rc = finish(t))) return rc;
    if (ll_mode) {
        t->last_ll = *t->ll_host;
        t->last_ll_tokens = t->range_tokens();
        t->ll_valid = true;
    }
    return LDA_OK;
}

extern "C" int lda_iterate_host(lda_trainer* t, const uint16_t* zin, uint16_t* zout, int32_t ll_mode, double* ll_sum) {
    if (!t || !zin || !zout) return fail(LDA_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(t->device));
    t->begin_stage(5);
    CUDA_TRY(cudaMemcpyAsync(t->z, zin, sizeof(uint16_t) * (size_t)t->N, cudaMemcpyHostToDevice, t->stream));
    t->end_stage();
    if (!t->copy_stream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&t->copy_stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&t->ev_chunk, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&t->ev_copied, cudaEventDisableTiming));
    }
    // A pinned output buffer gets each chunk's topics as soon as the chunk is sampled; a
    // device-to-host copy into pageable memory would block the host, so there the topics
    // come back in one copy after the sweep.
    cudaPointerAttributes pa{};
    const bool pinned = cudaPointerGetAttributes(&pa, zout) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();
    int rc;
    if (pinned) {
        // topics outside the sampled chunk range come back unchanged
        const int64_t r0 = t->chunk_tok[t->chunk_first], r1 = t->chunk_tok[t->chunk_last];
        if (r0 > 0) std::memcpy(zout, zin, sizeof(uint16_t) * (size_t)r0);
        if (r1 < t->N) std::memcpy(zout + r1, zin + r1, sizeof(uint16_t) * (size_t)(t->N - r1));
        if ((rc = sweep_async(t, ll_mode, zout))) return rc;
        // the sweep is complete when the last chunk's copy has landed
        CUDA_TRY(cudaEventRecord(t->ev_copied, t->copy_stream));
        CUDA_TRY(cudaStreamWaitEvent(t->stream, t->ev_copied, 0));
    } else {
        if ((rc = sweep_async(t, ll_mode))) return rc;
        t->begin_stage(5);
        CUDA_TRY(cudaMemcpyAsync(zout, t->z, sizeof(uint16_t) * (size_t)t->N, cudaMemcpyDeviceToHost, t->stream));
        t->end_stage();
    }
    if ((rc = finish(t))) return rc;
    if (ll_mode) {
        t->last_ll = *t->ll_host;
        t->last_ll_tokens = t->range_tokens();
        t->ll_valid = true;
        if (ll_sum) *ll_sum = t->last_ll;
    }
    return LDA_OK;
}

static int make_host_copy_stream(lda_trainer* t) {
    if (!t->copy_stream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&t->copy_stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&t->ev_chunk, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&t->ev_copied, cudaEventDisableTiming));
    }
    return LDA_OK;
}

extern "C" int lda_iterate_host_async(lda_trainer* t, const uint16_t* zin, uint16_t* zout) {
    if (!t || !zin || !zout) return fail(LDA_ERR_ARG, "null argument");
    if (zin == zout) return fail(LDA_ERR_ARG, "topics_in and topics_out must be different buffers");
    if (t->timing) return fail(LDA_ERR_STATE, "stage timing is on (it serialises the stages); use lda_iterate_host");
    CUDA_TRY(cudaSetDevice(t->device));
    for (const void* p : {(const void*)zin, (const void*)zout}) {
        cudaPointerAttributes pa{};
        const bool pinned = cudaPointerGetAttributes(&pa, p) == cudaSuccess && pa.type == cudaMemoryTypeHost;
        cudaGetLastError();
        if (!pinned) return fail(LDA_ERR_ARG, "lda_iterate_host_async needs pinned host buffers (cudaHostAlloc / cudaHostRegister)");
    }
    int rc;
    if ((rc = make_host_copy_stream(t))) return rc;
    if (!t->up_stream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&t->up_stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&t->ev_up, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&t->ev_tail, cudaEventDisableTiming));
        t->ev_down.assign(t->C, nullptr);
        for (auto& e : t->ev_down) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    // Chained: topics_in is the previous asynchronous sweep's topics_out, over the same
    // chunk range, and nothing else was enqueued since.  Chunk c's upload then waits only for that sweep's download of
    // chunk c (chunks read and write only their own tokens' topics; the word-topic rebuild,
    // which reads them all, ran first).  Otherwise it waits for all enqueued work.
    const bool chained = zin == t->last_out && t->stage_seq == t->last_seq && t->chunk_first == t->last_first &&
                         t->chunk_last == t->last_last;
    if (!chained) {
        CUDA_TRY(cudaEventRecord(t->ev_tail, t->stream));
        CUDA_TRY(cudaStreamWaitEvent(t->up_stream, t->ev_tail, 0));
        CUDA_TRY(cudaEventRecord(t->ev_copied, t->copy_stream));
        CUDA_TRY(cudaStreamWaitEvent(t->up_stream, t->ev_copied, 0));
    }
    // topics outside the sampled chunk range come back unchanged
    const int64_t r0 = t->chunk_tok[t->chunk_first], r1 = t->chunk_tok[t->chunk_last];
    if (r0 > 0) std::memcpy(zout, zin, sizeof(uint16_t) * (size_t)r0);
    if (r1 < t->N) std::memcpy(zout + r1, zin + r1, sizeof(uint16_t) * (size_t)(t->N - r1));
    for (int ch = t->chunk_first; ch < t->chunk_last; ++ch) {
        const int64_t t0 = t->chunk_tok[ch], n = t->chunk_tok[ch + 1] - t0;
        if (n <= 0) continue;
        if (chained) CUDA_TRY(cudaStreamWaitEvent(t->up_stream, t->ev_down[ch], 0));
        CUDA_TRY(cudaMemcpyAsync(t->z + t0, zin + t0, sizeof(uint16_t) * (size_t)n, cudaMemcpyHostToDevice, t->up_stream));
    }
    CUDA_TRY(cudaEventRecord(t->ev_up, t->up_stream));
    CUDA_TRY(cudaStreamWaitEvent(t->stream, t->ev_up, 0));
    t->record_down = true;
    rc = sweep_async(t, 0, zout);
    t->record_down = false;
    t->copies_pending = true;  // also on failure: some downloads may be enqueued
    if (rc) return rc;
    t->ll_valid = false;
    t->last_out = zout;
    t->last_seq = t->stage_seq;
    t->last_first = t->chunk_first;
    t->last_last = t->chunk_last;
    return LDA_OK;
}

extern "C" int lda_trainer_wait(lda_trainer* t) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    CUDA_TRY(cudaSetDevice(t->device));
    if (t->up_stream) CUDA_TRY(cudaStreamSynchronize(t->up_stream));
    if (t->copy_stream) CUDA_TRY(cudaStreamSynchronize(t->copy_stream));
    t->copies_pending = false;
    return finish(t);
}

extern "C" int lda_trainer_loglik(lda_trainer* t, double* ll, int64_t* n) {
    if (!t || !ll) return fail(LDA_ERR_ARG, "null argument");
    if (!t->ll_valid) return fail(LDA_ERR_STATE, "no log-likelihood has been evaluated (run a sweep with ll_mode=1)");
    *ll = t->last_ll;
    if (n) *n = t->last_ll_tokens;
    return LDA_OK;
}

extern "C" int lda_trainer_get_topics(lda_trainer* t, uint16_t* out, int64_t count) {
    if (!t || !out || count != t->N) return fail(LDA_ERR_ARG, "bad output buffer (need %lld topics)", (long long)(t ? t->N : 0));
    CUDA_TRY(cudaSetDevice(t->device));
    CUDA_TRY(cudaStreamSynchronize(t->stream));
    CUDA_TRY(cudaMemcpy(out, t->z, sizeof(uint16_t) * (size_t)count, cudaMemcpyDeviceToHost));
    return LDA_OK;
}

extern "C" int lda_trainer_set_topics(lda_trainer* t, const uint16_t* in, int64_t count) {
    if (!t || !in || count != t->N) return fail(LDA_ERR_ARG, "bad input buffer (need %lld topics)", (long long)(t ? t->N : 0));
    for (int64_t i = 0; i < count; ++i)
        if (in[i] >= t->K) return fail(LDA_ERR_ARG, "topic %d of token %lld >= K=%d", in[i], (long long)i, t->K);
    CUDA_TRY(cudaSetDevice(t->device));
    CUDA_TRY(cudaStreamSynchronize(t->stream));
    if (t->copy_stream) CUDA_TRY(cudaStreamSynchronize(t->copy_stream));
    t->copies_pending = false;
    CUDA_TRY(cudaMemcpy(t->z, in, sizeof(uint16_t) * (size_t)count, cudaMemcpyHostToDevice));
    return LDA_OK;
}

extern "C" int lda_trainer_get_iteration(const lda_trainer* t, uint32_t* it) {
    if (!t || !it) return fail(LDA_ERR_ARG, "null argument");
    *it = t->iter;
    return LDA_OK;
}

extern "C" int lda_trainer_set_iteration(lda_trainer* t, uint32_t it) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    t->iter = it;
    return LDA_OK;
}

extern "C" int lda_trainer_counters(lda_trainer* t, lda_sweep_counters* o) {
    if (!t || !o) return fail(LDA_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(t->device));
    CUDA_TRY(cudaStreamSynchronize(t->stream));
    unsigned long long h[kCounters];
    CUDA_TRY(cudaMemcpy(h, t->ctr, sizeof(h), cudaMemcpyDeviceToHost));
    o->tokens = (int64_t)h[0]; o->early_accept = (int64_t)h[1]; o->full = (int64_t)h[2]; o->sum_nnz_full = (int64_t)h[3];
    o->branch_max = (int64_t)h[4]; o->branch_s = (int64_t)h[5]; o->branch_q = (int64_t)h[6]; o->sum_word_nnz = (int64_t)h[7];
    o->word_tiles_dense = (int64_t)h[8]; o->word_tiles_sparse = (int64_t)h[9];
    o->rows_evaluated = (int64_t)h[10]; o->row_entries_read = (int64_t)h[11];
    return LDA_OK;
}

extern "C" int lda_trainer_reset_stats(lda_trainer* t) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    CUDA_TRY(cudaSetDevice(t->device));
    CUDA_TRY(cudaStreamSynchronize(t->stream));
    CUDA_TRY(cudaMemset(t->ctr, 0, sizeof(unsigned long long) * kCounters));
    t->collect_timing();
    t->tm = lda_stage_timing{};
    return LDA_OK;
}

extern "C" int lda_trainer_set_timing(lda_trainer* t, int32_t on) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    t->timing = on != 0;
    return LDA_OK;
}

extern "C" int lda_trainer_timing(lda_trainer* t, lda_stage_timing* o) {
    if (!t || !o) return fail(LDA_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(t->device));
    CUDA_TRY(cudaStreamSynchronize(t->stream));
    t->collect_timing();
    *o = t->tm;
    return LDA_OK;
}

// ---------------------------------------------------------------- checkpoint

namespace {
struct CkptHeader {
    char magic[8];
    uint32_t version, K;
    uint64_t N, seed;
    uint32_t iter, pad;
};
}  // namespace

extern "C" int lda_trainer_checkpoint(lda_trainer* t, const char* path) {
    if (!t || !path) return fail(LDA_ERR_ARG, "null argument");
    std::vector<uint16_t> z((size_t)t->N);
    int rc = lda_trainer_get_topics(t, z.data(), t->N);
    if (rc) return rc;
    CkptHeader h{};
    std::memcpy(h.magic, "LDAB200", 8);
    h.version = 1; h.K = (uint32_t)t->K; h.N = (uint64_t)t->N; h.seed = t->seed; h.iter = t->iter;
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(LDA_ERR_IO, "cannot open %s for writing", path);
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 && std::fwrite(z.data(), sizeof(uint16_t), z.size(), f) == z.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? LDA_OK : fail(LDA_ERR_IO, "short write to %s", path);
}

extern "C" int lda_trainer_restore(lda_trainer* t, const char* path) {
    if (!t || !path) return fail(LDA_ERR_ARG, "null argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(LDA_ERR_IO, "cannot open %s", path);
    CkptHeader h{};
    if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, "LDAB200", 8) != 0 || h.version != 1) {
        std::fclose(f);
        return fail(LDA_ERR_FORMAT, "%s is not a checkpoint of this library", path);
    }
    if (h.N != (uint64_t)t->N || h.K != (uint32_t)t->K) {
        std::fclose(f);
        return fail(LDA_ERR_FORMAT, "checkpoint holds N=%llu K=%u, trainer has N=%lld K=%d", (unsigned long long)h.N, h.K, (long long)t->N, t->K);
    }
    std::vector<uint16_t> z((size_t)t->N);
    const bool ok = std::fread(z.data(), sizeof(uint16_t), z.size(), f) == z.size();
    std::fclose(f);
    if (!ok) return fail(LDA_ERR_FORMAT, "%s is truncated", path);
    int rc = lda_trainer_set_topics(t, z.data(), t->N);
    if (rc) return rc;
    t->seed = h.seed;
    t->iter = h.iter;
    return LDA_OK;
}

// ---------------------------------------------------------------- readback

int lda::trainer_model_source(lda_trainer* t, ModelSource* o) {
    if (!t || !o) return fail(LDA_ERR_ARG, "null argument");
    o->device = t->device;
    o->K = t->K;
    o->Vd = t->Vd;
    o->V = t->V;
    o->alpha = t->alpha;
    o->beta = t->beta;
    o->n_k = t->n_k;
    o->dwt = t->dwt;
    o->swt_off = t->swt_off;
    o->swt_nnz = t->swt_nnz;
    o->swt_ent = t->swt_ent;
    o->top2 = t->st_top2;
    o->phi4 = t->st_phi;
    o->ql = t->st_ql;
    o->stream = t->stream;
    return LDA_OK;
}

int lda::trainer_view(lda_trainer* t, TrainerView* v) {
    if (!t || !v) return fail(LDA_ERR_ARG, "null argument");
    if (t->streaming) return fail(LDA_ERR_STATE, "a streaming trainer cannot join a batch");
    v->wt = wt_args(t);
    v->st = stats_args(t);
    v->dt = dt_args(t, 0, 0);
    v->dt.d_begin = 0;
    v->dt.d_end = (uint32_t)t->D;
    v->sm = sample_args(t, 0, 0, 0);
    v->sm.ntiles = t->s_tile_base[t->C];
    v->device = t->device;
    v->K = t->K;
    v->Vd = t->Vd;
    v->warps = t->warps;
    v->N = t->N;
    v->V = t->V;
    v->D = t->D;
    v->n_k = t->n_k;
    v->dwt = t->dwt;
    v->dwt_count = (int64_t)t->Vd * t->K;
    v->tile_ll = t->tile_ll;
    v->n_stiles = t->s_tile_base[t->C];
    v->n_wtiles = t->n_wtiles;
    v->s_tiles = t->h_stiles;
    v->w_tiles = t->h_wtiles;
    return LDA_OK;
}

int lda::trainer_note_sweeps(lda_trainer* t, int n, int ll_mode, double ll_sum) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    t->iter += (uint32_t)n;
    if (n > 0) {
        for (int ch = 0; ch < t->C; ++ch) t->chunk_sampled_ll[ch] = ll_mode != 0;
        if (ll_mode) {
            t->last_ll = ll_sum;
            t->last_ll_tokens = t->N;
            t->ll_valid = true;
        }
    }
    return LDA_OK;
}

extern "C" int lda_get_topic_totals(lda_trainer* t, int32_t* nk) {
    if (!t || !nk) return fail(LDA_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(t->device));
    CUDA_TRY(cudaStreamSynchronize(t->stream));
    CUDA_TRY(cudaMemcpy(nk, t->n_k, sizeof(int) * (size_t)t->K, cudaMemcpyDeviceToHost));
    return LDA_OK;
}

extern "C" int lda_get_dense_wt(lda_trainer* t, int32_t* out) {
    if (!t || !out) return fail(LDA_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(t->device));
    CUDA_TRY(cudaStreamSynchronize(t->stream));
    if (t->Vd > 0) CUDA_TRY(cudaMemcpy(out, t->dwt, sizeof(int) * (size_t)t->Vd * t->K, cudaMemcpyDeviceToHost));
    return LDA_OK;
}

extern "C" int64_t lda_get_sparse_wt(lda_trainer* t, int64_t* off, uint32_t* ent, int64_t cap) {
    if (!t || !off) return fail(LDA_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(t->device));
    CUDA_TRY(cudaStreamSynchronize(t->stream));
    const int64_t Vs = t->V - t->Vd;
    std::vector<uint32_t> hoff(std::max<int64_t>(Vs, 1)), hnnz(std::max<int64_t>(Vs, 1)), hent(std::max<int64_t>(t->swt_cap, 1));
    if (Vs > 0) {
        CUDA_TRY(cudaMemcpy(hoff.data(), t->swt_off, sizeof(uint32_t) * (size_t)Vs, cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(hnnz.data(), t->swt_nnz, sizeof(uint32_t) * (size_t)Vs, cudaMemcpyDeviceToHost));
    }
    if (t->swt_cap > 0) CUDA_TRY(cudaMemcpy(hent.data(), t->swt_ent, sizeof(uint32_t) * (size_t)t->swt_cap, cudaMemcpyDeviceToHost));
    int64_t n = 0;
    off[0] = 0;
    for (int64_t s = 0; s < Vs; ++s) {
        if (ent) {
            if (n + hnnz[s] > cap) return fail(LDA_ERR_ARG, "sparse WT buffer too small");
            std::memcpy(ent + n, hent.data() + hoff[s], sizeof(uint32_t) * hnnz[s]);
        }
        n += hnnz[s];
        off[s + 1] = n;
    }
    return n;
}

extern "C" int lda_get_word_stats(lda_trainer* t, uint32_t* top2, uint32_t* k3, float* phi4, float* ql) {
    if (!t) return fail(LDA_ERR_ARG, "null trainer");
    CUDA_TRY(cudaSetDevice(t->device));
    CUDA_TRY(cudaStreamSynchronize(t->stream));
    if (top2) CUDA_TRY(cudaMemcpy(top2, t->st_top2, sizeof(uint32_t) * (size_t)t->V, cudaMemcpyDeviceToHost));
    if (k3) CUDA_TRY(cudaMemcpy(k3, t->st_k3, sizeof(uint32_t) * (size_t)t->V, cudaMemcpyDeviceToHost));
    if (phi4) CUDA_TRY(cudaMemcpy(phi4, t->st_phi, sizeof(float4) * (size_t)t->V, cudaMemcpyDeviceToHost));
    if (ql) CUDA_TRY(cudaMemcpy(ql, t->st_ql, sizeof(float) * 32 * (size_t)t->V, cudaMemcpyDeviceToHost));
    return LDA_OK;
}

extern "C" int64_t lda_get_doc_rows(lda_trainer* t, int64_t* off, uint32_t* ent, int64_t cap) {
    if (t && t->streaming) return fail(LDA_ERR_STATE, "doc rows are not kept when the corpus is streamed");
    if (!t || !off) return fail(LDA_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(t->device));
    CUDA_TRY(cudaStreamSynchronize(t->stream));
    std::vector<uint32_t> hoff(t->D), hnnz(t->D), hent(std::max<int64_t>(t->dt_cap, 1));
    CUDA_TRY(cudaMemcpy(hoff.data(), t->dt_off, sizeof(uint32_t) * (size_t)t->D, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(hnnz.data(), t->dt_nnz, sizeof(uint32_t) * (size_t)t->D, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(hent.data(), t->dt_ent, sizeof(uint32_t) * (size_t)t->dt_cap, cudaMemcpyDeviceToHost));
    int64_t n = 0;
    off[0] = 0;
    for (int64_t d = 0; d < t->D; ++d) {
        if (ent) {
            if (n + hnnz[d] > cap) return fail(LDA_ERR_ARG, "doc-row buffer too small");
            const uint32_t* src = hent.data() + hoff[d];
            for (uint32_t j = 0; j < hnnz[d]; ++j) {
                // up to kLargeK topics the device rows carry word-column slot indices
                const uint32_t key = src[j] >> 16;
                const uint32_t k = t->K <= dev::kLargeK ? (uint32_t)dev::col_unskew((int)key) : key;
                ent[n + j] = (k << 16) | (src[j] & 0xffffu);
            }
        }
        n += hnnz[d];
        off[d + 1] = n;
    }
    return n;
}

extern "C" int lda_get_token_meta(lda_trainer* t, uint32_t* meta) {
    if (t && t->streaming) return fail(LDA_ERR_STATE, "token metadata is not kept when the corpus is streamed");
    if (!t || !meta) return fail(LDA_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(t->device));
    CUDA_TRY(cudaStreamSynchronize(t->stream));
    CUDA_TRY(cudaMemcpy(meta, t->meta, sizeof(uint32_t) * (size_t)t->N, cudaMemcpyDeviceToHost));
    return LDA_OK;
}

// ------------------------------------------------------- allocation-free sampling
//
// lda_sample_chunk_noalloc runs the same k_sample / k_ll_reduce kernels on buffers the
// caller owns.  Its scratch lives in one file-scope device array: bytes [0,4) the tile
// counter, [8,136) the sweep counters, [256, 256 + 8*kNoAllocMaxTiles) the per-tile LL
// partials, then (K > 2048) the smoothing table of the split Q bucket, K floats.  In host
// code the symbol is only a host-side stand-in, so the device address is looked up once
// per device (with that device current) and cached.

namespace {
constexpr int kNoAllocMaxTiles = 65536;
constexpr size_t kNoAllocHeader = 256;
// above 2048 topics the split Q bucket's smoothing table (K floats) follows the LL partials;
// K is bounded below this by the sampler's shared memory anyway
constexpr int kNoAllocMaxK = 29696;
constexpr size_t kNoAllocSmooth = kNoAllocHeader + sizeof(double) * (size_t)kNoAllocMaxTiles;
constexpr size_t kNoAllocBytes = kNoAllocSmooth + sizeof(float) * (size_t)kNoAllocMaxK;
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_addr[kMaxDevices] = {};
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {
// What k_check_sample_io reads: the indices of an allocation-free call that the sampler
// would follow, with the lengths of the buffers they index.
struct IoCheck {
    const int4* tiles;
    int ntiles, K, V, Vd, D;
    const uint32_t* top2;
    const uint32_t* swt_off;
    const uint32_t* swt_nnz;
    const uint32_t* swt_ent;
    const uint32_t* tok_doc;
    const uint32_t* dt_off;
    const uint32_t* dt_nnz;
    const uint32_t* dt_ent;
    int64_t N, n_dt, n_sp;
    int* status;
    unsigned* tile_counter;
};
}  // namespace

// Range checks before an allocation-free sampling launch: warp per tile (its word, token
// range, the word's max topic and sparse row, its tokens' doc ids), thread per doc (its
// row's extent and topics).  A failure ORs LDA_IO_* bits into *status and moves the tile
// counter past any tile index, so the sampling kernel that follows on the stream takes no
// tile (its warps' first claim returns >= ntiles; the counter stays below 2^31).
__global__ void __launch_bounds__(256) k_check_sample_io(IoCheck c) {
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    int bad = 0;
    for (int t = gw; t < c.ntiles; t += nw) {
        const int4 tl = c.tiles[t];
        if (tl.x < 0 || tl.x >= c.V || tl.y < 0 || tl.z < 0 || (int64_t)tl.y + tl.z > c.N) {
            bad |= LDA_IO_TILE;
            continue;
        }
        const int w = tl.x;
        if ((c.top2[w] & 0xffffu) >= (uint32_t)c.K) bad |= LDA_IO_MAX_TOPIC;
        if (w >= c.Vd) {
            const int sw = w - c.Vd;
            const uint64_t off = c.swt_off[sw], nnz = c.swt_nnz[sw];
            if (off + nnz > (uint64_t)c.n_sp) {
                bad |= LDA_IO_WORD_ROW;
            } else {
                for (uint64_t e = (uint64_t)lane; e < nnz; e += 32u)
                    if ((c.swt_ent[off + e] >> 16) >= (uint32_t)c.K) bad |= LDA_IO_WORD_ROW;
            }
        }
        for (int i = lane; i < tl.z; i += 32)
            if (c.tok_doc[(int64_t)tl.y + i] >= (uint32_t)c.D) bad |= LDA_IO_TOKEN_DOC;
    }
    for (int d = (int)(blockIdx.x * blockDim.x + threadIdx.x); d < c.D; d += (int)(gridDim.x * blockDim.x)) {
        const uint64_t off = c.dt_off[d], nnz = c.dt_nnz[d];
        if (off + nnz > (uint64_t)c.n_dt) {
            bad |= LDA_IO_DOC_ROW;
            continue;
        }
        for (uint64_t e = 0; e < nnz; ++e) {
            if ((c.dt_ent[off + e] >> 16) >= (uint32_t)c.K) {
                bad |= LDA_IO_DOC_ROW;
                break;
            }
        }
    }
    if (bad) {
        atomicOr(c.status, bad);
        atomicExch(c.tile_counter, 1u << 30);
    }
}

static int noalloc_scratch(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return fail(LDA_ERR_ARG, "device %d out of range", device);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));  // `device` is current here
        g_noalloc_addr[device] = (unsigned char*)p;
    }
    *out = g_noalloc_addr[device];
    return LDA_OK;
}

extern "C" int lda_sample_chunk_noalloc(const lda_sample_io* io, int32_t device, void* stream_ptr) {
    if (!io) return fail(LDA_ERR_ARG, "null io");
    if (io->K < 4 || io->K > kNoAllocMaxK)
        return fail(LDA_ERR_ARG, "K=%d outside [4, %d] (the allocation-free limit)", io->K, kNoAllocMaxK);
    if (io->num_tiles < 0 || io->num_tiles > kNoAllocMaxTiles)
        return fail(LDA_ERR_ARG, "num_tiles=%d exceeds the allocation-free limit of %d tiles per call",
                    io->num_tiles, kNoAllocMaxTiles);
    if (io->vocab <= 0 || io->num_dense < 0 || io->num_dense > io->vocab)
        return fail(LDA_ERR_ARG, "bad vocab / num_dense");
    if (!(io->alpha > 0.f) || !(io->beta > 0.f)) return fail(LDA_ERR_ARG, "alpha and beta must be > 0");
    if (io->num_tiles > 0 &&
        (!io->tiles || !io->n_k || !io->top2 || !io->phi4 || !io->ql || !io->tok_doc || !io->meta || !io->topics ||
         !io->doc_len || !io->dt_off || !io->dt_nnz || !io->dt_ent || (io->num_dense > 0 && !io->dense_wt) ||
         (io->num_dense < io->vocab && (!io->sparse_off || !io->sparse_nnz || !io->sparse_ent)) ||
         (io->ll_mode && !io->ll_sum)))
        return fail(LDA_ERR_ARG, "null device buffer in lda_sample_io");
    if (((uintptr_t)io->tiles & 15u) || ((uintptr_t)io->dt_ent & 15u) || ((uintptr_t)io->phi4 & 15u))
        return fail(LDA_ERR_ARG, "tiles, phi4 and dt_ent must be 16-byte aligned");
    if (!io->status) return fail(LDA_ERR_ARG, "null status word in lda_sample_io");
    if (io->num_tokens < 0 || io->num_docs < 0 || io->num_dt_entries < 0 || io->num_sparse_entries < 0)
        return fail(LDA_ERR_ARG, "negative buffer length in lda_sample_io");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return fail(LDA_ERR_CUDA, "CUDA device %d not available", device);
    }
    CUDA_TRY(cudaSetDevice(device));
    unsigned char* scratch = nullptr;
    int rc = noalloc_scratch(device, &scratch);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream_ptr;
    CUDA_TRY(cudaMemsetAsync(scratch, 0, kNoAllocHeader, st));  // tile counter + sweep counters
    CUDA_TRY(cudaMemsetAsync(io->status, 0, sizeof(int32_t), st));
    if (io->num_tiles == 0) {
        if (io->ll_mode) CUDA_TRY(cudaMemsetAsync(io->ll_sum, 0, sizeof(double), st));
        return LDA_OK;
    }
    int max_smem = 0, num_sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    const int64_t row = (int64_t)io->K * 4;
    const int warps = (int)std::min<int64_t>(std::min(8, dev::kSampleWarps), ((int64_t)max_smem - 2048) / (row + 256) - 1);
    if (warps < 1) return fail(LDA_ERR_ARG, "K=%d does not fit in shared memory", io->K);
    const size_t smem = (size_t)io->K * 4 + (size_t)warps * (dev::col_words(io->K) * 4 + 16 * sizeof(uint32_t));
    if (warps < 1 || smem > (size_t)max_smem) return fail(LDA_ERR_ARG, "K=%d does not fit in shared memory", io->K);
    const void* kfn = sample_kernel(io->ll_mode != 0, io->K, false);
    CUDA_TRY(raise_smem_limit(kfn, smem));
    int grid = 0;
    if ((rc = occupancy_grid(kfn, 32 * warps, smem, num_sms, &grid))) return rc;
    grid = std::max(1, std::min(grid, (io->num_tiles + warps - 1) / warps));
    dev::SampleArgs a;
    a.tiles = reinterpret_cast<const int4*>(io->tiles);
    a.ntiles = io->num_tiles;
    a.tile_counter = reinterpret_cast<unsigned*>(scratch);
    a.tile_ll = reinterpret_cast<double*>(scratch + kNoAllocHeader);
    a.K = io->K; a.Vd = io->num_dense; a.ll_mode = io->ll_mode ? 1 : 0;
    a.alpha = io->alpha; a.beta = io->beta; a.Vbeta = (float)io->vocab * io->beta;
    a.den_add = (double)io->K * (double)io->alpha;
    a.seed_lo = (uint32_t)io->seed; a.seed_hi = (uint32_t)(io->seed >> 32); a.iter = io->iter;
    a.n_k = io->n_k; a.dwt = io->dense_wt;
    a.swt_off = io->sparse_off; a.swt_nnz = io->sparse_nnz; a.swt_ent = io->sparse_ent;
    a.st_top2 = io->top2; a.st_phi = reinterpret_cast<const float4*>(io->phi4); a.st_ql = io->ql;
    a.tok_doc = io->tok_doc; a.meta = io->meta; a.z = io->topics; a.doc_len = io->doc_len;
    a.dt_off = io->dt_off; a.dt_nnz = io->dt_nnz; a.dt_ent = io->dt_ent;
    a.ctr = reinterpret_cast<unsigned long long*>(scratch + 8);
    a.tok_base = 0;
    a.dt_base = 0;
    if (io->K > dev::kLargeK) {
        a.smooth = reinterpret_cast<const float*>(scratch + kNoAllocSmooth);
        dev::k_smooth_table<<<1, 1024, 0, st>>>(io->n_k, io->K, a.Vbeta, io->alpha, io->beta,
                                              reinterpret_cast<float*>(scratch + kNoAllocSmooth));
        CUDA_TRY(cudaGetLastError());
    }
    IoCheck chk;
    chk.tiles = a.tiles; chk.ntiles = io->num_tiles; chk.K = io->K; chk.V = io->vocab; chk.Vd = io->num_dense;
    chk.D = io->num_docs; chk.top2 = io->top2; chk.swt_off = io->sparse_off; chk.swt_nnz = io->sparse_nnz;
    chk.swt_ent = io->sparse_ent; chk.tok_doc = io->tok_doc; chk.dt_off = io->dt_off; chk.dt_nnz = io->dt_nnz;
    chk.dt_ent = io->dt_ent; chk.N = io->num_tokens; chk.n_dt = io->num_dt_entries;
    chk.n_sp = io->num_sparse_entries; chk.status = io->status; chk.tile_counter = a.tile_counter;
    k_check_sample_io<<<4 * num_sms, 256, 0, st>>>(chk);
    CUDA_TRY(cudaGetLastError());
    launch_sample(a.ll_mode != 0, io->K, grid, 32 * warps, smem, st, a, false);
    CUDA_TRY(cudaGetLastError());
    if (io->ll_mode) {
        dev::k_ll_reduce<<<1, 1024, 0, st>>>(a.tile_ll, io->num_tiles, io->ll_sum);
        CUDA_TRY(cudaGetLastError());
    }
    return LDA_OK;
}
