// batch.cu -- many independent corpora swept together: one work list per stage spanning
// every model, persistent kernels that take work from it, and the sweeps of a run
// captured as one CUDA graph.
//
// No counterpart in the reference: EZLDA trains one corpus per process.  A batch is built
// over resident trainers (one per corpus, each with its own K, alpha, beta, seed and
// device arrays); the batched kernels run the same per-unit bodies as the single-corpus
// kernels (sweep_body.cuh) with each model's arguments read from a device table, so every
// model's topics after a batched sweep are identical to its own trainer's.  Per-model
// state that a CTA would otherwise share (the reciprocal table, topic totals) is kept per
// warp or updated in global memory, because one CTA serves several models.
#include <algorithm>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

#include "launch_util.h"
#include "trainer_internal.h"

using namespace lda;

namespace lda {
namespace dev {

struct ZeroSeg {
    int* p;
    long long n;
};

struct BatchArgs {
    const WtArgs* wt;
    const StatsArgs* st;
    const DtArgs* dt;
    const SampleArgs* sm;
    const uint2* wt_work;  // {model, word tile}
    int n_wt;
    const uint4* st_work;  // {model, first word, words, 0}
    int n_st;
    const uint4* dt_work;  // {model, first doc, docs, 0}
    int n_dt;
    const uint2* sm_work;  // {model, sampler tile}
    int n_sm;
    unsigned* counters;    // [4] work counters of the stages, zeroed at the start of a sweep
    const uint32_t* sweeps_done;  // sweeps this batch has run, added to each model's base iteration
    int Kmax;
};

__device__ __forceinline__ int grab(unsigned* counter, int lane) {
    int i = 0;
    if (lane == 0) i = (int)atomicAdd(counter, 1u);
    return __shfl_sync(FULL, i, 0);
}

// Zeroes every model's topic totals and dense word-topic rows, and the stage counters.
__global__ void kb_zero(const ZeroSeg* segs, int nseg, unsigned* counters) {
    if (blockIdx.x == 0 && threadIdx.x < 4) counters[threadIdx.x] = 0u;
    for (int s = blockIdx.x; s < nseg; s += gridDim.x) {
        const ZeroSeg z = segs[s];
        for (long long i = threadIdx.x; i < z.n; i += blockDim.x) z.p[i] = 0;
    }
}

// Word-topic rebuild; topic totals go straight to each model's global n_k.
__global__ void __launch_bounds__(256) kb_wt(BatchArgs b) {
    extern __shared__ uint32_t smu[];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = b.Kmax + wt_bit_words(b.Kmax);
    uint32_t* hist = smu + (size_t)per * wid;
    uint32_t* bits = hist + b.Kmax;
    for (int k = lane; k < per; k += 32) hist[k] = 0u;
    __syncwarp();
    for (;;) {
        const int i = grab(b.counters + 0, lane);
        if (i >= b.n_wt) break;
        const uint2 w = b.wt_work[i];
        const WtArgs& a = b.wt[w.x];
        wt_tile(a, a.tiles[w.y], Hist<false>{hist}, bits, reinterpret_cast<unsigned*>(a.n_k), lane);
    }
}

// 1 / ((float)n_k + V*beta) of one model into a warp-private table.
__device__ __forceinline__ void warp_recip(float* r, const int* n_k, int K, float Vbeta, int lane) {
    __syncwarp();
    for (int k = lane; k < K; k += 32) r[k] = __fdiv_rn(1.0f, fadd(__int2float_rn(n_k[k]), Vbeta));
    __syncwarp();
}

__global__ void __launch_bounds__(256) kb_stats(BatchArgs b) {
    extern __shared__ float smf[];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* r = smf + (size_t)b.Kmax * 2 * wid;
    float* col = r + b.Kmax;
    int cur = -1;
    for (;;) {
        const int i = grab(b.counters + 1, lane);
        if (i >= b.n_st) break;
        const uint4 u = b.st_work[i];
        const StatsArgs& a = b.st[u.x];
        if ((int)u.x != cur) {
            cur = (int)u.x;
            warp_recip(r, a.n_k, a.K, a.Vbeta, lane);
        }
        for (uint32_t w = u.y; w < u.y + u.z; ++w) word_stats_word(a, (int)w, r, col, lane);
    }
}

__global__ void __launch_bounds__(256) kb_dt(BatchArgs b) {
    extern __shared__ uint32_t smu[];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = b.Kmax + dt_bit_words(b.Kmax);
    uint32_t* hist = smu + (size_t)per * wid;
    uint32_t* bits = hist + b.Kmax;
    for (int k = lane; k < per; k += 32) hist[k] = 0u;
    __syncwarp();
    for (;;) {
        const int i = grab(b.counters + 2, lane);
        if (i >= b.n_dt) break;
        const uint4 u = b.dt_work[i];
        const DtArgs& a = b.dt[u.x];
        for (uint32_t d = u.y; d < u.y + u.z; ++d) dt_doc(a, d, Hist<false>{hist}, bits, lane);
    }
}

template <bool LL, int QB>
__global__ void __launch_bounds__(256) kb_sample(BatchArgs b) {
    extern __shared__ float smf[];
    const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = b.Kmax + col_words(b.Kmax);
    float* r = smf + (size_t)per * wid;
    float* col = r + b.Kmax;
    uint32_t* ctr = reinterpret_cast<uint32_t*>(smf + (size_t)per * warps) + C_NUM * wid;
    if (lane < C_NUM) ctr[lane] = 0u;
    __syncwarp();
    const uint32_t done = *b.sweeps_done;
    int cur = -1;
    const SampleArgs* ca = nullptr;
    for (;;) {
        const int i = grab(b.counters + 3, lane);
        if (i >= b.n_sm) break;
        const uint2 w = b.sm_work[i];
        if ((int)w.x != cur) {
            __syncwarp();
            if (ca && lane < C_NUM && ctr[lane]) atomicAdd(ca->ctr + lane, (unsigned long long)ctr[lane]);
            __syncwarp();
            if (lane < C_NUM) ctr[lane] = 0u;
            cur = (int)w.x;
            ca = b.sm + cur;
            warp_recip(r, ca->n_k, ca->K, ca->Vbeta, lane);
        }
        const SampleArgs& a = *ca;
        sample_tile<LL, QB>(a, (int)w.y, a.tiles[w.y], a.iter + done, r, col, ctr, lane);
    }
    __syncwarp();
    if (ca && lane < C_NUM && ctr[lane]) atomicAdd(ca->ctr + lane, (unsigned long long)ctr[lane]);
}

// Block per model: the fixed-order FP64 reduction of its sampler tiles' LL partials
// (the same order as the single-corpus reduction over the same partials).
__global__ void __launch_bounds__(1024) kb_ll(const SampleArgs* sm, double* out) {
    __shared__ double s[1024];
    const SampleArgs& a = sm[blockIdx.x];
    const double acc = strided_sum(a.tile_ll, a.ntiles);
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int h = blockDim.x >> 1; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

__global__ void kb_advance(uint32_t* sweeps_done) { *sweeps_done += 1u; }

// ORs the models' device error flags into one and clears them.
__global__ void kb_errors(int* const* errs, int n, int* out) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int e = *errs[i];
        if (e) {
            atomicOr(out, e);
            *errs[i] = 0;
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

namespace {

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    ~DevBuf() { cudaFree(p); }
    int put(const std::vector<T>& v) {
        cudaFree(p);
        p = nullptr;
        n = v.size();
        if (n == 0) return LDA_OK;
        cudaError_t e = cudaMalloc(&p, sizeof(T) * n);
        if (e == cudaSuccess) e = cudaMemcpy(p, v.data(), sizeof(T) * n, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(LDA_ERR_DEVICE_MEM, "batch table of %zu bytes: %s", sizeof(T) * n, cudaGetErrorString(e));
        }
        return LDA_OK;
    }
};

}  // namespace

struct lda_batch {
    int device = 0;
    cudaStream_t st = nullptr;
    std::vector<lda_trainer*> trainers;
    std::vector<TrainerView> views;
    lda_batch_tuning tuning{8, 0, 512};
    int Kmax = 0, num_sms = 0;
    // tables
    DevBuf<dev::WtArgs> wt;
    DevBuf<dev::StatsArgs> stt;
    DevBuf<dev::DtArgs> dt;
    DevBuf<dev::SampleArgs> sm;
    DevBuf<uint2> wt_work, sm_work;
    DevBuf<uint4> st_work, dt_work;
    DevBuf<dev::ZeroSeg> zero;
    DevBuf<int*> errs;
    DevBuf<int4> sub_tiles;      // sampler tiles split to tile_tokens
    DevBuf<double> sub_ll;       // their LL partials
    unsigned* counters = nullptr;
    uint32_t* sweeps_done = nullptr;
    double* ll_dev = nullptr;
    int* err_dev = nullptr;
    std::vector<double> ll_host;
    uint32_t host_sweeps = 0;
    // launch shapes
    size_t smem_hist = 0, smem_stats = 0, smem_sample = 0, smem_dt = 0;
    int grid_wt = 0, grid_stats = 0, grid_dt = 0, grid_sample = 0, grid_sample_ll = 0;
    // cached graph of (sweeps, ll)
    cudaGraphExec_t graph = nullptr;
    int graph_sweeps = -1, graph_ll = -1;
    int64_t kernel_launches = 0;

    ~lda_batch() {
        cudaSetDevice(device);
        if (st) cudaStreamSynchronize(st);
        if (graph) cudaGraphExecDestroy(graph);
        cudaFree(counters);
        cudaFree(sweeps_done);
        cudaFree(ll_dev);
        cudaFree(err_dev);
        if (st) cudaStreamDestroy(st);
    }
};

// Batched sampler instantiation: Q-bucket rounds four per batch when some model has K > 1024.
static const void* batch_sample_kernel(bool ll, int Kmax) {
    if (Kmax > 1024) return ll ? (const void*)dev::kb_sample<true, 4> : (const void*)dev::kb_sample<false, 4>;
    return ll ? (const void*)dev::kb_sample<true, 1> : (const void*)dev::kb_sample<false, 1>;
}

static int occupancy(const void* fn, int threads, size_t smem, int num_sms, int* grid) {
    int per_sm = 0;
    CUDA_TRY(raise_smem_limit(fn, smem));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
    if (per_sm < 1) return fail(LDA_ERR_ARG, "batched kernel cannot be resident with %zu bytes of shared memory", smem);
    *grid = per_sm * num_sms;
    return LDA_OK;
}

// Builds the tables, work lists and launch shapes for the current tuning.
static int batch_build(lda_batch* b) {
    const int M = (int)b->trainers.size();
    const lda_batch_tuning& tu = b->tuning;
    std::vector<dev::WtArgs> wt(M);
    std::vector<dev::StatsArgs> stt(M);
    std::vector<dev::DtArgs> dt(M);
    std::vector<dev::SampleArgs> sm(M);
    std::vector<dev::ZeroSeg> zero;
    std::vector<int*> errs;
    std::vector<int4> sub;
    std::vector<int64_t> sub_base(M + 1, 0);
    for (int m = 0; m < M; ++m) {
        const TrainerView& v = b->views[m];
        for (const int4& t : v.s_tiles)
            for (int p = 0; p < t.z; p += tu.tile_tokens) sub.push_back(make_int4(t.x, t.y + p, std::min(tu.tile_tokens, t.z - p), t.w));
        sub_base[m + 1] = (int64_t)sub.size();
    }
    int rc;
    if ((rc = b->sub_tiles.put(sub))) return rc;
    {
        std::vector<double> zeros(sub.size(), 0.0);
        if ((rc = b->sub_ll.put(zeros))) return rc;
    }
    for (int m = 0; m < M; ++m) {
        const TrainerView& v = b->views[m];
        wt[m] = v.wt;
        stt[m] = v.st;
        dt[m] = v.dt;
        sm[m] = v.sm;
        sm[m].tiles = b->sub_tiles.p + sub_base[m];
        sm[m].ntiles = (int)(sub_base[m + 1] - sub_base[m]);
        sm[m].tile_ll = b->sub_ll.p + sub_base[m];
        zero.push_back({v.n_k, (long long)v.K});
        if (v.dwt_count > 0) zero.push_back({v.dwt, (long long)v.dwt_count});
        errs.push_back(v.wt.err);
    }
    // work lists
    std::vector<uint2> wt_work, sm_work;
    std::vector<uint4> st_work, dt_work;
    std::vector<int> wt_cnt, sm_cnt;
    for (int m = 0; m < M; ++m) {
        const TrainerView& v = b->views[m];
        for (int j = 0; j < v.n_wtiles; ++j) {
            wt_work.push_back(make_uint2((unsigned)m, (unsigned)j));
            wt_cnt.push_back(v.w_tiles[j].z);
        }
        for (int64_t j = 0; j < sub_base[m + 1] - sub_base[m]; ++j) {
            sm_work.push_back(make_uint2((unsigned)m, (unsigned)j));
            sm_cnt.push_back(sub[sub_base[m] + j].z);
        }
        for (int64_t w = 0; w < v.V; w += 32) st_work.push_back(make_uint4((unsigned)m, (unsigned)w, (unsigned)std::min<int64_t>(32, v.V - w), 0u));
        for (int64_t d = 0; d < v.D; d += 16) dt_work.push_back(make_uint4((unsigned)m, (unsigned)d, (unsigned)std::min<int64_t>(16, v.D - d), 0u));
    }
    if (tu.schedule == 0) {
        // largest tiles first across all models (each model's lists are already largest first)
        auto by_size = [](std::vector<uint2>& work, const std::vector<int>& cnt) {
            std::vector<size_t> idx(work.size());
            std::iota(idx.begin(), idx.end(), 0);
            std::stable_sort(idx.begin(), idx.end(), [&](size_t x, size_t y) { return cnt[x] > cnt[y]; });
            std::vector<uint2> out(work.size());
            for (size_t i = 0; i < idx.size(); ++i) out[i] = work[idx[i]];
            work.swap(out);
        };
        by_size(wt_work, wt_cnt);
        by_size(sm_work, sm_cnt);
    }
    if ((rc = b->wt.put(wt)) || (rc = b->stt.put(stt)) || (rc = b->dt.put(dt)) || (rc = b->sm.put(sm)) ||
        (rc = b->wt_work.put(wt_work)) || (rc = b->sm_work.put(sm_work)) || (rc = b->st_work.put(st_work)) ||
        (rc = b->dt_work.put(dt_work)) || (rc = b->zero.put(zero)) || (rc = b->errs.put(errs)))
        return rc;
    // launch shapes
    const int threads = 32 * tu.warps;
    b->smem_hist = (size_t)tu.warps * (b->Kmax + (b->Kmax + 31) / 32) * 4;
    b->smem_stats = (size_t)tu.warps * b->Kmax * 8;
    b->smem_sample = (size_t)tu.warps * ((b->Kmax + dev::col_words(b->Kmax)) * 4 + dev::C_NUM * 4);
    b->smem_dt = (size_t)tu.warps * (b->Kmax + (b->Kmax + 31) / 32) * 4;
    if ((rc = occupancy((const void*)dev::kb_wt, threads, b->smem_hist, b->num_sms, &b->grid_wt)) ||
        (rc = occupancy((const void*)dev::kb_stats, threads, b->smem_stats, b->num_sms, &b->grid_stats)) ||
        (rc = occupancy((const void*)dev::kb_dt, threads, b->smem_dt, b->num_sms, &b->grid_dt)) ||
        (rc = occupancy(batch_sample_kernel(false, b->Kmax), threads, b->smem_sample, b->num_sms, &b->grid_sample)) ||
        (rc = occupancy(batch_sample_kernel(true, b->Kmax), threads, b->smem_sample, b->num_sms, &b->grid_sample_ll)))
        return rc;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        b->graph_sweeps = b->graph_ll = -1;
    }
    return LDA_OK;
}

static dev::BatchArgs batch_args(const lda_batch* b) {
    dev::BatchArgs a;
    a.wt = b->wt.p; a.st = b->stt.p; a.dt = b->dt.p; a.sm = b->sm.p;
    a.wt_work = b->wt_work.p; a.n_wt = (int)b->wt_work.n;
    a.st_work = b->st_work.p; a.n_st = (int)b->st_work.n;
    a.dt_work = b->dt_work.p; a.n_dt = (int)b->dt_work.n;
    a.sm_work = b->sm_work.p; a.n_sm = (int)b->sm_work.n;
    a.counters = b->counters;
    a.sweeps_done = b->sweeps_done;
    a.Kmax = b->Kmax;
    return a;
}

static int grid_for(int grid, int64_t work, int warps) {
    return (int)std::max<int64_t>(1, std::min<int64_t>(grid, (work + warps - 1) / warps));
}

// Enqueues `sweeps` batched sweeps on the batch's stream (LL on the last one when ll).
static int enqueue_sweeps(lda_batch* b, int sweeps, int ll) {
    const dev::BatchArgs a = batch_args(b);
    const int W = b->tuning.warps, threads = 32 * W;
    const int M = (int)b->trainers.size();
    for (int s = 0; s < sweeps; ++s) {
        const bool last_ll = ll && s == sweeps - 1;
        dev::kb_zero<<<std::min<int>((int)b->zero.n, 4 * b->num_sms), 256, 0, b->st>>>(b->zero.p, (int)b->zero.n, b->counters);
        dev::kb_wt<<<grid_for(b->grid_wt, a.n_wt, W), threads, b->smem_hist, b->st>>>(a);
        dev::kb_stats<<<grid_for(b->grid_stats, a.n_st, W), threads, b->smem_stats, b->st>>>(a);
        dev::kb_dt<<<grid_for(b->grid_dt, a.n_dt, W), threads, b->smem_dt, b->st>>>(a);
        const int gs = last_ll ? grid_for(b->grid_sample_ll, a.n_sm, W) : grid_for(b->grid_sample, a.n_sm, W);
        if (b->Kmax > 1024) {
            if (last_ll) dev::kb_sample<true, 4><<<gs, threads, b->smem_sample, b->st>>>(a);
            else dev::kb_sample<false, 4><<<gs, threads, b->smem_sample, b->st>>>(a);
        } else {
            if (last_ll) dev::kb_sample<true, 1><<<gs, threads, b->smem_sample, b->st>>>(a);
            else dev::kb_sample<false, 1><<<gs, threads, b->smem_sample, b->st>>>(a);
        }
        if (last_ll) dev::kb_ll<<<M, 1024, 0, b->st>>>(b->sm.p, b->ll_dev);
        dev::kb_advance<<<1, 1, 0, b->st>>>(b->sweeps_done);
        CUDA_TRY(cudaGetLastError());
        b->kernel_launches += last_ll ? 8 : 7;
    }
    return LDA_OK;
}

extern "C" int lda_batch_create(lda_trainer* const* trainers, int32_t n, const lda_batch_tuning* tuning,
                                lda_batch** out) {
    if (!trainers || !out || n < 1) return fail(LDA_ERR_ARG, "need at least one trainer");
    *out = nullptr;
    std::unique_ptr<lda_batch> b(new lda_batch());
    b->trainers.assign(trainers, trainers + n);
    b->views.resize(n);
    int rc;
    for (int m = 0; m < n; ++m) {
        if (!trainers[m]) return fail(LDA_ERR_ARG, "trainer %d is null", m);
        if ((rc = trainer_view(trainers[m], &b->views[m]))) return rc;
        if ((rc = lda_trainer_sync(trainers[m]))) return rc;
        if (b->views[m].device != b->views[0].device) return fail(LDA_ERR_ARG, "trainers of a batch share one device");
        for (int j = 0; j < m; ++j)
            if (trainers[j] == trainers[m]) return fail(LDA_ERR_ARG, "trainer %d appears twice", m);
        b->Kmax = std::max(b->Kmax, b->views[m].K);
        if (b->views[m].K > dev::kLargeK)
            return fail(LDA_ERR_ARG, "trainer %d has K=%d; batched models take K <= %d", m, b->views[m].K, dev::kLargeK);
    }
    b->device = b->views[0].device;
    if (tuning) b->tuning = *tuning;
    if (b->tuning.warps < 1 || b->tuning.warps > 8 || b->tuning.schedule < 0 || b->tuning.schedule > 1 ||
        b->tuning.tile_tokens < 32)
        return fail(LDA_ERR_ARG, "tuning: warps in [1,8], schedule 0 or 1, tile_tokens >= 32");
    CUDA_TRY(cudaSetDevice(b->device));
    CUDA_TRY(cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device));
    CUDA_TRY(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
    cudaError_t e = cudaMalloc(&b->counters, 4 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&b->sweeps_done, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(b->sweeps_done, 0, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->ll_dev, sizeof(double) * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&b->err_dev, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->err_dev, 0, sizeof(int));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(LDA_ERR_DEVICE_MEM, "batch allocation failed: %s", cudaGetErrorString(e));
    }
    b->ll_host.assign(n, 0.0);
    if ((rc = batch_build(b.get()))) return rc;
    *out = b.release();
    return LDA_OK;
}

extern "C" int lda_batch_destroy(lda_batch* b) {
    delete b;
    return LDA_OK;
}

extern "C" int lda_batch_set_tuning(lda_batch* b, const lda_batch_tuning* tuning) {
    if (!b || !tuning) return fail(LDA_ERR_ARG, "null argument");
    if (tuning->warps < 1 || tuning->warps > 8 || tuning->schedule < 0 || tuning->schedule > 1 || tuning->tile_tokens < 32)
        return fail(LDA_ERR_ARG, "tuning: warps in [1,8], schedule 0 or 1, tile_tokens >= 32");
    CUDA_TRY(cudaSetDevice(b->device));
    CUDA_TRY(cudaStreamSynchronize(b->st));
    b->tuning = *tuning;
    return batch_build(b);
}

extern "C" int lda_batch_get_tuning(const lda_batch* b, lda_batch_tuning* tuning) {
    if (!b || !tuning) return fail(LDA_ERR_ARG, "null argument");
    *tuning = b->tuning;
    return LDA_OK;
}

static int batch_finish(lda_batch* b, int sweeps, int ll) {
    dev::kb_errors<<<1, 256, 0, b->st>>>(b->errs.p, (int)b->errs.n, b->err_dev);
    CUDA_TRY(cudaGetLastError());
    int herr = 0;
    CUDA_TRY(cudaMemcpyAsync(&herr, b->err_dev, sizeof(int), cudaMemcpyDeviceToHost, b->st));
    if (ll) CUDA_TRY(cudaMemcpyAsync(b->ll_host.data(), b->ll_dev, sizeof(double) * b->ll_host.size(), cudaMemcpyDeviceToHost, b->st));
    CUDA_TRY(cudaStreamSynchronize(b->st));
    b->host_sweeps += (uint32_t)sweeps;
    for (size_t m = 0; m < b->trainers.size(); ++m) {
        int rc = trainer_note_sweeps(b->trainers[m], sweeps, ll, ll ? b->ll_host[m] : 0.0);
        if (rc) return rc;
    }
    if (herr) {
        CUDA_TRY(cudaMemset(b->err_dev, 0, sizeof(int)));
        return fail(LDA_ERR_DEVICE, "a batched kernel found a topic >= K in a model's topic array");
    }
    return LDA_OK;
}

extern "C" int lda_batch_iterate(lda_batch* b, int32_t sweeps, int32_t ll_mode) {
    if (!b) return fail(LDA_ERR_ARG, "null batch");
    if (sweeps < 0) return fail(LDA_ERR_ARG, "negative sweep count");
    if (sweeps == 0) return LDA_OK;
    CUDA_TRY(cudaSetDevice(b->device));
    const int ll = ll_mode ? 1 : 0;
    // the models' iterations must still be the ones the tables hold
    for (size_t m = 0; m < b->trainers.size(); ++m) {
        uint32_t it = 0;
        lda_trainer_get_iteration(b->trainers[m], &it);
        if (it != b->views[m].sm.iter + b->host_sweeps)
            return fail(LDA_ERR_STATE, "trainer %zu was swept outside the batch; rebuild the batch", m);
    }
    if (!b->graph || b->graph_sweeps != sweeps || b->graph_ll != ll) {
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
        const int64_t before = b->kernel_launches;
        int rc = enqueue_sweeps(b, sweeps, ll);
        cudaError_t e = cudaStreamEndCapture(b->st, &g);
        b->kernel_launches = before;
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(LDA_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
        }
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            cudaGetLastError();
            b->graph = nullptr;
            return fail(LDA_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
        }
        b->graph_sweeps = sweeps;
        b->graph_ll = ll;
    }
    CUDA_TRY(cudaGraphLaunch(b->graph, b->st));
    b->kernel_launches += (int64_t)sweeps * 7 + (ll ? 1 : 0);
    return batch_finish(b, sweeps, ll);
}

extern "C" int lda_batch_loglik(const lda_batch* b, double* ll, int32_t n) {
    if (!b || !ll || n != (int32_t)b->trainers.size()) return fail(LDA_ERR_ARG, "need one entry per model");
    std::memcpy(ll, b->ll_host.data(), sizeof(double) * (size_t)n);
    return LDA_OK;
}

extern "C" int lda_batch_stats(const lda_batch* b, int64_t* kernel_launches, int64_t* work_items) {
    if (!b) return fail(LDA_ERR_ARG, "null batch");
    if (kernel_launches) *kernel_launches = b->kernel_launches;
    if (work_items) *work_items = (int64_t)(b->wt_work.n + b->st_work.n + b->dt_work.n + b->sm_work.n);
    return LDA_OK;
}

// Times each candidate tuning on the live batch and keeps the fastest.  The models'
// topics, iterations and counters are restored after every trial, so tuning leaves no
// trace in the results.
extern "C" int lda_batch_autotune(lda_batch* b, int32_t sweeps_per_trial, lda_batch_tuning* best_out,
                                  double* best_ms_per_sweep) {
    if (!b || sweeps_per_trial < 1) return fail(LDA_ERR_ARG, "need a batch and >= 1 sweep per trial");
    CUDA_TRY(cudaSetDevice(b->device));
    CUDA_TRY(cudaStreamSynchronize(b->st));
    const int M = (int)b->trainers.size();
    // save every model's topics and counters, the batch's sweep count
    std::vector<std::vector<uint16_t>> z(M);
    std::vector<std::vector<unsigned long long>> ctr(M);
    int rc;
    for (int m = 0; m < M; ++m) {
        const TrainerView& v = b->views[m];
        z[m].resize((size_t)v.N);
        if ((rc = lda_trainer_get_topics(b->trainers[m], z[m].data(), v.N))) return rc;
        ctr[m].resize(16);
        CUDA_TRY(cudaMemcpy(ctr[m].data(), v.sm.ctr, sizeof(unsigned long long) * 16, cudaMemcpyDeviceToHost));
    }
    uint32_t done0 = 0;
    CUDA_TRY(cudaMemcpy(&done0, b->sweeps_done, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    const uint32_t host0 = b->host_sweeps;
    std::vector<uint32_t> it0(M);
    for (int m = 0; m < M; ++m) lda_trainer_get_iteration(b->trainers[m], &it0[m]);
    auto restore = [&]() -> int {
        for (int m = 0; m < M; ++m) {
            int r = lda_trainer_set_topics(b->trainers[m], z[m].data(), (int64_t)z[m].size());
            if (r) return r;
            lda_trainer_set_iteration(b->trainers[m], it0[m]);
            CUDA_TRY(cudaMemcpy(b->views[m].sm.ctr, ctr[m].data(), sizeof(unsigned long long) * 16, cudaMemcpyHostToDevice));
        }
        CUDA_TRY(cudaMemcpy(b->sweeps_done, &done0, sizeof(uint32_t), cudaMemcpyHostToDevice));
        b->host_sweeps = host0;
        return LDA_OK;
    };
    const lda_batch_tuning start = b->tuning;
    lda_batch_tuning best = start;
    double best_ms = 1e300;
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    std::vector<lda_batch_tuning> cands;
    for (int w : {4, 8})
        for (int sch : {0, 1})
            for (int tt : {128, 256, 512}) cands.push_back(lda_batch_tuning{w, sch, tt});
    rc = LDA_OK;
    for (const lda_batch_tuning& cand : cands) {
        b->tuning = cand;
        if ((rc = batch_build(b)) || (rc = enqueue_sweeps(b, 1, 0))) break;  // build + warm-up sweep
        float ms = 0.f;
        cudaError_t e = cudaEventRecord(e0, b->st);
        if (e == cudaSuccess && (rc = enqueue_sweeps(b, sweeps_per_trial, 0))) break;
        if (e == cudaSuccess) e = cudaEventRecord(e1, b->st);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) {
            cudaGetLastError();
            rc = fail(LDA_ERR_CUDA, "autotune trial failed: %s", cudaGetErrorString(e));
            break;
        }
        if (ms / sweeps_per_trial < best_ms) {
            best_ms = ms / sweeps_per_trial;
            best = cand;
        }
        if ((rc = restore())) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->kernel_launches = 0;
    if (rc) {
        restore();
        b->tuning = start;
        batch_build(b);
        return rc;
    }
    b->tuning = best;
    if ((rc = batch_build(b))) return rc;
    if (best_out) *best_out = best;
    if (best_ms_per_sweep) *best_ms_per_sweep = best_ms;
    return LDA_OK;
}
