/*
 * lda_b200.h -- C ABI of the B200-native collapsed-Gibbs LDA sweep.
 *
 * Drop-in boundary for EZLDA's hot path (asherliu/LDA_SC20).  EZLDA has no
 * FFI: its boundary is (1) the C++ kernel-launch wrappers of its L2 layer
 * (EZLDA/<stage>Kernel.cuh), called by the driver loop in EZLDA/mainKernel.cu, and
 * (2) the on-disk chunk directory plus the K/alpha/beta/iteration parameters
 * and the per-iteration log-likelihood line.  Every entry point below names the
 * reference interface it replaces.  Conventions:
 *   - plain pointers and sizes only; every function returns an int status
 *     (LDA_OK = 0, negative on error) and never exits the process; the text of
 *     the last error on the calling thread is in lda_last_error();
 *   - host buffers are owned by the caller, device buffers by the library;
 *   - one handle per host thread (handles are not internally locked);
 *   - topics are 0-based here (the chunk files hold 1-based topics).
 */
#ifndef LDA_B200_H_
#define LDA_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LDA_OK 0
#define LDA_ERR_ARG (-1)        /* bad argument or out-of-range value */
#define LDA_ERR_IO (-2)         /* missing / unreadable / unwritable file */
#define LDA_ERR_FORMAT (-3)     /* malformed or truncated chunk file */
#define LDA_ERR_NOMEM (-4)      /* host allocation failed */
#define LDA_ERR_DEVICE_MEM (-5) /* device memory budget or cudaMalloc exceeded */
#define LDA_ERR_CUDA (-6)       /* CUDA runtime error (no device, launch failure, ...) */
#define LDA_ERR_STATE (-7)      /* call not valid in the handle's current state */
#define LDA_ERR_DEVICE (-8)     /* a kernel reported an out-of-range value */

typedef struct lda_corpus lda_corpus;
typedef struct lda_trainer lda_trainer;

const char* lda_last_error(void);
const char* lda_version(void);

/* ------------------------------------------------------------------ corpus */

/* Synthetic corpus drawn from the LDA generative process. */
typedef struct {
    int64_t num_docs;    /* D */
    int64_t vocab;       /* V */
    int32_t gen_topics;  /* generating topics */
    int32_t len_kind;    /* 0: Poisson(len_p1); 1: lognormal(mu=len_p1, sigma=len_p2) */
    double len_p1, len_p2;
    int32_t len_min, len_max; /* clip */
    int32_t phi_kind;    /* 0: phi_k ~ Dir(phi_conc * 1_V);
                            1: phi_k ~ Dir(phi_conc * V * z), z_r ∝ (r+1)^-phi_zipf_s, sum z = 1;
                            2: kind 1 drawn in its Polya-urn form (phi integrated out), for
                               gen_topics * V too large to hold explicit distributions */
    double phi_conc, phi_zipf_s;
    double theta_conc;   /* theta_d ~ Dir(theta_conc * 1_T) */
    int32_t K;           /* model topics: initial topics are uniform in [0,K) */
    int32_t dense_kind;  /* 0: words with count >= K are dense (EZLDA's rule);
                            1: top dense_param fraction of words; 2: top dense_param words */
    double dense_param;
    int32_t num_chunks;  /* contiguous doc ranges with balanced token counts */
    uint64_t corpus_seed; /* std::mt19937_64 seed of the generative draws */
    uint64_t topic_seed;  /* Philox seed of the initial topics */
} lda_gen_config;

typedef struct {
    int64_t num_tokens; /* N */
    int64_t vocab;      /* V (words are frequency ranks 0..V-1) */
    int64_t num_docs;   /* D */
    int32_t num_chunks; /* C */
    int32_t num_dense;  /* words [0, num_dense) use the dense word-topic path */
    int32_t max_doc_len;
    int32_t K_hint;     /* K the topics were drawn for (0 if unknown) */
} lda_corpus_info;

/* Array fields readable with lda_corpus_get (element type, count). */
enum {
    LDA_F_TOK_WORD = 0,   /* int32 [N]   word of word-sorted token i */
    LDA_F_TOK_DOC = 1,    /* int32 [N]   global doc of token i */
    LDA_F_TOPICS = 2,     /* uint16 [N]  initial topic of token i */
    LDA_F_DOC_OFF = 3,    /* int64 [D+1] doc-order token offsets */
    LDA_F_DTOK_POS = 4,   /* int64 [N]   word-sorted index of doc-order token j */
    LDA_F_DTOK_WORD = 5,  /* int32 [N]   word of doc-order token j */
    LDA_F_CHUNK_TOK = 6,  /* int64 [C+1] first token of each chunk */
    LDA_F_CHUNK_DOC = 7,  /* int64 [C+1] first doc of each chunk */
    LDA_F_WORD_COUNT = 8, /* int64 [V]   corpus count of each word */
    LDA_F_SEG_OFF = 9,    /* int64 [C*V] first token of word w in chunk c (global index) */
    LDA_F_SEG_CNT = 10    /* int64 [C*V] tokens of word w in chunk c */
};

int lda_corpus_generate(const lda_gen_config* cfg, lda_corpus** out);
/* New documents from the generative process of a generated corpus (no counterpart in the
 * reference): its topic-word distributions, fresh theta ~ Dir(theta_conc), lengths
 * lognormal(len_mu, len_sigma) clipped to [len_min, len_max], all from request_seed;
 * words are the corpus' frequency ranks.  doc_off gets n+1 offsets; with words NULL only
 * the offsets are drawn (sizing call), else words needs doc_off[n] <= cap entries. */
int lda_corpus_generate_requests(const lda_corpus* c, uint64_t request_seed, int64_t n, double len_mu,
                                 double len_sigma, int32_t len_min, int32_t len_max, int64_t* doc_off,
                                 int32_t* words, int64_t cap);
/* Reads an EZLDA chunk directory (lengthVec.txt, docLength.txt, TLLength.txt,
 * TLSplit.txt, chunk<c>/{TL,word2DocMap,wordCountOffset,docCountOffset}.txt),
 * replacing Document::loadDocument / DocChunk::loadChunk (EZLDA/Doc.cu:45-108,
 * EZLDA/DataChunk.cu:50-100) and WTAll::loadWTCountOffset (EZLDA/WT.cu:155-186). */
int lda_corpus_load_ezlda(const char* dir, lda_corpus** out);
/* Writes the EZLDA chunk format (the files preprocess/streamTestBalance.cpp:356-547
 * writes); K sets the DT/WT capacities the format records. */
int lda_corpus_write_ezlda(const lda_corpus* c, const char* dir, int32_t K);
/* Builds the word-sorted chunk layout from doc-ordered tokens: words[j] is the
 * raw word id (0..V-1) of doc-order token j, doc d owns [doc_off[d], doc_off[d+1]).
 * Words are renumbered by descending frequency (stable); topics may be NULL
 * (then drawn from Philox(topic_seed)) and are given in doc order. */
int lda_corpus_from_docs(int64_t num_docs, const int64_t* doc_off, const int32_t* words,
                         int64_t vocab, const uint16_t* topics_doc_order, int32_t K,
                         int32_t num_chunks, int32_t dense_kind, double dense_param,
                         uint64_t topic_seed, lda_corpus** out);
int lda_corpus_info_get(const lda_corpus* c, lda_corpus_info* out);
int lda_corpus_get(const lda_corpus* c, int32_t field, void* out, int64_t count);
/* Replaces the corpus' initial topics (word-sorted order, 0-based, < K). */
int lda_corpus_set_topics(lda_corpus* c, const uint16_t* topics, int64_t count);
void lda_corpus_free(lda_corpus* c);

/* ----------------------------------------------------------------- trainer */

typedef struct {
    int32_t K;
    float alpha;            /* EZLDA: 50/K (EZLDA/Argument.cuh:9) */
    float beta;             /* EZLDA: 0.01 (EZLDA/Argument.cuh:8) */
    uint64_t seed;          /* Philox seed of the sweep randoms */
    int32_t device;         /* CUDA device ordinal */
    int64_t device_budget;  /* bytes the trainer may allocate (0: no limit) */
    int32_t stream_mode;    /* 0: keep the corpus resident when it fits device_budget, else
                               stream it; 1: always resident; 2: always stream */
    int32_t num_streams;    /* streaming: chunk slots on the device, one CUDA stream each (0: 4);
                               above 2048 topics the chunks are sampled in turn and a slot
                               keeps its chunk across sweeps */
    int32_t num_dense;      /* 0: the corpus' dense/sparse split; n > 0: words [0, n) use the
                               dense word-topic path; -1: none (results do not depend on it) */
} lda_train_config;

/* Sweep counters accumulated since the trainer was created or lda_trainer_reset_stats. */
typedef struct {
    int64_t tokens;        /* tokens sampled */
    int64_t early_accept;  /* settled by the max-topic bound */
    int64_t full;          /* S evaluated over the doc row */
    int64_t sum_nnz_full;  /* doc-row entries read by evaluated tokens */
    int64_t branch_max, branch_s, branch_q;
    int64_t sum_word_nnz;  /* sparse word-row entries read building word columns */
    int64_t word_tiles_dense, word_tiles_sparse;
    int64_t rows_evaluated;   /* doc rows evaluated (consecutive tokens of one (word, doc) share one) */
    int64_t row_entries_read; /* doc-row entries read by those evaluations */
} lda_sweep_counters;

/* Accumulated device time (CUDA events on the trainer's stream) per stage. */
typedef struct {
    double ms_wt;      /* word-topic + topic-total rebuild */
    double ms_stats;   /* per-word max topics / Q */
    double ms_dt;      /* doc-topic rebuild + per-token metadata */
    double ms_sample;  /* sampler */
    double ms_ll;      /* log-likelihood reduction */
    double ms_copy;    /* host<->device copies of lda_iterate_host */
    int64_t launches_wt, launches_stats, launches_dt, launches_sample, launches_ll;
} lda_stage_timing;

/* Allocates the device copy of the corpus (Document/DTChunk/WTAll/WTD
 * GPUMemAllocate, EZLDA/Doc.cu:179-246, DT.cu:53-70, WT.cu:76-97,
 * WTDense.cu:27-43) and uploads it.  Fails with LDA_ERR_DEVICE_MEM when the
 * allocation would exceed cfg->device_budget or cudaMalloc fails. */
int lda_trainer_create(const lda_corpus* c, const lda_train_config* cfg, lda_trainer** out);
/* Whether the trainer streams its chunks (EZLDA's DataChunk/WTChunk streaming,
 * EZLDA/mainKernel.cu:203-314), through how many streams, and the bytes it has copied
 * host->device for chunks since creation. */
int lda_trainer_stream_info(const lda_trainer* t, int32_t* streaming, int32_t* streams, int64_t* h2d_bytes);
int lda_trainer_destroy(lda_trainer* t);
/* Makes the trainer launch on an external cudaStream_t (NULL: its own stream). */
int lda_trainer_set_stream(lda_trainer* t, void* cuda_stream);
int lda_trainer_get_stream(lda_trainer* t, void** cuda_stream);
/* Bytes of device memory held by the trainer. */
int lda_trainer_device_bytes(const lda_trainer* t, int64_t* bytes);
/* Restricts lda_trainer_iterate's doc-topic rebuild, sampling and log-likelihood to
 * chunks [first, last) (default: all).  The word-topic rebuild always reads every
 * chunk's topics.  A document-sharded run gives each rank a disjoint range and
 * exchanges the ranges' topics after every sweep (EZLDA is single-GPU; this is the
 * exchange step of its multi-GPU form). */
int lda_trainer_set_chunk_range(lda_trainer* t, int32_t first, int32_t last);
/* Device address and length of the trainer's topic array (uint16, word-sorted), for a
 * collective that exchanges topic slices in place between sweeps. */
int lda_trainer_topics_device(lda_trainer* t, void** ptr, int64_t* count);
/* Restricts lda_update_wt and lda_max_topic to the words [w0, w1) (default: all): the
 * rebuild zeroes and refills only the range's dense rows and sparse rows, and n_k receives
 * only the range's tokens; the statistics are computed for the range's words only.  A
 * word-sharded run gives each rank a disjoint range, sums n_k over the ranks before
 * lda_max_topic, gathers every range's rows and statistics afterwards, and then calls
 * lda_trainer_sweep_chunks.  Replaces the replicated UpdateWT / MaxTopic pass that every
 * GPU of a multi-GPU form would otherwise run (EZLDA/mainKernel.cu:282-290). */
int lda_trainer_set_word_range(lda_trainer* t, int32_t w0, int32_t w1);
/* Device addresses of the word side a word-sharded run exchanges.  Words [0, num_dense)
 * have dense rows (dense_wt, K int32 each); word num_dense + s has the sparse row
 * sparse_ent[sparse_off[s] .. sparse_off[s] + sparse_nnz[s]) inside a fixed slot that ends
 * at sparse_off[s + 1] (sparse_capacity for the last word).  Per word: top2 and k3
 * (uint32), phi4 (4 floats), ql (32 floats); per dense word its Q-round table. */
typedef struct lda_word_side {
    int32_t* n_k;
    int32_t* dense_wt;
    uint32_t* sparse_ent;
    uint32_t* sparse_nnz;
    const uint32_t* sparse_off;
    uint32_t* top2;
    uint32_t* k3;
    float* phi4;
    float* ql;
    /* above 2048 topics: each dense word's Q-round table (32 * qtab_rounds pairs of floats),
     * built with its statistics; NULL (and qtab_rounds 0) otherwise */
    float* qtab;
    int64_t K, vocab, num_dense, sparse_capacity, qtab_rounds;
} lda_word_side;
int lda_trainer_word_side(lda_trainer* t, lda_word_side* out);
/* One sweep without its word side: the caller has run lda_update_wt and lda_max_topic (and
 * exchanged their results) for this sweep's starting topics.  Runs the chunk range's
 * doc-topic rebuilds and sampling, the LL when ll_mode is set, and advances the
 * iteration; returns when the sweep is done. */
int lda_trainer_sweep_chunks(lda_trainer* t, int32_t ll_mode);

/* n full sweeps of the driver loop EZLDA/mainKernel.cu:158-380 on resident
 * data; ll_mode=1 also evaluates the FP64 log-likelihood of every sweep.
 * Blocks until the sweeps finish. */
int lda_trainer_iterate(lda_trainer* t, int32_t n_iters, int32_t ll_mode);
/* End-to-end sweep through host buffers: uploads topics_in (word-sorted, N),
 * runs one sweep, downloads the new topics to topics_out and the LL sum to
 * *ll_sum (when ll_mode), as EZLDA's per-chunk Document::CPU2GPU /
 * Document::GPU2CPU (EZLDA/Doc.cu:266-308) do around every sweep. */
int lda_iterate_host(lda_trainer* t, const uint16_t* topics_in, uint16_t* topics_out,
                     int32_t ll_mode, double* ll_sum);
/* lda_iterate_host without waiting, for a loop of sweeps through host buffers (the same
 * per-chunk uploads and downloads, EZLDA/Doc.cu:266-308, overlapped across sweeps).  Both
 * buffers must be pinned host memory (cudaHostAlloc / cudaHostRegister) and stay untouched
 * until lda_trainer_wait returns.  When topics_in is the previous call's topics_out and
 * nothing else ran on the trainer since, chunk c of it is uploaded as soon as the previous
 * sweep has downloaded chunk c, while that sweep samples its later chunks.  No
 * log-likelihood; not with stage timing on. */
int lda_iterate_host_async(lda_trainer* t, const uint16_t* topics_in, uint16_t* topics_out);
/* Waits for every sweep and copy enqueued on the trainer; reports a device error any of
 * them found. */
int lda_trainer_wait(lda_trainer* t);
/* FP64 sum and token count of the last log-likelihood evaluation; EZLDA's
 * PerplexityKernel / LDATrainPerplexityReduce (EZLDA/SamplingKernel.cu:172-180,
 * profilePerp/utility.cu:2883-2925).  Mean per-token LL = ll_sum / n_tokens. */
int lda_trainer_loglik(lda_trainer* t, double* ll_sum, int64_t* n_tokens);
int lda_trainer_get_topics(lda_trainer* t, uint16_t* out, int64_t count);
int lda_trainer_set_topics(lda_trainer* t, const uint16_t* in, int64_t count);
int lda_trainer_get_iteration(const lda_trainer* t, uint32_t* iter);
int lda_trainer_set_iteration(lda_trainer* t, uint32_t iter);
int lda_trainer_counters(lda_trainer* t, lda_sweep_counters* out);
/* Per-stage CUDA-event timing.  While it is on, a resident trainer runs its chunks'
 * doc-topic rebuilds and sampling one at a time on its stream; while it is off, chunk i of
 * the range runs on work stream i mod 2, overlapping the next chunk's work with this one's
 * (the results are the same either way). */
int lda_trainer_set_timing(lda_trainer* t, int32_t enabled);
int lda_trainer_timing(lda_trainer* t, lda_stage_timing* out);
int lda_trainer_reset_stats(lda_trainer* t);

/* Checkpoint = (topics, iteration, seed): every count is a function of the
 * topics and every random of (seed, iteration, token), so resume is exact. */
int lda_trainer_checkpoint(lda_trainer* t, const char* path);
int lda_trainer_restore(lda_trainer* t, const char* path);

/* -------------------------------------------- stage entry points (L2 layer) */
/* Each runs one stage of a sweep on the trainer's stream (asynchronously). */

/* Rebuilds the dense and sparse word-topic counts and the topic totals n_k
 * from the current topics.  Replaces UpdateWTDenKernel + UpdateWTDenRowSumKernel
 * (EZLDA/WTDenUpdateKernel.cuh:25-26), UpdateWTKernel (EZLDA/WTUpdateKernel.cuh:23)
 * and WTAdditionKernel (EZLDA/WTAddKernel.cuh:24). */
int lda_update_wt(lda_trainer* t);
/* Per-word max / 2nd / 3rd topic of phi and the Q bucket.  Replaces
 * MaxTopicKernel (EZLDA/SamplingKernel.cuh:12). */
int lda_max_topic(lda_trainer* t);
/* Doc-topic rows of one chunk plus each token's counts of its word's max and
 * 2nd topic.  Replaces UpdateDTKernel (EZLDA/DTUpdateKernel.cuh:13). */
int lda_update_dt(lda_trainer* t, int32_t chunk);
/* Samples every token of one chunk (dense and sparse words, early accept and
 * full evaluation in one kernel).  Replaces UpdateProbKernelD, SampleKernelD
 * and SampleKernel (EZLDA/SamplingKernel.cuh:10-14). */
int lda_sample_chunk(lda_trainer* t, int32_t chunk, int32_t ll_mode);
/* Reduces the per-tile LL partials of the sampled chunks to *ll_sum (blocks).
 * Replaces PerplexityKernel (EZLDA/SamplingKernel.cuh:15). */
int lda_perplexity(lda_trainer* t, double* ll_sum);
/* Advances the sweep counter (the iteration key of the randoms). */
int lda_end_sweep(lda_trainer* t);
int lda_trainer_sync(lda_trainer* t);

/* Device-state readback (blocking copies into caller buffers). */
int lda_get_topic_totals(lda_trainer* t, int32_t* n_k /*K*/);
int lda_get_dense_wt(lda_trainer* t, int32_t* out /*num_dense*K*/);
/* Sparse word rows (words num_dense..V-1) compacted: off has V-num_dense+1
 * entries, ent holds (k<<16 | count) ascending k.  Returns entries or <0. */
int64_t lda_get_sparse_wt(lda_trainer* t, int64_t* off, uint32_t* ent, int64_t cap);
int lda_get_word_stats(lda_trainer* t, uint32_t* top2, uint32_t* k3, float* phi4, float* ql);
/* Doc rows of every doc (valid for chunks whose lda_update_dt ran). */
int64_t lda_get_doc_rows(lda_trainer* t, int64_t* off, uint32_t* ent, int64_t cap);
int lda_get_token_meta(lda_trainer* t, uint32_t* meta /*N*/);

/* ------------------------------------------------ allocation-free sampling */

/* Device buffers of one sampling call (all device pointers; sizes implied by the
 * corpus layout): tiles is num_tiles x {word, first token, token count, dense flag}
 * (16-byte aligned); the rest follow the layout lda_get_* return, with every doc row
 * starting at a multiple of 4 entries of dt_ent (16-byte aligned rows). */
typedef struct {
    int32_t K, num_dense, vocab;
    float alpha, beta;
    uint64_t seed;
    uint32_t iter;
    int32_t ll_mode;
    int32_t num_tiles;
    const int32_t* tiles;
    const int32_t* n_k;            /* [K] */
    const int32_t* dense_wt;       /* [num_dense*K] */
    const uint32_t* sparse_off;    /* [vocab-num_dense] */
    const uint32_t* sparse_nnz;    /* [vocab-num_dense] */
    const uint32_t* sparse_ent;    /* (k<<16 | count) */
    const uint32_t* top2;          /* [vocab] */
    const float* phi4;             /* [vocab*4] */
    const float* ql;               /* [vocab*32] */
    const uint32_t* tok_doc;       /* [N] */
    const uint32_t* meta;          /* [N] */
    uint16_t* topics;              /* [N], updated for the tiles' tokens */
    const uint32_t* doc_len;       /* [D] */
    const uint32_t* dt_off;        /* [D] */
    const uint32_t* dt_nnz;        /* [D] */
    const uint32_t* dt_ent;
    double* ll_sum;                /* device scalar, written when ll_mode */
    /* lengths of the caller's buffers, for the range checks below */
    int64_t num_tokens;            /* entries of tok_doc, meta and topics */
    int32_t num_docs;              /* entries of doc_len, dt_off and dt_nnz */
    int64_t num_dt_entries;        /* entries of dt_ent */
    int64_t num_sparse_entries;    /* entries of sparse_ent */
    int32_t* status;               /* device int32, written every call (LDA_IO_* bits; 0 = sampled) */
} lda_sample_io;

/* Bits of *io->status: a check that failed on the device.  When any is set no token is
 * sampled (topics are left as they were) and ll_sum is not meaningful. */
#define LDA_IO_TILE 1        /* a tile's word is outside [0, vocab) or its tokens outside [0, num_tokens) */
#define LDA_IO_MAX_TOPIC 2   /* a tile word's max topic (top2 & 0xffff) is >= K */
#define LDA_IO_WORD_ROW 4    /* a sparse word's row leaves sparse_ent or holds a topic >= K */
#define LDA_IO_TOKEN_DOC 8   /* a tile token's doc id is >= num_docs */
#define LDA_IO_DOC_ROW 16    /* a doc row leaves dt_ent or holds a topic >= K */

/* Samples the tokens of io->tiles exactly as lda_sample_chunk does, but allocates
 * nothing: no cudaMalloc, cudaFree or allocating library call.  It exists for callers
 * that own all device memory through their own allocator or a pre-reserved arena (a
 * serving process that has handed HBM to its pool, an embedding framework with its own
 * caching allocator), where a library-side cudaMalloc/cudaFree would synchronise the
 * device, fragment the pool, or fail with out-of-memory in the middle of a request.
 * No counterpart in the reference: EZLDA allocates everything up front in its classes.
 *
 * Its scratch (tile counter, sweep counters, per-tile LL partials and, above 2048 topics,
 * the smoothing table of the sparse words' split Q bucket) is one file-scope device array
 * of 643,328 bytes that every GPU loading the library holds until the process exits.
 * Limits: num_tiles <= 65536 (LDA_ERR_ARG beyond); K at most what one warp's word column
 * plus the CTA's reciprocal table fit in shared memory, about 28,000 topics on a B200
 * (LDA_ERR_ARG beyond).  Every K runs the per-warp-column sampler the trainer uses up to
 * 2048 topics; above that the trainer splits dense and sparse words over two other
 * kernels, and this entry point draws the same topics with one.  Doc-row keys are topics
 * (the layout lda_get_doc_rows returns).
 *
 * The caller's indices are checked on the device before any token is sampled: a kernel
 * checks every tile, the max topic and sparse row of every tile's word, every tile
 * token's doc id and every doc row against K and the buffer lengths above, and writes the
 * failed checks to *io->status (0 when all pass; read it after the stream's work).  A
 * failure stops the sampling kernel from taking any tile, so bad input never indexes
 * memory.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress with that device current) and keeps it for the process; make that
 * first call before any stream capture, and do not reset the device (cudaDeviceReset)
 * after it.  Every call shares the array, so calls that overlap on the GPU (on different
 * streams or devices sharing a context) race; serialise them.  The call is asynchronous on
 * `stream` (NULL: the legacy default stream) and sets `device` current. */
int lda_sample_chunk_noalloc(const lda_sample_io* io, int32_t device, void* stream);

/* ------------------------------------------------ batched training */
/* No counterpart in the reference (EZLDA trains one corpus per process).  A batch sweeps
 * many resident trainers together: per stage, one persistent kernel takes work items of
 * every model from a shared list (each model keeps its own K, alpha, beta, seed and device
 * arrays), and the sweeps of one lda_batch_iterate call are one CUDA graph launch.  Every
 * model's topics after a batched sweep equal its own trainer's after the same sweep.  The
 * batch owns its trainers' state while it exists: sweeping a trainer on its own in between
 * makes lda_batch_iterate fail with LDA_ERR_STATE. */
typedef struct lda_batch lda_batch;
typedef struct {
    int32_t warps;        /* warps per CTA of the batched kernels, 1..8 */
    int32_t schedule;     /* 0: largest work items first across models; 1: model by model */
    int32_t tile_tokens;  /* tokens per sampler work item (>= 32): warps per frequent word */
} lda_batch_tuning;
/* tuning NULL: {8, 0, 512}.  The trainers must outlive the batch. */
int lda_batch_create(lda_trainer* const* trainers, int32_t n, const lda_batch_tuning* tuning, lda_batch** out);
int lda_batch_destroy(lda_batch* b);
int lda_batch_set_tuning(lda_batch* b, const lda_batch_tuning* tuning);
int lda_batch_get_tuning(const lda_batch* b, lda_batch_tuning* tuning);
/* `sweeps` sweeps of every model in one graph launch; with ll_mode the FP64 LL of the last
 * sweep per model (lda_batch_loglik, and each trainer's lda_trainer_loglik). */
int lda_batch_iterate(lda_batch* b, int32_t sweeps, int32_t ll_mode);
int lda_batch_loglik(const lda_batch* b, double* ll /*n*/, int32_t n);
int lda_batch_stats(const lda_batch* b, int64_t* kernel_launches, int64_t* work_items);
/* Times every candidate tuning (warps {4,8} x schedule {0,1} x tile_tokens {128,256,512})
 * for sweeps_per_trial sweeps on the live batch, restoring the models' topics, iterations
 * and counters after each trial, and keeps the fastest. */
int lda_batch_autotune(lda_batch* b, int32_t sweeps_per_trial, lda_batch_tuning* best, double* best_ms_per_sweep);

/* ------------------------------------------------ fold-in serving */
/* No counterpart in the reference: EZLDA trains only.  A model is the frozen word side
 * of a trainer (phi_wk = (n_wk+beta)/(n_k+V*beta) as a dense [V][K] float matrix plus
 * the per-word max topics and Q partials); fold-in of a new document runs `sweeps`
 * sweeps of the training sampler with the word side frozen and returns
 * theta_k = (n_dk+alpha)/(len+K*alpha).  A request's randoms are keyed on
 * (server seed, request id, sweep, token position): the same request gives the same
 * topics and theta whatever it is batched with. */
typedef struct lda_model lda_model;
typedef struct lda_server lda_server;

/* Freezes the trainer's current topics into a model (rebuilds the word-topic counts and
 * the per-word statistics first).  device_budget > 0 bounds the model's bytes. */
int lda_model_from_trainer(lda_trainer* t, int64_t device_budget, lda_model** out);
int lda_model_info(const lda_model* m, int32_t* K, int64_t* V, int64_t* bytes);
int lda_model_get_phi(const lda_model* m, int32_t w, float* out /*K*/);
void lda_model_free(lda_model* m);

/* A continuous-batching server over one model: a token pool of max_tokens tokens
 * (0: a quarter of the free device memory), at most max_active requests in flight.
 * The model must outlive the server. */
int lda_server_create(lda_model* m, int64_t max_tokens, int32_t max_active, int32_t sweeps, uint64_t seed,
                      lda_server** out);
int lda_server_destroy(lda_server* s);
/* Queues a document (word ranks of the model's vocabulary, 1..65535 tokens). */
int lda_server_submit(lda_server* s, uint32_t rid, const int32_t* words, int32_t len);
/* One step: admits queued requests that fit (FIFO), queues one sweep of every active
 * request on the server's stream, and retires requests whose last sweep has completed.
 * Up to two steps are queued on the device before a step waits for the older one; with
 * nothing to issue, a step waits for every queued step.  *n_done = requests retired. */
int lda_server_step(lda_server* s, int32_t* n_done);
/* Pops one finished request: returns 1 and fills rid / theta (K floats) / latency
 * (seconds from submit to completion), or 0 when none is waiting. */
int lda_server_poll(lda_server* s, uint32_t* rid, float* theta, double* latency_s);
int lda_server_status(const lda_server* s, int32_t* queued, int32_t* active, int64_t* free_tokens);
/* Current topics of an active request (len must match; synchronises the server's stream). */
int lda_server_get_topics(lda_server* s, uint32_t rid, uint16_t* out, int32_t len);
/* Tokens per work item (a multiple of 32, default 32): a request is split into items of
 * this many tokens, each sampled by one warp.  Only while the server is idle. */
int lda_server_set_item_tokens(lda_server* s, int32_t n);
/* Steps issued and fold-in kernel launches since creation. */
int lda_server_stats(const lda_server* s, int64_t* steps, int64_t* kernel_launches);
/* Real-time replay on an idle server: document i (words[doc_off[i]..doc_off[i+1]))
 * arrives arrival_s[i] seconds after the start (non-decreasing) and gets request id i;
 * latency_s[i] = completion - scheduled arrival; theta (n x K) optional. */
int lda_serve_replay(lda_server* s, int32_t n, const int64_t* doc_off, const int32_t* words,
                     const double* arrival_s, double* latency_s, float* theta, double* wall_s);

#ifdef __cplusplus
}
#endif
#endif
