/*
 * lda_oracle.h -- serial/threaded C restatement of EZLDA's collapsed-Gibbs sweep.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA path in
 * lda_sc20_b200/csrc; only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs may load it.  The product never links,
 * imports or calls anything here.
 *
 * Parity status: the count rebuilds, per-word top-3/Q and per-token doc
 * metadata follow EZLDA's kernels exactly (integer results are unique).  The
 * reference has no tests, golden vectors or CPU path, and its RNG is curand
 * XORWOW seeded from clock(), so per-token sampling is pinned against this
 * oracle's own Philox stream and distributionally (exact p(k) chi-square, LL
 * curve) against the reference.  See the header of lda_oracle.c for the full
 * arithmetic specification shared with the CUDA kernels.
 */
#ifndef LDA_ORACLE_H_
#define LDA_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Uniform in [0,1) for token `tok` at sweep `iter`. */
float orc_token_uniform(uint64_t seed, uint32_t iter, uint64_t tok);
/* Initial topic in [0,K) for token `tok`. */
uint16_t orc_init_topic(uint64_t seed, uint64_t tok, int32_t K);

typedef struct orc_state orc_state;

/* tok_word[i], tok_doc[i]: word rank and global doc id of token i, where i is
 * the global word-sorted token index that also keys the RNG. */
orc_state* orc_create(int64_t N, int32_t V, int32_t D, int32_t K,
                      const int32_t* tok_word, const int32_t* tok_doc,
                      float alpha, float beta, int32_t nthreads);
void orc_destroy(orc_state* s);

/* Rebuild every iteration-start count from topics z: n_k, doc rows (DT CSR),
 * per-word top-3 / Q.  Returns 0 on success, <0 on bad input. */
int orc_rebuild(orc_state* s, const uint16_t* z);

int orc_get_topic_totals(const orc_state* s, int32_t* n_k /*K*/);
/* Dense counts of word w (K entries). */
int orc_get_word_row(const orc_state* s, int32_t w, int32_t* row /*K*/);
/* Sparse word rows, packed (k<<16 | count), ascending k, for words
 * [w_begin, w_end); rows laid out back to back.  off has (w_end-w_begin+1). */
int64_t orc_get_word_rows_packed(const orc_state* s, int32_t w_begin, int32_t w_end,
                                 int64_t* off, uint32_t* ent, int64_t cap);
/* Per word: top2 = (k2<<16 | maxK), k3, phi4 = {phi_max, phi_2nd, phi_3rd, Q},
 * ql = 32 per-lane partial sums of alpha*phi (maxK excluded). */
int orc_get_word_stats(const orc_state* s, uint32_t* top2, uint32_t* k3,
                       float* phi4, float* ql);
/* Doc rows: nnz per doc and packed entries (k<<16 | count) ascending k,
 * concatenated in doc order (off = prefix of nnz, D+1 entries). */
int64_t orc_get_doc_rows(const orc_state* s, int64_t* off, uint32_t* ent, int64_t cap);
/* Per-token metadata (count of word's 2nd topic in the doc)<<16 | (count of
 * word's max topic in the doc). */
int orc_get_token_meta(const orc_state* s, uint32_t* meta /*N*/);
/* Reciprocal table r_k = 1/(n_k + V*beta). */
int orc_get_recip(const orc_state* s, float* r /*K*/);

typedef struct {
    int64_t tokens;       /* tokens sampled */
    int64_t early_accept; /* tokens settled by the max-topic bound */
    int64_t full;         /* tokens whose S was evaluated */
    int64_t sum_nnz_full; /* sum of doc-row nnz over evaluated tokens */
    int64_t branch_max, branch_s, branch_q;
    double  loglik;       /* sum over sampled tokens of log p(w|d) (ll_mode) */
} orc_sample_stats;

/* One sweep over the counts of the last orc_rebuild.  z_out must hold the
 * previous topics; only tokens of words w with (w % word_stride)==0 are
 * resampled (word_stride=1: all).  ll_mode=1 also evaluates S for
 * early-accepted tokens and accumulates the FP64 log-likelihood. */
int orc_sample(orc_state* s, uint16_t* z_out, uint64_t seed, uint32_t iter,
               int32_t ll_mode, int32_t word_stride, orc_sample_stats* st);

/* Words [0, Vd) are the trainer's dense words (default 0).  Above 2048 topics a sparse
 * word (w >= Vd) splits its Q bucket into its own topics and a word-independent smoothing
 * part; the rebuild's statistics and the draws follow.  Call before orc_rebuild. */
int orc_set_num_dense(orc_state* s, int32_t Vd);

/* Restricts orc_sample / orc_iterate to the tokens of docs [d0, d1) (the documents of a
 * range of chunks: what one rank of a document-sharded sweep samples); the others keep
 * their topics.  The default is every document. */
int orc_set_doc_range(orc_state* s, int32_t d0, int32_t d1);

/* Rebuild + sample: one full iteration, z updated in place. */
int orc_iterate(orc_state* s, uint16_t* z, uint64_t seed, uint32_t iter,
                int32_t ll_mode, orc_sample_stats* st);

/* Exact FP64 conditional p(k) (normalised) of token i under the current
 * counts: p(k) ∝ (n_dk+alpha)(n_wk+beta)/(n_k+V*beta).  Used to classify
 * disagreements and for distribution tests. */
int orc_token_probs(const orc_state* s, int64_t tok, double* p /*K*/);

/* Fold-in of one new document (words of the trained vocabulary) against the frozen
 * counts of the last orc_rebuild: `sweeps` sweeps from Philox initial topics keyed on
 * (seed, rid), then theta_k = ((float)n_dk + alpha) / ((float)len + (float)K * alpha). */
float orc_foldin_uniform(uint64_t seed, uint32_t rid, uint32_t sweep, uint32_t pos);
uint16_t orc_foldin_init(uint64_t seed, uint32_t rid, uint32_t pos, int32_t K);
int orc_foldin(const orc_state* s, const int32_t* words, int32_t len, uint32_t rid, uint64_t seed,
               int32_t sweeps, uint16_t* z, float* theta /*K or NULL*/);
/* phi_k of word w under the counts of the last orc_rebuild. */
int orc_get_phi_row(const orc_state* s, int32_t w, float* out /*K*/);

#ifdef __cplusplus
}
#endif
#endif
