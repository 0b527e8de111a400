/*
 * lda_oracle.c -- CPU oracle for the EZLDA collapsed-Gibbs sweep.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product; see lda_oracle.h).
 *
 * What it restates (EZLDA = asherliu/LDA_SC20, paths relative to that project):
 *   - iteration-start count snapshot: EZLDA/mainKernel.cu:158-380 rebuilds the
 *     sparse WT / n_k before the sweep (:163-185), the DT CSR per chunk from the
 *     chunk's previous topics (:228), and samples into a copy of the dense WT
 *     (utility.cu:1998,2937).  No "-1" exclusion of the current token
 *     (utility.cu:1347-1349,1400,2896-2898).
 *   - phi_k = (n_wk+beta)/(n_k+V*beta) (utility.cu:1259,1267,1700).
 *   - per-word max / 2nd / 3rd topic of phi (utility.cu:305-1062), Q =
 *     alpha*sum_{k!=max} phi_k (utility.cu:1272-1311).
 *   - DT rows: per-doc histogram compacted to (k,count) ascending k
 *     (utility.cu:79-284); per-token counts of the word's max and 2nd topic in
 *     the doc (utility.cu:125-161).
 *   - sampler: p_max=(n_d,max+alpha)phi_max, S over the doc row with
 *     phi_max zeroed, Q bucket; early accept when u < p_max/(p_max+Shat+Q)
 *     with Shat an upper bound of S (utility.cu:1341-1373, 2896-2898);
 *     three-way branch and two-level bin search (utility.cu:1447-1559).
 *   - LL: (1/N) sum_i log((S_i+Q_i)/(n_d+K*alpha)) with S,Q the full bucket
 *     masses (profilePerp/utility.cu:2398,2810,2883-2925), summed in FP64.
 *
 * Arithmetic specification shared with the CUDA kernels (every float op is a
 * single IEEE-754 binary32 operation, round to nearest; fmaf is fused):
 *   Vb      = (float)V * beta
 *   r_k     = 1.0f / ((float)n_k + Vb)
 *   phi_k   = ((float)n_wk + beta) * r_k
 *   maxK/k2/k3: argmax of phi, ties to the lower k, excluding the previous
 *   QL[l]   = serial fmaf(alpha, phi_k, acc) over k = l, l+32, ... < K, k != maxK
 *   QP      = inclusive Kogge-Stone scan of QL over 32 lanes; Q = QP[31]
 *   cmax,c2 = n_d,maxK and n_d,k2; rest = n_d - cmax - c2
 *   pmax    = ((float)cmax + alpha) * phi_max
 *   shat    = fmaf((float)c2, phi_2nd, (float)rest * phi_3rd)
 *   bound   = (pmax + shat) + Q;   early accept  <=>  u*bound < pmax
 *   colz    = phi with colz[maxK] = 0
 *   SL[l]   = serial fmaf((float)cnt_e, colz[k_e], acc) over the row entries
 *             e = l, l+32, l+64, ... < nnz (row ascending in k)
 *   SP      = Kogge-Stone scan of SL; S = SP[31]
 *   pS      = pmax + S; total = pS + Q; target = u*total
 *   target < pmax -> maxK;
 *   target < pS   -> S bucket, t = target - pmax, lanes (SL, SP); in lane l the
 *                    serial partial sums of SL[l]'s fmaf chain are compared with t2;
 *   otherwise     -> Q bucket, t = target - pS, lanes (QL, QP), slots of lane l:
 *                    k = l, l+32, ... < K, term = alpha * colz[k], in rounds of 32
 *                    slots: prefix = carry + Kogge-Stone scan of the round's terms
 *                    (empty slots 0), carry = the round's last prefix.
 *   Lane choice: the first lane l with t < P[l] and L[l] > 0 (else the last lane
 *   with L[l] > 0); t2 = t - P[l-1].  In the lane: the first entry/slot with
 *   colz > 0 whose partial sum / prefix exceeds t2, else the last one with
 *   colz > 0, else maxK.
 *   Split Q (K > 2048 and a sparse word, w >= Vd; SparseLDA's smoothing / word split):
 *   sm_k    = alpha * (beta * r_k); T[k] = carry + Kogge-Stone scan of sm over rounds
 *             of 32 topics (carry = the previous round's last prefix), Tsum = T[K-1]
 *   Qw      = the same rounds over the word's own topics (ascending k) with terms
 *             alpha * ((float)n_wk * r_k), the max topic's term 0; Qs = Tsum - sm_max;
 *             Q = Qw + Qs (QL = {Qw, Qs, 0, ...})
 *   Q draw  : t < Qw -> the first own topic with a non-zero term whose prefix exceeds t
 *             (else the last such topic); otherwise t' = t - Qw: the first k < maxK with
 *             t' < T[k] if t' < T[maxK-1], else the first k > maxK with t' + sm_max < T[k],
 *             else the last topic other than maxK.  Fold-in keeps the lane form (its
 *             frozen model has no word rows): QL from the column as above.
 *   LL_i    = log((double)total / ((double)n_d + (double)K * (double)alpha))
 * Randoms: u = (float)(x0 >> 8) * 2^-24 with x = Philox4x32-10(ctr = {tok_lo,
 * tok_hi, iter, 0x4C444131}, key = {seed_lo, seed_hi}); initial topic =
 * (x0 * K) >> 32 with ctr = {tok_lo, tok_hi, 0xFFFFFFFF, 0x494E4954}.
 */
#include "lda_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define LANES 32

/* ------------------------------------------------------------------ Philox */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * (uint64_t)c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * (uint64_t)c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

float orc_token_uniform(uint64_t seed, uint32_t iter, uint64_t tok) {
    uint32_t ctr[4] = {(uint32_t)tok, (uint32_t)(tok >> 32), iter, 0x4C444131u};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t x[4];
    orc_philox4x32_10(ctr, key, x);
    return (float)(x[0] >> 8) * 0x1p-24f;
}

uint16_t orc_init_topic(uint64_t seed, uint64_t tok, int32_t K) {
    uint32_t ctr[4] = {(uint32_t)tok, (uint32_t)(tok >> 32), 0xFFFFFFFFu, 0x494E4954u};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t x[4];
    orc_philox4x32_10(ctr, key, x);
    return (uint16_t)(((uint64_t)x[0] * (uint64_t)(uint32_t)K) >> 32);
}

/* ------------------------------------------------------------------- state */
/* Above this many topics a sparse word (w >= Vd) splits its Q bucket into the word's own
 * topics and a word-independent smoothing part (see the specification above). */
#define ORC_LARGE_K 2048

struct orc_state {
    int64_t N;
    int32_t doc_lo, doc_hi; /* orc_sample draws only tokens of docs in [doc_lo, doc_hi) */
    int32_t Vd;             /* words [0, Vd) are dense (the trainer's split) */
    float* T;               /* K > ORC_LARGE_K: smoothing prefix table, T[K-1] = Tsum */
    float Tsum;
    int32_t V, D, K, nthreads;
    float alpha, beta;
    const int32_t* tok_word;
    const int32_t* tok_doc;
    /* static indices */
    int64_t* woff; /* V+1 */
    int64_t* wtok; /* N: token ids grouped by word, ascending */
    int64_t* doff; /* D+1 */
    int64_t* dtok; /* N: token ids grouped by doc, ascending */
    int64_t* rcap; /* D+1: doc-row capacity offsets, cap = min(len, K) */
    /* rebuilt per iteration */
    const uint16_t* z;
    int32_t* n_k;
    float* r;
    int32_t* rnnz;  /* D */
    uint32_t* rent; /* rcap[D] */
    uint32_t* top2; /* V */
    uint32_t* k3;   /* V */
    float* phi4;    /* V*4 */
    float* ql;      /* V*32 */
    int built;
};

static int64_t* counting_index(int64_t N, int32_t n_keys, const int32_t* key, int64_t** out_idx) {
    int64_t* off = (int64_t*)calloc((size_t)n_keys + 1, sizeof(int64_t));
    int64_t* idx = (int64_t*)malloc((size_t)(N > 0 ? N : 1) * sizeof(int64_t));
    if (!off || !idx) { free(off); free(idx); return NULL; }
    for (int64_t i = 0; i < N; ++i) off[key[i] + 1]++;
    for (int32_t k = 0; k < n_keys; ++k) off[k + 1] += off[k];
    int64_t* fill = (int64_t*)malloc(((size_t)n_keys + 1) * sizeof(int64_t));
    if (!fill) { free(off); free(idx); return NULL; }
    memcpy(fill, off, ((size_t)n_keys + 1) * sizeof(int64_t));
    for (int64_t i = 0; i < N; ++i) idx[fill[key[i]]++] = i;
    free(fill);
    *out_idx = idx;
    return off;
}

orc_state* orc_create(int64_t N, int32_t V, int32_t D, int32_t K, const int32_t* tok_word,
                      const int32_t* tok_doc, float alpha, float beta, int32_t nthreads) {
    if (N < 0 || V <= 0 || D <= 0 || K < 4 || K > 65535) return NULL;
    for (int64_t i = 0; i < N; ++i) {
        if (tok_word[i] < 0 || tok_word[i] >= V || tok_doc[i] < 0 || tok_doc[i] >= D) return NULL;
    }
    orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
    if (!s) return NULL;
    s->N = N; s->V = V; s->D = D; s->K = K;
    s->nthreads = nthreads > 0 ? nthreads : 1;
    s->alpha = alpha; s->beta = beta;
    s->tok_word = tok_word; s->tok_doc = tok_doc;
    s->doc_lo = 0; s->doc_hi = D;
    s->Vd = 0;
    s->woff = counting_index(N, V, tok_word, &s->wtok);
    s->doff = counting_index(N, D, tok_doc, &s->dtok);
    s->rcap = (int64_t*)calloc((size_t)D + 1, sizeof(int64_t));
    s->n_k = (int32_t*)calloc((size_t)K, sizeof(int32_t));
    s->r = (float*)calloc((size_t)K, sizeof(float));
    s->rnnz = (int32_t*)calloc((size_t)D, sizeof(int32_t));
    s->top2 = (uint32_t*)calloc((size_t)V, sizeof(uint32_t));
    s->k3 = (uint32_t*)calloc((size_t)V, sizeof(uint32_t));
    s->phi4 = (float*)calloc((size_t)V * 4, sizeof(float));
    s->ql = (float*)calloc((size_t)V * LANES, sizeof(float));
    s->T = (float*)calloc((size_t)K, sizeof(float));
    if (!s->woff || !s->doff || !s->rcap || !s->n_k || !s->r || !s->rnnz || !s->top2 || !s->k3 ||
        !s->phi4 || !s->ql || !s->T) {
        orc_destroy(s);
        return NULL;
    }
    for (int32_t d = 0; d < D; ++d) {
        int64_t len = s->doff[d + 1] - s->doff[d];
        if (len > 65535) { orc_destroy(s); return NULL; } /* counts are packed in 16 bits */
        s->rcap[d + 1] = s->rcap[d] + (len < K ? len : K);
    }
    s->rent = (uint32_t*)calloc((size_t)(s->rcap[D] > 0 ? s->rcap[D] : 1), sizeof(uint32_t));
    if (!s->rent) { orc_destroy(s); return NULL; }
    return s;
}

void orc_destroy(orc_state* s) {
    if (!s) return;
    free(s->woff); free(s->wtok); free(s->doff); free(s->dtok); free(s->rcap);
    free(s->n_k); free(s->r); free(s->rnnz); free(s->rent);
    free(s->top2); free(s->k3); free(s->phi4); free(s->ql); free(s->T);
    free(s);
}

int orc_set_num_dense(orc_state* s, int32_t Vd) {
    if (!s || Vd < 0 || Vd > s->V) return -1;
    s->Vd = Vd;
    s->built = 0;
    return 0;
}

/* Whether word w draws its Q bucket in two parts (the word's topics, then smoothing). */
static int split_word(const orc_state* s, int32_t w) { return s->K > ORC_LARGE_K && w >= s->Vd; }

/* ------------------------------------------------------------- thread pool */
typedef void (*task_fn)(void* ctx, int64_t begin, int64_t end, int tid);
typedef struct {
    task_fn fn; void* ctx; int64_t n, grain; int64_t next; int tid;
} pf_arg;
typedef struct { pf_arg* shared; int tid; } pf_worker;

static void* pf_run(void* p) {
    pf_worker* w = (pf_worker*)p;
    pf_arg* a = w->shared;
    for (;;) {
        int64_t b = __atomic_fetch_add(&a->next, a->grain, __ATOMIC_RELAXED);
        if (b >= a->n) break;
        int64_t e = b + a->grain < a->n ? b + a->grain : a->n;
        a->fn(a->ctx, b, e, w->tid);
    }
    return NULL;
}

static void parallel_for(int nthreads, int64_t n, int64_t grain, task_fn fn, void* ctx) {
    pf_arg a = {fn, ctx, n, grain > 0 ? grain : 1, 0, 0};
    if (nthreads <= 1 || n <= grain) {
        pf_worker w = {&a, 0};
        pf_run(&w);
        return;
    }
    pthread_t th[256];
    pf_worker ws[256];
    int nt = nthreads > 256 ? 256 : nthreads;
    for (int t = 0; t < nt; ++t) { ws[t].shared = &a; ws[t].tid = t; }
    for (int t = 1; t < nt; ++t) pthread_create(&th[t], NULL, pf_run, &ws[t]);
    pf_run(&ws[0]);
    for (int t = 1; t < nt; ++t) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------ shared */
/* Inclusive Kogge-Stone scan over 32 lanes, the order a warp's shfl_up scan
 * adds in: round `off` adds lane l-off into lane l for l >= off. */
static void ks_scan32(const float* in, float* out) {
    float v[LANES], nv[LANES];
    memcpy(v, in, sizeof(v));
    for (int off = 1; off < LANES; off <<= 1) {
        for (int l = 0; l < LANES; ++l) nv[l] = l >= off ? v[l] + v[l - off] : v[l];
        memcpy(v, nv, sizeof(v));
    }
    memcpy(out, v, sizeof(v));
}

/* n_dk from the doc row (binary search; rows are ascending in k). */
static int32_t row_count(const uint32_t* ent, int32_t nnz, int32_t k) {
    int32_t lo = 0, hi = nnz - 1;
    while (lo <= hi) {
        int32_t mid = (lo + hi) >> 1;
        int32_t km = (int32_t)(ent[mid] >> 16);
        if (km == k) return (int32_t)(ent[mid] & 0xffffu);
        if (km < k) lo = mid + 1; else hi = mid - 1;
    }
    return 0;
}

/* Word column phi_k = ((float)n_wk + beta) * r_k (utility.cu:1259,1267,1700). */
static void word_column(const orc_state* s, int32_t w, int32_t* cnt, float* col) {
    const int32_t K = s->K;
    memset(cnt, 0, sizeof(int32_t) * (size_t)K);
    for (int64_t j = s->woff[w]; j < s->woff[w + 1]; ++j) cnt[s->z[s->wtok[j]]]++;
    for (int32_t k = 0; k < K; ++k) col[k] = ((float)cnt[k] + s->beta) * s->r[k];
}

/* ------------------------------------------------------------------ rebuild */
typedef struct {
    orc_state* s;
    int32_t** icnt;  /* per-thread K ints */
    float** fcol;    /* per-thread K floats */
    uint32_t** list; /* per-thread K touched topics */
    int32_t** nkp;   /* per-thread partial n_k */
} rb_ctx;

static void rb_topic_totals(void* c, int64_t b, int64_t e, int tid) {
    rb_ctx* x = (rb_ctx*)c;
    int32_t* nk = x->nkp[tid];
    for (int64_t i = b; i < e; ++i) nk[x->s->z[i]]++;
}

static int cmp_u32(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x < y ? -1 : x > y;
}

/* DT row of doc d: per-doc histogram compacted to (k<<16 | count) ascending k
 * (EZLDA/utility.cu:102-123 histogram, :183-236 ballot compaction). */
static void rb_doc_rows(void* c, int64_t b, int64_t e, int tid) {
    rb_ctx* x = (rb_ctx*)c;
    orc_state* s = x->s;
    int32_t* h = x->icnt[tid];
    uint32_t* list = x->list[tid];
    for (int64_t d = b; d < e; ++d) {
        int32_t n = 0;
        for (int64_t j = s->doff[d]; j < s->doff[d + 1]; ++j) {
            uint16_t k = s->z[s->dtok[j]];
            if (h[k]++ == 0) list[n++] = k;
        }
        qsort(list, (size_t)n, sizeof(uint32_t), cmp_u32);
        uint32_t* out = s->rent + s->rcap[d];
        for (int32_t i = 0; i < n; ++i) {
            out[i] = (list[i] << 16) | (uint32_t)h[list[i]];
            h[list[i]] = 0;
        }
        s->rnnz[d] = n;
    }
}

/* Per-word top-3 of phi and the 32 lane partials of Q (EZLDA/utility.cu:305-678
 * dense, :679-1062 sparse; Q = alpha*(sum phi - phi_max), :1272-1311). */
static void rb_word_stats(void* c, int64_t b, int64_t e, int tid) {
    rb_ctx* x = (rb_ctx*)c;
    orc_state* s = x->s;
    const int32_t K = s->K;
    int32_t* cnt = x->icnt[tid];
    float* col = x->fcol[tid];
    for (int64_t w = b; w < e; ++w) {
        word_column(s, (int32_t)w, cnt, col);
        int32_t m1 = 0;
        for (int32_t k = 1; k < K; ++k) if (col[k] > col[m1]) m1 = k;
        int32_t m2 = -1;
        for (int32_t k = 0; k < K; ++k) {
            if (k == m1) continue;
            if (m2 < 0 || col[k] > col[m2]) m2 = k;
        }
        int32_t m3 = -1;
        for (int32_t k = 0; k < K; ++k) {
            if (k == m1 || k == m2) continue;
            if (m3 < 0 || col[k] > col[m3]) m3 = k;
        }
        float* ql = s->ql + w * LANES;
        float qp[LANES];
        if (split_word(s, (int32_t)w)) {
            /* Q = Qw + Qs: Qw over the word's own topics in rounds of 32 entries (ascending
             * k, the max topic's term 0), Qs = Tsum - sm_max; ql holds {Qw, Qs, 0, ...} */
            float carry = 0.0f, tr[LANES], P[LANES];
            int n = 0;
            for (int32_t k = 0; k <= K; ++k) {
                if (k < K) {
                    if (!cnt[k]) continue;
                    tr[n++] = k == m1 ? 0.0f : s->alpha * ((float)cnt[k] * s->r[k]);
                }
                if (n == LANES || (k == K && n > 0)) {
                    for (int i = n; i < LANES; ++i) tr[i] = 0.0f;
                    ks_scan32(tr, P);
                    carry = carry + P[LANES - 1];
                    n = 0;
                }
            }
            memset(ql, 0, sizeof(float) * LANES);
            ql[0] = carry;
            ql[1] = s->Tsum - s->alpha * (s->beta * s->r[m1]);
            qp[LANES - 1] = ql[0] + ql[1];
        } else {
            for (int l = 0; l < LANES; ++l) {
                float acc = 0.0f;
                for (int32_t k = l; k < K; k += LANES)
                    if (k != m1) acc = fmaf(s->alpha, col[k], acc);
                ql[l] = acc;
            }
            ks_scan32(ql, qp);
        }
        s->top2[w] = ((uint32_t)m2 << 16) | (uint32_t)m1;
        s->k3[w] = (uint32_t)m3;
        s->phi4[w * 4 + 0] = col[m1];
        s->phi4[w * 4 + 1] = col[m2];
        s->phi4[w * 4 + 2] = col[m3];
        s->phi4[w * 4 + 3] = qp[LANES - 1];
    }
}

int orc_rebuild(orc_state* s, const uint16_t* z) {
    if (!s || !z) return -1;
    for (int64_t i = 0; i < s->N; ++i) if (z[i] >= s->K) return -2;
    s->z = z;
    const int nt = s->nthreads;
    rb_ctx x;
    x.s = s;
    x.icnt = (int32_t**)calloc((size_t)nt, sizeof(int32_t*));
    x.fcol = (float**)calloc((size_t)nt, sizeof(float*));
    x.list = (uint32_t**)calloc((size_t)nt, sizeof(uint32_t*));
    x.nkp = (int32_t**)calloc((size_t)nt, sizeof(int32_t*));
    for (int t = 0; t < nt; ++t) {
        x.icnt[t] = (int32_t*)calloc((size_t)s->K, sizeof(int32_t));
        x.fcol[t] = (float*)calloc((size_t)s->K, sizeof(float));
        x.list[t] = (uint32_t*)calloc((size_t)s->K, sizeof(uint32_t));
        x.nkp[t] = (int32_t*)calloc((size_t)s->K, sizeof(int32_t));
    }
    /* n_k (EZLDA/utility.cu:1104-1126 dense part, :1163-1169 sparse part) */
    parallel_for(nt, s->N, 1 << 20, rb_topic_totals, &x);
    memset(s->n_k, 0, sizeof(int32_t) * (size_t)s->K);
    for (int t = 0; t < nt; ++t)
        for (int32_t k = 0; k < s->K; ++k) s->n_k[k] += x.nkp[t][k];
    const float Vb = (float)s->V * s->beta;
    for (int32_t k = 0; k < s->K; ++k) s->r[k] = 1.0f / ((float)s->n_k[k] + Vb);
    if (s->K > ORC_LARGE_K) {
        /* smoothing table: T[k] = carry + Kogge-Stone scan of sm in rounds of 32 topics,
         * sm_k = alpha * (beta * r_k); the carry is the previous round's last prefix */
        float carry = 0.0f;
        for (int32_t base = 0; base < s->K; base += LANES) {
            float tr[LANES], P[LANES];
            for (int i = 0; i < LANES; ++i)
                tr[i] = base + i < s->K ? s->alpha * (s->beta * s->r[base + i]) : 0.0f;
            ks_scan32(tr, P);
            for (int i = 0; i < LANES && base + i < s->K; ++i) s->T[base + i] = carry + P[i];
            carry = carry + P[LANES - 1];
        }
        s->Tsum = carry;
    }
    parallel_for(nt, s->D, 256, rb_doc_rows, &x);
    parallel_for(nt, s->V, 64, rb_word_stats, &x);
    for (int t = 0; t < nt; ++t) { free(x.icnt[t]); free(x.fcol[t]); free(x.list[t]); free(x.nkp[t]); }
    free(x.icnt); free(x.fcol); free(x.list); free(x.nkp);
    s->built = 1;
    return 0;
}

/* ------------------------------------------------------------------ getters */
int orc_get_topic_totals(const orc_state* s, int32_t* n_k) {
    if (!s || !s->built) return -1;
    memcpy(n_k, s->n_k, sizeof(int32_t) * (size_t)s->K);
    return 0;
}

int orc_get_recip(const orc_state* s, float* r) {
    if (!s || !s->built) return -1;
    memcpy(r, s->r, sizeof(float) * (size_t)s->K);
    return 0;
}

int orc_get_word_row(const orc_state* s, int32_t w, int32_t* row) {
    if (!s || !s->built || w < 0 || w >= s->V) return -1;
    memset(row, 0, sizeof(int32_t) * (size_t)s->K);
    for (int64_t j = s->woff[w]; j < s->woff[w + 1]; ++j) row[s->z[s->wtok[j]]]++;
    return 0;
}

int64_t orc_get_word_rows_packed(const orc_state* s, int32_t w_begin, int32_t w_end, int64_t* off,
                                 uint32_t* ent, int64_t cap) {
    if (!s || !s->built || w_begin < 0 || w_end > s->V || w_begin > w_end) return -1;
    int32_t* row = (int32_t*)malloc(sizeof(int32_t) * (size_t)s->K);
    if (!row) return -1;
    int64_t n = 0;
    off[0] = 0;
    for (int32_t w = w_begin; w < w_end; ++w) {
        orc_get_word_row(s, w, row);
        for (int32_t k = 0; k < s->K; ++k) {
            if (!row[k]) continue;
            if (n >= cap) { free(row); return -2; }
            ent[n++] = ((uint32_t)k << 16) | (uint32_t)row[k];
        }
        off[w - w_begin + 1] = n;
    }
    free(row);
    return n;
}

int orc_get_word_stats(const orc_state* s, uint32_t* top2, uint32_t* k3, float* phi4, float* ql) {
    if (!s || !s->built) return -1;
    if (top2) memcpy(top2, s->top2, sizeof(uint32_t) * (size_t)s->V);
    if (k3) memcpy(k3, s->k3, sizeof(uint32_t) * (size_t)s->V);
    if (phi4) memcpy(phi4, s->phi4, sizeof(float) * (size_t)s->V * 4);
    if (ql) memcpy(ql, s->ql, sizeof(float) * (size_t)s->V * LANES);
    return 0;
}

int64_t orc_get_doc_rows(const orc_state* s, int64_t* off, uint32_t* ent, int64_t cap) {
    if (!s || !s->built) return -1;
    int64_t n = 0;
    off[0] = 0;
    for (int32_t d = 0; d < s->D; ++d) {
        if (n + s->rnnz[d] > cap) return -2;
        memcpy(ent + n, s->rent + s->rcap[d], sizeof(uint32_t) * (size_t)s->rnnz[d]);
        n += s->rnnz[d];
        off[d + 1] = n;
    }
    return n;
}

/* Per-token counts of the word's max and 2nd topic in its doc
 * (EZLDA/utility.cu:125-161: (docId+1)<<32 | DT[2nd]<<16 | DT[max]). */
int orc_get_token_meta(const orc_state* s, uint32_t* meta) {
    if (!s || !s->built) return -1;
    for (int64_t i = 0; i < s->N; ++i) {
        int32_t w = s->tok_word[i], d = s->tok_doc[i];
        uint32_t t2 = s->top2[w];
        const uint32_t* row = s->rent + s->rcap[d];
        int32_t cmax = row_count(row, s->rnnz[d], (int32_t)(t2 & 0xffffu));
        int32_t c2 = row_count(row, s->rnnz[d], (int32_t)(t2 >> 16));
        meta[i] = ((uint32_t)c2 << 16) | (uint32_t)cmax;
    }
    return 0;
}

int orc_token_probs(const orc_state* s, int64_t tok, double* p) {
    if (!s || !s->built || tok < 0 || tok >= s->N) return -1;
    const int32_t K = s->K;
    int32_t w = s->tok_word[tok], d = s->tok_doc[tok];
    int32_t* row = (int32_t*)malloc(sizeof(int32_t) * (size_t)K);
    if (!row) return -1;
    orc_get_word_row(s, w, row);
    const uint32_t* drow = s->rent + s->rcap[d];
    double tot = 0.0, Vb = (double)s->V * (double)s->beta;
    for (int32_t k = 0; k < K; ++k) {
        double ndk = (double)row_count(drow, s->rnnz[d], k);
        p[k] = (ndk + (double)s->alpha) * ((double)row[k] + (double)s->beta) / ((double)s->n_k[k] + Vb);
        tot += p[k];
    }
    for (int32_t k = 0; k < K; ++k) p[k] /= tot;
    free(row);
    return 0;
}

/* ------------------------------------------------------------------- sample */
typedef struct {
    orc_state* s;
    uint16_t* z_out;
    uint64_t seed;
    uint32_t iter;
    int32_t ll_mode, word_stride;
    int32_t** icnt;
    float** fcol;
    double* wll;            /* per-word LL partial */
    orc_sample_stats* part; /* per-thread counters */
} sp_ctx;

/* Bucket search shared by S and Q (EZLDA/utility.cu:1456-1552): first lane
 * with t < P[l] and L[l] > 0, else the last lane with L[l] > 0. */
static int pick_lane(float t, const float* P, const float* L) {
    for (int l = 0; l < LANES; ++l) if (t < P[l] && L[l] > 0.0f) return l;
    for (int l = LANES - 1; l >= 0; --l) if (L[l] > 0.0f) return l;
    return -1;
}

/* The per-word state a draw reads. */
typedef struct {
    int32_t K, maxK;
    float alpha, phi1, phi2, phi3, Q;
    const float* QL;   /* 32 lane partials of Q */
    const float* QP;   /* their Kogge-Stone scan */
    const float* colz; /* the word's column with colz[maxK] = 0 */
    /* split Q (K > ORC_LARGE_K, sparse word): Q = Qw + Qs */
    int split;
    float Qw, Qs, beta, Tsum;
    const int32_t* wk; /* the word's topics, ascending */
    const int32_t* wn; /* their counts */
    int32_t nw;
    const float* r;    /* r_k */
    const float* T;    /* smoothing prefix table */
} word_ctx;

/* First k in [lo, hi) with x < T[k] (T non-decreasing, so a binary search), else -1. */
static int32_t first_above(const float* T, int32_t lo, int32_t hi, float x) {
    if (lo >= hi || !(x < T[hi - 1])) return -1;
    while (lo < hi) {
        const int32_t mid = lo + (hi - lo) / 2;
        if (x < T[mid]) hi = mid; else lo = mid + 1;
    }
    return lo;
}

/* The Q-bucket draw of a split word for t = target - pS: the word's own topics first (rounds
 * of 32 entries: carry + Kogge-Stone scan of alpha * (n_wk * r_k), the max topic's term 0;
 * the first entry with a non-zero term whose prefix exceeds t, else the last such entry),
 * then smoothing for t' = t - Qw against the table T with the max topic left out: the first
 * k < maxK with t' < T[k] when t' < T[maxK-1], else the first k > maxK with
 * t' + sm_max < T[k], else the last topic other than maxK. */
static int32_t draw_q_split(const word_ctx* w, float t) {
    if (t < w->Qw) {
        float carry = 0.0f;
        int32_t last = -1;
        for (int32_t base = 0; base < w->nw; base += LANES) {
            float tr[LANES], P[LANES];
            for (int i = 0; i < LANES; ++i) {
                const int32_t e = base + i;
                tr[i] = (e < w->nw && w->wk[e] != w->maxK) ? w->alpha * ((float)w->wn[e] * w->r[w->wk[e]]) : 0.0f;
            }
            ks_scan32(tr, P);
            for (int i = 0; i < LANES; ++i) P[i] = carry + P[i];
            for (int i = 0; i < LANES && base + i < w->nw; ++i)
                if (tr[i] > 0.0f && t < P[i]) return w->wk[base + i];
            for (int i = 0; i < LANES && base + i < w->nw; ++i)
                if (tr[i] > 0.0f) last = w->wk[base + i];
            carry = P[LANES - 1];
        }
        if (last >= 0) return last;
    }
    const float t1 = t - w->Qw;
    const int32_t m = w->maxK;
    if (m > 0 && t1 < w->T[m - 1]) return first_above(w->T, 0, m, t1);
    const float t2 = t1 + w->alpha * (w->beta * w->r[m]);
    const int32_t k = first_above(w->T, m + 1, w->K, t2);
    if (k >= 0) return k;
    return m == w->K - 1 ? w->K - 2 : w->K - 1;
}

enum { BR_MAX = 0, BR_S = 1, BR_Q = 2 };

/* One token's draw under the arithmetic specification at the top of this file.  The
 * doc row (ascending k), the counts of the word's max / 2nd topic in the doc and the
 * uniform are the token's inputs.  With force_eval the row mass is evaluated even when
 * the early-accept bound settles the draw (LL mode).  *total is the full mass when the
 * row was evaluated (else 0). */
static int32_t draw_token(const word_ctx* w, const uint32_t* row, int32_t nnz, int32_t cmax, int32_t c2,
                          int32_t nd, float u, int force_eval, int* ea_out, int* evaluated, float* total_out,
                          int* branch) {
    const float pmax = ((float)cmax + w->alpha) * w->phi1;
    const int32_t rest = nd - cmax - c2;
    const float shat = fmaf((float)c2, w->phi2, (float)rest * w->phi3);
    const float bound = (pmax + shat) + w->Q;
    const int ea = (u * bound < pmax);
    *ea_out = ea;
    *evaluated = 0;
    *total_out = 0.0f;
    *branch = BR_MAX;
    if (ea && !force_eval) return w->maxK;
    /* S: lane l sums the doc row's entries l, l+32, l+64, ...; the lane sums are
     * Kogge-Stone scanned (EZLDA likewise strides the row over a warp's lanes in 32-entry
     * steps, EZLDA/utility.cu:1376-1440) */
    float SL[LANES], SP[LANES];
    for (int l = 0; l < LANES; ++l) {
        float acc = 0.0f;
        for (int32_t q = l; q < nnz; q += LANES)
            acc = fmaf((float)(row[q] & 0xffffu), w->colz[row[q] >> 16], acc);
        SL[l] = acc;
    }
    ks_scan32(SL, SP);
    const float S = SP[LANES - 1];
    const float pS = pmax + S;
    const float total = pS + w->Q;
    *evaluated = 1;
    *total_out = total;
    if (ea) return w->maxK;
    const float target = u * total;
    if (target < pmax) return w->maxK;
    if (target < pS) {
        *branch = BR_S;
        const float tt = target - pmax;
        const int l = pick_lane(tt, SP, SL);
        const float t2 = tt - (l > 0 ? SP[l - 1] : 0.0f);
        if (l < 0) return w->maxK;
        /* the lane's serial partial sums (the fmaf chain of SL[l]) */
        float acc = 0.0f;
        int32_t last = -1;
        for (int32_t q = l; q < nnz; q += LANES) {
            const int32_t k = (int32_t)(row[q] >> 16);
            acc = fmaf((float)(row[q] & 0xffffu), w->colz[k], acc);
            if (w->colz[k] > 0.0f) {
                last = k;
                if (t2 < acc) return k;
            }
        }
        return last >= 0 ? last : w->maxK;
    }
    *branch = BR_Q;
    const float tt = target - pS;
    if (w->split) return draw_q_split(w, tt);
    const int l = pick_lane(tt, w->QP, w->QL);
    const float t2 = tt - (l > 0 ? w->QP[l - 1] : 0.0f);
    if (l < 0) return w->maxK;
    /* rounds of 32 of the lane's topics k = l, l+32, ...: carry + Kogge-Stone scan */
    const int32_t n = (w->K - l + LANES - 1) / LANES;
    float carry = 0.0f;
    int32_t last = -1;
    for (int32_t base = 0; base < n; base += LANES) {
        float tr[LANES], P[LANES];
        for (int i = 0; i < LANES; ++i) tr[i] = base + i < n ? w->alpha * w->colz[l + LANES * (base + i)] : 0.0f;
        ks_scan32(tr, P);
        for (int i = 0; i < LANES; ++i) P[i] = carry + P[i];
        for (int i = 0; i < LANES && base + i < n; ++i) {
            const int32_t k = l + LANES * (base + i);
            if (w->colz[k] > 0.0f && t2 < P[i]) return k;
        }
        for (int i = 0; i < LANES && base + i < n; ++i) {
            const int32_t k = l + LANES * (base + i);
            if (w->colz[k] > 0.0f) last = k;
        }
        carry = P[LANES - 1];
    }
    return last >= 0 ? last : w->maxK;
}

/* Fills the word context of word w (its column with colz[maxK] = 0).  A split word gets
 * its own topics and counts in wk / wn (K entries each).  With lane_q a split word instead
 * draws its Q bucket by lane partials formed here from the column (the fold-in's
 * specification, which has no sparse word rows), into ql. */
static void word_ctx_of(const orc_state* s, int32_t w, int32_t* cnt, float* colz, float* QP, word_ctx* wc,
                        int32_t* wk, int32_t* wn, float* ql, int lane_q) {
    word_column(s, w, cnt, colz);
    wc->K = s->K;
    wc->alpha = s->alpha;
    wc->beta = s->beta;
    wc->maxK = (int32_t)(s->top2[w] & 0xffffu);
    wc->phi1 = s->phi4[(int64_t)w * 4 + 0];
    wc->phi2 = s->phi4[(int64_t)w * 4 + 1];
    wc->phi3 = s->phi4[(int64_t)w * 4 + 2];
    wc->split = split_word(s, w) && !lane_q;
    wc->QL = s->ql + (int64_t)w * LANES;
    if (split_word(s, w) && lane_q) {
        for (int l = 0; l < LANES; ++l) {
            float acc = 0.0f;
            for (int32_t k = l; k < s->K; k += LANES)
                if (k != wc->maxK) acc = fmaf(s->alpha, colz[k], acc);
            ql[l] = acc;
        }
        wc->QL = ql;
    }
    ks_scan32(wc->QL, QP);
    wc->QP = QP;
    wc->Q = QP[LANES - 1];
    if (wc->split) {
        wc->Qw = s->ql[(int64_t)w * LANES];
        wc->Qs = s->ql[(int64_t)w * LANES + 1];
        wc->Q = s->phi4[(int64_t)w * 4 + 3];
        int32_t n = 0;
        for (int32_t k = 0; k < s->K; ++k)
            if (cnt[k]) { wk[n] = k; wn[n] = cnt[k]; ++n; }
        wc->wk = wk;
        wc->wn = wn;
        wc->nw = n;
        wc->r = s->r;
        wc->T = s->T;
        wc->Tsum = s->Tsum;
    }
    colz[wc->maxK] = 0.0f;
    wc->colz = colz;
}

static void sp_words(void* c, int64_t b, int64_t e, int tid) {
    sp_ctx* x = (sp_ctx*)c;
    orc_state* s = x->s;
    const double den_add = (double)s->K * (double)s->alpha;
    int32_t* cnt = x->icnt[tid];
    float* colz = x->fcol[tid];
    orc_sample_stats* st = &x->part[tid];
    for (int64_t w = b; w < e; ++w) {
        if (w % x->word_stride) continue;
        if (s->woff[w + 1] == s->woff[w]) continue;
        float QP[LANES];
        word_ctx wc;
        word_ctx_of(s, (int32_t)w, cnt, colz, QP, &wc, cnt + s->K, cnt + 2 * (size_t)s->K, NULL, 0);
        double wll = 0.0;
        for (int64_t j = s->woff[w]; j < s->woff[w + 1]; ++j) {
            const int64_t t = s->wtok[j];
            const int32_t d = s->tok_doc[t];
            if (d < s->doc_lo || d >= s->doc_hi) continue;
            const int32_t nd = (int32_t)(s->doff[d + 1] - s->doff[d]);
            const uint32_t* row = s->rent + s->rcap[d];
            const int32_t nnz = s->rnnz[d];
            const int32_t cmax = row_count(row, nnz, wc.maxK);
            const int32_t c2 = row_count(row, nnz, (int32_t)(s->top2[w] >> 16));
            const float u = orc_token_uniform(x->seed, x->iter, (uint64_t)t);
            int ea, evald, br;
            float total;
            const int32_t z = draw_token(&wc, row, nnz, cmax, c2, nd, u, x->ll_mode, &ea, &evald, &total, &br);
            st->tokens++;
            if (ea) st->early_accept++;
            if (evald) {
                st->full++;
                st->sum_nnz_full += nnz;
                if (x->ll_mode) wll += log((double)total / ((double)nd + den_add));
            }
            if (br == BR_S) st->branch_s++;
            else if (br == BR_Q) st->branch_q++;
            else st->branch_max++;
            x->z_out[t] = (uint16_t)z;
        }
        x->wll[w] = wll;
    }
}

int orc_sample(orc_state* s, uint16_t* z_out, uint64_t seed, uint32_t iter, int32_t ll_mode,
               int32_t word_stride, orc_sample_stats* st) {
    if (!s || !s->built || !z_out || word_stride < 1) return -1;
    const int nt = s->nthreads;
    sp_ctx x;
    x.s = s; x.z_out = z_out; x.seed = seed; x.iter = iter;
    x.ll_mode = ll_mode; x.word_stride = word_stride;
    x.icnt = (int32_t**)calloc((size_t)nt, sizeof(int32_t*));
    x.fcol = (float**)calloc((size_t)nt, sizeof(float*));
    x.part = (orc_sample_stats*)calloc((size_t)nt, sizeof(orc_sample_stats));
    x.wll = (double*)calloc((size_t)s->V, sizeof(double));
    for (int t = 0; t < nt; ++t) {
        x.icnt[t] = (int32_t*)calloc((size_t)s->K * 3, sizeof(int32_t)); /* counts, split topics, split counts */
        x.fcol[t] = (float*)calloc((size_t)s->K, sizeof(float));
    }
    parallel_for(nt, s->V, 16, sp_words, &x);
    orc_sample_stats tot;
    memset(&tot, 0, sizeof(tot));
    for (int t = 0; t < nt; ++t) {
        tot.tokens += x.part[t].tokens;
        tot.early_accept += x.part[t].early_accept;
        tot.full += x.part[t].full;
        tot.sum_nnz_full += x.part[t].sum_nnz_full;
        tot.branch_max += x.part[t].branch_max;
        tot.branch_s += x.part[t].branch_s;
        tot.branch_q += x.part[t].branch_q;
        free(x.icnt[t]); free(x.fcol[t]);
    }
    for (int32_t w = 0; w < s->V; ++w) tot.loglik += x.wll[w];
    free(x.icnt); free(x.fcol); free(x.part); free(x.wll);
    if (st) *st = tot;
    return 0;
}

int orc_set_doc_range(orc_state* s, int32_t d0, int32_t d1) {
    if (!s || d0 < 0 || d1 < d0 || d1 > s->D) return -1;
    s->doc_lo = d0;
    s->doc_hi = d1;
    return 0;
}

int orc_iterate(orc_state* s, uint16_t* z, uint64_t seed, uint32_t iter, int32_t ll_mode,
                orc_sample_stats* st) {
    if (!s || !z) return -1;
    /* Counts must be a snapshot of the iteration-start topics: sample into a
     * copy, as EZLDA samples into WTDenseCopy (utility.cu:1998,2937). */
    uint16_t* zin = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)(s->N > 0 ? s->N : 1));
    if (!zin) return -1;
    memcpy(zin, z, sizeof(uint16_t) * (size_t)s->N);
    int rc = orc_rebuild(s, zin);
    if (rc == 0) rc = orc_sample(s, z, seed, iter, ll_mode, 1, st);
    s->built = 0;
    s->z = NULL;
    free(zin);
    return rc;
}

/* ------------------------------------------------------------------- fold-in */
/* Fold-in of a new document against frozen counts (the word-topic counts and n_k of the
 * last orc_rebuild stay fixed; only the document's own topic counts move).  Each sweep
 * draws every token with draw_token() from the document's sweep-start counts, as the
 * training sweep does (EZLDA's sampler with the word-topic side frozen). */
float orc_foldin_uniform(uint64_t seed, uint32_t rid, uint32_t sweep, uint32_t pos) {
    uint32_t ctr[4] = {pos, rid, sweep, 0x464F4C44u};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t x[4];
    orc_philox4x32_10(ctr, key, x);
    return (float)(x[0] >> 8) * 0x1p-24f;
}

uint16_t orc_foldin_init(uint64_t seed, uint32_t rid, uint32_t pos, int32_t K) {
    uint32_t ctr[4] = {pos, rid, 0xFFFFFFFFu, 0x46494E49u};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t x[4];
    orc_philox4x32_10(ctr, key, x);
    return (uint16_t)(((uint64_t)x[0] * (uint64_t)(uint32_t)K) >> 32);
}

int orc_foldin(const orc_state* s, const int32_t* words, int32_t len, uint32_t rid, uint64_t seed,
               int32_t sweeps, uint16_t* z, float* theta) {
    if (!s || !s->built || !words || !z || len < 1 || len > 65535 || sweeps < 0) return -1;
    const int32_t K = s->K;
    for (int32_t i = 0; i < len; ++i)
        if (words[i] < 0 || words[i] >= s->V) return -2;
    int32_t* cnt = (int32_t*)malloc(sizeof(int32_t) * (size_t)K * 3);
    int32_t* hist = (int32_t*)calloc((size_t)K, sizeof(int32_t));
    float* colz = (float*)malloc(sizeof(float) * (size_t)K);
    uint32_t* row = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)K);
    uint16_t* zn = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)len);
    if (!cnt || !hist || !colz || !row || !zn) {
        free(cnt); free(hist); free(colz); free(row); free(zn);
        return -3;
    }
    for (int32_t i = 0; i < len; ++i) z[i] = orc_foldin_init(seed, rid, (uint32_t)i, K);
    for (int32_t sw = 0; sw < sweeps; ++sw) {
        memset(hist, 0, sizeof(int32_t) * (size_t)K);
        for (int32_t i = 0; i < len; ++i) hist[z[i]]++;
        int32_t nnz = 0;
        for (int32_t k = 0; k < K; ++k)
            if (hist[k]) row[nnz++] = ((uint32_t)k << 16) | (uint32_t)hist[k];
        for (int32_t i = 0; i < len; ++i) {
            float QP[LANES], qlf[LANES];
            word_ctx wc;
            word_ctx_of(s, words[i], cnt, colz, QP, &wc, cnt + K, cnt + 2 * (size_t)K, qlf, 1);
            const int32_t cmax = hist[wc.maxK];
            const int32_t c2 = hist[s->top2[words[i]] >> 16];
            const float u = orc_foldin_uniform(seed, rid, (uint32_t)sw, (uint32_t)i);
            int ea, evald, br;
            float total;
            zn[i] = (uint16_t)draw_token(&wc, row, nnz, cmax, c2, len, u, 0, &ea, &evald, &total, &br);
        }
        memcpy(z, zn, sizeof(uint16_t) * (size_t)len);
    }
    if (theta) {
        memset(hist, 0, sizeof(int32_t) * (size_t)K);
        for (int32_t i = 0; i < len; ++i) hist[z[i]]++;
        const float den = (float)len + (float)K * s->alpha;
        for (int32_t k = 0; k < K; ++k) theta[k] = ((float)hist[k] + s->alpha) / den;
    }
    free(cnt); free(hist); free(colz); free(row); free(zn);
    return 0;
}

int orc_get_phi_row(const orc_state* s, int32_t w, float* out) {
    if (!s || !s->built || w < 0 || w >= s->V) return -1;
    int32_t* cnt = (int32_t*)malloc(sizeof(int32_t) * (size_t)s->K);
    if (!cnt) return -3;
    word_column(s, w, cnt, out);
    free(cnt);
    return 0;
}
