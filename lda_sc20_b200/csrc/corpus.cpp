// corpus.cpp -- corpus layout, synthetic generator and the EZLDA chunk-file format.
//
// Layout (EZLDA DocChunk, EZLDA/DataChunk.cuh:22): the corpus is cut into C chunks of
// contiguous documents; inside a chunk tokens are sorted by word rank, stably in doc
// order (preprocess/streamTestBalance.cpp:375-398), and words are ranked by descending
// corpus frequency with ties to the lower raw id (streamTestBalance.cpp:288-301).
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <memory>
#include <numeric>
#include <random>
#include <sys/stat.h>

#include "common.h"

namespace lda {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

const char* last_error_text() { return g_err.c_str(); }

uint16_t initial_topic(uint64_t seed, uint64_t tok, int32_t K) {
    uint32_t c0 = (uint32_t)tok, c1 = (uint32_t)(tok >> 32), c2 = 0xFFFFFFFFu, c3 = 0x494E4954u;
    Philox::round10(c0, c1, c2, c3, (uint32_t)seed, (uint32_t)(seed >> 32));
    return (uint16_t)(((uint64_t)c0 * (uint64_t)(uint32_t)K) >> 32);
}

int build_layout(lda_corpus& c, int64_t D, const int64_t* doc_off, const int32_t* w,
                 int64_t V, int32_t V_dense, const uint16_t* topics, int32_t K,
                 int32_t num_chunks, uint64_t topic_seed) {
    if (D <= 0 || V <= 0 || num_chunks <= 0 || num_chunks > D)
        return fail(LDA_ERR_ARG, "build_layout: bad sizes D=%lld V=%lld C=%d", (long long)D,
                    (long long)V, num_chunks);
    const int64_t N = doc_off[D];
    if (N >= (int64_t)UINT32_MAX)
        return fail(LDA_ERR_ARG, "corpus of %lld tokens exceeds 2^32-1", (long long)N);
    c.N = N; c.V = V; c.D = D; c.C = num_chunks; c.V_dense = V_dense;
    c.K_hint = K;
    c.doc_off.assign(doc_off, doc_off + D + 1);
    c.max_doc_len = 0;
    for (int64_t d = 0; d < D; ++d) {
        int64_t len = doc_off[d + 1] - doc_off[d];
        if (len < 0) return fail(LDA_ERR_ARG, "doc offsets not ascending at doc %lld", (long long)d);
        if (len > 65535) return fail(LDA_ERR_ARG, "doc %lld has %lld tokens (limit 65535)", (long long)d, (long long)len);
        c.max_doc_len = std::max<int32_t>(c.max_doc_len, (int32_t)len);
    }
    // contiguous doc ranges with balanced token counts
    c.chunk_doc.assign(num_chunks + 1, 0);
    c.chunk_doc[num_chunks] = D;
    {
        int64_t d = 0;
        for (int32_t k = 1; k < num_chunks; ++k) {
            const int64_t target = (N * k + num_chunks - 1) / num_chunks;
            while (d < D && doc_off[d] < target) ++d;
            d = std::max<int64_t>(d, c.chunk_doc[k - 1] + 1);
            d = std::min<int64_t>(d, D - (num_chunks - k));
            c.chunk_doc[k] = d;
        }
    }
    c.chunk_tok.assign(num_chunks + 1, 0);
    for (int32_t k = 0; k <= num_chunks; ++k) c.chunk_tok[k] = doc_off[c.chunk_doc[k]];
    c.tok_word.assign(N, 0);
    c.tok_doc.assign(N, 0);
    c.z.assign(N, 0);
    c.dtok_pos.assign(N, 0);
    c.dtok_word.assign(w, w + N);
    c.word_count.assign(V, 0);
    c.seg_off.assign((size_t)num_chunks * V, 0);
    c.seg_cnt.assign((size_t)num_chunks * V, 0);
    for (int64_t j = 0; j < N; ++j) {
        if (w[j] < 0 || w[j] >= V) return fail(LDA_ERR_ARG, "word %d out of range at token %lld", w[j], (long long)j);
        if (topics && topics[j] >= K) return fail(LDA_ERR_ARG, "topic %d >= K at token %lld", topics[j], (long long)j);
    }
    std::vector<int64_t> fill(V);
    for (int32_t ch = 0; ch < num_chunks; ++ch) {
        int64_t* cnt = &c.seg_cnt[(size_t)ch * V];
        int64_t* off = &c.seg_off[(size_t)ch * V];
        const int64_t j0 = c.chunk_tok[ch], j1 = c.chunk_tok[ch + 1];
        for (int64_t j = j0; j < j1; ++j) cnt[w[j]]++;
        int64_t run = j0;
        for (int64_t v = 0; v < V; ++v) { off[v] = run; fill[v] = run; run += cnt[v]; c.word_count[v] += cnt[v]; }
        for (int64_t d = c.chunk_doc[ch]; d < c.chunk_doc[ch + 1]; ++d) {
            for (int64_t j = doc_off[d]; j < doc_off[d + 1]; ++j) {
                const int64_t pos = fill[w[j]]++;
                c.tok_word[pos] = w[j];
                c.tok_doc[pos] = (int32_t)d;
                c.dtok_pos[j] = pos;
                c.z[pos] = topics ? topics[j] : 0;
            }
        }
    }
    if (!topics) {
        if (K < 1 || K > 65535) return fail(LDA_ERR_ARG, "K=%d out of range", K);
        for (int64_t i = 0; i < N; ++i) c.z[i] = initial_topic(topic_seed, (uint64_t)i, K);
    }
    return LDA_OK;
}

// Frequency ranks: descending count, ties to the lower raw id.
static void rank_words(int64_t V, const std::vector<int64_t>& cnt, std::vector<int32_t>& rank_of) {
    std::vector<int32_t> order(V);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return cnt[a] > cnt[b]; });
    rank_of.assign(V, 0);
    for (int64_t r = 0; r < V; ++r) rank_of[order[r]] = (int32_t)r;
}

static int32_t dense_count(const std::vector<int64_t>& sorted_cnt, int32_t K, int32_t kind, double param) {
    const int64_t V = (int64_t)sorted_cnt.size();
    int64_t nd = 0;
    if (kind == 0) {
        while (nd < V && sorted_cnt[nd] >= K) ++nd;  // streamTestBalance.cpp:100,291
    } else if (kind == 1) {
        nd = (int64_t)std::llround(param * (double)V);
    } else {
        nd = (int64_t)param;
    }
    nd = std::max<int64_t>(0, std::min<int64_t>(nd, V));
    // sparse rows pack counts in 16 bits
    while (nd < V && sorted_cnt[nd] > 65535) ++nd;
    return (int32_t)nd;
}

// ------------------------------------------------------------- generator

namespace {
struct Rng {
    std::mt19937_64 g;
    explicit Rng(uint64_t s) : g(s) {}
    inline double u01() { return ((double)(g() >> 11) + 0.5) * 0x1p-53; }  // (0,1)
    double normal() {  // Marsaglia polar
        for (;;) {
            double a = 2.0 * u01() - 1.0, b = 2.0 * u01() - 1.0, s = a * a + b * b;
            if (s > 0.0 && s < 1.0) return a * std::sqrt(-2.0 * std::log(s) / s);
        }
    }
    // log of a Gamma(a,1) draw (Marsaglia & Tsang 2000; a<1 boosted by U^(1/a))
    double log_gamma_draw(double a) {
        double boost = 0.0;
        if (a < 1.0) { boost = std::log(u01()) / a; a += 1.0; }
        const double d = a - 1.0 / 3.0, cc = 1.0 / std::sqrt(9.0 * d);
        for (;;) {
            double x = normal(), v = 1.0 + cc * x;
            if (v <= 0.0) continue;
            v = v * v * v;
            double u = u01();
            if (u < 1.0 - 0.0331 * x * x * x * x || std::log(u) < 0.5 * x * x + d * (1.0 - v + std::log(v)))
                return std::log(d * v) + boost;
        }
    }
    int64_t poisson(double lam) {  // Knuth's product of uniforms (lam <= 700)
        const double L = std::exp(-lam);
        int64_t k = 0;
        double p = 1.0;
        do { ++k; p *= u01(); } while (p > L);
        return k - 1;
    }
};

// Vose alias table over one topic's word distribution.
struct Alias {
    std::vector<float> prob;
    std::vector<int32_t> alias;
    void build(const std::vector<double>& p) {
        const int64_t n = (int64_t)p.size();
        prob.assign(n, 0.f);
        alias.assign(n, 0);
        std::vector<double> q(n);
        std::vector<int32_t> small, large;
        for (int64_t i = 0; i < n; ++i) { q[i] = p[i] * (double)n; (q[i] < 1.0 ? small : large).push_back((int32_t)i); }
        while (!small.empty() && !large.empty()) {
            int32_t s = small.back(), l = large.back();
            small.pop_back();
            prob[s] = (float)q[s];
            alias[s] = l;
            q[l] = (q[l] + q[s]) - 1.0;
            if (q[l] < 1.0) { large.pop_back(); small.push_back(l); }
        }
        for (int32_t i : large) { prob[i] = 1.0f; alias[i] = i; }
        for (int32_t i : small) { prob[i] = 1.0f; alias[i] = i; }
    }
    inline int32_t draw(double u) const {  // one uniform: slot + coin
        const double x = u * (double)prob.size();
        int64_t s = (int64_t)x;
        if (s >= (int64_t)prob.size()) s = (int64_t)prob.size() - 1;
        return (x - (double)s) < (double)prob[s] ? (int32_t)s : alias[s];
    }
};
}  // namespace

}  // namespace lda

using namespace lda;

namespace {

int check_gen_config(const lda_gen_config* g) {
    if (g->num_docs <= 0 || g->vocab <= 0 || g->gen_topics <= 0 || g->len_min < 1 ||
        g->len_max < g->len_min || g->len_max > 65535 || g->theta_conc <= 0 || g->phi_conc <= 0 ||
        g->K < 1 || g->K > 65535 || g->num_chunks < 1 || g->num_chunks > g->num_docs)
        return fail(LDA_ERR_ARG, "lda_corpus_generate: invalid configuration");
    if (g->len_kind == 0 && (g->len_p1 <= 0 || g->len_p1 > 700))
        return fail(LDA_ERR_ARG, "Poisson mean must be in (0,700]");
    if (g->phi_kind < 0 || g->phi_kind > 2) return fail(LDA_ERR_ARG, "phi_kind must be 0, 1 or 2");
    return LDA_OK;
}

int64_t draw_length(Rng& rng, int32_t kind, double p1, double p2, int32_t lo, int32_t hi) {
    int64_t L;
    if (kind == 0) L = rng.poisson(p1);
    else L = (int64_t)std::llround(std::exp(p1 + p2 * rng.normal()));
    return std::max<int64_t>(lo, std::min<int64_t>(hi, L));
}

// The Dirichlet parameter of phi_t: a_w = phi_conc (kind 0) or phi_conc * V * z_w with z a
// Zipf(phi_zipf_s) base over word rank (kinds 1 and 2).
std::vector<double> phi_base(const lda_gen_config* g) {
    const int64_t V = g->vocab;
    std::vector<double> a(V);
    if (g->phi_kind == 0) {
        std::fill(a.begin(), a.end(), g->phi_conc);
    } else {
        double zs = 0.0;
        for (int64_t r = 0; r < V; ++r) zs += std::pow((double)(r + 1), -g->phi_zipf_s);
        for (int64_t r = 0; r < V; ++r) a[r] = g->phi_conc * (double)V * std::pow((double)(r + 1), -g->phi_zipf_s) / zs;
    }
    return a;
}

// Word draws of the generating topics.  Kinds 0 and 1 draw phi_t ~ Dir(a) explicitly (one
// alias table per topic, T*V gamma draws).  Kind 2 draws the same process in its Polya-urn
// form, for T*V too large to materialise: topic t's n-th word is a copy of one of its n
// earlier words with probability n/(n+A), else a fresh draw from the base a/A (A = sum a),
// which is the predictive of words drawn i.i.d. from phi_t ~ Dir(a) with phi_t integrated out.
struct TopicWords {
    std::vector<Alias> phi;                  // kinds 0, 1
    Alias base;                              // kind 2
    double A = 0.0;
    std::vector<std::vector<int32_t>> drawn; // kind 2: words drawn so far per topic
    bool urn = false;

    void init(Rng& rng, const lda_gen_config* g) {
        const int64_t V = g->vocab;
        const int32_t T = g->gen_topics;
        std::vector<double> a = phi_base(g);
        if (g->phi_kind == 2) {
            urn = true;
            A = 0.0;
            for (double x : a) A += x;
            std::vector<double> p(V);
            for (int64_t v = 0; v < V; ++v) p[v] = a[v] / A;
            base.build(p);
            drawn.assign(T, {});
            return;
        }
        phi.resize(T);
        std::vector<double> lg(V), p(V);
        for (int32_t t = 0; t < T; ++t) {
            double mx = -INFINITY;
            for (int64_t v = 0; v < V; ++v) { lg[v] = rng.log_gamma_draw(a[v]); mx = std::max(mx, lg[v]); }
            double s = 0.0;
            for (int64_t v = 0; v < V; ++v) { p[v] = std::exp(lg[v] - mx); s += p[v]; }
            for (int64_t v = 0; v < V; ++v) p[v] /= s;
            phi[t].build(p);
        }
    }

    int32_t draw(Rng& rng, int32_t t) {
        if (!urn) return phi[t].draw(rng.u01());
        std::vector<int32_t>& L = drawn[t];
        const double n = (double)L.size();
        const double x = rng.u01() * (n + A);
        const int32_t w = x < n ? L[(size_t)x] : base.draw(rng.u01());
        L.push_back(w);
        return w;
    }
};

// Tokens of one document of length L: topics by the Polya urn of theta ~ Dir(theta_conc),
// words from the topics' word draws.
void draw_doc(Rng& rng, TopicWords& tw, int32_t T, double theta_conc, int64_t L, std::vector<int32_t>& tt,
              int32_t* out) {
    const double Ta = (double)T * theta_conc;
    tt.resize(L);
    for (int64_t i = 0; i < L; ++i) {
        const double x = rng.u01() * ((double)i + Ta);
        int32_t t;
        if (x < (double)i) t = tt[(int64_t)x];
        else t = std::min<int32_t>(T - 1, (int32_t)((x - (double)i) / theta_conc));
        tt[i] = t;
        out[i] = tw.draw(rng, t);
    }
}

}  // namespace

extern "C" int lda_corpus_generate(const lda_gen_config* g, lda_corpus** out) {
    if (!g || !out) return fail(LDA_ERR_ARG, "null argument");
    *out = nullptr;
    int rc = check_gen_config(g);
    if (rc) return rc;
    const int64_t D = g->num_docs, V = g->vocab;
    try {
        Rng rng(g->corpus_seed);
        // 1. doc lengths
        std::vector<int64_t> doc_off(D + 1, 0);
        for (int64_t d = 0; d < D; ++d)
            doc_off[d + 1] = doc_off[d] + draw_length(rng, g->len_kind, g->len_p1, g->len_p2, g->len_min, g->len_max);
        const int64_t N = doc_off[D];
        // 2. topic-word distributions
        TopicWords tw;
        tw.init(rng, g);
        // 3. tokens
        std::vector<int32_t> raw(N), tt;
        for (int64_t d = 0; d < D; ++d)
            draw_doc(rng, tw, g->gen_topics, g->theta_conc, doc_off[d + 1] - doc_off[d], tt, raw.data() + doc_off[d]);
        tw = TopicWords();
        // 4. frequency ranks, dense split, layout
        std::vector<int64_t> cnt(V, 0);
        for (int64_t j = 0; j < N; ++j) cnt[raw[j]]++;
        std::vector<int32_t> rank_of;
        rank_words(V, cnt, rank_of);
        std::vector<int64_t> sorted(V);
        for (int64_t v = 0; v < V; ++v) sorted[rank_of[v]] = cnt[v];
        for (int64_t j = 0; j < N; ++j) raw[j] = rank_of[raw[j]];
        const int32_t Vd = dense_count(sorted, g->K, g->dense_kind, g->dense_param);
        auto* c = new lda_corpus();
        rc = build_layout(*c, D, doc_off.data(), raw.data(), V, Vd, nullptr, g->K, g->num_chunks, g->topic_seed);
        if (rc != LDA_OK) { delete c; return rc; }
        c->generated = true;
        c->gen = *g;
        c->rank_of = std::move(rank_of);
        *out = c;
        return LDA_OK;
    } catch (const std::bad_alloc&) {
        return fail(LDA_ERR_NOMEM, "host allocation failed while generating the corpus");
    }
}

extern "C" int lda_corpus_generate_requests(const lda_corpus* c, uint64_t request_seed, int64_t n, double len_mu,
                                            double len_sigma, int32_t len_min, int32_t len_max, int64_t* doc_off,
                                            int32_t* words, int64_t cap) {
    if (!c || !doc_off || n < 0) return fail(LDA_ERR_ARG, "null argument");
    if (!c->generated) return fail(LDA_ERR_STATE, "the corpus was not made by lda_corpus_generate");
    if (len_min < 1 || len_max < len_min || len_max > 65535 || len_sigma < 0)
        return fail(LDA_ERR_ARG, "request lengths must satisfy 1 <= len_min <= len_max <= 65535");
    try {
        // lengths from their own stream, so that the sizing call draws nothing else
        Rng lrng(request_seed ^ 0x4C454E47544853ull);
        doc_off[0] = 0;
        for (int64_t i = 0; i < n; ++i) doc_off[i + 1] = doc_off[i] + draw_length(lrng, 1, len_mu, len_sigma, len_min, len_max);
        if (!words) return LDA_OK;
        if (cap < doc_off[n]) return fail(LDA_ERR_ARG, "words holds %lld entries, %lld needed", (long long)cap, (long long)doc_off[n]);
        // the corpus' generating phi: replay its stream through the doc lengths
        const lda_gen_config* g = &c->gen;
        if (g->phi_kind == 2)
            return fail(LDA_ERR_STATE, "requests need an explicit phi (phi_kind 0 or 1); this corpus used the urn form");
        Rng rng(g->corpus_seed);
        for (int64_t d = 0; d < g->num_docs; ++d) draw_length(rng, g->len_kind, g->len_p1, g->len_p2, g->len_min, g->len_max);
        TopicWords tw;
        tw.init(rng, g);
        Rng drng(request_seed);
        std::vector<int32_t> tt;
        for (int64_t i = 0; i < n; ++i) {
            int32_t* w = words + doc_off[i];
            const int64_t L = doc_off[i + 1] - doc_off[i];
            draw_doc(drng, tw, g->gen_topics, g->theta_conc, L, tt, w);
            for (int64_t j = 0; j < L; ++j) w[j] = c->rank_of[w[j]];
        }
        return LDA_OK;
    } catch (const std::bad_alloc&) {
        return fail(LDA_ERR_NOMEM, "host allocation failed while generating requests");
    }
}

extern "C" int lda_corpus_from_docs(int64_t D, const int64_t* doc_off, const int32_t* words, int64_t V,
                                    const uint16_t* topics, int32_t K, int32_t num_chunks,
                                    int32_t dense_kind, double dense_param, uint64_t topic_seed,
                                    lda_corpus** out) {
    if (!doc_off || !words || !out) return fail(LDA_ERR_ARG, "null argument");
    *out = nullptr;
    if (D <= 0 || V <= 0 || doc_off[0] != 0) return fail(LDA_ERR_ARG, "bad doc offsets / vocab");
    try {
        const int64_t N = doc_off[D];
        std::vector<int64_t> cnt(V, 0);
        for (int64_t j = 0; j < N; ++j) {
            if (words[j] < 0 || words[j] >= V) return fail(LDA_ERR_ARG, "word id %d out of range", words[j]);
            cnt[words[j]]++;
        }
        std::vector<int32_t> rank_of;
        rank_words(V, cnt, rank_of);
        std::vector<int64_t> sorted(V);
        for (int64_t v = 0; v < V; ++v) sorted[rank_of[v]] = cnt[v];
        std::vector<int32_t> ranked(N);
        for (int64_t j = 0; j < N; ++j) ranked[j] = rank_of[words[j]];
        const int32_t Vd = dense_count(sorted, K, dense_kind, dense_param);
        auto* c = new lda_corpus();
        int rc = build_layout(*c, D, doc_off, ranked.data(), V, Vd, topics, K, num_chunks, topic_seed);
        if (rc != LDA_OK) { delete c; return rc; }
        *out = c;
        return LDA_OK;
    } catch (const std::bad_alloc&) {
        return fail(LDA_ERR_NOMEM, "host allocation failed");
    }
}

extern "C" int lda_corpus_info_get(const lda_corpus* c, lda_corpus_info* o) {
    if (!c || !o) return fail(LDA_ERR_ARG, "null argument");
    o->num_tokens = c->N; o->vocab = c->V; o->num_docs = c->D; o->num_chunks = c->C;
    o->num_dense = c->V_dense; o->max_doc_len = c->max_doc_len; o->K_hint = c->K_hint;
    return LDA_OK;
}

template <class T>
static int copy_out(const std::vector<T>& v, void* out, int64_t count) {
    if ((int64_t)v.size() != count) return fail(LDA_ERR_ARG, "count %lld != field size %lld", (long long)count, (long long)v.size());
    std::memcpy(out, v.data(), sizeof(T) * v.size());
    return LDA_OK;
}

extern "C" int lda_corpus_get(const lda_corpus* c, int32_t field, void* out, int64_t count) {
    if (!c || !out) return fail(LDA_ERR_ARG, "null argument");
    switch (field) {
        case LDA_F_TOK_WORD: return copy_out(c->tok_word, out, count);
        case LDA_F_TOK_DOC: return copy_out(c->tok_doc, out, count);
        case LDA_F_TOPICS: return copy_out(c->z, out, count);
        case LDA_F_DOC_OFF: return copy_out(c->doc_off, out, count);
        case LDA_F_DTOK_POS: return copy_out(c->dtok_pos, out, count);
        case LDA_F_DTOK_WORD: return copy_out(c->dtok_word, out, count);
        case LDA_F_CHUNK_TOK: return copy_out(c->chunk_tok, out, count);
        case LDA_F_CHUNK_DOC: return copy_out(c->chunk_doc, out, count);
        case LDA_F_WORD_COUNT: return copy_out(c->word_count, out, count);
        case LDA_F_SEG_OFF: return copy_out(c->seg_off, out, count);
        case LDA_F_SEG_CNT: return copy_out(c->seg_cnt, out, count);
        default: return fail(LDA_ERR_ARG, "unknown corpus field %d", field);
    }
}

extern "C" int lda_corpus_set_topics(lda_corpus* c, const uint16_t* topics, int64_t count) {
    if (!c || !topics || count != c->N) return fail(LDA_ERR_ARG, "bad topics array");
    std::memcpy(c->z.data(), topics, sizeof(uint16_t) * (size_t)count);
    return LDA_OK;
}

extern "C" void lda_corpus_free(lda_corpus* c) { delete c; }

// ------------------------------------------------------------ EZLDA format

namespace {
struct TextOut {
    FILE* f = nullptr;
    std::vector<char> buf;
    bool open(const std::string& p) {
        f = std::fopen(p.c_str(), "wb");
        buf.reserve(1 << 20);
        return f != nullptr;
    }
    void put(int64_t v) {
        char tmp[24];
        int n = 0;
        bool neg = v < 0;
        uint64_t u = neg ? (uint64_t)(-v) : (uint64_t)v;
        do { tmp[n++] = (char)('0' + u % 10); u /= 10; } while (u);
        if (neg) buf.push_back('-');
        while (n) buf.push_back(tmp[--n]);
        if (buf.size() > (1 << 20)) flush();
    }
    void ch(char x) { buf.push_back(x); }
    void line1(int64_t a) { put(a); ch('\n'); }
    void line2(int64_t a, int64_t b) { put(a); ch(' '); put(b); ch('\n'); }
    void flush() { if (!buf.empty()) { std::fwrite(buf.data(), 1, buf.size(), f); buf.clear(); } }
    bool close() { flush(); bool ok = std::ferror(f) == 0; ok = (std::fclose(f) == 0) && ok; f = nullptr; return ok; }
};

struct TextIn {
    std::vector<char> data;
    size_t p = 0;
    int load(const std::string& path) {
        FILE* f = std::fopen(path.c_str(), "rb");
        if (!f) return fail(LDA_ERR_IO, "cannot open %s: %s", path.c_str(), std::strerror(errno));
        std::fseek(f, 0, SEEK_END);
        long n = std::ftell(f);
        std::fseek(f, 0, SEEK_SET);
        data.resize((size_t)(n > 0 ? n : 0));
        size_t got = n > 0 ? std::fread(data.data(), 1, (size_t)n, f) : 0;
        std::fclose(f);
        if ((long)got != n) return fail(LDA_ERR_IO, "short read of %s", path.c_str());
        p = 0;
        return LDA_OK;
    }
    bool next(int64_t& v) {
        while (p < data.size() && (data[p] == ' ' || data[p] == '\n' || data[p] == '\r' || data[p] == '\t')) ++p;
        if (p >= data.size()) return false;
        bool neg = false;
        if (data[p] == '-') { neg = true; ++p; }
        if (p >= data.size() || data[p] < '0' || data[p] > '9') return false;
        int64_t x = 0;
        while (p < data.size() && data[p] >= '0' && data[p] <= '9') x = x * 10 + (data[p++] - '0');
        v = neg ? -x : x;
        return true;
    }
    int64_t count_all() {
        size_t save = p;
        int64_t n = 0, v;
        while (next(v)) ++n;
        p = save;
        return n;
    }
};

static bool make_dir(const std::string& d) {
    if (mkdir(d.c_str(), 0755) == 0) return true;
    return errno == EEXIST;
}
}  // namespace

extern "C" int lda_corpus_write_ezlda(const lda_corpus* c, const char* dir, int32_t K) {
    if (!c || !dir) return fail(LDA_ERR_ARG, "null argument");
    if (K < 1 || K > 65535) return fail(LDA_ERR_ARG, "K=%d out of range", K);
    const std::string root(dir);
    if (!make_dir(root)) return fail(LDA_ERR_IO, "cannot create %s", dir);
    const int64_t V = c->V, Vd = c->V_dense, Vs = V - Vd;
    auto cap32 = [&](int64_t len) { int64_t r = ((len - 1) / 32 + 1) * 32; if (len == 0) r = 32; return std::min<int64_t>(r, K); };
    std::vector<int64_t> dtlen(c->C), wtlen(c->C), nd(c->C), ns(c->C);
    int64_t maxTL = 0, maxDT = 0, maxChunkWT = 0, maxDocs = 0;
    for (int32_t ch = 0; ch < c->C; ++ch) {
        const std::string cd = root + "/chunk" + std::to_string(ch);
        if (!make_dir(cd)) return fail(LDA_ERR_IO, "cannot create %s", cd.c_str());
        const int64_t t0 = c->chunk_tok[ch], t1 = c->chunk_tok[ch + 1];
        const int64_t d0 = c->chunk_doc[ch], d1 = c->chunk_doc[ch + 1];
        maxTL = std::max(maxTL, t1 - t0);
        maxDocs = std::max(maxDocs, d1 - d0);
        TextOut tl, w2d, d2w, wco, dco, dtco, wtco;
        if (!tl.open(cd + "/TL.txt") || !w2d.open(cd + "/word2DocMap.txt") || !d2w.open(cd + "/doc2WordMap.txt") ||
            !wco.open(cd + "/wordCountOffset.txt") || !dco.open(cd + "/docCountOffset.txt") ||
            !dtco.open(cd + "/DTCountOffset.txt") || !wtco.open(cd + "/WTCountOffset.txt"))
            return fail(LDA_ERR_IO, "cannot write chunk files in %s", cd.c_str());
        for (int64_t i = t0; i < t1; ++i) {
            tl.line1((int64_t)c->z[i] + 1);                       // streamTestBalance.cpp:469
            d2w.line1((int64_t)c->tok_doc[i] - d0 + 1);            // :436
        }
        for (int64_t j = t0; j < t1; ++j) w2d.line1(c->dtok_pos[j] - t0);  // :470
        int64_t dt = 0;
        for (int64_t d = d0; d < d1; ++d) {
            const int64_t len = c->doc_off[d + 1] - c->doc_off[d];
            dco.line2(len, c->doc_off[d] - t0);                    // :421
            dtco.line2(cap32(len), dt);                             // :409-410,422
            dt += cap32(len);
        }
        dtlen[ch] = dt;
        maxDT = std::max(maxDT, dt);
        int64_t wt = 0;
        nd[ch] = ns[ch] = 0;
        for (int64_t v = 0; v < V; ++v) {
            const int64_t n = c->seg_cnt[(size_t)ch * V + v];
            wco.line2(n, c->seg_off[(size_t)ch * V + v] - t0);  // :477
            if (v < Vd) nd[ch] += n;
            else {
                ns[ch] += n;
                const int64_t capw = std::min<int64_t>(n, K);       // :451
                wtco.line2(capw, wt);                               // :461
                wt += capw;
            }
        }
        wtlen[ch] = wt;
        maxChunkWT = std::max(maxChunkWT, wt);
        if (!tl.close() || !w2d.close() || !d2w.close() || !wco.close() || !dco.close() || !dtco.close() || !wtco.close())
            return fail(LDA_ERR_IO, "write error in %s", cd.c_str());
    }
    TextOut f;
    int64_t off = 0, sparseStart = 0;
    if (!f.open(root + "/WTCountOffset.txt")) return fail(LDA_ERR_IO, "cannot write WTCountOffset.txt");
    for (int64_t v = 0; v < V; ++v) {
        const int64_t capw = std::min<int64_t>(c->word_count[v], K);
        if (v == Vd) sparseStart = off;
        f.line2(capw, off);                                          // :487-505
        off += capw;
    }
    if (Vd == V) sparseStart = off;
    if (!f.close()) return fail(LDA_ERR_IO, "write error");
    const int64_t maxWT = off - sparseStart;
    struct { const char* name; int which; } per[] = {{"docLength.txt", 0}, {"TLLength.txt", 1}, {"DTLength.txt", 2},
                                                     {"WTLength.txt", 3}, {"TLSplit.txt", 4}};
    for (auto& e : per) {
        if (!f.open(root + "/" + e.name)) return fail(LDA_ERR_IO, "cannot write %s", e.name);
        for (int32_t ch = 0; ch < c->C; ++ch) {
            switch (e.which) {
                case 0: f.line1(c->chunk_doc[ch + 1] - c->chunk_doc[ch]); break;
                case 1: f.line1(c->chunk_tok[ch + 1] - c->chunk_tok[ch]); break;
                case 2: f.line1(dtlen[ch]); break;
                case 3: f.line1(wtlen[ch]); break;
                default: f.line2(nd[ch], ns[ch]); break;
            }
        }
        if (!f.close()) return fail(LDA_ERR_IO, "write error");
    }
    if (!f.open(root + "/lengthVec.txt")) return fail(LDA_ERR_IO, "cannot write lengthVec.txt");
    // maxTLLength maxDTLength maxWTLength maxDocLength W maxChunkWTLength numOfWordD numOfWordS (:546)
    f.put(maxTL); f.ch(' '); f.put(maxDT); f.ch(' '); f.put(maxWT); f.ch(' '); f.put(maxDocs); f.ch(' ');
    f.put(V); f.ch(' '); f.put(maxChunkWT); f.ch(' '); f.put(Vd); f.ch(' '); f.put(Vs);
    if (!f.close()) return fail(LDA_ERR_IO, "write error");
    return LDA_OK;
}

extern "C" int lda_corpus_load_ezlda(const char* dir, lda_corpus** out) {
    if (!dir || !out) return fail(LDA_ERR_ARG, "null argument");
    *out = nullptr;
    const std::string root(dir);
    try {
        TextIn lv;
        int rc = lv.load(root + "/lengthVec.txt");
        if (rc) return rc;
        int64_t L[8];
        for (int i = 0; i < 8; ++i)
            if (!lv.next(L[i])) return fail(LDA_ERR_FORMAT, "lengthVec.txt: expected 8 integers");
        const int64_t V = L[4], Vd = L[6], Vs = L[7];
        if (V <= 0 || Vd < 0 || Vs < 0 || Vd + Vs != V)
            return fail(LDA_ERR_FORMAT, "lengthVec.txt: inconsistent W=%lld numOfWordD=%lld numOfWordS=%lld",
                        (long long)V, (long long)Vd, (long long)Vs);
        TextIn fd, ft, fs;
        if ((rc = fd.load(root + "/docLength.txt")) || (rc = ft.load(root + "/TLLength.txt")) ||
            (rc = fs.load(root + "/TLSplit.txt")))
            return rc;
        const int64_t C = fd.count_all();
        if (C <= 0 || ft.count_all() != C || fs.count_all() != 2 * C)
            return fail(LDA_ERR_FORMAT, "docLength/TLLength/TLSplit disagree on the chunk count");
        std::vector<int64_t> Dc(C), Nc(C);
        int64_t D = 0, N = 0;
        for (int64_t ch = 0; ch < C; ++ch) {
            int64_t a = -1, b = -1;
            fd.next(Dc[ch]); ft.next(Nc[ch]); fs.next(a); fs.next(b);
            if (Dc[ch] <= 0 || Nc[ch] < 0 || a + b != Nc[ch] || a < 0 || b < 0)
                return fail(LDA_ERR_FORMAT, "chunk %lld: bad doc/token counts", (long long)ch);
            D += Dc[ch];
            N += Nc[ch];
        }
        if (N >= (int64_t)UINT32_MAX) return fail(LDA_ERR_FORMAT, "corpus exceeds 2^32-1 tokens");
        auto* c = new lda_corpus();
        std::unique_ptr<lda_corpus> guard(c);
        c->N = N; c->V = V; c->D = D; c->C = (int32_t)C; c->V_dense = (int32_t)Vd; c->K_hint = 0;
        c->tok_word.assign(N, 0); c->tok_doc.assign(N, -1); c->z.assign(N, 0);
        c->doc_off.assign(D + 1, 0); c->dtok_pos.assign(N, -1); c->dtok_word.assign(N, 0);
        c->chunk_tok.assign(C + 1, 0); c->chunk_doc.assign(C + 1, 0);
        c->word_count.assign(V, 0);
        c->seg_off.assign((size_t)C * V, 0); c->seg_cnt.assign((size_t)C * V, 0);
        for (int64_t ch = 0; ch < C; ++ch) { c->chunk_tok[ch + 1] = c->chunk_tok[ch] + Nc[ch]; c->chunk_doc[ch + 1] = c->chunk_doc[ch] + Dc[ch]; }
        c->max_doc_len = 0;
        for (int64_t ch = 0; ch < C; ++ch) {
            const std::string cd = root + "/chunk" + std::to_string(ch);
            const int64_t t0 = c->chunk_tok[ch], d0 = c->chunk_doc[ch], n = Nc[ch];
            TextIn tl, w2d, wco, dco;
            if ((rc = wco.load(cd + "/wordCountOffset.txt")) || (rc = dco.load(cd + "/docCountOffset.txt")) ||
                (rc = tl.load(cd + "/TL.txt")) || (rc = w2d.load(cd + "/word2DocMap.txt")))
                return rc;
            int64_t run = 0;
            for (int64_t v = 0; v < V; ++v) {
                int64_t cnt, off;
                if (!wco.next(cnt) || !wco.next(off))
                    return fail(LDA_ERR_FORMAT, "%s/wordCountOffset.txt truncated at word %lld", cd.c_str(), (long long)v);
                if (cnt < 0 || (cnt > 0 && off != run))
                    return fail(LDA_ERR_FORMAT, "%s/wordCountOffset.txt: word %lld offset %lld, expected %lld", cd.c_str(), (long long)v, (long long)off, (long long)run);
                c->seg_cnt[(size_t)ch * V + v] = cnt;
                c->seg_off[(size_t)ch * V + v] = t0 + run;
                for (int64_t i = 0; i < cnt; ++i) {
                    if (run + i >= n) return fail(LDA_ERR_FORMAT, "%s: word segments exceed TLLength", cd.c_str());
                    c->tok_word[t0 + run + i] = (int32_t)v;
                }
                run += cnt;
                c->word_count[v] += cnt;
            }
            if (run != n) return fail(LDA_ERR_FORMAT, "%s: word counts sum to %lld, TLLength is %lld", cd.c_str(), (long long)run, (long long)n);
            for (int64_t i = 0; i < n; ++i) {
                int64_t t, p;
                if (!tl.next(t)) return fail(LDA_ERR_FORMAT, "%s/TL.txt truncated at token %lld", cd.c_str(), (long long)i);
                if (t < 1 || t > 65535) return fail(LDA_ERR_FORMAT, "%s/TL.txt: topic %lld out of range", cd.c_str(), (long long)t);
                c->z[t0 + i] = (uint16_t)(t - 1);
                if (!w2d.next(p)) return fail(LDA_ERR_FORMAT, "%s/word2DocMap.txt truncated at token %lld", cd.c_str(), (long long)i);
                if (p < 0 || p >= n) return fail(LDA_ERR_FORMAT, "%s/word2DocMap.txt: position %lld out of range", cd.c_str(), (long long)p);
                c->dtok_pos[t0 + i] = t0 + p;
            }
            int64_t drun = 0;
            for (int64_t i = 0; i < Dc[ch]; ++i) {
                int64_t cnt, off;
                if (!dco.next(cnt) || !dco.next(off))
                    return fail(LDA_ERR_FORMAT, "%s/docCountOffset.txt truncated at doc %lld", cd.c_str(), (long long)i);
                if (cnt < 0 || cnt > 65535 || off != drun)
                    return fail(LDA_ERR_FORMAT, "%s/docCountOffset.txt: doc %lld count %lld offset %lld", cd.c_str(), (long long)i, (long long)cnt, (long long)off);
                c->doc_off[d0 + i] = t0 + drun;
                for (int64_t j = 0; j < cnt; ++j) {
                    const int64_t pos = c->dtok_pos[t0 + drun + j];
                    if (c->tok_doc[pos] != -1) return fail(LDA_ERR_FORMAT, "%s/word2DocMap.txt is not a permutation", cd.c_str());
                    c->tok_doc[pos] = (int32_t)(d0 + i);
                }
                drun += cnt;
                c->max_doc_len = std::max<int32_t>(c->max_doc_len, (int32_t)cnt);
            }
            if (drun != n) return fail(LDA_ERR_FORMAT, "%s: doc counts sum to %lld, TLLength is %lld", cd.c_str(), (long long)drun, (long long)n);
        }
        c->doc_off[D] = N;
        for (int64_t j = 0; j < N; ++j) c->dtok_word[j] = c->tok_word[c->dtok_pos[j]];
        for (int64_t v = Vd; v < V; ++v)
            if (c->word_count[v] > 65535) return fail(LDA_ERR_FORMAT, "sparse word %lld has %lld tokens (limit 65535)", (long long)v, (long long)c->word_count[v]);
        *out = guard.release();
        return LDA_OK;
    } catch (const std::bad_alloc&) {
        return fail(LDA_ERR_NOMEM, "host allocation failed while loading %s", dir);
    }
}

extern "C" const char* lda_last_error(void) { return lda::last_error_text(); }
