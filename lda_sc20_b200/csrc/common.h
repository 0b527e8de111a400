// common.h -- status codes, thread-local error text and the host corpus type.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "lda_b200.h"

namespace lda {

void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);  // set_error + return code
const char* last_error_text();

}  // namespace lda

// Host corpus in the word-sorted chunk layout (EZLDA DocChunk, EZLDA/DataChunk.cuh:22).
// Token i is the i-th token of the concatenation of the chunks' word-sorted lists;
// within a chunk, tokens are ordered by word rank and, inside a word, by doc order.
struct lda_corpus {
    int64_t N = 0, V = 0, D = 0;
    int32_t C = 0, V_dense = 0, max_doc_len = 0, K_hint = 0;
    std::vector<int32_t> tok_word;   // [N]
    std::vector<int32_t> tok_doc;    // [N]
    std::vector<uint16_t> z;         // [N]
    std::vector<int64_t> doc_off;    // [D+1] doc-order offsets
    std::vector<int64_t> dtok_pos;   // [N] doc-order token -> word-sorted index
    std::vector<int32_t> dtok_word;  // [N]
    std::vector<int64_t> chunk_tok;  // [C+1]
    std::vector<int64_t> chunk_doc;  // [C+1]
    std::vector<int64_t> word_count; // [V]
    std::vector<int64_t> seg_off;    // [C*V]
    std::vector<int64_t> seg_cnt;    // [C*V]
    // generated corpora: the generator configuration and raw word -> frequency rank
    bool generated = false;
    lda_gen_config gen{};
    std::vector<int32_t> rank_of;    // [V]
};

namespace lda {

// Builds the layout from doc-ordered tokens whose words are already frequency
// ranks.  topics_doc_order may be null (then Philox initial topics are drawn).
int build_layout(lda_corpus& c, int64_t D, const int64_t* doc_off, const int32_t* ranked_words,
                 int64_t V, int32_t V_dense, const uint16_t* topics_doc_order, int32_t K,
                 int32_t num_chunks, uint64_t topic_seed);

// Philox4x32-10 (Salmon et al., SC'11); shared by host code and kernels.
struct Philox {
    static inline void round10(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t& c3, uint32_t k0,
                               uint32_t k1) {
        for (int r = 0; r < 10; ++r) {
            uint64_t p0 = (uint64_t)0xD2511F53u * c0;
            uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
            uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
            uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
            c1 = (uint32_t)p1;
            c3 = (uint32_t)p0;
            c0 = n0;
            c2 = n2;
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
    }
};

uint16_t initial_topic(uint64_t seed, uint64_t tok, int32_t K);

// Device arrays of a trainer that a frozen fold-in model is built from (trainer.cu).
struct ModelSource {
    int device = 0, K = 0, Vd = 0;
    int64_t V = 0;
    float alpha = 0, beta = 0;
    const int* n_k = nullptr;
    const int* dwt = nullptr;
    const uint32_t *swt_off = nullptr, *swt_nnz = nullptr, *swt_ent = nullptr, *top2 = nullptr;
    const void* phi4 = nullptr;  // float4 per word
    const float* ql = nullptr;   // 32 per word
    void* stream = nullptr;
};
int trainer_model_source(lda_trainer* t, ModelSource* out);

}  // namespace lda
